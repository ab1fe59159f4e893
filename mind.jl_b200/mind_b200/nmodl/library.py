"""The generated-mechanism header compiled into libmindgpu.so.

`library_header(sources)` turns MOD sources into one CUDA header: a struct of device
functions per mechanism (mind_b200.nmodl.cuda), the dispatch the window kernel calls
for a generated kind (kind code MIND_MECH_GENERATED + its index), and the host table
behind mind_mechanism_info (name, kind, fields, defaults, NET_RECEIVE).  The header in
the package (csrc/generated_mechanisms.cuh) is made by csrc/gen_mechanisms.py.  A user
MOD file is compiled at run time instead: `runtime_header` emits it after the compiled-in
mechanisms, as a module of the window kernel's generated-mechanism variants
(mind_b200.mechanisms.register_mod, mind_load_mechanisms).
"""
from __future__ import annotations

import os
from typing import List, Sequence, Tuple

from .cuda import MechanismIR, compile_source, emit_mechanism

MIND_MECH_GENERATED = 64


def _c_string(text: str) -> str:
    return '"' + text.replace("\\", "\\\\").replace('"', '\\"') + '"'


def library_header(sources: Sequence[Tuple[str, str]]) -> str:
    """sources: (filename, MOD text) pairs, in the order that numbers the kinds."""
    irs: List[MechanismIR] = [compile_source(text, name) for name, text in sources]
    names = [ir.name for ir in irs]
    if len(set(names)) != len(names):
        raise ValueError("two MOD files declare the same mechanism name")
    return _header(irs)


def runtime_header(irs: Sequence[MechanismIR], first_id: int) -> str:
    """The header of a mechanism module compiled at run time (mind_load_mechanisms): the
    mechanisms `irs` as generated ids first_id, first_id + 1, ..., after the ones compiled
    into the library, whose header it includes with its dispatch renamed gen_builtin_*; its
    own dispatch serves the new ids and passes the others on."""
    out = ["/*",
           " * runtime_mechanisms.cuh -- CUDA C emitted from MOD files by mind_b200.nmodl at run time: the",
           f" * generated mechanisms {first_id}.. after those compiled into libmindgpu.so.",
           " */",
           "#pragma once",
           "",
           "#define MIND_GEN_BUILTIN_DISPATCH 1",
           '#include "generated_mechanisms.cuh"',
           "",
           "namespace mind {",
           "namespace gen {",
           ""]
    for k, ir in enumerate(irs):
        out.append(emit_mechanism(ir, f"M{first_id + k}_{ir.name}"))
        out.append("")
    out.append("}  // namespace gen")
    out.append("")
    _dispatch(out, irs, first_id, "gen_", "gen_builtin_")
    out.append("")
    out.append("}  // namespace mind")
    return "\n".join(out) + "\n"


def _dispatch(out: List[str], irs: Sequence[MechanismIR], first_id: int, prefix: str, fallback: str = None):
    """The window kernel's entry points for generated ids first_id..; other ids go to
    `fallback` (the compiled-in dispatch) or do nothing."""
    def one(name: str, params: str, args: str, call: str, ret: str, default: str, only=None):
        out.append(f"__device__ __forceinline__ {ret} {prefix}{name}({params}) {{")
        out.append("    switch (id) {")
        for k, ir in enumerate(irs):
            if only is not None and not only(ir):
                continue
            target = f"gen::M{first_id + k}_{ir.name}::{call}"
            stmt = f"return {target};" if ret != "void" else f"{target}; return;"
            out.append(f"        case {first_id + k}: {stmt}")
        out.append("        default: break;")
        out.append("    }")
        if fallback is not None:
            out.append(f"    {'return ' if ret != 'void' else ''}{fallback}{name}({args});")
        elif ret != "void":
            out.append(f"    return {default};")
        out.append("}")
    one("initial", "int32_t id, const MindGenRow &r", "id, r", "initial(r)", "void", "")
    one("current", "int32_t id, const MindGenRow &r", "id, r", "current(r)", "double", "0.0")
    one("advance", "int32_t id, const MindGenRow &r", "id, r", "advance(r)", "void", "")
    one("receive", "int32_t id, const MindGenRow &r, double w, double flag", "id, r, w, flag", "receive(r, w, flag)",
        "void", "", only=lambda ir: bool(ir.receive_args))


def _header(irs: Sequence[MechanismIR]) -> str:
    out = ["/*",
           " * generated_mechanisms.cuh -- CUDA C emitted from MOD files by mind_b200.nmodl.  Do not edit:",
           " * regenerate with mind.jl_b200/csrc/gen_mechanisms.py.  Each mechanism's kind code is",
           " * MIND_MECH_GENERATED + its index below; its fields are its columns in order.",
           " */",
           "#pragma once",
           "",
           '#include "gen_runtime.cuh"',
           "",
           "namespace mind {",
           "namespace gen {",
           ""]
    for k, ir in enumerate(irs):
        out.append(emit_mechanism(ir, f"M{k}_{ir.name}"))
        out.append("")
    out.append("}  // namespace gen")
    out.append("")
    out.append(f"constexpr int kGeneratedCount = {len(irs)};")
    # host table
    columns, defaults, offsets = [], [], [0]
    for ir in irs:
        columns += [_c_string(c) for c in ir.field_names]
        defaults += [repr(float(d)) for d in ir.defaults]
        offsets.append(len(columns))
    out.append("struct GenMechanism {")
    out.append("    const char *name;")
    out.append("    int32_t point;          // 1: POINT_PROCESS, 0: density (SUFFIX)")
    out.append("    int32_t net_receive;    // NET_RECEIVE arity (0: none)")
    out.append("    int32_t first_field;    // into kGenFieldNames / kGenDefaults")
    out.append("    int32_t n_fields;");
    out.append("    uint64_t digest;        // first 16 hex digits of the MOD source's SHA-256")
    out.append("    const char *ion_reads;  // \"field ion ...\" pairs a USEION READ fills from the ion species")
    out.append("};")
    out.append("static const char *const kGenFieldNames[] = {" + ", ".join(columns or ['""']) + "};")
    out.append("static const double kGenDefaults[] = {" + ", ".join(defaults or ["0.0"]) + "};")
    out.append("static const GenMechanism kGenMechanisms[] = {")
    for k, ir in enumerate(irs):
        reads = " ".join(f"{f} {ion}" for f, ion in ir.ion_reads)
        out.append(f"    {{{_c_string(ir.name)}, {int(ir.kind == 'point')}, {len(ir.receive_args)}, {offsets[k]}, "
                   f"{offsets[k + 1] - offsets[k]}, 0x{ir.digest:016X}ull, {_c_string(reads)}}},")
    out.append("};")
    out.append("")
    # device dispatch: a module compiled at run time (runtime_header) includes this header with
    # MIND_GEN_BUILTIN_DISPATCH defined, which renames these entry points gen_builtin_*
    out.append("#ifdef MIND_GEN_BUILTIN_DISPATCH")
    _dispatch(out, irs, 0, "gen_builtin_")
    out.append("#else")
    _dispatch(out, irs, 0, "gen_")
    out.append("#endif")
    out.append("")
    out.append("}  // namespace mind")
    return "\n".join(out) + "\n"


def read_sources(paths: Sequence[str]) -> List[Tuple[str, str]]:
    return [(os.path.basename(p), open(p).read()) for p in paths]
