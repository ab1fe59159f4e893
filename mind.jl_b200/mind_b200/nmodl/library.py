"""The generated-mechanism header compiled into libmindgpu.so.

`library_header(sources)` turns MOD sources into one CUDA header: a struct of device
functions per mechanism (mind_b200.nmodl.cuda), the dispatch the window kernel calls
for a generated kind (kind code MIND_MECH_GENERATED + its index), and the host table
behind mind_mechanism_info (name, kind, fields, defaults, NET_RECEIVE).  The header in
the package (csrc/generated_mechanisms.cuh) is made by csrc/gen_mechanisms.py; a user
MOD file goes through the same path and a rebuild (build_library).
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
    # device dispatch
    def dispatch(signature: str, call: str, ret: str, default: str, only=None):
        out.append(f"__device__ __forceinline__ {ret} gen_{signature} {{")
        out.append("    switch (id) {")
        for k, ir in enumerate(irs):
            if only is not None and not only(ir):
                continue
            stmt = f"return gen::M{k}_{ir.name}::{call};" if ret != "void" else \
                f"gen::M{k}_{ir.name}::{call}; return;"
            out.append(f"        case {k}: {stmt}")
        out.append("        default: break;")
        out.append("    }")
        if ret != "void":
            out.append(f"    return {default};")
        out.append("}")
    dispatch("initial(int32_t id, const MindGenRow &r)", "initial(r)", "void", "")
    dispatch("current(int32_t id, const MindGenRow &r)", "current(r)", "double", "0.0")
    dispatch("advance(int32_t id, const MindGenRow &r)", "advance(r)", "void", "")
    dispatch("receive(int32_t id, const MindGenRow &r, double w, double flag)", "receive(r, w, flag)", "void", "",
             only=lambda ir: bool(ir.receive_args))
    out.append("")
    out.append("}  // namespace mind")
    return "\n".join(out) + "\n"


def read_sources(paths: Sequence[str]) -> List[Tuple[str, str]]:
    return [(os.path.basename(p), open(p).read()) for p in paths]
