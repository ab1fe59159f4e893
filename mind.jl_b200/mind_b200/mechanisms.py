"""Builtin mechanism descriptors: the field tables the device kernels understand.

MIND.jl compiles each MOD file into a CompiledMechanism whose IR lists the
instance fields, their defaults and the NET_RECEIVE arity
(src/compiler/ir.jl:264-288, src/compiler/frontend.jl:58-72).  The hot path of
this library evaluates the six builtins the benchmark networks use with
hand-written sm_100a device code, so a mechanism here is a descriptor: its MOD
name, its kind, the C-ABI kind code, its fields with MOD defaults, and the
digest that keys its random streams.

The digest is the first 16 hex digits of the SHA-256 of the MOD source, as the
reference derives it for Philox keys (src/compiler/ir.jl:316-324,
src/runtime/initialize.jl:309).  The values below were computed from the
reference's mod/*.mod files; only NetStim draws random numbers.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Any, Dict, Tuple

# C-ABI kind codes (include/mindgpu.h).
MIND_MECH_HH = 1
MIND_MECH_PAS = 2
MIND_MECH_EXPSYN = 3
MIND_MECH_EXP2SYN = 4
MIND_MECH_NETSTIM = 5
MIND_MECH_ICLAMP = 6
MIND_MECH_ALPHASYN = 7
MIND_MECH_PATTERNSTIM = 8


@dataclass(frozen=True)
class Mechanism:
    """A compiled mechanism as the model builders see it (CompiledMechanism)."""

    name: str
    kind: str  # "density" | "point" | "artificial"
    code: int
    fields: Tuple[str, ...]
    defaults: Tuple[float, ...]
    digest: int
    receive_arity: int = 0
    # Fields filled from ion species at build time (USEION ... READ e<ion>).
    ion_reads: Tuple[Tuple[str, str], ...] = field(default_factory=tuple)
    # The lowered MOD (mind_b200.nmodl.cuda.MechanismIR) when this process compiled the
    # source (compile_mod, load_mod, register_mod); None for hand-written device code.
    ir: Any = field(default=None, compare=False, repr=False)

    def field_index(self, name: str) -> int:
        try:
            return self.fields.index(name)
        except ValueError:
            raise ValueError(f"{self.name} has no field {name}") from None

    @property
    def has_net_receive(self) -> bool:
        return self.receive_arity > 0


def _mechanism(name, kind, code, table, digest, arity=0, ion_reads=()):
    fields = tuple(name for name, _ in table)
    defaults = tuple(float(value) for _, value in table)
    return Mechanism(name, kind, code, fields, defaults, digest, arity, tuple(ion_reads))


# PARAMETER defaults from mod/*.mod; ASSIGNED and STATE fields start at 0.
_BUILTINS: Dict[str, Mechanism] = {
    "hh": _mechanism(
        "hh",
        "density",
        MIND_MECH_HH,
        [
            ("gnabar", 0.12), ("gkbar", 0.036), ("gl", 0.0003), ("el", -54.3),
            ("m", 0.0), ("h", 0.0), ("n", 0.0),
            ("ena", 50.0), ("ek", -77.0),
            ("gna", 0.0), ("gk", 0.0), ("ina", 0.0), ("ik", 0.0), ("il", 0.0),
            ("minf", 0.0), ("hinf", 0.0), ("ninf", 0.0),
            ("mtau", 0.0), ("htau", 0.0), ("ntau", 0.0),
        ],
        0x06A1D0784470B30B,
        ion_reads=(("ena", "na"), ("ek", "k")),
    ),
    "pas": _mechanism(
        "pas", "density", MIND_MECH_PAS,
        [("g", 0.001), ("e", -70.0), ("i", 0.0)],
        0x7C96D2C7CB7FE0C5,
    ),
    "ExpSyn": _mechanism(
        "ExpSyn", "point", MIND_MECH_EXPSYN,
        [("tau", 0.1), ("e", 0.0), ("g", 0.0), ("i", 0.0)],
        0x9704333E132D681C,
        arity=1,
    ),
    "Exp2Syn": _mechanism(
        "Exp2Syn", "point", MIND_MECH_EXP2SYN,
        [("tau1", 0.1), ("tau2", 10.0), ("e", 0.0), ("A", 0.0), ("B", 0.0),
         ("g", 0.0), ("i", 0.0), ("factor", 0.0)],
        0xC42E524B775C6D4D,
        arity=1,
    ),
    "NetStim": _mechanism(
        "NetStim", "artificial", MIND_MECH_NETSTIM,
        [("interval", 10.0), ("number", 10.0), ("start", 50.0), ("noise", 0.0),
         ("event", 0.0), ("on", 0.0), ("ispike", 0.0)],
        0xA186833B569FF3B2,
        arity=1,
    ),
    "AlphaSynapse": _mechanism(
        "AlphaSynapse", "point", MIND_MECH_ALPHASYN,
        [("onset", 0.0), ("tau", 0.1), ("gmax", 0.0), ("e", 0.0), ("i", 0.0), ("g", 0.0)],
        0x29B06B38B5009424,
    ),
    "IClamp": _mechanism(
        "IClamp", "point", MIND_MECH_ICLAMP,
        [("del", 0.0), ("dur", 0.0), ("amp", 0.0), ("i", 0.0)],
        0x6EB0551A76C267F8,
    ),
    # an artificial cell that fires at the spike_times given to add_pointprocess
    "PatternStim": _mechanism("PatternStim", "artificial", MIND_MECH_PATTERNSTIM, [], 0x053F906BDBA59243),
}


def compiled_mechanisms() -> Dict[str, Mechanism]:
    """The mechanisms whose CUDA C was emitted from MOD files (mind_b200.nmodl) and compiled
    into libmindgpu.so, by name (mind_mechanism_info; kind codes MIND_MECH_GENERATED + k)."""
    global _COMPILED
    if _COMPILED is None:
        import ctypes

        from . import abi

        lib = abi.load_library()
        n = ctypes.c_int32()
        abi.check(lib, None, lib.mind_mechanism_count(ctypes.byref(n)))
        table = {}
        for k in range(n.value):
            info = abi.MindMechanismInfo()
            abi.check(lib, None, lib.mind_mechanism_info(k, ctypes.byref(info)))
            name = info.name.decode()
            fields = tuple(info.field_names[j].decode() for j in range(info.n_fields))
            defaults = tuple(float(info.defaults[j]) for j in range(info.n_fields))
            words = (info.ion_reads or b"").decode().split()
            reads = tuple(zip(words[0::2], words[1::2]))
            table[name] = Mechanism(name, "point" if info.point else "density", int(info.kind), fields, defaults,
                                    int(info.digest), int(info.net_receive), reads)
        _COMPILED = table
    return _COMPILED


_COMPILED = None


def builtin(name) -> Mechanism:
    """Select a packaged builtin by its MOD name (frontend.jl:58-72): the hand-written device
    code for hh, pas, ExpSyn, Exp2Syn, NetStim, IClamp and AlphaSynapse, else a mechanism
    emitted from the reference's MOD directory into the library (SEClamp, VClamp)."""
    key = str(name)
    if key in _BUILTINS:
        return _BUILTINS[key]
    compiled = compiled_mechanisms()
    if key in compiled:
        return compiled[key]
    raise ValueError(f"unknown mechanism {key}; the library runs {sorted(set(_BUILTINS) | set(compiled))}; "
                     "load a MOD file with load_mod")


def emitted(name: str) -> Mechanism:
    """The mechanism `name` as CUDA C emitted from its MOD file and compiled into the library
    (for hh, pas, ExpSyn, Exp2Syn, IClamp and AlphaSynapse this is the same MOD that
    builtin() runs through hand-written device code)."""
    try:
        return compiled_mechanisms()[str(name)]
    except KeyError:
        raise ValueError(f"{name} is not compiled into this library as emitted code") from None


def compile_mod(source: str, filename: str = "<string>") -> Mechanism:
    """compile_mod (src/compiler/frontend.jl:85-110): parse and lower MOD source, and select
    the emitted mechanism the library knows for exactly this source (same name and SHA-256
    digest) -- compiled in, or compiled now (register_mod) when it is new.  The emitted CUDA
    C (mind_b200.nmodl.emit) runs through the window kernel's generated-mechanism path, even
    for names that also have hand-written code."""
    from .nmodl.cuda import compile_source

    ir = compile_source(source, filename)
    compiled = compiled_mechanisms().get(ir.name)
    if compiled is None:
        return _register(ir)
    if compiled.digest != ir.digest:
        raise ValueError(f"{ir.name} ({filename}) differs from the {ir.name} this process already knows "
                         "(a mechanism name is registered once)")
    if compiled.fields != ir.field_names:
        raise ValueError(f"{ir.name}: the library's fields differ from this source's")
    return Mechanism(ir.name, ir.kind, compiled.code, compiled.fields, compiled.defaults, ir.digest,
                     len(ir.receive_args), tuple(ir.ion_reads), ir)


_RUNTIME = []   # MechanismIR of the mechanisms compiled at run time, in registry order


def register_mod(source: str, filename: str = "<string>") -> Mechanism:
    """Compile MOD source that the library was not built with and register it
    (mind_load_mechanisms): its CUDA C is emitted after the compiled-in mechanisms
    (mind_b200.nmodl.library.runtime_header), the window kernel's generated-mechanism
    variants are compiled with it into a module (nvcc for sm_100a, csrc/gen_module.cu,
    cached by the header's digest under mind.jl_b200/lib/mechanisms/), and the library
    loads the module.  Handles created afterwards run it.  Returns its Mechanism."""
    from .nmodl.cuda import compile_source

    ir = compile_source(source, filename)
    known = compiled_mechanisms().get(ir.name)
    if known is not None:
        if known.digest != ir.digest:
            raise ValueError(f"{ir.name} ({filename}) differs from the {ir.name} this process already knows")
        return dataclasses.replace(known, ir=ir)
    return _register(ir)


def mechanism_module(irs, first_id: int) -> str:
    """The cubin of csrc/gen_module.cu for the mechanisms `irs` as generated ids first_id..
    (compiled with nvcc for sm_100a on first use, cached by the header's digest)."""
    import hashlib
    import os
    import subprocess

    from .nmodl.library import runtime_header

    header = runtime_header(irs, first_id)
    package = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    csrc = os.path.join(package, "csrc")
    # The key covers the kernel sources the module is compiled from, not only the emitted
    # header: a module built from other sources than the library's could disagree with it on
    # the launch parameters' layout.
    key = hashlib.sha256(header.encode())
    sources = sorted(f for f in os.listdir(csrc) if f.endswith((".cu", ".cuh", ".h")))
    for path in [os.path.join(csrc, f) for f in sources] + [os.path.join(package, "..", "include", "mindgpu.h")]:
        with open(path, "rb") as f:
            key.update(os.path.basename(path).encode() + b"\0" + f.read())
    out_dir = os.path.join(package, "lib", "mechanisms", key.hexdigest()[:16])
    module = os.path.join(out_dir, "module.cubin")
    if not os.path.exists(module):
        os.makedirs(out_dir, exist_ok=True)
        with open(os.path.join(out_dir, "runtime_mechanisms.cuh"), "w") as f:
            f.write(header)
        nvcc = os.environ.get("NVCC") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc")
                                         else "nvcc")
        cmd = [nvcc, "-cubin", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
               "-fmad=false", "-DMIND_RUNTIME_MECHANISMS", "-I", out_dir, "-I", csrc, "-o", module + ".tmp",
               os.path.join(csrc, "gen_module.cu")]
        done = subprocess.run(cmd, capture_output=True, text=True)
        if done.returncode != 0:
            raise RuntimeError(f"nvcc failed on the mechanism module ({done.returncode}):\n{done.stderr}")
        os.replace(module + ".tmp", module)
    return module


def _register(ir) -> Mechanism:
    import ctypes

    from . import abi

    global _COMPILED
    lib = abi.load_library()
    first_id = len(compiled_mechanisms()) - len(_RUNTIME)
    irs = _RUNTIME + [ir]
    module = mechanism_module(irs, first_id)
    keep = []   # ctypes buffers that must outlive the call
    infos = (abi.MindMechanismInfo * len(irs))()
    for k, m in enumerate(irs):
        names = (ctypes.c_char_p * max(1, len(m.field_names)))(*[n.encode() for n in m.field_names])
        defaults = (ctypes.c_double * max(1, len(m.defaults)))(*[float(d) for d in m.defaults])
        reads = " ".join(f"{f} {ion}" for f, ion in m.ion_reads).encode()
        keep += [names, defaults, reads]
        infos[k].name = m.name.encode()
        infos[k].point = int(m.kind == "point")
        infos[k].net_receive = len(m.receive_args)
        infos[k].n_fields = len(m.field_names)
        infos[k].field_names = names
        infos[k].defaults = defaults
        infos[k].digest = m.digest
        infos[k].ion_reads = reads
    status = lib.mind_load_mechanisms(module.encode(), infos, len(irs))
    if status != abi.MIND_OK:
        raise abi.MindError(status, (lib.mind_last_error(None) or b"").decode())
    _RUNTIME.append(ir)
    _COMPILED = None
    return dataclasses.replace(compiled_mechanisms()[ir.name], ir=ir)


def mechanism_ir(mechanism: Mechanism):
    """mechanism_ir (src/compiler/ir.jl:359): the lowered MOD of a mechanism this process
    compiled (compile_mod, load_mod, register_mod): its fields, currents, ion reads, NET_RECEIVE
    arguments and blocks."""
    if mechanism.ir is None:
        raise ValueError(f"{mechanism.name} has no IR in this process: it runs hand-written device code or "
                         "came from the library's registry; load its MOD file with load_mod")
    return mechanism.ir


def clear_mod_cache() -> None:
    """clear_mod_cache! (src/compiler/frontend.jl:113-120): forget this process's view of the
    library's mechanism registry, which the next lookup reads again.  Mechanisms compiled at
    run time stay registered: the registry is append-only, so handles and kind codes made
    from them stay valid."""
    global _COMPILED
    _COMPILED = None


def load_mod(path: str) -> Mechanism:
    """load_mod (src/compiler/frontend.jl:15-57) for one MOD file."""
    with open(path) as f:
        return compile_mod(f.read(), path)


def resolve_mechanism(mechanism) -> Mechanism:
    return mechanism if isinstance(mechanism, Mechanism) else builtin(mechanism)
