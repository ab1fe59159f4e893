"""ctypes wrapper of the CPU FP64 oracle (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module;
it is the checker for the CUDA path and the timed CPU baseline, never part of it.
`build_oracle()` compiles liboracle.so with the Makefile beside this file, and
liboracle_libm.so, the same restatement on the C library's exp, log and pow
(`run(..., libm=True)`), and liboracle_rev.so, which sums the order-dependent terms in
the opposite order (`run(..., reversed_order=True)`).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
LIBM_PATH = os.path.join(HERE, "liboracle_libm.so")
REV_PATH = os.path.join(HERE, "liboracle_rev.so")
_LIBS = {}


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def _load(libm: bool = False, reversed_order: bool = False):
    if libm and reversed_order:
        raise ValueError("one oracle variant at a time")
    path = LIBM_PATH if libm else REV_PATH if reversed_order else LIB_PATH
    if path not in _LIBS:
        if not os.path.exists(path):
            build_oracle()
        lib = ctypes.CDLL(path)
        lib.oracle_run.restype = ctypes.c_int32
        lib.oracle_run.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
            ctypes.POINTER(ctypes.c_int64), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_int32,
        ]
        lib.oracle_run_macro.restype = ctypes.c_int32
        lib.oracle_run_macro.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
            ctypes.POINTER(ctypes.c_int64), ctypes.c_int64, ctypes.POINTER(ctypes.c_int64),
            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_char_p, ctypes.c_int32,
            ctypes.c_int64,
        ]
        lib.oracle_region_input_count.restype = ctypes.c_int32
        lib.oracle_region_input_count.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int64, ctypes.c_double]
        lib.oracle_exp.restype = ctypes.c_double
        lib.oracle_exp.argtypes = [ctypes.c_double]
        lib.oracle_log.restype = ctypes.c_double
        lib.oracle_log.argtypes = [ctypes.c_double]
        lib.oracle_pow.restype = ctypes.c_double
        lib.oracle_pow.argtypes = [ctypes.c_double, ctypes.c_double]
        lib.oracle_div_milli.restype = None
        lib.oracle_div_milli.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        lib.oracle_philox.restype = None
        lib.oracle_philox.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, ctypes.c_uint32]
        lib.oracle_negexp_stream.restype = None
        lib.oracle_negexp_stream.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int64,
                                             ctypes.POINTER(ctypes.c_double)]
        _LIBS[path] = lib
    return _LIBS[path]


def exp(x: float) -> float:
    return _load().oracle_exp(x)


def log(x: float) -> float:
    return _load().oracle_log(x)


def pow(x: float, y: float) -> float:
    return _load().oracle_pow(x, y)


def div_milli(x):
    """The CUDA path's division-free x / 0.001 (mind_math.h), element-wise."""
    import numpy as np

    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    _load().oracle_div_milli(x.ctypes.data, out.ctypes.data, x.size)
    return out


def region_input_count(seed: int, input_index: int, k: int, mu: float) -> int:
    return _load().oracle_region_input_count(seed, input_index, k, mu)


def philox4x32_10(ctr, key0: int, key1: int):
    words = (ctypes.c_uint32 * 4)(*ctr)
    _load().oracle_philox(words, key0, key1)
    return list(words)


def negexp_stream(logical_id: int, digest: int, seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    _load().oracle_negexp_stream(logical_id, digest, seed, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


@dataclass
class OracleResult:
    status: int
    message: str
    trace: np.ndarray        # [steps+1, n_records]
    spike_times: np.ndarray
    spike_sids: np.ndarray
    run_ms: float
    macro_trace: np.ndarray = None   # [macro boundaries, regions], with regions


# Kind codes of this oracle's hand restatements of the clamps (mind_oracle.cpp).
ORACLE_SECLAMP, ORACLE_VCLAMP = 1001, 1002
_BUILTIN_CODES = {"hh": 1, "pas": 2, "ExpSyn": 3, "Exp2Syn": 4, "NetStim": 5, "IClamp": 6, "AlphaSynapse": 7,
                  "SEClamp": ORACLE_SECLAMP, "VClamp": ORACLE_VCLAMP}


def _oracle_kinds(layout, c_layout) -> None:
    """The oracle knows mechanisms by its own restatements: a group whose mechanism the
    library runs as CUDA C emitted from a MOD file (kind >= 64) is handed to the oracle as
    the restatement of the same MOD (hh, pas, ... by their hand-written oracle code, SEClamp
    and VClamp by the clamp restatements); fields are matched by name, so column order
    does not matter."""
    for i, g in enumerate(layout.groups):
        if g.mechanism.code >= 64:
            code = _BUILTIN_CODES.get(g.mechanism.name)
            if code is None:
                raise ValueError(f"the oracle has no restatement of {g.mechanism.name}")
            c_layout.mechanisms[i].kind = code


def run(layout, steps: int, record_nodes=(), threads: int = 0, spike_cap: int = 1 << 22, macro=None,
        records=None, timed_from: int = 0, libm: bool = False, reversed_order: bool = False) -> OracleResult:
    """Initialize the layout (and the regions of `macro`, a MacroModel) on the CPU and advance
    `steps` micro steps; with regions, `macro_trace` holds out(k) for k = 0 .. steps / (dt_macro/dt).
    `threads` worker threads (0: every host core) share the cells of each step; the result
    does not depend on their number.  `run_ms` times steps timed_from .. steps-1.
    `records` (objects with kind, node, group, row, field, such as RecordSpec) replaces
    `record_nodes` (voltages of 1-based nodes) when given.  libm=True runs the restatement
    built on the C library's exp, log and pow instead of the project's (liboracle_libm.so);
    reversed_order=True the one that sums mechanism rows into a node and children into a
    parent in the opposite order (liboracle_rev.so)."""
    import sys

    pkg = os.path.join(os.path.dirname(HERE), "mind.jl_b200")
    if pkg not in sys.path:
        sys.path.insert(0, pkg)
    from mind_b200 import abi

    lib = _load(libm, reversed_order)
    if threads <= 0:
        threads = os.cpu_count() or 1
    c_layout = layout.to_c()
    _oracle_kinds(layout, c_layout)
    if records is None:
        specs = [(abi.MIND_RECORD_VOLTAGE, int(node), 0, 0, 0) for node in record_nodes]
    else:
        specs = [(r.kind, r.node, r.group, r.row, r.field) for r in records]
    nodes = specs
    recs = (abi.MindRecord * max(1, len(specs)))()
    for i, spec in enumerate(specs):
        recs[i] = abi.MindRecord(*spec)
    trace = np.zeros((steps + 1, max(1, len(nodes))))
    spike_t = np.zeros(spike_cap)
    spike_sid = np.zeros(spike_cap, dtype=np.int64)
    count = ctypes.c_int64()
    ms = ctypes.c_double()
    message = ctypes.create_string_buffer(256)
    c_macro = macro.to_c() if macro is not None else None
    macro_trace = None
    if macro is not None:
        spm = int(round(macro.dt_macro / layout.dt))
        macro_trace = np.zeros((steps // spm + 1, macro.n_regions))
    status = lib.oracle_run_macro(
        ctypes.addressof(c_layout), ctypes.addressof(c_macro) if c_macro is not None else None, steps,
        ctypes.addressof(recs), len(nodes), threads,
        trace.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        spike_t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        spike_sid.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), spike_cap, ctypes.byref(count),
        macro_trace.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if macro_trace is not None else None,
        ctypes.byref(ms), message, 256, int(timed_from))
    n = min(count.value, spike_cap)
    result = OracleResult(status, message.value.decode(), trace[:, :len(nodes)],
                          spike_t[:n].copy(), spike_sid[:n].copy(), ms.value)
    result.macro_trace = macro_trace
    return result
