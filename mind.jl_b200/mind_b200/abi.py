"""ctypes view of include/mindgpu.h and the loader for libmindgpu.so.

This is the Python side of the same boundary the Julia adapter binds with
ccall (mind.jl_b200/julia/MINDGPU.jl): plain pointers and sizes, no torch types.
The library is built in-tree by mind.jl_b200/csrc/build.py; there is no
fallback — a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_int32, c_int64, c_uint64, c_void_p)

MIND_ABI_VERSION = 2

MIND_OK = 0
MIND_ECAPACITY = 3
MIND_ESELFEVENT = 5
MIND_ESINGULAR = 6
MIND_ENONFINITE = 8
MIND_ETIMEOUT = 9
MIND_ELAYOUT = 10
MIND_ECUDA = 11
MIND_EARG = 12

MIND_FP64 = 0
MIND_MIXED = 1

MIND_RECORD_VOLTAGE = 1
MIND_RECORD_MECHANISM = 2

STATUS_NAMES = {
    MIND_ECAPACITY: "capacity exhausted",
    MIND_ESELFEVENT: "invalid self-event delay or target",
    MIND_ESINGULAR: "singular or non-finite cable system",
    MIND_ENONFINITE: "non-finite numerical state",
    MIND_ETIMEOUT: "device wait timeout",
    MIND_ELAYOUT: "layout rejected",
    MIND_ECUDA: "CUDA runtime error",
    MIND_EARG: "invalid argument",
}


class MindMechanism(Structure):
    _fields_ = [
        ("kind", c_int32),
        ("n_fields", c_int32),
        ("rows", c_int64),
        ("data", POINTER(c_double)),
        ("field_names", POINTER(c_char_p)),
        ("nodes", POINTER(c_int32)),
        ("logical_ids", POINTER(c_uint64)),
        ("digest", c_uint64),
    ]


class MindLayout(Structure):
    _fields_ = [
        ("abi_version", c_int32),
        ("secondorder", c_int32),
        ("n_nodes", c_int64),
        ("parent", POINTER(c_int32)),
        ("voltage", POINTER(c_double)),
        ("area", POINTER(c_double)),
        ("capacitance", POINTER(c_double)),
        ("axial", POINTER(c_double)),
        ("axial_diagonal", POINTER(c_double)),
        ("n_mechanisms", c_int32),
        ("mechanisms", POINTER(MindMechanism)),
        ("n_points", c_int64),
        ("point_group", POINTER(c_int32)),
        ("point_row", POINTER(c_int32)),
        ("n_sources", c_int64),
        ("source_ids", POINTER(c_int64)),
        ("source_nodes", POINTER(c_int32)),
        ("source_thresholds", POINTER(c_double)),
        ("source_points", POINTER(c_int32)),
        ("n_edges", c_int64),
        ("fanout_offsets", POINTER(c_int64)),
        ("edge_targets", POINTER(c_int32)),
        ("edge_delays", POINTER(c_double)),
        ("edge_weights", POINTER(c_double)),
        ("dt", c_double),
        ("celsius", c_double),
        ("seed", c_uint64),
        ("event_capacity", c_int64),
        ("spike_capacity", c_int64),
        ("n_pattern", c_int64),
        ("pattern_times", POINTER(c_double)),
        ("pattern_points", POINTER(c_int32)),
    ]


class MindRecord(Structure):
    _fields_ = [("kind", c_int32), ("node", c_int32), ("group", c_int32), ("row", c_int32), ("field", c_int32)]


class MindMechanismInfo(Structure):
    _fields_ = [("name", c_char_p), ("kind", c_int32), ("point", c_int32), ("net_receive", c_int32),
                ("n_fields", c_int32), ("field_names", POINTER(c_char_p)), ("defaults", POINTER(c_double)),
                ("digest", ctypes.c_uint64), ("ion_reads", c_char_p)]


MIND_MECH_GENERATED = 64


class MindSection(Structure):
    _fields_ = [("parent", c_int32), ("nseg", c_int32), ("parent_x", c_double), ("child_x", c_double),
                ("length", c_double), ("diameter", c_double), ("Ra", c_double), ("cm", c_double),
                ("n_points", c_int32), ("points", POINTER(c_double))]


class MindMorphology(Structure):
    _fields_ = [("node_count", c_int64), ("parent", POINTER(c_int32)), ("area", POINTER(c_double)),
                ("diameter", POINTER(c_double)), ("axial", POINTER(c_double)), ("capacitance", POINTER(c_double)),
                ("edge_length", POINTER(c_double)), ("section_start", POINTER(c_int64)),
                ("section_end", POINTER(c_int64)), ("section_first", POINTER(c_int64))]


class MindRunStats(Structure):
    _fields_ = [
        ("run_ms", c_double),
        ("window_ms", c_double),
        ("launches", c_int64),
        ("window_launches", c_int64),
        ("steps", c_int64),
        ("window_steps", c_int32),
        ("bins", c_int32),
    ]


class MindMacroLayout(Structure):
    _fields_ = [
        ("n_regions", c_int32),
        ("params", POINTER(c_double)),
        ("y0", POINTER(c_double)),
        ("micro_gain", POINTER(c_double)),
        ("n_edges", c_int64),
        ("edge_src", POINTER(c_int32)),
        ("edge_dst", POINTER(c_int32)),
        ("edge_gain", POINTER(c_double)),
        ("edge_delay", POINTER(c_int32)),
        ("n_inputs", c_int64),
        ("input_region", POINTER(c_int32)),
        ("input_source", POINTER(c_int64)),
        ("input_scale", POINTER(c_double)),
        ("n_outputs", c_int64),
        ("output_region", POINTER(c_int32)),
        ("output_source", POINTER(c_int64)),
        ("dt_macro", c_double),
        ("bin_ms", c_double),
    ]


class MindMlpConfig(Structure):
    _fields_ = [("n_in", c_int32), ("hidden", c_int32), ("layers", c_int32), ("seed", c_uint64)]


class MindError(RuntimeError):
    """A non-zero status from libmindgpu, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"mindgpu status {status} ({STATUS_NAMES.get(status, 'error')}): {message}")


_LIB = None

PACKAGE_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBRARY_PATH = os.path.join(PACKAGE_ROOT, "lib", "libmindgpu.so")


def library_path() -> str:
    return os.environ.get("MINDGPU_LIBRARY", LIBRARY_PATH)


def load_library():
    """Load libmindgpu.so (built in-tree); raises if it is absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise OSError(f"{path} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(path)
    handle = c_void_p
    lib.mind_create.argtypes = [POINTER(MindLayout), POINTER(handle)]
    lib.mind_initialize.argtypes = [handle]
    lib.mind_set_precision.argtypes = [handle, c_int32]
    lib.mind_run.argtypes = [handle, c_int64, POINTER(MindRecord), c_int32, c_int32]
    lib.mind_step.argtypes = [handle]
    lib.mind_time.argtypes = [handle, POINTER(c_int64), POINTER(c_double)]
    lib.mind_get_trace.argtypes = [handle, POINTER(c_double), c_int64]
    lib.mind_get_trace_by_record.argtypes = [handle, POINTER(c_double), c_int64]
    lib.mind_get_spikes.argtypes = [handle, POINTER(c_double), POINTER(c_int64), c_int64, POINTER(c_int64)]
    lib.mind_read_voltage.argtypes = [handle, c_int32, POINTER(c_double)]
    lib.mind_read_value.argtypes = [handle, POINTER(MindRecord), POINTER(c_double)]
    lib.mind_set_surrogate_cells.argtypes = [handle, POINTER(ctypes.c_uint8)]
    lib.mind_set_surrogate_offsets.argtypes = [handle, POINTER(ctypes.c_float), c_int32]
    i32p = POINTER(c_int32)
    lib.mind_exchange_id.argtypes = [POINTER(ctypes.c_uint8)]
    lib.mind_attach_exchange.argtypes = [handle, POINTER(ctypes.c_uint8), c_int32, c_int32, c_int32, c_int32,
                                         i32p, i32p, c_int32, i32p, i32p, c_int32]
    lib.mind_exchange_pack.argtypes = [handle, c_void_p]
    lib.mind_exchange_inject.argtypes = [handle, c_void_p]
    lib.mind_autotune.argtypes = [handle, c_int32]
    lib.mind_bin_threads.argtypes = [handle, POINTER(c_int32), c_int32, POINTER(c_int32)]
    lib.mind_set_bin_threads.argtypes = [handle, POINTER(c_int32), c_int32]
    lib.mind_inject_event.argtypes = [handle, c_int64, c_double]
    lib.mind_last_error.argtypes = [handle]
    lib.mind_last_error.restype = c_char_p
    lib.mind_last_run_ms.argtypes = [handle, POINTER(c_double)]
    lib.mind_destroy.argtypes = [handle]
    lib.mind_run_stats.argtypes = [handle, POINTER(MindRunStats)]
    lib.mind_set_profiling.argtypes = [handle, c_int32]
    lib.mind_run_noalloc.argtypes = [handle, c_int64, POINTER(MindRecord), c_int32, POINTER(c_double)]
    lib.mind_inject_spikes.argtypes = [handle, c_int64, POINTER(c_int64), POINTER(c_double)]
    lib.mind_window_steps.argtypes = [handle, POINTER(c_int32)]
    lib.mind_attach_macro.argtypes = [handle, POINTER(MindMacroLayout)]
    lib.mind_get_macro_trace.argtypes = [handle, POINTER(c_double), c_int64, POINTER(c_int64)]
    f32 = POINTER(ctypes.c_float)
    lib.mind_set_drive_recording.argtypes = [handle, c_double]
    lib.mind_attach_surrogate.argtypes = [handle, handle, POINTER(ctypes.c_uint8), ctypes.c_float]
    lib.mind_get_drive.argtypes = [handle, f32, c_int64, POINTER(c_int64)]
    lib.mind_mlp_create.argtypes = [POINTER(MindMlpConfig), POINTER(handle)]
    lib.mind_mlp_destroy.argtypes = [handle]
    lib.mind_mlp_last_error.argtypes = [handle]
    lib.mind_mlp_last_error.restype = c_char_p
    lib.mind_mlp_last_ms.argtypes = [handle, f32]
    lib.mind_mlp_param_count.argtypes = [handle, POINTER(c_int64)]
    lib.mind_mlp_set_params.argtypes = [handle, f32, c_int64]
    lib.mind_mlp_get_params.argtypes = [handle, f32, c_int64]
    lib.mind_mlp_predict.argtypes = [handle, f32, c_int64, f32]
    lib.mind_mlp_gradients.argtypes = [handle, f32, f32, c_int64, f32, f32]
    lib.mind_mlp_set_data.argtypes = [handle, f32, f32, c_int64]
    lib.mind_mlp_train.argtypes = [handle, c_int32, c_int32, ctypes.c_float, f32, f32]
    lib.mind_mechanism_count.argtypes = [POINTER(c_int32)]
    lib.mind_mechanism_info.argtypes = [c_int32, POINTER(MindMechanismInfo)]
    lib.mind_mechanism_kind.argtypes = [c_char_p, POINTER(c_int32)]
    lib.mind_load_mechanisms.argtypes = [c_char_p, POINTER(MindMechanismInfo), c_int32]
    lib.mind_discretize.argtypes = [POINTER(MindSection), c_int32, c_int64, POINTER(MindMorphology), c_char_p,
                                    c_int32]
    for name in ("mind_create", "mind_initialize", "mind_set_precision", "mind_run", "mind_step",
                 "mind_time", "mind_get_trace", "mind_get_spikes", "mind_read_voltage", "mind_read_value",
                 "mind_inject_event", "mind_last_run_ms", "mind_destroy", "mind_run_stats",
                 "mind_set_profiling", "mind_run_noalloc", "mind_inject_spikes", "mind_window_steps",
                 "mind_autotune", "mind_bin_threads", "mind_set_bin_threads", "mind_set_surrogate_cells",
                 "mind_set_surrogate_offsets", "mind_exchange_id", "mind_attach_exchange",
                 "mind_exchange_pack", "mind_exchange_inject",
                 "mind_attach_macro", "mind_get_macro_trace", "mind_set_drive_recording", "mind_get_drive",
                 "mind_attach_surrogate",
                 "mind_mlp_create", "mind_mlp_destroy", "mind_mlp_last_ms",
                 "mind_mlp_param_count", "mind_mlp_set_params", "mind_mlp_get_params", "mind_mlp_predict",
                 "mind_mlp_gradients", "mind_mlp_set_data", "mind_mlp_train", "mind_mechanism_count",
                 "mind_mechanism_info", "mind_mechanism_kind", "mind_discretize", "mind_load_mechanisms",
                 "mind_get_trace_by_record"):
        getattr(lib, name).restype = c_int32
    _LIB = lib
    return lib


EXPORTED_SYMBOLS = (
    "mind_create", "mind_initialize", "mind_set_precision", "mind_run", "mind_step", "mind_time",
    "mind_get_trace", "mind_get_spikes", "mind_read_voltage", "mind_read_value", "mind_inject_event",
    "mind_last_error", "mind_last_run_ms", "mind_destroy", "mind_run_stats", "mind_set_profiling",
    "mind_run_noalloc", "mind_inject_spikes", "mind_window_steps", "mind_autotune", "mind_bin_threads",
    "mind_set_surrogate_cells", "mind_set_surrogate_offsets", "mind_exchange_id", "mind_attach_exchange",
    "mind_exchange_pack", "mind_exchange_inject", "mind_load_mechanisms", "mind_get_trace_by_record",
    "mind_set_bin_threads", "mind_attach_macro", "mind_get_macro_trace",
    "mind_set_drive_recording", "mind_get_drive", "mind_attach_surrogate", "mind_mlp_create", "mind_mlp_destroy", "mind_mlp_last_error", "mind_mlp_last_ms", "mind_mlp_param_count", "mind_mlp_set_params",
    "mind_mlp_get_params", "mind_mlp_predict", "mind_mlp_gradients", "mind_mlp_set_data", "mind_mlp_train",
    "mind_mechanism_count", "mind_mechanism_info", "mind_mechanism_kind", "mind_discretize",
)

MIND_NOALLOC_SCRATCH_BYTES = 16 << 20


def check(lib, handle, status: int) -> None:
    if status != MIND_OK:
        message = lib.mind_last_error(handle)
        raise MindError(status, message.decode() if message else "")
