"""The C-ABI library loads and exports every entry point include/mindgpu.h declares (CPU, no compute)."""
import ctypes
import os
import re

from mind_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mindgpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(mind_[a-z_]+)\s*\(", text, flags=re.M)))


def test_header_and_binding_agree():
    declared = declared_functions()
    assert "mind_create" in declared and "mind_run" in declared
    assert sorted(abi.EXPORTED_SYMBOLS) == declared


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(abi.library_path())
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_malformed_layout_rejected_before_any_device_work():
    """A parent index out of range is refused with status 10 (no CUDA call is reached)."""
    import mind_b200 as mb
    from mind_b200 import networks

    layout = mb.build(networks.config1(n_cells=1))
    layout.parent[5] = 10_000
    lib = abi.load_library()
    c_layout = layout.to_c()
    handle = ctypes.c_void_p()
    status = lib.mind_create(ctypes.byref(c_layout), ctypes.byref(handle))
    assert status == abi.MIND_ELAYOUT
    assert b"parent" in lib.mind_last_error(None)


def test_null_handles_are_refused_without_device_work():
    """Every entry point that takes a handle answers a null one with MIND_EARG (12)
    before any CUDA call; destroying nothing succeeds; the create error text is kept."""
    lib = abi.load_library()
    d = ctypes.c_double()
    i32 = ctypes.c_int32()
    i64 = ctypes.c_int64()
    rec = abi.MindRecord(abi.MIND_RECORD_VOLTAGE, 1, 0, 0, 0)
    calls = {
        "mind_set_precision": (None, 0), "mind_initialize": (None,), "mind_run": (None, 1, None, 0, 0),
        "mind_step": (None,), "mind_time": (None, ctypes.byref(i64), ctypes.byref(d)),
        "mind_get_trace": (None, None, 0), "mind_get_spikes": (None, None, None, 0, ctypes.byref(i64)),
        "mind_read_voltage": (None, 1, ctypes.byref(d)), "mind_read_value": (None, ctypes.byref(rec), ctypes.byref(d)),
        "mind_inject_event": (None, 1, 0.0), "mind_inject_spikes": (None, 0, None, None),
        "mind_window_steps": (None, ctypes.byref(i32)), "mind_autotune": (None, 0),
        "mind_bin_threads": (None, None, 0, ctypes.byref(i32)), "mind_set_bin_threads": (None, None, 0),
        "mind_attach_macro": (None, None), "mind_get_macro_trace": (None, None, 0, None),
        "mind_set_drive_recording": (None, 1.0), "mind_get_drive": (None, None, 0, None),
        "mind_attach_surrogate": (None, None, None, 1.0), "mind_set_surrogate_cells": (None, None),
            "mind_set_surrogate_offsets": (None, None, 0), "mind_exchange_id": (None,),
            "mind_attach_exchange": (None, None, 2, 0, 1, 1, None, None, 0, None, None, 0),
            "mind_exchange_pack": (None, None), "mind_exchange_inject": (None, None),
        "mind_last_run_ms": (None, ctypes.byref(d)), "mind_run_stats": (None, None),
        "mind_set_profiling": (None, 1), "mind_run_noalloc": (None, 1, None, 0, None),
        "mind_mlp_param_count": (None, ctypes.byref(i64)), "mind_mlp_last_ms": (None, None), "mind_mlp_set_params": (None, None, 0),
        "mind_mlp_get_params": (None, None, 0), "mind_mlp_predict": (None, None, 0, None),
        "mind_mlp_gradients": (None, None, None, 1, None, None), "mind_mlp_set_data": (None, None, None, 1),
        "mind_mlp_train": (None, 1, 1, ctypes.c_float(1e-3), None, None), "mind_mlp_create": (None, None),
        "mind_mechanism_count": (None,), "mind_mechanism_info": (0, None), "mind_mechanism_kind": (None, None),
        "mind_discretize": (None, 1, 0, None, None, 0), "mind_load_mechanisms": (None, None, 0), "mind_get_trace_by_record": (None, None, 0),
    }
    declared = set(declared_functions())
    for name, args in calls.items():
        assert name in declared, name
        assert getattr(lib, name)(*args) == abi.MIND_EARG, name
    assert lib.mind_destroy(None) == abi.MIND_OK and lib.mind_mlp_destroy(None) == abi.MIND_OK
    untested = declared - set(calls) - {"mind_create", "mind_destroy", "mind_mlp_destroy", "mind_last_error",
                                        "mind_mlp_last_error"}
    assert not untested, untested
