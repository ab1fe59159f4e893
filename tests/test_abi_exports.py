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
