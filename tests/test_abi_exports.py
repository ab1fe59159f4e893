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
