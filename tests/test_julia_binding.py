"""The Julia ccall adapter (mind.jl_b200/julia/MINDGPU.jl) against the C-ABI (CPU, text only).

Julia is not installed here, so the adapter cannot run; what can go wrong silently at the
boundary is checked from its source instead: every ccall names an entry point that
include/mindgpu.h declares and the built library exports, with as many argument types as
the C declaration has parameters, and the structs the adapter passes by pointer (MindLayout,
MindMechanism, MindRecord) have the C structs' fields, in the same order, with the Julia
type of each C type.
"""
import ctypes
import os
import re

from mind_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JULIA = open(os.path.join(ROOT, "mind.jl_b200", "julia", "MINDGPU.jl")).read()
HEADER = open(os.path.join(ROOT, "include", "mindgpu.h")).read()


def _strip_c_comments(text):
    return re.sub(r"/\*.*?\*/", "", text, flags=re.S)


def _split_top(text):
    """Split on commas outside (), {} and []."""
    parts, depth, cur = [], 0, ""
    for ch in text:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur.strip())
            cur = ""
        else:
            cur += ch
    parts.append(cur.strip())
    return [p for p in parts if p]


def _balanced(text, start):
    """The text inside the parenthesis that opens at text[start]."""
    depth = 0
    for k in range(start, len(text)):
        depth += text[k] == "("
        depth -= text[k] == ")"
        if depth == 0:
            return text[start + 1:k]
    raise AssertionError("unbalanced parenthesis")


def c_parameter_counts():
    text = _strip_c_comments(HEADER)
    counts = {}
    for m in re.finditer(r"^\s*(?:int|const char \*)\s*(mind_[a-z_0-9]+)\s*\(", text, flags=re.M):
        params = _split_top(_balanced(text, m.end() - 1))
        counts[m.group(1)] = 0 if params == ["void"] else len(params)
    return counts


def julia_ccalls():
    calls = []
    for m in re.finditer(r"ccall\(\(:(mind_[a-z_0-9]+),\s*libmindgpu\),\s*[A-Za-z{}]+,\s*\(", JULIA):
        calls.append((m.group(1), len(_split_top(_balanced(JULIA, m.end() - 1)))))
    return calls


def test_every_ccall_names_a_declared_exported_entry_point_with_its_arity():
    declared = c_parameter_counts()
    lib = ctypes.CDLL(abi.library_path())
    calls = julia_ccalls()
    assert len(calls) >= 15
    for name, n_args in calls:
        assert name in declared, f"{name} is not declared in include/mindgpu.h"
        assert hasattr(lib, name), f"{name} is not exported by libmindgpu.so"
        assert n_args == declared[name], f"{name}: {n_args} argument types, C declares {declared[name]}"


def _c_fields(struct):
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct), _strip_c_comments(HEADER), re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        name = re.search(r"([A-Za-z_0-9]+)$", decl).group(1)
        ctype = decl[: -len(name)].strip()
        fields.append((name, ctype))
    return fields


def _julia_fields(struct):
    body = re.search(r"\nstruct %s\n(.*?)\nend\n" % struct, JULIA, re.S).group(1)
    return [tuple(x.strip() for x in line.split("::")) for line in body.strip().splitlines()]


_SCALARS = {"int32_t": "Int32", "int64_t": "Int64", "uint64_t": "UInt64", "double": "Float64"}


def test_structs_passed_by_pointer_match_the_c_layout():
    for struct in ("MindMechanism", "MindLayout", "MindRecord"):
        c, jl = _c_fields(struct), _julia_fields(struct)
        assert [n for n, _ in c] == [n for n, _ in jl], struct
        for (name, ctype), (_, jtype) in zip(c, jl):
            if "*" in ctype:
                assert jtype.startswith("Ptr{"), f"{struct}.{name}: {ctype} is a pointer, Julia has {jtype}"
            else:
                assert jtype == _SCALARS[ctype], f"{struct}.{name}: {ctype} needs {_SCALARS[ctype]}, Julia has {jtype}"


def test_abi_version_matches():
    c = int(re.search(r"#define MIND_ABI_VERSION\s+(\d+)", HEADER).group(1))
    jl = int(re.search(r"const MIND_ABI_VERSION = Int32\((\d+)\)", JULIA).group(1))
    assert c == jl
