"""The NMODL front end (mind_b200.nmodl): parsing, lowering and the emitted CUDA C.

MOD sources here are small ones written for these tests.  Where the MIND.jl checkout is
present, its mod/ directory is parsed too and the committed generated header is checked
to be exactly what the generator makes from it.
"""
import os
import subprocess

import pytest

import mind_b200 as mb
from mind_b200.nmodl.cuda import compile_source, emit_mechanism
from mind_b200.nmodl.parser import Binary, ModError, Unary, parse_mod

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mind.jl_b200", "csrc")
MOD_DIR = "/root/reference/mod"

LEAKY = """
TITLE a leaky gate for the tests
NEURON {
    SUFFIX leaky
    USEION k READ ek WRITE ik
    NONSPECIFIC_CURRENT il
    RANGE gbar, gl, el
}
DEFINE NSTEP 2
PARAMETER {
    gbar = 0.01 (S/cm2) <0, 1e9>
    gl = 1e-4 el = -70 (mV)
    level[NSTEP] (mV)
}
STATE { w }
ASSIGNED { v (mV) ek (mV) ik (mA/cm2) il (mA/cm2) winf wtau (ms) celsius }
INITIAL { w = 0.5 }
BREAKPOINT {
    SOLVE gates METHOD cnexp
    ik = gbar * w^2 * (v - ek)
    il = gl * (v - el)
}
DERIVATIVE gates {
    winf = 1 / (1 + exp(-(v + 40) / 5))
    wtau = 2 + level[1] * 0
    w' = (winf - w) / wtau
}
"""

AFFINE = """
NEURON { POINT_PROCESS drift NONSPECIFIC_CURRENT i RANGE k }
PARAMETER { k = 0.5 }
STATE { x }
ASSIGNED { v i }
BREAKPOINT { SOLVE s METHOD cnexp i = x * 0 }
DERIVATIVE s { x' = -k * x + 2 * k }
NET_RECEIVE (w) { x = x + w }
"""


def test_precedence_power_binds_tighter_than_unary_minus():
    mod = parse_mod("NEURON { SUFFIX p } ASSIGNED { y } INITIAL { y = -2^2^3 + 1 }")
    assign = mod.blocks["initial"].body[0]
    top = assign.value
    assert isinstance(top, Binary) and top.op == "+"
    neg = top.left
    assert isinstance(neg, Unary) and isinstance(neg.arg, Binary) and neg.arg.op == "^"
    assert isinstance(neg.arg.right, Binary) and neg.arg.right.op == "^"   # right-associative


def test_lowering_columns_currents_and_ions():
    ir = compile_source(LEAKY, "leaky.mod")
    assert ir.name == "leaky" and ir.kind == "density"
    assert ir.field_names[:5] == ("gbar", "gl", "el", "level[0]", "level[1]")
    assert "v" not in ir.field_names and "celsius" not in ir.field_names
    assert ir.currents == ["il", "ik"] and ir.ion_reads == [("ek", "k")]
    code = emit_mechanism(ir, "Leaky")
    # the relaxation form takes cnexp's fast path; the current sums NONSPECIFIC then ions
    assert "s.w = s.w + (1.0 - mind_exp(s.dt * (-1.0 / s.wtau))) * (s.winf - s.w);" in code
    assert code.index("value += s.il;") < code.index("value += s.ik;")
    assert "mind_pow(s.w, 2.0)" in code


def test_general_affine_equation_and_net_receive():
    code = emit_mechanism(compile_source(AFFINE, "drift.mod"), "Drift")
    assert "mind_exponential_factor(r_.c * s.dt)" in code
    assert "void receive(const MindGenRow &r, double w_, double flag_)" in code
    assert "s.x = (s.x + w_);" in code


@pytest.mark.parametrize("source, message", [
    ("NEURON { SUFFIX k } KINETIC scheme { }", "KINETIC"),
    ("NEURON { SUFFIX k } ASSIGNED { y } INITIAL { y = q }", "unknown name"),
    ("NEURON { SUFFIX k } STATE { x } BREAKPOINT { SOLVE d METHOD cnexp } DERIVATIVE d { x' = x * x }",
     "affine"),
    ("NEURON { SUFFIX k } BREAKPOINT { SOLVE d METHOD sparse } DERIVATIVE d { }", "METHOD"),
])
def test_unsupported_constructs_are_rejected_with_their_line(source, message):
    with pytest.raises(ModError, match=message):
        emit_mechanism(compile_source(source, "bad.mod"), "Bad")


def test_emitted_code_compiles_for_sm_100a(tmp_path):
    """A user MOD's emitted struct compiles with nvcc against the runtime header (no GPU)."""
    src = tmp_path / "user.cu"
    body = emit_mechanism(compile_source(LEAKY, "leaky.mod"), "Leaky")
    src.write_text('#include "gen_runtime.cuh"\nnamespace mind {\n' + body + "\n"
                   "__global__ void k(MindGenRow r) { Leaky::initial(r); r.at(0) = Leaky::current(r); "
                   "Leaky::advance(r); }\n}\n")
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    out = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c", "-I", CSRC,
                          "-o", str(tmp_path / "user.o"), str(src)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_library_lists_its_emitted_mechanisms():
    table = mb.compiled_mechanisms()
    assert set(table) >= {"SEClamp", "VClamp", "hh", "pas", "ExpSyn", "Exp2Syn", "IClamp", "AlphaSynapse"}
    assert all(m.code >= 64 for m in table.values())
    assert table["VClamp"].fields[:3] == ("dur[0]", "dur[1]", "dur[2]")
    assert table["Exp2Syn"].receive_arity == 1 and table["hh"].ion_reads == (("ena", "na"), ("ek", "k"))
    # the emitted MODs are the same sources whose digests key the hand-written descriptors
    assert table["hh"].digest == mb.builtin("hh").digest
    assert mb.builtin("SEClamp").code == table["SEClamp"].code


@pytest.mark.skipif(not os.path.isdir(MOD_DIR), reason="MIND.jl checkout not present")
def test_reference_mod_directory_parses_and_regenerates_the_committed_header():
    import sys

    for name in os.listdir(MOD_DIR):
        if name.endswith(".mod"):
            parse_mod(open(os.path.join(MOD_DIR, name)).read(), name)
    sys.path.insert(0, CSRC)
    import gen_mechanisms
    from mind_b200.nmodl.library import library_header, read_sources

    paths = [os.path.join(MOD_DIR, f"{n}.mod") for n in gen_mechanisms.MECHANISMS]
    with open(os.path.join(CSRC, "generated_mechanisms.cuh")) as f:
        assert f.read() == library_header(read_sources(paths))
    for name in ("hh", "SEClamp"):
        assert mb.load_mod(os.path.join(MOD_DIR, f"{name}.mod")).code == mb.compiled_mechanisms()[name].code


@pytest.mark.skipif(not os.path.isdir(MOD_DIR), reason="MIND.jl checkout not present")
def test_mechanism_ir_of_a_compiled_mod_and_clear_mod_cache():
    """mechanism_ir gives the lowered MOD of what compile_mod returned; clear_mod_cache drops
    the cached view of the library's registry, which reads back the same."""
    seclamp = mb.load_mod(os.path.join(MOD_DIR, "SEClamp.mod"))
    ir = mb.mechanism_ir(seclamp)
    assert ir.name == "SEClamp" and ir.kind == "point"
    assert tuple(ir.field_names) == seclamp.fields and ir.digest == seclamp.digest
    before = mb.compiled_mechanisms()
    mb.clear_mod_cache()
    assert mb.compiled_mechanisms() == before


def test_hand_written_builtins_have_no_ir():
    with pytest.raises(ValueError, match="hand-written"):
        mb.mechanism_ir(mb.builtin("hh"))


def test_a_user_mod_compiles_into_a_mechanism_module_for_sm_100a():
    """register_mod's compile step, without a GPU: a MOD file the library was not built with
    is emitted after the compiled-in mechanisms and the window kernel's generated variants
    compile with it into a cubin (mind_load_mechanisms loads it on a GPU)."""
    import os

    from mind_b200 import mechanisms
    from mind_b200.nmodl.cuda import compile_source

    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, "mod", "UserExpSyn.mod")
    ir = compile_source(open(path).read(), path)
    assert ir.name == "UserExpSyn" and ir.kind == "point" and len(ir.receive_args) == 1
    first = len(mechanisms.compiled_mechanisms())
    module = mechanisms.mechanism_module([ir], first)
    assert os.path.getsize(module) > 10000
    header = open(os.path.join(os.path.dirname(module), "runtime_mechanisms.cuh")).read()
    assert f"M{first}_UserExpSyn" in header and "gen_builtin_current(id, r)" in header
