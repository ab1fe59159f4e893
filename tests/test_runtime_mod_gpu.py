"""MOD files compiled at run time (register_mod / load_mod, mind_load_mechanisms).

Two mechanisms the library was not built with, written for these tests (tests/mod): a
single-exponential synapse and a passive leak whose equations are those of ExpSyn and pas.
Each is emitted after the compiled-in mechanisms, compiled with the window kernel into a
module and loaded; a network that uses them must run exactly like the same network on the
builtin ExpSyn and pas.  A second registration appends to the first: handles made before
it keep running.
"""
import os

import numpy as np
import pytest

import mind_b200 as mb
import netcases
from mind_b200.runtime import DeviceState

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _run(layout, steps, nodes):
    state = DeviceState(layout, "fp64")
    state.initialize()
    result = state.run_steps(steps, [mb.RecordSpec(int(n), f"n{n}") for n in nodes])
    return state, result


def test_mods_registered_at_run_time_run_like_the_builtins_they_restate():
    steps = 1600
    known = len(mb.compiled_mechanisms())
    syn = mb.load_mod(os.path.join(HERE, "mod", "UserExpSyn.mod"))
    assert syn.name == "UserExpSyn" and syn.code == 64 + known and syn.receive_arity == 1
    hand = mb.build(netcases.mechanism_mix(mb.builtin))
    nodes = netcases.soma_nodes(hand)
    s_hand, want = _run(hand, steps, nodes)
    s_hand.close()
    first = mb.build(netcases.mechanism_mix(lambda n: syn if n == "ExpSyn" else mb.builtin(n)))
    s_first, got = _run(first, steps, nodes)
    np.testing.assert_array_equal(got.traces.by_record, want.traces.by_record)
    np.testing.assert_array_equal(got.spike_times, want.spike_times)
    # a second mechanism: the new module holds both; the earlier handle keeps its kernels
    leak = mb.load_mod(os.path.join(HERE, "mod", "UserLeak.mod"))
    assert leak.code == syn.code + 1 and leak.kind == "density"
    both = mb.build(netcases.mechanism_mix(
        lambda n: syn if n == "ExpSyn" else leak if n == "pas" else mb.builtin(n)))
    s_both, got2 = _run(both, steps, nodes)
    np.testing.assert_array_equal(got2.traces.by_record, want.traces.by_record)
    s_first.initialize()
    again = s_first.run_steps(steps, [mb.RecordSpec(int(n), f"n{n}") for n in nodes])
    np.testing.assert_array_equal(again.traces.by_record, want.traces.by_record)
    assert np.sum(want.spike_sources < hand.n_cells) > 5
    # the registry knows them by name, and a source that differs from a registered one is refused
    assert leak.name == "userleak"   # a density mechanism is named by its SUFFIX
    assert mb.compiled_mechanisms()["userleak"].fields == ("g", "e", "i")
    with pytest.raises(ValueError):
        mb.compile_mod(open(os.path.join(HERE, "mod", "UserLeak.mod")).read().replace("-70", "-60"), "x.mod")
    s_first.close()
    s_both.close()
