"""Mechanisms as CUDA C emitted from their MOD files (mind_b200.nmodl), on the GPU.

* hh, pas, ExpSyn, Exp2Syn, IClamp and AlphaSynapse emitted from mod/*.mod reproduce the
  hand-written device code bit for bit: the same network with mb.emitted(...) and with
  mb.builtin(...) gives identical traces and rasters, and both equal the CPU FP64 oracle.
* SEClamp and VClamp, which run only as emitted code, match the oracle's hand restatement
  of mod/SEClamp.mod and mod/VClamp.mod bit for bit, and hold the soma at their commands.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200.runtime import DeviceState

pytestmark = pytest.mark.gpu


def gpu_run(layout, steps, nodes, precision="fp64"):
    state = DeviceState(layout, precision)
    state.initialize()
    result = state.run_steps(steps, [mb.RecordSpec(int(n), f"n{n}") for n in nodes])
    state.close()
    return result.traces.by_record.T, result


def test_emitted_cell_mechanisms_equal_the_hand_written_ones_bit_for_bit():
    steps = 1600
    hand = mb.build(netcases.mechanism_mix(mb.builtin))
    gen = mb.build(netcases.mechanism_mix(mb.emitted))
    assert {g.mechanism.code for g in gen.groups} - {5} >= {66, 67, 68, 69, 70, 71}
    nodes = netcases.soma_nodes(hand)
    ref = oracle.run(gen, steps, nodes)
    assert ref.status == 0, ref.message
    t_hand, r_hand = gpu_run(hand, steps, nodes)
    t_gen, r_gen = gpu_run(gen, steps, nodes)
    assert np.array_equal(t_gen, ref.trace), float(np.max(np.abs(t_gen - ref.trace)))
    assert np.array_equal(t_gen, t_hand)
    np.testing.assert_array_equal(r_gen.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(r_gen.spike_times, ref.spike_times)
    np.testing.assert_array_equal(r_gen.spike_sources, r_hand.spike_sources)
    assert np.sum(ref.spike_sids < gen.n_cells) > 5


def test_emitted_clamps_match_the_oracle_and_hold_their_commands():
    steps = 1200   # 30 ms: every command level of both clamps and their release
    layout = mb.build(netcases.mechanism_mix(mb.emitted, clamps=True))
    nodes = netcases.soma_nodes(layout)
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    trace, result = gpu_run(layout, steps, nodes)
    assert np.array_equal(trace, ref.trace), float(np.max(np.abs(trace - ref.trace)))
    np.testing.assert_array_equal(result.spike_times, ref.spike_times)
    at = lambda ms: int(round(ms / layout.dt))
    assert abs(trace[at(12.0), 0] - (-20.0)) < 0.5      # SEClamp level 2 (5-15 ms), rs = 0.01 MOhm
    assert abs(trace[at(4.0), 1] - (-68.0)) < 0.1       # VClamp level 1 (0-6 ms)
    assert abs(trace[at(12.0), 1] - (-25.0)) < 0.1      # VClamp level 2 (6-15 ms)


def test_emitted_fields_are_recorded_and_read():
    """An emitted mechanism's fields are layout columns: recordable and readable by name."""
    model = netcases.mechanism_mix(mb.emitted, clamps=True)
    layout = mb.build(model)
    mb.initialize(model)
    ref = mb.mechanism_ref(model, "SEClamp", 1, "vc")
    result = mb.run(model, 12.0, records=[ref])
    vc = result.traces[ref.name]
    assert vc[int(round(3.0 / layout.dt))] == -70.0 and vc[-1] == -20.0
    assert mb.read_value(model, ref) == -20.0
