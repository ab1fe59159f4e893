"""CUDA path vs the CPU FP64 oracle, through the C-ABI (libmindgpu.so).

FP64 mode: voltage traces bit-identical (so max |dV| = 0 <= 1e-9 mV) and the
spike raster identical (sids and times).  Mixed mode: bounded |dV| and spike
times within one dt of FP64, with the tolerance written in each test.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import model as M
from mind_b200 import networks

pytestmark = pytest.mark.gpu


def run_gpu(model, t_stop, nodes, precision="fp64"):
    records = [mb.RecordSpec(node, f"n{node}") for node in nodes]
    mb.initialize(model, precision=precision)
    result = mb.run(model, t_stop, records=records)
    trace = np.stack([result.traces[r.name] for r in records], axis=1)
    return result, trace


def assert_fp64_parity(model, t_stop):
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    steps = int(round(t_stop / layout.dt))
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    result, trace = run_gpu(model, t_stop, nodes)
    assert trace.shape == ref.trace.shape
    dv = np.max(np.abs(trace - ref.trace))
    assert dv <= 1e-9, f"max |dV| = {dv} mV"
    np.testing.assert_array_equal(result.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(result.spike_times, ref.spike_times)
    return ref, result, trace


def test_config1_full_fp64():
    """The benchmark's config 1 (64 cells, 100 ms) reproduces the oracle exactly."""
    ref, result, trace = assert_fp64_parity(networks.config1(), 100.0)
    assert np.array_equal(trace, ref.trace)  # bit-exact, not just within 1e-9
    assert len(result.spike_times) > 600     # the 640 NetStim trains fired


def test_spiking_ball_and_stick_fp64():
    ref, result, _ = assert_fp64_parity(netcases.strong_config1(), 50.0)
    n_cells = 16
    assert np.sum(result.spike_sources < n_cells) > 10


def test_recurrent_trees_fp64():
    """Branched cells, Exp2Syn, recurrent NetCons with delays, IClamp drive."""
    ref, result, _ = assert_fp64_parity(netcases.recurrent_trees(), 50.0)
    assert np.sum(result.spike_sources < 24) > 10


def test_split_run_matches_single_run():
    """run!(50) then run!(100) equals one run!(100): the state persists across calls."""
    model = netcases.recurrent_trees()
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    records = [mb.RecordSpec(node, f"n{node}") for node in nodes]
    mb.initialize(model)
    whole = mb.run(model, 40.0, records=records)
    mb.initialize(model)
    first = mb.run(model, 20.0, records=records)
    second = mb.run(model, 40.0, records=records)
    for r in records:
        joined = np.concatenate([first.traces[r.name], second.traces[r.name][1:]])
        np.testing.assert_array_equal(joined, whole.traces[r.name])
    np.testing.assert_array_equal(np.concatenate([first.spike_times, second.spike_times]), whole.spike_times)


def test_mixed_precision_close_to_fp64():
    """FP32 gating/synapses with FP64 cable: |dV| bounded, spikes within 1 dt.

    Tolerance: max |dV| <= 5 mV outside spikes is not meaningful for spiking
    traces, so the test bounds the subthreshold RMS difference (<= 0.5 mV) and
    requires >= 90% of FP64 cell spikes to have a mixed-mode spike of the same
    cell within 1 dt, on a 40 ms recurrent run.
    """
    model = netcases.recurrent_trees()
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    fp64, t64 = run_gpu(model, 40.0, nodes, "fp64")
    mixed, t32 = run_gpu(model, 40.0, nodes, "mixed")
    sub = (t64 < -50.0) & (t32 < -50.0)
    rms = np.sqrt(np.mean((t64[sub] - t32[sub]) ** 2))
    assert rms <= 0.5, rms
    cells = fp64.spike_sources < layout.n_cells
    matched = 0
    for sid, t in zip(fp64.spike_sources[cells], fp64.spike_times[cells]):
        same = mixed.spike_times[mixed.spike_sources == sid]
        matched += np.any(np.abs(same - t) <= layout.dt + 1e-12)
    assert matched >= 0.9 * np.sum(cells)


@pytest.mark.parametrize("order", [1, 2])
def test_secondorder_crank_nicolson_fp64(order):
    """build!(secondorder=1 or 2): the cable matrix with C/(dt/2) and v += 2 x, bit-exact
    against the oracle on the recurrent tree network (spikes included)."""
    from mind_b200.runtime import DeviceState

    layout = mb.build(netcases.recurrent_trees(), secondorder=order)
    nodes = netcases.soma_nodes(layout)
    steps = 1600
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    state = DeviceState(layout, "fp64")
    state.initialize()
    result = state.run_steps(steps, [mb.RecordSpec(n, f"n{n}") for n in nodes])
    state.close()
    assert np.array_equal(result.traces.by_record.T, ref.trace)
    np.testing.assert_array_equal(result.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(result.spike_times, ref.spike_times)
    assert np.sum(ref.spike_sids < layout.n_cells) > 10


def test_patternstim_trains_fp64():
    """PatternStim firings replayed at initialize match the oracle bit for bit, twice (the
    second initialize replays them again)."""
    model, trains = netcases.pattern_driven()
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    ref = oracle.run(layout, 1400, nodes)
    assert ref.status == 0, ref.message
    for _ in range(2):
        result, trace = run_gpu(model, 1400 * layout.dt, nodes)
        assert np.array_equal(trace, ref.trace)
        np.testing.assert_array_equal(result.spike_sources, ref.spike_sids)
        np.testing.assert_array_equal(result.spike_times, ref.spike_times)
    for sid, times in trains.items():
        np.testing.assert_array_equal(result.spike_times[result.spike_sources == sid], np.sort(times))


def test_mixed_long_chains_close_to_fp64():
    """Chains of 24 nodes or more are eliminated and back-substituted by a whole warp in the
    mixed mode (segment scans).  On cells whose dendrites are single chains of 60 to 400
    nodes, driven to spike: subthreshold |dV| against FP64 stays below 1e-3 mV and every
    FP64 spike has a mixed-mode spike of the same cell within one dt (tolerances of this
    test); two mixed runs are identical."""
    model = M.MicroModel(celsius=6.3)
    for nseg in (60, 150, 400):
        soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
        dend = mb.Section("dend", label="dend", parent="soma", parent_x=1.0, length=2.0 * nseg, diameter=2.0,
                          nseg=nseg)
        side = mb.Section("side", label="dend", parent="dend", parent_x=0.5, length=100.0, diameter=1.0, nseg=40)
        cell = M.add_population(model, [soma, dend, side], 1, voltage=-65.0)[0]
        M.insert(cell, mb.builtin("hh"), sections="soma")
        M.insert(cell, mb.builtin("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
    M.add_pointprocesses(model, mb.builtin("IClamp"), np.array([1, 2, 3]), "soma", np.full(3, 0.5),
                         {"del": 2.0, "dur": 40.0, "amp": 0.4})
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    fp64, t64 = run_gpu(model, 50.0, nodes, "fp64")
    mixed, t32 = run_gpu(model, 50.0, nodes, "mixed")
    again, t32b = run_gpu(model, 50.0, nodes, "mixed")
    assert np.array_equal(t32, t32b)
    sub = (t64 < -55.0) & (t32 < -55.0)
    assert np.max(np.abs(t64[sub] - t32[sub])) <= 1e-3
    assert np.sum(fp64.spike_sources < 3) >= 6
    for sid, t in zip(fp64.spike_sources, fp64.spike_times):
        same = mixed.spike_times[mixed.spike_sources == sid]
        assert np.any(np.abs(same - t) <= layout.dt + 1e-12)
