"""Parity at the benchmark's own sizes, and on a node order like MIND.jl's DHS layout.

* FP64 at full size: config 3 (1,000 cells, 949k compartments) for 800 steps and
  config 2 (10,000 cells, 5.5M compartments) for 1,200 steps, long enough for
  recurrent cell spikes, routed events and NET_RECEIVE: every soma trace and the
  raster bit-identical to the CPU FP64 oracle (all host threads).
* Mixed mode against FP64 on config 3 for 1 s: max |dV| <= 0.1 mV over every soma
  sample, and >= 99% of FP64 cell spikes matched by a spike of the same cell
  within one dt -- the accuracy bound the mixed mode is specified to meet.
* A layout in DHS order (children before parents, cells interleaved round by round,
  src/model/micro/model.jl:906-1077): the GPU reproduces the oracle bit for bit on it,
  and both stay within 1e-9 mV of the same network in discretization order.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import networks
from mind_b200.runtime import DeviceState

pytestmark = pytest.mark.gpu


def fp64_parity(layout, steps, nodes):
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    state = DeviceState(layout, "fp64")
    state.initialize()
    records = [mb.RecordSpec(int(n), f"n{n}") for n in nodes]
    result = state.run_steps(steps, records)
    state.close()
    trace = result.traces.by_record.T
    assert trace.shape == ref.trace.shape
    assert np.array_equal(trace, ref.trace), f"max |dV| = {np.max(np.abs(trace - ref.trace))} mV"
    np.testing.assert_array_equal(result.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(result.spike_times, ref.spike_times)
    return ref


def test_config3_full_1000cells_800steps_fp64():
    layout = mb.build(networks.config3(n_cells=1000), seed=1)
    ref = fp64_parity(layout, 800, netcases.soma_nodes(layout))
    assert np.sum(ref.spike_sids < layout.n_cells) >= 5   # recurrent cell spikes inside the prefix


def test_config2_full_10000cells_1200steps_fp64():
    layout = mb.build(networks.config2(n_cells=10000), seed=1)
    ref = fp64_parity(layout, 1200, netcases.soma_nodes(layout))
    assert np.sum(ref.spike_sids < layout.n_cells) >= 1


def test_config3_full_1000cells_1s_mixed_accuracy():
    """Tolerance: max |dV| <= 0.1 mV against FP64 over 1 s, >= 99% of spikes within 1 dt."""
    layout = mb.build(networks.config3(n_cells=1000), seed=1)
    nodes = netcases.soma_nodes(layout)
    records = [mb.RecordSpec(int(n), f"n{n}") for n in nodes]
    runs = {p: DeviceState(layout, p) for p in ("fp64", "mixed")}
    for state in runs.values():
        state.initialize()
    chunk, total = 4000, 40000
    worst = 0.0
    rasters = {p: ([], []) for p in runs}
    for _ in range(total // chunk):
        out = {p: s.run_steps(chunk, records) for p, s in runs.items()}
        worst = max(worst, float(np.max(np.abs(out["fp64"].traces.by_record - out["mixed"].traces.by_record))))
        for p, r in out.items():
            rasters[p][0].append(r.spike_sources)
            rasters[p][1].append(r.spike_times)
    for state in runs.values():
        state.close()
    sid64, t64 = (np.concatenate(x) for x in rasters["fp64"])
    sid32, t32 = (np.concatenate(x) for x in rasters["mixed"])
    cells = sid64 < layout.n_cells
    matched = sum(np.any(np.abs(t32[sid32 == s] - t) <= layout.dt + 1e-9) for s, t in zip(sid64[cells], t64[cells]))
    n = int(np.sum(cells))
    assert n > 100
    assert worst <= 0.1, f"max |dV| = {worst} mV"
    assert matched >= 0.99 * n, f"{matched} of {n} spikes within 1 dt"


def test_dhs_ordered_layout_24cells_40ms_fp64():
    model = netcases.recurrent_trees()
    layout = mb.build(model)
    perm, new_of = netcases.permute_layout(layout, netcases.dhs_order(layout))
    assert np.mean(perm.parent > np.arange(1, perm.n_nodes + 1)) > 0.9   # children before parents
    nodes = netcases.soma_nodes(layout)
    ref = fp64_parity(perm, 1600, [int(new_of[n]) for n in nodes])
    plain = oracle.run(layout, 1600, nodes)
    assert np.max(np.abs(ref.trace - plain.trace)) <= 1e-9
    np.testing.assert_array_equal(ref.spike_sids, plain.spike_sids)
    assert np.sum(ref.spike_sids < layout.n_cells) > 10
