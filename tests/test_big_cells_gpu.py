"""A cell whose shared-memory image would exceed one CTA keeps it in HBM.

The reference solves cells of any size in global memory; here such a cell runs in its
own size bin with the same window kernel reading its image from an HBM slot.  FP64 runs
stay bit-identical to the CPU oracle (voltages of every soma and of nodes deep in the big
tree, and the raster), and the mixed mode stays within its tolerances.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle

pytestmark = pytest.mark.gpu


def test_oversized_cell_runs_from_hbm_and_matches_the_oracle():
    model = netcases.big_and_small_cells()
    layout = mb.build(model)
    off = np.asarray(layout.cell_offsets)
    assert off[1] - off[0] > 7000          # ~34 B per node: beyond 227 KB of shared memory
    nodes = netcases.soma_nodes(layout) + [int(off[0]) + k for k in (500, 3000, 9000)]
    steps = 1600
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    mb.initialize(model, precision="fp64")
    recs = [mb.RecordSpec(n, f"n{n}") for n in nodes]
    res = mb.run(model, steps * layout.dt, records=recs)
    got = np.stack([res.traces[r.name] for r in recs], axis=1)
    assert np.array_equal(got, ref.trace)
    np.testing.assert_array_equal(res.spike_times, ref.spike_times)
    np.testing.assert_array_equal(res.spike_sources, ref.spike_sids)
    assert np.sum(ref.spike_sids < 4) > 0      # the cells fired (sids 0-3 are the cells)
    mb.initialize(model, precision="mixed")
    mixed = mb.run(model, steps * layout.dt, records=recs)
    mx = np.stack([mixed.traces[r.name] for r in recs], axis=1)
    assert np.max(np.abs(mx - ref.trace)) < 0.5    # mV; spikes may shift by a step
