"""Several handles in one process: the window kernel's shared-memory opt-in is an attribute
of the kernel function, shared by every handle, so a handle created later with smaller
cells must not shrink what an earlier handle with larger cells launches with."""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
from mind_b200 import networks
from mind_b200.runtime import DeviceState

pytestmark = pytest.mark.gpu


def test_a_later_handle_with_smaller_cells_leaves_an_earlier_one_running():
    big = mb.build(networks.config3(n_cells=4, synapses_per_cell=20))
    small = mb.build(networks.config1(n_cells=2, synapses_per_cell=2))
    nodes = [big.voltage_node(c) for c in range(1, big.n_cells + 1)]
    recs = [mb.RecordSpec(n, f"n{n}") for n in nodes]
    alone = DeviceState(big)
    alone.initialize()
    want = alone.run_steps(400, recs, True)
    alone.close()
    first = DeviceState(big)
    first.initialize()
    second = DeviceState(small)       # made after the first, with far smaller cells
    second.initialize()
    got = first.run_steps(400, recs, True)
    second.run_steps(400, [], True)
    for r in recs:
        np.testing.assert_array_equal(got.traces[r.name], want.traces[r.name])
    np.testing.assert_array_equal(got.spike_times, want.spike_times)
    first.close()
    second.close()
