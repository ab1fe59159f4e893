"""A cell's events of one window have no limit of their own (the reference grows its
event pages instead of failing, src/runtime/cuda/micro.jl:811-882): a burst of hundreds or
thousands of events onto one cell within one window is delivered in heap order and matches
the CPU FP64 oracle bit for bit, where a fixed per-cell inbox used to return status 3."""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_events", [200, 2000])
def test_burst_onto_one_cell_matches_the_oracle(n_events):
    model = netcases.burst_onto_one_cell(n_events=n_events)
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    steps = 400   # 10 ms: the burst lands at 2.5-3.0 ms
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    mb.initialize(model)
    records = [mb.RecordSpec(n, f"n{n}") for n in nodes]
    result = mb.run(model, steps * layout.dt, records=records)
    trace = result.traces.by_record.T
    assert np.array_equal(trace, ref.trace), float(np.max(np.abs(trace - ref.trace)))
    np.testing.assert_array_equal(result.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(result.spike_times, ref.spike_times)
    assert np.max(ref.trace[:, 0]) - ref.trace[0, 0] > 1.0   # the burst moved cell 1's soma
