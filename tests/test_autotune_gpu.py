"""Launch shapes of the size bins (mind_set_bin_threads, mind_autotune) on the device.

A bin's cells run one per CTA of 128 threads or of 64 threads serving two owner slots
each; the arithmetic and its order do not depend on the shape, so FP64 runs stay
bit-identical to the CPU oracle and mixed runs are identical between shapes.  Autotune
times trial windows, keeps the faster shape per bin and leaves the state at t = 0.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle

pytestmark = pytest.mark.gpu


def _trace(model, t_stop, nodes, precision):
    mb.initialize(model, precision=precision)
    recs = [mb.RecordSpec(n, f"n{n}") for n in nodes]
    res = mb.run(model, t_stop, records=recs)
    return np.stack([res.traces[r.name] for r in recs], axis=1), res


def test_half_size_ctas_reproduce_the_oracle():
    model = netcases.recurrent_trees(n_cells=12, synapses=10)
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    steps = 1200
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    mb.initialize(model)
    bins = model.state.bin_threads()
    assert bins and all(t == 128 for t in bins)
    model.state.set_bin_threads([64] * len(bins))
    got, res = _trace(model, steps * layout.dt, nodes, "fp64")
    assert model.state.bin_threads() == [64] * len(bins)
    assert np.array_equal(got, ref.trace)
    np.testing.assert_array_equal(res.spike_times, ref.spike_times)
    np.testing.assert_array_equal(res.spike_sources, ref.spike_sids)
    # mixed: the same bits with either shape
    mixed64, _ = _trace(model, steps * layout.dt, nodes, "mixed")
    model.state.set_bin_threads([128] * len(bins))
    mixed128, _ = _trace(model, steps * layout.dt, nodes, "mixed")
    assert np.array_equal(mixed64, mixed128)


def test_autotune_keeps_results_and_restarts_at_zero():
    model = netcases.recurrent_trees(n_cells=16, synapses=8)
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    steps = 800
    ref = oracle.run(layout, steps, nodes)
    mb.initialize(model)
    shapes = mb.autotune(model, windows=2)
    assert all(t in (64, 128) for t in shapes)
    assert mb.simulation_time(model) == 0.0
    recs = [mb.RecordSpec(n, f"n{n}") for n in nodes]
    res = mb.run(model, steps * layout.dt, records=recs)
    got = np.stack([res.traces[r.name] for r in recs], axis=1)
    assert np.array_equal(got, ref.trace)
    with pytest.raises(mb.abi.MindError):
        mb.autotune(model)     # not at step 0 any more
    with pytest.raises(mb.abi.MindError):
        model.state.set_bin_threads([96] * len(shapes))
