"""The spike-output surrogate on the GPU: gradients against the FP64 oracle, and training on
windows the cable solver produced, against the method without it (a constant rate)."""
import numpy as np
import pytest

import mind_b200 as mb
import mlp as oracle_mlp
import netcases
from mind_b200 import surrogate

pytestmark = pytest.mark.gpu


def test_gradients_and_predictions_match_the_fp64_oracle():
    """BF16 products with FP32 accumulation against FP64: relative L2 error of the gradient
    below 5e-2, cosine above 0.995, probabilities within 1e-2."""
    rng = np.random.default_rng(5)
    net = surrogate.Mlp(seed=3)
    dims = [surrogate.N_FEATURES, 256, 256, 256, 1]
    x = rng.normal(0.0, 1.0, (512, surrogate.N_FEATURES)).astype(np.float32)
    y = (rng.uniform(size=512) < 0.2).astype(np.float32)
    params = net.params.astype(np.float64)
    want_loss, want = oracle_mlp.loss_and_gradients(params, dims, x, y)
    got, loss = net.gradients(x, y)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    cos = float(got @ want / (np.linalg.norm(got) * np.linalg.norm(want)))
    assert err < 5e-2 and cos > 0.995, (err, cos)
    assert abs(loss - want_loss) < 1e-2 * want_loss
    np.testing.assert_allclose(net.predict(x), oracle_mlp.predict(params, dims, x), atol=1e-2)
    net.close()


@pytest.mark.parametrize("n_in,hidden,layers,rows", [(45, 48, 2, 37), (645, 256, 3, 300), (70, 16, 1, 129),
                                                     (645, 128, 2, 1000)])
def test_tensor_core_products_on_tile_edges(n_in, hidden, layers, rows):
    """The tcgen05 products at tile edges: inputs that end inside a 64-column K block,
    hidden widths below one N tile, one hidden layer (the head reads the inputs directly),
    batches that end inside a 128-row tile and weight-gradient K slices that end inside a
    64-row block; gradients and probabilities against the FP64 oracle."""
    rng = np.random.default_rng(11 + rows)
    net = surrogate.Mlp(n_in=n_in, hidden=hidden, layers=layers, seed=4)
    dims = [n_in] + [hidden] * layers + [1]
    x = rng.normal(0.0, 1.0, (rows, n_in)).astype(np.float32)
    y = (rng.uniform(size=rows) < 0.3).astype(np.float32)
    params = net.params.astype(np.float64)
    want_loss, want = oracle_mlp.loss_and_gradients(params, dims, x, y)
    got, loss = net.gradients(x, y)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    cos = float(got @ want / (np.linalg.norm(got) * np.linalg.norm(want)))
    assert err < 5e-2 and cos > 0.995, (err, cos)
    assert abs(loss - want_loss) < 1e-2 * want_loss
    np.testing.assert_allclose(net.predict(x), oracle_mlp.predict(params, dims, x), atol=1e-2)
    # a second, smaller call reuses the buffers sized for the first
    np.testing.assert_allclose(net.predict(x[:5]), oracle_mlp.predict(params, dims, x[:5]), atol=1e-2)
    net.close()


def test_trained_surrogate_beats_a_constant_rate():
    """200 cells of a region-coupled network, 600 ms: train on the first 70% of the 1 ms bins,
    test on the rest; the held-out cross-entropy must be 15% below the constant-probability
    predictor's (the training set's spike fraction)."""
    model, _ = netcases.coupled_regions(n_regions=4, cells_per_region=50, synapses=32, seed=21)
    layout = model.layout
    mb.initialize(model)
    model.state.set_drive_recording(1.0)
    result = mb.run(model, 600.0)
    drive = result.drive
    spikes = surrogate.cell_spike_bins(layout, result, drive.shape[0])
    assert drive.shape == (600, layout.n_cells, 32)
    assert spikes.sum() > 200 and drive.sum() > 0
    split = 420
    x_tr, y_tr = surrogate.windows(drive, spikes, last_bin=split)
    x_te, y_te = surrogate.windows(drive, spikes, first_bin=split)
    scale = 1.0 / (x_tr[:, :-surrogate.HISTORY_BINS].std() + 1e-12)
    x_tr[:, :-surrogate.HISTORY_BINS] *= scale
    x_te[:, :-surrogate.HISTORY_BINS] *= scale
    net = surrogate.Mlp(seed=1)
    losses, ms = net.train(x_tr, y_tr, steps=150, batch=1024, lr=1e-3)
    assert losses[-50:].mean() < losses[:10].mean()
    p = np.clip(net.predict(x_te), 1e-6, 1 - 1e-6)
    q = np.clip(y_tr.mean(), 1e-6, 1 - 1e-6)
    ce = -np.mean(y_te * np.log(p) + (1 - y_te) * np.log(1 - p))
    base = -np.mean(y_te * np.log(q) + (1 - y_te) * np.log(1 - q))
    assert ce < 0.85 * base, (ce, base)
    net.close()


def test_surrogate_cells_drive_the_regions():
    """Train on a detailed run, then let the network stand in for 90% of the cells: the run
    stays finite, surrogate cells fire at the detailed cells' order of magnitude, the regions
    keep moving, and the same seed gives the same run."""
    model, macro = netcases.coupled_regions(n_regions=4, cells_per_region=50, synapses=32, seed=21)
    layout = model.layout
    net, scale, detailed = surrogate.train_from_run(model, 400.0, steps=150)
    mask = np.ones(layout.n_cells, dtype=bool)
    mask[::10] = False                      # every tenth cell stays detailed
    runs = []
    for _ in range(2):
        state = mb.runtime.DeviceState(layout)
        state.attach_macro(macro)
        state.attach_surrogate(net, mask, scale)
        state.initialize()
        runs.append(state.run_steps(int(round(400.0 / layout.dt)), []))
        state.close()
    a, b = runs
    np.testing.assert_array_equal(a.spike_times, b.spike_times)
    np.testing.assert_array_equal(a.macro_trace, b.macro_trace)
    assert np.all(np.isfinite(a.macro_trace)) and np.ptp(a.macro_trace) > 0.1
    n_detailed = np.sum(detailed.spike_sources <= layout.n_cells)
    n_sur = np.sum(a.spike_sources <= layout.n_cells)
    assert n_detailed / 4 < n_sur < 4 * n_detailed, (n_sur, n_detailed)
    net.close()


def test_judge_reverts_a_failing_surrogate_to_the_cable_solver():
    """A network that predicts a spike in every bin: after the first judge window every
    population is reverted, and from then on its cells fire like detailed cells."""
    model, macro = netcases.coupled_regions(n_regions=4, cells_per_region=50, synapses=32, seed=21)
    layout = model.layout
    net = surrogate.Mlp()
    params = net.params
    params[-1] = 20.0                       # output bias: p = 1 in every bin
    net.params = params
    mask = np.ones(layout.n_cells, dtype=bool)
    mask[::10] = False
    state = mb.runtime.DeviceState(layout)
    state.attach_macro(macro)
    state.attach_surrogate(net, mask, 1.0)
    with pytest.raises(mb.abi.MindError):
        state.set_surrogate_cells(np.ones(layout.n_cells, dtype=bool))   # cells that were never attached
    state.initialize()
    results, log, final = surrogate.judged_run(state, layout, macro, mask, 200.0, window_ms=20.0)
    assert log and log[0][0] == 20.0 and sorted(log[0][1]) == [0, 1, 2, 3]
    assert not final.any()
    region = surrogate.cell_regions(layout, macro)
    first = np.sum(results[0].spike_sources < layout.n_cells)
    later = sum(np.sum(r.spike_sources < layout.n_cells) for r in results[2:]) / (len(results) - 2)
    assert first > 0.5 * 20 * np.count_nonzero(mask)   # the failing surrogate fired (almost) every bin
    assert later < 0.5 * first                          # reverted cells fire at their own rate
    assert np.all(region >= 0)
    state.close()
    net.close()


def test_surrogate_offsets_shift_the_spike_probability():
    """mind_set_surrogate_offsets: an offset of -20 on the logit silences the surrogate cells,
    +20 makes them fire in (almost) every bin; offsets of 0 give back the uncalibrated run,
    spike for spike."""
    model, macro = netcases.coupled_regions(n_regions=4, cells_per_region=50, synapses=32, seed=21)
    layout = model.layout
    net = surrogate.Mlp(seed=2)
    mask = np.ones(layout.n_cells, dtype=bool)
    mask[::10] = False
    steps = int(round(40.0 / layout.dt))
    state = mb.runtime.DeviceState(layout)
    state.attach_macro(macro)
    state.attach_surrogate(net, mask, 1.0)
    counts, rasters = {}, {}
    for shift in (0.0, -20.0, 20.0, 0.0):
        state.set_surrogate_offsets(np.full(layout.n_cells, shift))
        state.initialize()
        res = state.run_steps(steps, [])
        rates = surrogate.population_rates(layout, macro, res, 40.0, mask)
        counts.setdefault(shift, []).append(float(np.nansum(rates)))
        rasters.setdefault(shift, []).append(res.spike_times.copy())
    assert counts[-20.0][0] == 0.0
    assert np.nanmin(counts[20.0][0]) > 0.9 * 4 * 1000.0   # four populations near 1 spike per 1 ms bin
    np.testing.assert_array_equal(rasters[0.0][0], rasters[0.0][1])
    with pytest.raises(mb.abi.MindError):
        state.set_surrogate_offsets(np.full(layout.n_cells, np.inf))
    state.close()
    net.close()


def test_rotating_judge_sample_sees_more_cells_and_still_reverts_a_failing_surrogate():
    """judged_run(rotate=True): every cell attached to the surrogate, a 10% sample that
    rotates by half each window.  Over the run the judge samples several times the cells
    its sample holds at once, the run is reproducible, and a network that predicts a spike
    in every bin is still reverted everywhere."""
    model, macro = netcases.coupled_regions(n_regions=4, cells_per_region=50, synapses=32, seed=21)
    layout = model.layout
    net = surrogate.Mlp()
    params = net.params
    params[-1] = 20.0                       # p = 1 in every bin: a failing surrogate
    net.params = params
    mask = np.ones(layout.n_cells, dtype=bool)
    mask[::10] = False
    outs = []
    for _ in range(2):
        state = mb.runtime.DeviceState(layout)
        state.attach_macro(macro)
        state.attach_surrogate(net, np.ones(layout.n_cells, dtype=bool), 1.0)
        state.set_surrogate_cells(mask)
        state.initialize()
        results, log, final = surrogate.judged_run(state, layout, macro, mask, 100.0, window_ms=10.0,
                                                   rotate=True, seed=3)
        outs.append((np.concatenate([r.spike_times for r in results]), log, final))
        state.close()
    (t0, log0, final0), (t1, log1, final1) = outs
    np.testing.assert_array_equal(t0, t1)
    assert log0 == log1 and log0 and sorted(sum((regs for _, regs in log0), [])) == [0, 1, 2, 3]
    assert not final0.any()

    # a sane network: the rotation moves the sample through the populations
    net2 = surrogate.Mlp(seed=5)
    p2 = net2.params
    p2[-1] = -3.0
    net2.params = p2
    state = mb.runtime.DeviceState(layout)
    state.attach_macro(macro)
    state.attach_surrogate(net2, np.ones(layout.n_cells, dtype=bool), 1.0)
    state.set_surrogate_cells(mask)
    state.initialize()
    masks = []
    real = state.set_surrogate_cells

    def spy(m):
        masks.append(np.asarray(m, dtype=bool).copy())
        real(m)

    state.set_surrogate_cells = spy
    results, log, final = surrogate.judged_run(state, layout, macro, mask, 60.0, window_ms=10.0, rotate=True,
                                               bound=10.0, z=50.0)
    sampled = np.zeros(layout.n_cells, dtype=bool)
    for m in [mask] + masks:
        sampled |= ~m
    assert len(masks) >= 4
    assert sampled.sum() >= 2.5 * (~mask).sum()
    assert all(int((~m).sum()) == int((~mask).sum()) for m in masks)   # the sample keeps its size
    state.close()
    net.close()
    net2.close()
