"""The surrogate network's CPU oracle (FP64) against finite differences, and its layout."""
import numpy as np

import mlp as oracle_mlp


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    dims = [7, 5, 5, 1]
    n_params = sum(i * o + o for i, o in zip(dims[:-1], dims[1:]))
    params = rng.normal(0, 0.5, n_params)
    x = rng.normal(0, 1, (11, dims[0]))
    y = (rng.uniform(size=11) < 0.3).astype(float)
    loss, grad = oracle_mlp.loss_and_gradients(params, dims, x, y)
    eps = 1e-6
    for k in rng.choice(n_params, 25, replace=False):
        p = params.copy()
        p[k] += eps
        up, _ = oracle_mlp.loss_and_gradients(p, dims, x, y)
        p[k] -= 2 * eps
        down, _ = oracle_mlp.loss_and_gradients(p, dims, x, y)
        assert abs((up - down) / (2 * eps) - grad[k]) < 1e-7 * max(1.0, abs(grad[k]))
    assert loss > 0


def test_judge_reverts_on_rate_error_not_on_counting_noise():
    from mind_b200.surrogate import judge_populations

    # 100 surrogate and 2 sample cells per population, 1 s observed
    sur_cells, det_cells = np.array([100.0] * 4), np.array([2.0] * 4)
    det = np.array([20.0, 20.0, 2.0, 20.0])            # 10 Hz samples (1 Hz in population 2)
    sur = np.array([1000.0, 3000.0, 200.0, 1040.0])    # 10, 30, 2, 10.4 Hz
    revert = judge_populations(sur, sur_cells, det, det_cells, 1.0, bound=0.05, z=3.0)
    # population 1 fires 3x its sample: reverted; population 3 is 4% off: kept; population 2
    # is 2x off but its sample saw 2 spikes: within the counting noise
    assert revert.tolist() == [False, True, False, False]
    # populations without surrogate cells or without a sample are not judged
    assert not judge_populations([5.0], [0.0], [50.0], [2.0], 1.0, 0.05).any()
    assert not judge_populations([500.0], [100.0], [0.0], [0.0], 1.0, 0.05).any()


class _FakeState:
    """A DeviceState stand-in: each run_steps returns a raster in which every surrogate
    cell fires `sur_hz` and every detailed cell `det_hz` (regular spikes), and
    set_surrogate_cells records the masks it is given."""

    def __init__(self, layout, mask, sur_hz, det_hz):
        self.layout, self.mask, self.sur_hz, self.det_hz = layout, mask.copy(), sur_hz, det_hz
        self.t, self.calls = 0.0, []

    def run_steps(self, steps, records):
        from mind_b200.runtime import SimulationResult

        dt = self.layout.dt
        t0, t1 = self.t, self.t + steps * dt
        times, sids = [], []
        for c in range(self.layout.n_cells):
            hz = self.sur_hz if self.mask[c] else self.det_hz
            k = np.arange(np.ceil(t0 * hz / 1000.0), np.ceil(t1 * hz / 1000.0))
            times += list(k * 1000.0 / hz)
            sids += [c] * len(k)
        self.t = t1
        order = np.argsort(times, kind="stable")
        return SimulationResult(np.zeros(1), {}, np.asarray(times)[order], np.asarray(sids, np.int64)[order], 1.0)

    def set_surrogate_cells(self, mask):
        self.mask = np.asarray(mask, dtype=bool).copy()
        self.calls.append(self.mask.copy())


def test_judged_run_reverts_only_the_failing_population():
    import netcases
    from mind_b200 import surrogate

    model, macro = netcases.coupled_regions(n_regions=2, cells_per_region=50, synapses=2, seed=3)
    layout = model.layout
    region = surrogate.cell_regions(layout, macro)
    assert sorted(set(region.tolist())) == [0, 1]
    mask = np.ones(layout.n_cells, dtype=bool)
    mask[::10] = False                                   # 10% detailed sample
    # population 0's surrogate fires 4x its sample; population 1's matches its sample
    state = _FakeState(layout, mask, sur_hz=40.0, det_hz=10.0)
    good = region == 1
    state.sur_hz = 40.0

    def run_steps(steps, records, _orig=state.run_steps):
        res = _orig(steps, records)
        keep = np.ones(len(res.spike_sources), dtype=bool)
        for i, sid in enumerate(res.spike_sources):
            c = int(sid)
            if good[c] and state.mask[c] and (i % 4 != 0):
                keep[i] = False                          # population 1 surrogate: 10 Hz
        res.spike_times, res.spike_sources = res.spike_times[keep], res.spike_sources[keep]
        return res

    state.run_steps = run_steps
    results, log, final = surrogate.judged_run(state, layout, macro, mask, 200.0, window_ms=20.0)
    assert len(results) == 10
    assert log and all(regs == [0] for _, regs in log) and len(log) == 1
    assert not final[region == 0].any()                  # population 0 reverted
    assert np.array_equal(final[region == 1], mask[region == 1])   # population 1 kept
    assert len(state.calls) == 1 and np.array_equal(state.calls[0], final)


def test_network_shapes_the_tensor_core_kernels_cannot_tile_are_refused():
    """mind_mlp_create checks its configuration before it touches the device: the hidden
    width must be a multiple of 16 in [16, 256] (one tensor-core tile spans a hidden layer)."""
    import ctypes

    from mind_b200 import abi

    lib = abi.load_library()
    for n_in, hidden, layers in [(645, 20, 3), (645, 272, 3), (645, 0, 3), (0, 256, 3), (645, 256, 0)]:
        h = ctypes.c_void_p()
        cfg = abi.MindMlpConfig(n_in, hidden, layers, 1)
        assert lib.mind_mlp_create(ctypes.byref(cfg), ctypes.byref(h)) == abi.MIND_EARG
        assert not h.value


class _LoopState:
    """Stands in for a coupled run on the host: each population's surrogate cells fire at
    base_hz * exp(offset) * gain (a closed loop that scales every population's bias), the
    detailed sample at sample_hz; spike counts are the expected counts, rounded."""

    def __init__(self, layout, macro, mask, base_hz, sample_hz, gain):
        from mind_b200 import surrogate

        self.layout, self.mask = layout, np.asarray(mask, dtype=bool)
        self.region = surrogate.cell_regions(layout, macro)
        self.base, self.sample, self.gain = np.asarray(base_hz), np.asarray(sample_hz), gain
        self.offsets = np.zeros(layout.n_cells)
        offsets = np.asarray(layout.cell_offsets)
        self.sid_of_cell = {}
        for s, node in enumerate(np.asarray(layout.source_nodes)):
            if node > 0:
                self.sid_of_cell[int(np.searchsorted(offsets, node - 1, side="right") - 1)] = int(layout.source_ids[s])

    def set_surrogate_offsets(self, offsets):
        self.offsets = np.asarray(offsets, dtype=float)

    def initialize(self):
        pass

    def run_steps(self, steps, records):
        from types import SimpleNamespace

        seconds = steps * self.layout.dt * 1e-3
        sids = []
        for c, sid in self.sid_of_cell.items():
            p = self.region[c]
            if p < 0:
                continue
            hz = self.base[p] * np.exp(self.offsets[c]) * self.gain if self.mask[c] else self.sample[p]
            sids += [sid] * int(round(hz * seconds))
        return SimpleNamespace(spike_sources=np.asarray(sids, dtype=np.int64),
                               spike_times=np.zeros(len(sids)))


def test_calibration_moves_each_population_to_its_target_rate():
    """surrogate.calibrate on a host stand-in for the coupled run: per-population offsets
    bring populations that start 3x too low or 2x too high to their targets; the pooled
    mode fits one offset to the detailed sample's pooled rate."""
    import netcases
    from mind_b200 import surrogate

    model, macro = netcases.coupled_regions(n_regions=4, cells_per_region=50, synapses=4, seed=21)
    layout = model.layout
    mask = np.ones(layout.n_cells, dtype=bool)
    mask[::10] = False
    target = np.array([5.0, 8.0, 3.0, 6.0])
    loop = _LoopState(layout, macro, mask, base_hz=[5.0 / 3, 16.0, 3.0, 2.0], sample_hz=target, gain=1.0)
    offsets, history = surrogate.calibrate(loop, layout, macro, mask, target, t_ms=1000.0, rounds=3)
    final = surrogate.population_rates(layout, macro, loop.run_steps(40000, []), 1000.0, mask)
    np.testing.assert_allclose(final, target, rtol=0.03)
    assert len(history) == 3 and np.all(np.isfinite(offsets))
    # detailed sample as the target, one offset for all populations
    loop = _LoopState(layout, macro, mask, base_hz=[2.0, 2.0, 2.0, 2.0], sample_hz=[4.0] * 4, gain=1.0)
    offsets, _ = surrogate.calibrate(loop, layout, macro, mask, None, t_ms=1000.0, rounds=3, pooled=True)
    assert np.allclose(offsets[mask], np.log(2.0), atol=0.02)
