"""The spike-output surrogate: an MLP that predicts a cell's spike in the next 1 ms bin.

Inputs per cell and bin (645 features): the cell's synaptic drive in the last 20 bins of
1 ms over 32 synapse groups (the summed NetCon weights of the events its synapses
received, synapse k in group k mod 32), then its own spike counts in the last 5 bins.  (The
configuration names the last 5 ms of somatic voltage as the last five features; a cell
that the surrogate replaces has no membrane voltage, so its recent output takes that
place.)  Output: the spike probability of the next bin.  Training data come from the
cable solver's own runs (`windows_from_run`); training and inference run in
libmindgpu.so (BF16 products on the tensor cores, FP32 masters, fused kernels around
them).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi

WINDOW_BINS = 20
GROUPS = 32
HISTORY_BINS = 5
N_FEATURES = WINDOW_BINS * GROUPS + HISTORY_BINS


def _f32(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Mlp:
    """mind_mlp_*: n_in -> hidden (SiLU) x layers -> sigmoid."""

    def __init__(self, n_in: int = N_FEATURES, hidden: int = 256, layers: int = 3, seed: int = 1):
        self.lib = abi.load_library()
        cfg = abi.MindMlpConfig(n_in, hidden, layers, seed)
        h = ctypes.c_void_p()
        status = self.lib.mind_mlp_create(ctypes.byref(cfg), ctypes.byref(h))
        self.handle = h
        self._check(status)
        n = ctypes.c_int64()
        self._check(self.lib.mind_mlp_param_count(self.handle, ctypes.byref(n)))
        self.n_params = n.value
        self.n_in, self.hidden, self.layers = n_in, hidden, layers

    def _check(self, status):
        if status != abi.MIND_OK:
            msg = self.lib.mind_mlp_last_error(self.handle) if self.handle else b""
            raise abi.MindError(status, msg.decode() if msg else "")

    def last_ms(self) -> float:
        """Device time of the last predict / gradients / train call's network work."""
        ms = ctypes.c_float()
        self._check(self.lib.mind_mlp_last_ms(self.handle, ctypes.byref(ms)))
        return ms.value

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        self._check(self.lib.mind_mlp_get_params(self.handle, _f32(out), self.n_params))
        return out

    @params.setter
    def params(self, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32)
        self._check(self.lib.mind_mlp_set_params(self.handle, _f32(v), v.size))

    def predict(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros(x.shape[0], dtype=np.float32)
        self._check(self.lib.mind_mlp_predict(self.handle, _f32(x), x.shape[0], _f32(out)))
        return out

    def gradients(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.mind_mlp_gradients(self.handle, _f32(x), _f32(y), x.shape[0], _f32(g),
                                                ctypes.byref(loss)))
        return g, float(loss.value)

    def train(self, x, y, steps: int, batch: int = 4096, lr: float = 1e-3):
        """Adam on batches drawn from (x, y); returns (per-step batch losses, device ms)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        self._check(self.lib.mind_mlp_set_data(self.handle, _f32(x), _f32(y), x.shape[0]))
        losses = np.zeros(steps, dtype=np.float32)
        ms = ctypes.c_float()
        self._check(self.lib.mind_mlp_train(self.handle, steps, batch, lr, _f32(losses), ctypes.byref(ms)))
        return losses, float(ms.value)

    def close(self):
        if self.handle:
            self.lib.mind_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def unpack(params: np.ndarray, dims):
    """[(W [out x in], b [out]) per linear map] views of a flat parameter vector."""
    out, k = [], 0
    for i, o in zip(dims[:-1], dims[1:]):
        W = params[k:k + i * o].reshape(o, i)
        k += i * o
        b = params[k:k + o]
        k += o
        out.append((W, b))
    return out


def cell_spike_bins(layout, result, bins: int, bin_ms: float = 1.0, start_ms: float = 0.0) -> np.ndarray:
    """[bins, cells] spike counts of the cells' detectors from a run's raster."""
    counts = np.zeros((bins, layout.n_cells), dtype=np.float32)
    nodes = np.asarray(layout.source_nodes)
    offsets = np.asarray(layout.cell_offsets)
    sid_cell = {}
    for s, node in enumerate(nodes):
        if node > 0:
            sid_cell[int(layout.source_ids[s])] = int(np.searchsorted(offsets, node - 1, side="right") - 1)
    for t, sid in zip(result.spike_times, result.spike_sources):
        c = sid_cell.get(int(sid))
        b = int((t - start_ms) // bin_ms)
        if c is not None and 0 <= b < bins:
            counts[b, c] += 1.0
    return counts


def windows(drive: np.ndarray, spikes: np.ndarray, first_bin: int = WINDOW_BINS, last_bin: int = None,
            cells=None):
    """(x [n, 645], y [n]) for every cell and target bin b in [first_bin, last_bin): the drive of
    bins b-20..b-1, the cell's spikes in bins b-5..b-1, and whether it spikes in bin b."""
    bins, n_cells, groups = drive.shape
    assert groups == GROUPS
    last_bin = bins if last_bin is None else last_bin
    cells = np.arange(n_cells) if cells is None else np.asarray(cells)
    xs, ys = [], []
    for b in range(max(first_bin, WINDOW_BINS), last_bin):
        d = drive[b - WINDOW_BINS:b][:, cells, :].transpose(1, 0, 2).reshape(len(cells), -1)
        h = spikes[b - HISTORY_BINS:b][:, cells].T
        xs.append(np.concatenate([d, h], axis=1))
        ys.append((spikes[b, cells] > 0).astype(np.float32))
    return np.concatenate(xs).astype(np.float32), np.concatenate(ys)


def train_from_run(model, t_ms: float, steps: int = 150, batch: int = 1024, lr: float = 1e-3, seed: int = 1,
                   hidden: int = 256, layers: int = 3):
    """Run the detailed network for t_ms with drive recording (from initialize), build the
    windows of every cell and bin, and train a surrogate on them.  Returns (mlp, drive_scale,
    result of the detailed run)."""
    from . import runtime

    runtime.initialize(model)
    model.state.set_drive_recording(1.0)
    result = runtime.run(model, t_ms)
    model.state.set_drive_recording(0.0)
    spikes = cell_spike_bins(model.layout, result, result.drive.shape[0])
    x, y = windows(result.drive, spikes)
    scale = float(1.0 / (x[:, :-HISTORY_BINS].std() + 1e-12))
    x[:, :-HISTORY_BINS] *= scale
    net = Mlp(hidden=hidden, layers=layers, seed=seed)
    net.train(x, y, steps=steps, batch=batch, lr=lr)
    return net, scale, result


def region_rates(layout, result, macro, t_ms: float, bin_ms: float = 10.0) -> np.ndarray:
    """[bins, regions] spike rate (Hz per cell) of each region's cells from a run's raster."""
    region_of = {}
    for region, source in macro.outputs:
        region_of[int(layout.source_ids[source - 1])] = region - 1
    cells = np.zeros(macro.n_regions)
    for region, _ in macro.outputs:
        cells[region - 1] += 1
    bins = int(round(t_ms / bin_ms))
    rates = np.zeros((bins, macro.n_regions))
    for t, sid in zip(result.spike_times, result.spike_sources):
        r = region_of.get(int(sid))
        b = int(t // bin_ms)
        if r is not None and 0 <= b < bins:
            rates[b, r] += 1.0
    return rates / np.maximum(cells, 1.0) / (bin_ms * 1e-3)


def cell_regions(layout, macro) -> np.ndarray:
    """Region (0-based) whose rate bin each cell's detector feeds, -1 for none."""
    offsets = np.asarray(layout.cell_offsets)
    nodes = np.asarray(layout.source_nodes)
    out = np.full(layout.n_cells, -1, dtype=np.int64)
    for region, source in macro.outputs:
        node = int(nodes[source - 1])
        if node > 0:
            out[int(np.searchsorted(offsets, node - 1, side="right") - 1)] = region - 1
    return out


def judge_populations(sur_spikes, sur_cells, det_spikes, det_cells, seconds: float, bound: float,
                      z: float = 3.0) -> np.ndarray:
    """Populations to revert to the cable solver: where the surrogate cells' mean rate differs
    from the detailed sample's by more than `bound` of the sample's rate plus z standard
    errors of the two Poisson estimates (so a population with few sample spikes is not
    reverted on counting noise alone).  Arguments are per population; returns a bool mask."""
    sur_spikes = np.asarray(sur_spikes, dtype=float)
    det_spikes = np.asarray(det_spikes, dtype=float)
    ns = np.maximum(np.asarray(sur_cells, dtype=float), 1.0) * seconds
    nd = np.maximum(np.asarray(det_cells, dtype=float), 1.0) * seconds
    r_s, r_d = sur_spikes / ns, det_spikes / nd
    se = np.sqrt(np.maximum(sur_spikes, 1.0) / ns ** 2 + np.maximum(det_spikes, 1.0) / nd ** 2)
    judged = (np.asarray(sur_cells) > 0) & (np.asarray(det_cells) > 0)
    return judged & (np.abs(r_s - r_d) > bound * r_d + z * se)


def population_rates(layout, macro, result, t_ms: float, cells=None) -> np.ndarray:
    """Per region: spikes per cell per second over a run of t_ms, counting only the cells
    flagged in `cells` (every cell when None); NaN for a region without such cells."""
    region = cell_regions(layout, macro)
    chosen = np.ones(layout.n_cells, dtype=bool) if cells is None else np.asarray(cells, dtype=bool)
    offsets = np.asarray(layout.cell_offsets)
    nodes = np.asarray(layout.source_nodes)
    sid_cell = {int(layout.source_ids[s]): int(np.searchsorted(offsets, node - 1, side="right") - 1)
                for s, node in enumerate(nodes) if node > 0}
    counts = np.zeros(macro.n_regions)
    for sid in result.spike_sources:
        c = sid_cell.get(int(sid))
        if c is not None and chosen[c] and region[c] >= 0:
            counts[region[c]] += 1.0
    members = np.array([np.count_nonzero(chosen & (region == p)) for p in range(macro.n_regions)], dtype=float)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(members > 0, counts / members / (t_ms * 1e-3), np.nan)


def calibrate(state, layout, macro, surrogate_cells, target_hz, t_ms: float = 100.0, rounds: int = 4,
              max_shift: float = 4.0, pooled: bool = False):
    """Per-population calibration of the surrogate in its closed loop (no counterpart in the
    reference).  A coupled run feeds the surrogate's spikes back through the regions, so a
    small bias of the network grows into a large rate error; the remedy here is one logit
    offset per population, fitted on the coupled run itself: `rounds` runs of t_ms from
    mind_initialize, after each of which every population's offset moves by
    log(target / measured) of its surrogate cells' rate (the shift that scales a small
    spike probability by that ratio), clipped to +-max_shift in total.  `state` has the
    macro model and the surrogate attached; `target_hz` holds each population's rate in the
    detailed run the network was trained on over the same t_ms from initialize (a run's
    early rates differ from its later ones), or is None: then each population's target is
    the rate of its detailed sample (the cells not in `surrogate_cells`) pooled over the
    rounds so far.  pooled=True fits one offset for every population, from the rates of
    all surrogate cells and all sample cells (for samples too small to judge one
    population).  Returns (per-cell offsets, per-round rates)."""
    mask = np.asarray(surrogate_cells, dtype=bool)
    region = cell_regions(layout, macro)
    shift = np.zeros(macro.n_regions)
    history = []
    sample = []
    steps = int(round(t_ms / layout.dt))
    for _ in range(rounds):
        per_cell = np.where(region >= 0, shift[np.maximum(region, 0)], 0.0)
        state.set_surrogate_offsets(per_cell)
        state.initialize()
        res = state.run_steps(steps, [])
        measured = population_rates(layout, macro, res, t_ms, mask)
        history.append(measured)
        if target_hz is None:
            sample.append(population_rates(layout, macro, res, t_ms, ~mask))
            target = np.nanmean(np.array(sample), axis=0)
        else:
            target = np.asarray(target_hz, dtype=float)
        if pooled:   # cell-weighted means over the populations
            w_sur = np.array([np.count_nonzero(mask & (region == p)) for p in range(macro.n_regions)], float)
            w_det = np.array([np.count_nonzero(~mask & (region == p)) for p in range(macro.n_regions)], float)
            if target_hz is not None:
                w_det = w_sur + w_det
            m_all = np.nansum(np.nan_to_num(measured) * w_sur) / max(w_sur.sum(), 1.0)
            t_all = np.nansum(np.nan_to_num(target) * w_det) / max(w_det.sum(), 1.0)
            measured = np.full(macro.n_regions, m_all)
            target = np.full(macro.n_regions, t_all)
        live = np.isfinite(measured) & np.isfinite(target) & (target > 0)
        safe_target = np.where(live, target, 1.0)
        ratio = np.where(measured > 0, safe_target / np.where(measured > 0, measured, 1.0), np.e)
        shift = np.where(live, np.clip(shift + np.log(ratio), -max_shift, max_shift), shift)
    per_cell = np.where(region >= 0, shift[np.maximum(region, 0)], 0.0)
    state.set_surrogate_offsets(per_cell)
    return per_cell, history


def judged_run(state, layout, macro, surrogate_cells, t_ms: float, window_ms: float = 20.0,
               bound: float = 0.05, z: float = 3.0, rotate: bool = False, seed: int = 0):
    """Run t_ms in windows with the cable solver as judge: the cells of each population that
    stay detailed (the sample) are compared, after every window and over the run so far,
    with the population's surrogate cells (judge_populations); a population that fails is
    reverted (mind_set_surrogate_cells) and simulated from the next window on.  `state` is an
    initialized DeviceState with the surrogate attached for `surrogate_cells` (for a
    rotating sample: attached for every cell, then set to `surrogate_cells`).

    rotate=True rotates the sample: after every window, half of each population's sample
    (its longest-serving cells) returns to the surrogate and as many surrogate cells of the
    population, drawn at random, join it, so that over a run the judge sees many more cells
    than the sample holds at once.  A joining cell resumes from the membrane state it had
    when it last left detailed simulation (from initialize, if never detailed), so it counts
    toward its population's sample rate only from its second window in the sample.
    Returns (per-window results, [(time ms, reverted population indices)], final mask)."""
    mask = np.asarray(surrogate_cells, dtype=bool).copy()
    region = cell_regions(layout, macro)
    n_pop = macro.n_regions
    offsets = np.asarray(layout.cell_offsets)
    nodes = np.asarray(layout.source_nodes)
    sid_cell = {int(layout.source_ids[s]): int(np.searchsorted(offsets, node - 1, side="right") - 1)
                for s, node in enumerate(nodes) if node > 0}
    steps = int(round(window_ms / layout.dt))
    total = int(round(t_ms / layout.dt))
    sur_count = np.zeros(n_pop)
    det_count = np.zeros(n_pop)
    sur_time = np.zeros(n_pop)   # cell-seconds observed in each role
    det_time = np.zeros(n_pop)
    joined = np.full(layout.n_cells, -1)   # window a cell joined the sample (-1: from the start)
    reverted = np.zeros(n_pop, dtype=bool)
    rng = np.random.default_rng(seed)
    results, log, done, w = [], [], 0, 0
    while done < total:
        k = min(steps, total - done)
        res = state.run_steps(k, [])
        results.append(res)
        seconds = k * layout.dt * 1e-3
        counted = ~mask & (w - joined >= 1)   # sample cells past their burn-in window
        for sid in res.spike_sources:
            c = sid_cell.get(int(sid))
            if c is None or region[c] < 0:
                continue
            if mask[c]:
                sur_count[region[c]] += 1.0
            elif counted[c]:
                det_count[region[c]] += 1.0
        for p in range(n_pop):
            members = region == p
            sur_time[p] += seconds * np.count_nonzero(mask & members)
            det_time[p] += seconds * np.count_nonzero(counted & members)
        done += k
        w += 1
        live = np.array([np.any(mask & (region == p)) for p in range(n_pop)])
        revert = live & judge_populations(sur_count, sur_time, det_count, det_time, 1.0, bound, z)
        changed = False
        if np.any(revert):
            for p in np.nonzero(revert)[0]:
                mask[region == p] = False
            reverted |= revert
            changed = True
            log.append((done * layout.dt, [int(p) for p in np.nonzero(revert)[0]]))
        if rotate and done < total:
            for p in np.nonzero(~reverted)[0]:
                sample = np.nonzero(~mask & (region == p))[0]
                pool = np.nonzero(mask & (region == p))[0]
                n_out = min((len(sample) + 1) // 2, len(pool))
                if n_out == 0:
                    continue
                leaving = sample[np.argsort(joined[sample], kind="stable")[:n_out]]
                entering = rng.choice(pool, size=n_out, replace=False)
                mask[leaving] = True
                mask[entering] = False
                joined[entering] = w
                changed = True
        if changed:
            state.set_surrogate_cells(mask)
    return results, log, mask


def flops_per_row(n_in: int = N_FEATURES, hidden: int = 256, layers: int = 3) -> int:
    """Forward FLOPs of one row (2 per multiply-add of the linear maps); training is 3x."""
    dims = [n_in] + [hidden] * layers + [1]
    return 2 * sum(i * o for i, o in zip(dims[:-1], dims[1:]))


def throughput(train_steps: int = 40, batch: int = 4096, rows: int = 1 << 16, infer_rows: int = 100_000,
               seed: int = 1) -> dict:
    """Training and inference speed of the network on synthetic windows (rows of uniform
    drive features and 3% positive labels): device ms per Adam step, per inference call,
    and the tensor-core FLOP rates they imply."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, (rows, N_FEATURES)).astype(np.float32)
    y = (rng.uniform(size=rows) < 0.03).astype(np.float32)
    net = Mlp(seed=seed)
    net.train(x, y, 5, batch)                      # warm-up
    _, ms = net.train(x, y, train_steps, batch)
    per_step = ms / train_steps
    xi = rng.uniform(0.0, 1.0, (infer_rows, N_FEATURES)).astype(np.float32)
    net.predict(xi)                                # warm-up (buffers sized)
    net.predict(xi)
    infer_ms = net.last_ms()
    f = flops_per_row()
    return {"train_ms_per_step": per_step, "batch": batch,
            "train_tflops": 3 * f * batch / (per_step / 1000.0) / 1e12,
            "infer_rows": infer_rows, "infer_device_ms": infer_ms,
            "infer_tflops": f * infer_rows / (infer_ms / 1000.0) / 1e12,
            "flops_per_row_forward": f}


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="surrogate MLP training/inference throughput")
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--batch", type=int, default=4096)
    args = ap.parse_args()
    print(json.dumps(throughput(args.steps, args.batch)))
