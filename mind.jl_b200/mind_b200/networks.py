"""Seeded synthetic networks for the benchmark configurations, built through the public API.

Each generator uses numpy's PCG64 stream seeded with 0x4D494E44 + config number
and the builders of this package exactly as a MIND.jl user script would use
the Julia builders.  Choices the configuration text leaves open are fixed here
and stated in each docstring.  No external dataset is involved.

Units: lengths um, Ra ohm cm, cm uF/cm2, conductances S/cm2, synaptic weights
uS (NET_RECEIVE weights are uS in mod/ExpSyn.mod and mod/Exp2Syn.mod, so nS
draws are divided by 1000).
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from . import model as M
from .mechanisms import builtin
from .morphology import Section

SEED_BASE = 0x4D494E44


def _rng(config: int) -> np.random.Generator:
    return np.random.default_rng(SEED_BASE + config)


def config1(n_cells: int = 64, synapses_per_cell: int = 10) -> M.MicroModel:
    """Ball-and-stick cells with Poisson-driven ExpSyn (64 cells in the benchmark).

    Soma 1 compartment (L = diam = 20 um, hh); dendrite 50 compartments
    (L = 500 um, diam = 2 um, pas g = 1e-4 S/cm2, e = -65 mV); Ra 100, cm 1.
    Each cell has a soma(0.5) detector at -10 mV and `synapses_per_cell`
    ExpSyn (tau 2 ms, e 0 mV) at uniform-random dendritic x, each driven by its
    own NetStim (10 Hz: interval 100 ms, noise 1, start 0, number 1e9) through a
    NetCon with delay 0 and weight lognormal(ln 0.5 nS, 0.5).
    Point order: all ExpSyn (cell-major), then all NetStims in the same order.
    """
    rng = _rng(1)
    model = M.MicroModel(celsius=6.3)
    soma = Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1, Ra=100.0, cm=1.0)
    dend = Section("dend", label="dend", parent="soma", parent_x=1.0, length=500.0, diameter=2.0,
                   nseg=50, Ra=100.0, cm=1.0)
    cells = M.add_population(model, [soma, dend], n_cells, voltage=-65.0)
    for cell in cells:
        M.insert(cell, builtin("hh"), sections="soma")
        M.insert(cell, builtin("pas"), sections="dend", params={"g": 1.0e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
    n = n_cells * synapses_per_cell
    xs = rng.uniform(0.0, 1.0, n)
    weights = rng.lognormal(math.log(0.5), 0.5, n) / 1000.0
    owners = np.repeat(np.arange(1, n_cells + 1), synapses_per_cell)
    first_syn = M.add_pointprocesses(model, builtin("ExpSyn"), owners, "dend", xs,
                                     {"tau": 2.0, "e": 0.0})
    first_stim = M.add_pointprocesses(model, builtin("NetStim"), np.zeros(n, np.int64), "none",
                                      np.zeros(n), {"interval": 100.0, "number": 1e9, "start": 0.0,
                                                    "noise": 1.0})
    sources = M.register_point_sources(model, np.arange(first_stim, first_stim + n))
    M.connect_many(model, sources, np.arange(first_syn, first_syn + n), weights, np.zeros(n))
    return model


def _binary_tree(rng, compartments: int, soma: Section) -> List[Section]:
    """Random binary dendritic tree with exactly `compartments` dendritic compartments.

    Branch lengths lognormal(ln 50 um, 0.5) at 10 um per compartment (nseg =
    max(1, round(L/10))); the first branch starts at soma(1) with diam 3 um and
    each generation tapers 0.9x.  A random leaf is split into two children until
    the budget is spent; the last branch is shortened to fit (L = 10 um x nseg).
    """
    sections = [soma]
    budget = compartments

    def branch(name, parent, diameter):
        nonlocal budget
        length = float(rng.lognormal(math.log(50.0), 0.5))
        nseg = max(1, int(round(length / 10.0)))
        if nseg >= budget:
            nseg = budget
            length = 10.0 * nseg
        budget -= nseg
        sections.append(Section(name, label="dend", parent=parent, parent_x=1.0, length=length,
                                diameter=diameter, nseg=nseg, Ra=100.0, cm=1.0))
        return name

    leaves = [(branch("d0", soma.name, 3.0), 3.0)]
    count = 1
    while budget > 0:
        pick = int(rng.integers(len(leaves)))
        name, diameter = leaves.pop(pick)
        for _ in range(2):
            if budget <= 0:
                break
            child = branch(f"d{count}", name, diameter * 0.9)
            count += 1
            leaves.append((child, diameter * 0.9))
    return sections


def _dendritic_sites(rng, sections: List[Section], count: int, labels=None):
    """Uniform-random dendritic positions: section with probability proportional to nseg, x ~ U(0,1)."""
    dends = [s for s in sections if s.label != "soma" and (labels is None or s.label in labels)]
    weights = np.array([s.nseg for s in dends], dtype=np.float64)
    picks = rng.choice(len(dends), size=count, p=weights / weights.sum())
    xs = rng.uniform(0.0, 1.0, count)
    return [dends[i].name for i in picks], xs


def config2(n_cells: int = 10000, synapses_per_cell: int = 100, background_hz: float = 5.0,
            compartment_range: Tuple[int, int] = (100, 1000), *, rank: int = 0, world: int = 1) -> M.MicroModel:
    """Uneven random binary trees in a recurrent Exp2Syn network (10,000 cells per rank).

    The network has `n_cells * world` cells; this call builds rank `rank`'s block of
    `n_cells` consecutive cells (world = 1: the whole network).  Every cell draws from its
    own stream, numpy PCG64 seeded with (0x4D494E44 + 2, global cell index), so a rank
    builds its cells alone and the cells do not depend on the rank count.

    Each cell: soma (1 compartment, L = diam = 20 um, hh) plus a random binary
    tree (`_binary_tree`) so that the total compartment count is uniform in
    `compartment_range`; pas (g 1e-4 S/cm2, e -65 mV) on every dendrite.
    100 Exp2Syn per cell (tau1 0.5 ms, tau2 5 ms; 80% e = 0 mV, 20% e = -80 mV)
    at uniform-random dendritic positions; each gets one NetCon from a
    uniform-random presynaptic cell of the whole network (soma(0.5) detector, -10 mV)
    with delay U[1,5] ms and weight lognormal(ln 0.3 nS, 0.7), and its own 5 Hz Poisson
    NetStim (interval 200 ms, noise 1, start 0) through a NetCon with delay 0
    and a weight from the same lognormal.  A presynaptic cell on another rank enters as
    an external spike input with the cell's sid.
    Source ids: cell g's detector is g + 1; synapse k of cell g's NetStim is
    cells + g * synapses_per_cell + k + 1.  Point order: all Exp2Syn (cell-major), then all
    NetStims.
    """
    total = n_cells * world
    first_cell = rank * n_cells
    model = M.MicroModel(celsius=6.3)
    S = synapses_per_cell
    cells = []
    draws = []
    for k in range(n_cells):
        g = first_cell + k
        rng = np.random.default_rng([SEED_BASE + 2, g])
        size = int(rng.integers(compartment_range[0], compartment_range[1] + 1))
        soma = Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1, Ra=100.0, cm=1.0)
        secs = _binary_tree(rng, size - 1, soma)
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, builtin("hh"), sections="soma")
        M.insert(cell, builtin("pas"), sections="dend", params={"g": 1.0e-4, "e": -65.0})
        M.register_spike_source(cell, sid=g + 1, threshold=-10.0)
        names, xs = _dendritic_sites(rng, secs, S)
        e_rev = np.where(rng.uniform(size=S) < 0.8, 0.0, -80.0)
        presyn = rng.integers(1, total + 1, S)
        delays = rng.uniform(1.0, 5.0, S)
        weights = rng.lognormal(math.log(0.3), 0.7, S) / 1000.0
        bg_weights = rng.lognormal(math.log(0.3), 0.7, S) / 1000.0
        cells.append(cell)
        draws.append((names, xs, e_rev, presyn, delays, weights, bg_weights))
    n = n_cells * S
    owners = np.repeat(np.arange(1, n_cells + 1), S)
    names = [nm for d in draws for nm in d[0]]
    first_syn = M.add_pointprocesses(model, builtin("Exp2Syn"), owners, names, np.concatenate([d[1] for d in draws]),
                                     {"tau1": 0.5, "tau2": 5.0, "e": np.concatenate([d[2] for d in draws])})
    presyn = np.concatenate([d[3] for d in draws])
    local = (presyn > first_cell) & (presyn <= first_cell + n_cells)
    sources = np.empty(n, dtype=np.int64)
    sources[local] = presyn[local] - first_cell          # detector of local cell c is source c
    for gid in np.unique(presyn[~local]):
        sources[presyn == gid] = M.register_spike_source(model, sid=int(gid)).index
    targets = np.arange(first_syn, first_syn + n)
    M.connect_many(model, sources, targets, np.concatenate([d[5] for d in draws]), np.concatenate([d[4] for d in draws]))
    first_stim = M.add_pointprocesses(model, builtin("NetStim"), np.zeros(n, np.int64), "none",
                                      np.zeros(n), {"interval": 1000.0 / background_hz,
                                                    "number": 1e9, "start": 0.0, "noise": 1.0})
    stim_sids = total + first_cell * S + np.arange(n) + 1
    stim_sources = M.register_point_sources(model, np.arange(first_stim, first_stim + n), sids=stim_sids)
    M.connect_many(model, stim_sources, targets, np.concatenate([d[6] for d in draws]), np.zeros(n))
    return model


def _pyramidal(rng, target: int) -> List[Section]:
    """Pyramidal-like morphology with about `target` compartments (10 um each).

    Soma (1 compartment, 20x20 um); apical trunk of 600 um split into a
    proximal 100 um section (`trunk0`, label "prox") and the rest; 10-20
    oblique branches on the trunk and 5-10 tuft branches at its end; 4-8 basal
    dendrites of 150-250 um from soma(0), each with a proximal 100 um section
    (label "prox").  Diameters are seeded draws in [0.6, 4] um.  Oblique and
    tuft lengths share the compartments left after trunk and basals.
    """
    soma = Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1, Ra=100.0, cm=1.0)
    secs = [soma]
    trunk_d = float(rng.uniform(2.5, 4.0))
    secs.append(Section("trunk0", label="prox", parent="soma", parent_x=1.0, length=100.0,
                        diameter=trunk_d, nseg=10))
    secs.append(Section("trunk1", label="apical", parent="trunk0", parent_x=1.0, length=500.0,
                        diameter=trunk_d * 0.6, nseg=50))
    used = 1 + 60
    n_basal = int(rng.integers(4, 9))
    for b in range(n_basal):
        length = float(rng.uniform(150.0, 250.0))
        nseg = int(round(length / 10.0))
        d = float(rng.uniform(0.8, 2.0))
        secs.append(Section(f"basal{b}p", label="prox", parent="soma", parent_x=0.0, length=100.0,
                            diameter=d, nseg=10))
        secs.append(Section(f"basal{b}d", label="basal", parent=f"basal{b}p", parent_x=1.0,
                            length=length - 100.0, diameter=d * 0.8, nseg=nseg - 10))
        used += nseg
    n_oblique = int(rng.integers(10, 21))
    n_tuft = int(rng.integers(5, 11))
    remaining = max(target - used, n_oblique + n_tuft)
    shares = rng.dirichlet(np.ones(n_oblique + n_tuft)) * remaining
    nsegs = np.maximum(1, np.round(shares).astype(int))
    for k in range(n_oblique):
        x = float(rng.uniform(0.05, 0.95))
        secs.append(Section(f"obl{k}", label="apical", parent="trunk1", parent_x=x,
                            length=10.0 * nsegs[k], diameter=float(rng.uniform(0.6, 1.5)),
                            nseg=int(nsegs[k])))
    for k in range(n_tuft):
        nseg = int(nsegs[n_oblique + k])
        secs.append(Section(f"tuft{k}", label="apical", parent="trunk1", parent_x=1.0,
                            length=10.0 * nseg, diameter=float(rng.uniform(0.6, 1.5)), nseg=nseg))
    return secs


def config3(n_cells: int = 1000, synapses_per_cell: int = 300, connectivity: float = 0.03,
            background_hz: float = 2.0, iclamp_onset: float = 100.0) -> M.MicroModel:
    """Pyramidal-like micro network (1,000 cells of 700-1,200 compartments).

    hh at the soma and on the proximal 100 um sections (trunk0, basal*p), pas
    (g 1e-4, e -65) elsewhere.  300 Exp2Syn per cell (tau1 0.5, tau2 5 ms; 85%
    e = 0 mV, 15% e = -80 mV; 80% on basal, 20% on apical sections); 3%
    recurrent connectivity (each cell receives from round(0.03 N) distinct
    random presynaptic cells, each NetCon to a random synapse of the target)
    with delays U[0.5,3] ms and weights lognormal(ln 0.3 nS, 0.7); a 2 Hz
    Poisson NetStim per synapse (delay 0, same weight law); IClamp 0.1 nA for
    50 ms from `iclamp_onset` ms at soma(0.5) on the first 10% of cells.
    """
    rng = _rng(3)
    model = M.MicroModel(celsius=6.3)
    targets_n = rng.integers(700, 1201, n_cells)
    morph = []
    for c in range(n_cells):
        secs = _pyramidal(rng, int(targets_n[c]))
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, builtin("hh"), sections=["soma", "prox"])
        M.insert(cell, builtin("pas"), sections=["apical", "basal"], params={"g": 1.0e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
        morph.append((cell, secs))
    n = n_cells * synapses_per_cell
    owners = np.repeat(np.arange(1, n_cells + 1), synapses_per_cell)
    names, xs = [], []
    n_basal = int(round(0.8 * synapses_per_cell))
    for cell, secs in morph:
        nb, xb = _dendritic_sites(rng, secs, n_basal, labels=("basal", "prox"))
        na, xa = _dendritic_sites(rng, secs, synapses_per_cell - n_basal, labels=("apical",))
        names.extend(nb + na)
        xs.append(np.concatenate([xb, xa]))
    xs = np.concatenate(xs)
    e_rev = np.where(rng.uniform(size=n) < 0.85, 0.0, -80.0)
    first_syn = M.add_pointprocesses(model, builtin("Exp2Syn"), owners, names, xs,
                                     {"tau1": 0.5, "tau2": 5.0, "e": e_rev})
    k_in = int(round(connectivity * n_cells))
    pre, post = [], []
    for c in range(n_cells):
        choices = rng.choice(n_cells - 1, size=k_in, replace=False)
        choices = np.where(choices >= c, choices + 1, choices)
        pre.append(choices + 1)
        post.append(first_syn + c * synapses_per_cell + rng.integers(0, synapses_per_cell, k_in))
    pre = np.concatenate(pre) if pre else np.zeros(0, np.int64)
    post = np.concatenate(post) if post else np.zeros(0, np.int64)
    M.connect_many(model, pre, post, rng.lognormal(math.log(0.3), 0.7, len(pre)) / 1000.0,
                   rng.uniform(0.5, 3.0, len(pre)))
    first_stim = M.add_pointprocesses(model, builtin("NetStim"), np.zeros(n, np.int64), "none",
                                      np.zeros(n), {"interval": 1000.0 / background_hz,
                                                    "number": 1e9, "start": 0.0, "noise": 1.0})
    sources = M.register_point_sources(model, np.arange(first_stim, first_stim + n))
    M.connect_many(model, sources, np.arange(first_syn, first_syn + n),
                   rng.lognormal(math.log(0.3), 0.7, n) / 1000.0, np.zeros(n))
    n_clamp = max(1, n_cells // 10) if n_cells >= 1 else 0
    M.add_pointprocesses(model, builtin("IClamp"), np.arange(1, n_clamp + 1), "soma",
                         np.full(n_clamp, 0.5), {"del": iclamp_onset, "dur": 50.0, "amp": 0.1})
    return model


def config4(n_cells: int = 2000, populations: int = 20, synapses_per_cell: int = 300, connectivity: float = 0.03,
            input_scale: float = 2.0, micro_gain: float = 1.0, iclamp_onset: float = 100.0) -> M.MicroModel:
    """Micro-macro coupling: 2,000 pyramidal-like cells (300-600 compartments) in 20
    populations of 100, each population coupled to a Jansen-Rit region.

    Cells, synapses, recurrent NetCons and IClamps follow config 3 (hh soma and proximal,
    pas elsewhere; 300 Exp2Syn; 3% recurrence, delays U[0.5,3] ms), except that the
    synapses are driven by their population's region instead of NetStims: every synapse has
    its own external spike input (NetCon delay 0, weight lognormal(ln 0.3 nS, 0.7)) firing as
    a Poisson process at `input_scale` x the region's output (s^-1 -> Hz).  Regions: the
    Jansen-Rit defaults of mind_b200.macro (A 3.25 mV, B 22 mV, a 100 /s, b 50 /s, e0 2.5 /s,
    r 0.56 /mV, v0 6 mV, C 135, p0 120 /s), states from 0; region input += `micro_gain` x
    the population's spike rate (Hz per cell, 1 ms bins); a random region graph of density
    0.2 with gains U[0,1] and delays of U{1..20} macro steps (0.1-2 ms, a choice: the
    configuration leaves delays open); RK4 at dt_macro = 0.1 ms.  The model's `macro`
    attribute holds the MacroModel.
    """
    from .macro import MacroModel

    rng = _rng(4)
    model = M.MicroModel(celsius=6.3)
    targets_n = rng.integers(300, 601, n_cells)
    morph = []
    detectors = np.empty(n_cells, dtype=np.int64)
    for c in range(n_cells):
        secs = _pyramidal(rng, int(targets_n[c]))
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, builtin("hh"), sections=["soma", "prox"])
        M.insert(cell, builtin("pas"), sections=["apical", "basal"], params={"g": 1.0e-4, "e": -65.0})
        detectors[c] = M.register_spike_source(cell, threshold=-10.0).index
        morph.append((cell, secs))
    S = synapses_per_cell
    n = n_cells * S
    owners = np.repeat(np.arange(1, n_cells + 1), S)
    names, xs = [], []
    n_basal = int(round(0.8 * S))
    for cell, secs in morph:
        nb, xb = _dendritic_sites(rng, secs, n_basal, labels=("basal", "prox"))
        na, xa = _dendritic_sites(rng, secs, S - n_basal, labels=("apical",))
        names.extend(nb + na)
        xs.append(np.concatenate([xb, xa]))
    e_rev = np.where(rng.uniform(size=n) < 0.85, 0.0, -80.0)
    first_syn = M.add_pointprocesses(model, builtin("Exp2Syn"), owners, names, np.concatenate(xs),
                                     {"tau1": 0.5, "tau2": 5.0, "e": e_rev})
    k_in = int(round(connectivity * n_cells))
    pre, post = [], []
    for c in range(n_cells):
        choices = rng.choice(n_cells - 1, size=k_in, replace=False)
        choices = np.where(choices >= c, choices + 1, choices)
        pre.append(detectors[choices])
        post.append(first_syn + c * S + rng.integers(0, S, k_in))
    M.connect_many(model, np.concatenate(pre), np.concatenate(post),
                   rng.lognormal(math.log(0.3), 0.7, n_cells * k_in) / 1000.0, rng.uniform(0.5, 3.0, n_cells * k_in))
    inputs = M.register_external_sources(model, n)
    M.connect_many(model, inputs, np.arange(first_syn, first_syn + n), rng.lognormal(math.log(0.3), 0.7, n) / 1000.0,
                   np.zeros(n))
    n_clamp = max(1, n_cells // 10)
    M.add_pointprocesses(model, builtin("IClamp"), np.arange(1, n_clamp + 1), "soma",
                         np.full(n_clamp, 0.5), {"del": iclamp_onset, "dur": 50.0, "amp": 0.1})
    macro = MacroModel(dt_macro=0.1, bin_ms=1.0)
    for _ in range(populations):
        macro.add_region(micro_gain=micro_gain)
    for src in range(1, populations + 1):
        for dst in range(1, populations + 1):
            if src != dst and rng.uniform() < 0.2:
                macro.connect(src, dst, float(rng.uniform(0.0, 1.0)), int(rng.integers(1, 21)))
    per_pop = n_cells // populations
    for c in range(n_cells):
        region = min(c // per_pop, populations - 1) + 1
        macro.add_inputs(region, inputs[c * S:(c + 1) * S], input_scale)
        macro.add_outputs(region, [detectors[c]])
    model.macro = macro
    return model


def config5(n_cells: int = 100_000, populations: int = 200, **kwargs) -> M.MicroModel:
    """Surrogate-coupled micro-macro: config 4 scaled to 100,000 cells in 200 populations of
    500, each coupled to its own Jansen-Rit region (200 regions, the same random region graph
    rule).  Each cell keeps config 4's recurrent in-degree (3% of 2,000 cells: 60 NetCons from
    random cells), so that a cell's input statistics, and with them the surrogate trained on
    config 4, carry over.  The surrogate that stands in for most of its cells is trained on
    config 4."""
    kwargs.setdefault("connectivity", 0.03 * 2000 / n_cells)
    return config4(n_cells=n_cells, populations=populations, **kwargs)


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}


def compartment_count(layout) -> int:
    """Number of compartments (segments) in a built layout: the metric's unit."""
    return layout.segment_count
