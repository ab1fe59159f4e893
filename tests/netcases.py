"""Small seeded networks for parity tests, built through the public API.

Each returns a built model whose cells fire (the benchmark's config 1 drive is
sub-threshold), so rasters and traces both carry information.
"""
import math

import numpy as np

import mind_b200 as mb
from mind_b200 import model as M
from mind_b200 import networks


def strong_config1(n_cells=16, synapses=10, weight_scale=40.0):
    """Config 1 geometry with weights scaled so the somata spike."""
    model = networks.config1(n_cells=n_cells, synapses_per_cell=synapses)
    for chunk in model.connection_chunks:
        chunk.weights = chunk.weights * weight_scale
    return model


def recurrent_trees(n_cells=24, synapses=20, seed=7, min_delay=0.6):
    """Random binary trees (config 2 style) with recurrent Exp2Syn and IClamp drive."""
    rng = np.random.default_rng(seed)
    model = M.MicroModel(celsius=6.3)
    cells = []
    for c in range(n_cells):
        soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
        secs = networks._binary_tree(rng, int(rng.integers(30, 120)), soma)
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, mb.builtin("hh"), sections="soma")
        M.insert(cell, mb.builtin("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
        cells.append((cell, secs))
    n = n_cells * synapses
    owners = np.repeat(np.arange(1, n_cells + 1), synapses)
    names, xs = [], []
    for cell, secs in cells:
        nm, x = networks._dendritic_sites(rng, secs, synapses)
        names += nm
        xs.append(x)
    first = M.add_pointprocesses(model, mb.builtin("Exp2Syn"), owners, names, np.concatenate(xs),
                                 {"tau1": 0.5, "tau2": 5.0, "e": np.where(rng.uniform(size=n) < 0.8, 0.0, -80.0)})
    M.connect_many(model, rng.integers(1, n_cells + 1, n), np.arange(first, first + n),
                   rng.lognormal(math.log(3.0), 0.5, n) / 1000.0, rng.uniform(min_delay, 3.0, n))
    stims = M.add_pointprocesses(model, mb.builtin("NetStim"), np.zeros(n, np.int64), "none", np.zeros(n),
                                 {"interval": 50.0, "number": 1e9, "start": 0.0, "noise": 1.0})
    sources = M.register_point_sources(model, np.arange(stims, stims + n))
    M.connect_many(model, sources, np.arange(first, first + n),
                   rng.lognormal(math.log(6.0), 0.5, n) / 1000.0, rng.uniform(0.0, 1.0, n))
    k = max(1, n_cells // 4)
    M.add_pointprocesses(model, mb.builtin("IClamp"), np.arange(1, k + 1), "soma", np.full(k, 0.5),
                         {"del": 5.0, "dur": 20.0, "amp": 0.3})
    return model


def soma_nodes(layout):
    return [layout.voltage_node(c) for c in range(1, layout.n_cells + 1)]


def coupled_regions(n_regions=3, cells_per_region=4, synapses=8, seed=11, input_scale=300.0, min_cell_delay=0.6):
    """Ball-and-stick populations coupled to Jansen-Rit regions (config 4 in miniature).

    Every synapse (Exp2Syn) gets its own external spike input driven by its population's
    region; every cell's soma detector feeds the region's rate bin; regions are coupled by
    random edges with delays of 1-5 macro steps; recurrent NetCons between cells
    (min_cell_delay-2 ms).
    Returns (model, macro) with model built.
    """
    from mind_b200.macro import MacroModel

    rng = np.random.default_rng(seed)
    model = M.MicroModel(celsius=6.3)
    soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
    dend = mb.Section("dend", label="dend", parent="soma", parent_x=1.0, length=300.0, diameter=2.0, nseg=15)
    n_cells = n_regions * cells_per_region
    cells = M.add_population(model, [soma, dend], n_cells, voltage=-65.0)
    detectors = []
    for cell in cells:
        M.insert(cell, mb.builtin("hh"), sections="soma")
        M.insert(cell, mb.builtin("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        detectors.append(M.register_spike_source(cell, threshold=-10.0).index)
    n = n_cells * synapses
    owners = np.repeat(np.arange(1, n_cells + 1), synapses)
    first = M.add_pointprocesses(model, mb.builtin("Exp2Syn"), owners, "dend", rng.uniform(0, 1, n),
                                 {"tau1": 0.5, "tau2": 5.0, "e": np.where(rng.uniform(size=n) < 0.8, 0.0, -80.0)})
    inputs = [M.register_spike_source(model).index for _ in range(n)]
    M.connect_many(model, inputs, np.arange(first, first + n), rng.lognormal(math.log(4.0), 0.4, n) / 1000.0,
                   np.zeros(n))
    k = n // 4
    M.connect_many(model, rng.choice(detectors, k), rng.integers(first, first + n, k),
                   rng.lognormal(math.log(2.0), 0.4, k) / 1000.0, rng.uniform(min_cell_delay, 2.0, k))
    macro = MacroModel(dt_macro=0.1, bin_ms=1.0)
    for r in range(n_regions):
        macro.add_region(micro_gain=2.0, y0=[0.0, rng.uniform(0, 5), rng.uniform(0, 5), 0.0, 0.0, 0.0])
    for src in range(1, n_regions + 1):
        for dst in range(1, n_regions + 1):
            if src != dst and rng.uniform() < 0.5:
                macro.connect(src, dst, float(rng.uniform(0, 1)) * 50.0, int(rng.integers(1, 6)))
    for c in range(n_cells):
        region = c // cells_per_region + 1
        macro.add_inputs(region, inputs[c * synapses:(c + 1) * synapses], input_scale)
        macro.add_outputs(region, [detectors[c]])
    model.macro = macro
    mb.build(model)
    return model, macro


def big_and_small_cells(big_compartments=8000, n_small=3, synapses=12, seed=5):
    """One cell too large for a CTA's shared memory (its image lives in HBM) beside small
    ones, with hh somata, pas dendrites, Exp2Syn driven by NetStims and recurrent NetCons."""
    rng = np.random.default_rng(seed)
    model = M.MicroModel(celsius=6.3)
    cells = []
    for c in range(1 + n_small):
        soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
        size = big_compartments if c == 0 else int(rng.integers(40, 120))
        secs = networks._binary_tree(rng, size, soma)
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, mb.builtin("hh"), sections="soma")
        M.insert(cell, mb.builtin("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
        cells.append((cell, secs))
    n_cells = len(cells)
    n = n_cells * synapses
    owners = np.repeat(np.arange(1, n_cells + 1), synapses)
    names, xs = [], []
    for cell, secs in cells:
        nm, x = networks._dendritic_sites(rng, secs, synapses)
        names += nm
        xs.append(x)
    first = M.add_pointprocesses(model, mb.builtin("Exp2Syn"), owners, names, np.concatenate(xs),
                                 {"tau1": 0.5, "tau2": 5.0, "e": 0.0})
    M.connect_many(model, rng.integers(1, n_cells + 1, n), np.arange(first, first + n),
                   rng.lognormal(math.log(3.0), 0.5, n) / 1000.0, rng.uniform(0.6, 3.0, n))
    stims = M.add_pointprocesses(model, mb.builtin("NetStim"), np.zeros(n, np.int64), "none", np.zeros(n),
                                 {"interval": 10.0, "number": 1e9, "start": 0.0, "noise": 1.0})
    sources = M.register_point_sources(model, np.arange(stims, stims + n))
    M.connect_many(model, sources, np.arange(first, first + n),
                   rng.lognormal(math.log(8.0), 0.5, n) / 1000.0, rng.uniform(0.0, 1.0, n))
    M.add_pointprocesses(model, mb.builtin("IClamp"), np.array([1, 2]), "soma", np.full(2, 0.5),
                         {"del": 2.0, "dur": 30.0, "amp": 0.8})
    return model


def dhs_order(layout, lanes=32):
    """A node order of the kind MIND.jl's DHS planner hands the runtime
    (src/model/micro/model.jl:906-1077): each cell's nodes in elimination order -- reverse
    breadth-first, children before their parent -- and the cells of each group of `lanes`
    interleaved round by round, largest cell first.  Returns the old 1-based node of every
    new position (0-based array)."""
    parent = np.asarray(layout.parent, dtype=np.int64)
    n = len(parent)
    children = [[] for _ in range(n + 1)]
    for i in range(n):
        children[parent[i]].append(i + 1)
    cells = []
    for root in children[0]:
        bfs = [root]
        k = 0
        while k < len(bfs):
            bfs.extend(children[bfs[k]])
            k += 1
        cells.append(bfs[::-1])
    order = []
    for g in range(0, len(cells), lanes):
        group = sorted(cells[g:g + lanes], key=len, reverse=True)
        for r in range(len(group[0])):
            order.extend(c[r] for c in group if r < len(c))
    return np.asarray(order, dtype=np.int64)


def permute_layout(layout, order):
    """The same network with node new = position of old in `order` (1-based): parents,
    node arrays, mechanism nodes and detector nodes renumbered; rows, points and edges kept."""
    import dataclasses

    new_of = np.zeros(len(order) + 1, dtype=np.int64)
    new_of[order] = np.arange(1, len(order) + 1)
    idx = order - 1
    parent = np.asarray(layout.parent, dtype=np.int64)[idx]
    groups = []
    for g in layout.groups:
        nodes = np.asarray(g.nodes, dtype=np.int64)
        renumbered = np.where(nodes > 0, new_of[nodes], 0).astype(np.int32)
        groups.append(dataclasses.replace(g, nodes=renumbered))
    src = np.asarray(layout.source_nodes, dtype=np.int64)
    return dataclasses.replace(
        layout, parent=new_of[parent].astype(np.int32), voltage=np.asarray(layout.voltage)[idx],
        area=np.asarray(layout.area)[idx], capacitance=np.asarray(layout.capacitance)[idx],
        axial=np.asarray(layout.axial)[idx], axial_diagonal=np.asarray(layout.axial_diagonal)[idx],
        groups=groups, source_nodes=np.where(src > 0, new_of[src], 0).astype(np.int32), _keep=[]), new_of


def burst_onto_one_cell(n_events=200, n_cells=3, seed=4):
    """One NetStim that fires once (t = 2 ms, no noise) with `n_events` NetCons onto the
    Exp2Syn of cell 1, delays U[0.5, 1.0] ms: every event lands in one window of cell 1's
    inbox.  The other cells get a few ordinary synapses, so their inboxes stay small."""
    rng = np.random.default_rng(seed)
    model = M.MicroModel(celsius=6.3)
    cells = []
    for c in range(n_cells):
        soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
        secs = networks._binary_tree(rng, 60, soma)
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, mb.builtin("hh"), sections="soma")
        M.insert(cell, mb.builtin("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
        cells.append((cell, secs))
    counts = [n_events] + [8] * (n_cells - 1)
    owners = np.repeat(np.arange(1, n_cells + 1), counts)
    names, xs = [], []
    for (cell, secs), k in zip(cells, counts):
        nm, x = networks._dendritic_sites(rng, secs, k)
        names += nm
        xs.append(x)
    n = int(sum(counts))
    first = M.add_pointprocesses(model, mb.builtin("Exp2Syn"), owners, names, np.concatenate(xs),
                                 {"tau1": 0.5, "tau2": 5.0, "e": 0.0})
    stim = M.add_pointprocesses(model, mb.builtin("NetStim"), np.zeros(1, np.int64), "none", np.zeros(1),
                                {"interval": 10.0, "number": 1.0, "start": 2.0, "noise": 0.0})
    source = M.register_point_sources(model, np.array([stim]))
    M.connect_many(model, np.repeat(source, n), np.arange(first, first + n),
                   rng.lognormal(math.log(0.05), 0.3, n) / 1000.0, rng.uniform(0.5, 1.0, n))
    return model


def mechanism_mix(select, n_cells=12, synapses=12, seed=9, clamps=False):
    """Branched cells with every cell mechanism of the MOD directory, each taken from
    `select(name)` -- mb.builtin (hand-written device code) or mb.emitted (CUDA C emitted
    from the MOD file): hh somata, pas dendrites, Exp2Syn and ExpSyn synapses driven by
    NetStims and recurrent NetCons, IClamp and AlphaSynapse on some somata; with `clamps`,
    an SEClamp on cell 1's soma and a VClamp on cell 2's (three command levels each)."""
    rng = np.random.default_rng(seed)
    model = M.MicroModel(celsius=6.3)
    cells = []
    for c in range(n_cells):
        soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
        secs = networks._binary_tree(rng, int(rng.integers(30, 90)), soma)
        cell = M.add_population(model, secs, 1, voltage=-65.0)[0]
        M.insert(cell, select("hh"), sections="soma")
        M.insert(cell, select("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
        cells.append((cell, secs))
    n = n_cells * synapses
    owners = np.repeat(np.arange(1, n_cells + 1), synapses)
    names, xs = [], []
    for cell, secs in cells:
        nm, x = networks._dendritic_sites(rng, secs, synapses)
        names += nm
        xs.append(x)
    xs = np.concatenate(xs)
    half = n // 2
    first2 = M.add_pointprocesses(model, select("Exp2Syn"), owners[:half], names[:half], xs[:half],
                                  {"tau1": 0.5, "tau2": 5.0, "e": np.where(rng.uniform(size=half) < 0.8, 0.0, -80.0)})
    first1 = M.add_pointprocesses(model, select("ExpSyn"), owners[half:], names[half:], xs[half:],
                                  {"tau": 2.0, "e": 0.0})
    targets = np.concatenate([np.arange(first2, first2 + half), np.arange(first1, first1 + n - half)])
    M.connect_many(model, rng.integers(1, n_cells + 1, n), targets,
                   rng.lognormal(math.log(3.0), 0.5, n) / 1000.0, rng.uniform(0.6, 3.0, n))
    stims = M.add_pointprocesses(model, mb.builtin("NetStim"), np.zeros(n, np.int64), "none", np.zeros(n),
                                 {"interval": 40.0, "number": 1e9, "start": 0.0, "noise": 1.0})
    sources = M.register_point_sources(model, np.arange(stims, stims + n))
    M.connect_many(model, sources, targets, rng.lognormal(math.log(6.0), 0.5, n) / 1000.0, rng.uniform(0.0, 1.0, n))
    k = max(1, n_cells // 4)
    M.add_pointprocesses(model, select("IClamp"), np.arange(3, 3 + k), "soma", np.full(k, 0.5),
                         {"del": 5.0, "dur": 20.0, "amp": 0.3})
    M.add_pointprocesses(model, select("AlphaSynapse"), np.arange(4, 4 + k), "soma", np.full(k, 0.5),
                         {"onset": 8.0, "tau": 2.0, "gmax": 0.02, "e": 0.0})
    if clamps:
        M.add_pointprocesses(model, select("SEClamp"), np.array([1]), "soma", np.array([0.5]),
                             {"dur1": 5.0, "amp1": -70.0, "dur2": 10.0, "amp2": -20.0, "dur3": 8.0, "amp3": -60.0,
                              "rs": 0.01})
        M.add_pointprocesses(model, select("VClamp"), np.array([2]), "soma", np.array([0.5]),
                             {"dur[0]": 6.0, "dur[1]": 9.0, "dur[2]": 6.0, "amp[0]": -68.0, "amp[1]": -25.0,
                              "amp[2]": -55.0})
    return model


def pattern_driven(n_cells=4, seed=6):
    """Ball-and-stick cells driven only by two PatternStims (prescribed spike trains) through
    Exp2Syn NetCons; returns (model, {PatternStim source sid: its spike times})."""
    rng = np.random.default_rng(seed)
    model = M.MicroModel(celsius=6.3)
    soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
    dend = mb.Section("dend", label="dend", parent="soma", parent_x=1.0, length=200.0, diameter=2.0, nseg=10)
    cells = M.add_population(model, [soma, dend], n_cells, voltage=-65.0)
    for cell in cells:
        M.insert(cell, mb.builtin("hh"), sections="soma")
        M.insert(cell, mb.builtin("pas"), sections="dend", params={"g": 1e-4, "e": -65.0})
        M.register_spike_source(cell, threshold=-10.0)
    syn = M.add_pointprocesses(model, mb.builtin("Exp2Syn"), np.arange(1, n_cells + 1), "dend", np.full(n_cells, 0.3),
                               {"tau1": 0.5, "tau2": 5.0, "e": 0.0})
    trains = {}
    for k, times in enumerate(([1.0, 4.0, 4.0, 9.5, 20.0], np.sort(rng.uniform(0.0, 30.0, 12)))):
        stim = M.add_pointprocess(model, mb.builtin("PatternStim"), spike_times=times)
        source = M.register_spike_source(stim)
        trains[source.sid] = np.asarray(times, dtype=float)
        M.connect_many(model, np.full(n_cells, source.index), np.arange(syn, syn + n_cells),
                       np.full(n_cells, 0.012 if k == 0 else 0.004), rng.uniform(0.5, 2.0, n_cells))
    return model, trains
