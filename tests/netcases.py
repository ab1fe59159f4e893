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
