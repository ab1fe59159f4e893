"""AlphaSynapse (mod/AlphaSynapse.mod) on the device against the CPU oracle.

Branched cells with hh somata, recurrent Exp2Syn and, on every cell, AlphaSynapses at
dendritic sites with staggered onsets: FP64 voltages and raster bit-identical to the
oracle, the mixed mode within its tolerances, and a recorded AlphaSynapse parameter.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import model as M
from mind_b200 import networks

pytestmark = pytest.mark.gpu


def _model(n_cells=10, per_cell=4, seed=3):
    model = netcases.recurrent_trees(n_cells=n_cells, synapses=8, seed=seed)
    rng = np.random.default_rng(seed)
    owners = np.repeat(np.arange(1, n_cells + 1), per_cell)
    n = len(owners)
    M.add_pointprocesses(model, mb.builtin("AlphaSynapse"), owners, "soma", np.full(n, 0.5),
                         {"onset": rng.uniform(1.0, 20.0, n), "tau": rng.uniform(0.5, 3.0, n),
                          "gmax": rng.uniform(0.002, 0.02, n), "e": np.where(rng.uniform(size=n) < 0.8, 0.0, -80.0)})
    return model


def test_alpha_synapses_match_the_oracle():
    model = _model()
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    steps = 1400
    gmax = mb.mechanism_ref(model, "AlphaSynapse", 3, "gmax")
    recs = [mb.RecordSpec(n, f"n{n}") for n in nodes] + [gmax]
    ref = oracle.run(layout, steps, records=recs)
    assert ref.status == 0, ref.message
    mb.initialize(model, precision="fp64")
    res = mb.run(model, steps * layout.dt, records=recs)
    got = np.stack([res.traces[r.name] for r in recs], axis=1)
    assert np.array_equal(got, ref.trace)
    np.testing.assert_array_equal(res.spike_times, ref.spike_times)
    np.testing.assert_array_equal(res.spike_sources, ref.spike_sids)
    assert np.sum(ref.spike_sids < layout.n_cells) > 5          # the synapses made cells fire
    mb.initialize(model, precision="mixed")
    mixed = mb.run(model, steps * layout.dt, records=recs[:-1])
    mx = np.stack([mixed.traces[r.name] for r in recs[:-1]], axis=1)
    sub = (ref.trace[:, :-1] < -50.0) & (mx < -50.0)
    assert np.max(np.abs(mx - ref.trace[:, :-1])[sub]) < 0.05   # mV, below threshold
