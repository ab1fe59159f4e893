"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the oracle reproduces its committed fixtures bit for bit (regression pin).
GPU: libmindgpu.so reproduces the same fixtures bit for bit through the C-ABI.
"""
import os

import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {
    "ball_and_stick_4cells_10ms": lambda: netcases.strong_config1(n_cells=4),
    "recurrent_trees_8cells_20ms": lambda: netcases.recurrent_trees(n_cells=8, synapses=12),
}


def load(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as f:
        return {k: f[k] for k in f.files}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(name):
    gold = load(name)
    layout = mb.build(CASES[name]())
    nodes = netcases.soma_nodes(layout)
    np.testing.assert_array_equal(nodes, gold["nodes"])
    ref = oracle.run(layout, int(gold["steps"]), nodes)
    np.testing.assert_array_equal(ref.trace[::int(gold["every"])], gold["trace"])
    np.testing.assert_array_equal(ref.spike_times, gold["spike_times"])
    np.testing.assert_array_equal(ref.spike_sids, gold["spike_sids"])
    assert len(gold["spike_times"]) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_reproduces_golden(name):
    gold = load(name)
    model = CASES[name]()
    layout = mb.build(model)
    records = [mb.RecordSpec(int(n), f"n{n}") for n in gold["nodes"]]
    mb.initialize(model)
    result = mb.run(model, int(gold["steps"]) * layout.dt, records=records)
    trace = np.stack([result.traces[r.name] for r in records], axis=1)
    np.testing.assert_array_equal(trace[::int(gold["every"])], gold["trace"])
    np.testing.assert_array_equal(result.spike_times, gold["spike_times"])
    np.testing.assert_array_equal(result.spike_sources, gold["spike_sids"])
