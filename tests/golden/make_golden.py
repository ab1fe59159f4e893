"""Generate the golden fixtures of tests/golden/ from the CPU FP64 oracle.

    python tests/golden/make_golden.py

Each fixture is a small seeded network built through the public API, run by the
oracle; it stores soma voltages every 10 steps and the full spike raster.  The
fixtures pin the oracle against regressions and give the CUDA tests a target
that does not need the oracle at run time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "mind.jl_b200"), os.path.join(ROOT, "oracle"), os.path.dirname(HERE)]

import mind_b200 as mb  # noqa: E402
import netcases  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "ball_and_stick_4cells_10ms": (lambda: netcases.strong_config1(n_cells=4), 400),
    "recurrent_trees_8cells_20ms": (lambda: netcases.recurrent_trees(n_cells=8, synapses=12), 800),
}


def generate(name):
    build, steps = CASES[name]
    layout = mb.build(build())
    nodes = netcases.soma_nodes(layout)
    ref = oracle.run(layout, steps, nodes)
    assert ref.status == 0, ref.message
    return dict(steps=steps, nodes=np.array(nodes), trace=ref.trace[::10].copy(), every=10,
                spike_times=ref.spike_times, spike_sids=ref.spike_sids)


if __name__ == "__main__":
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **generate(name))
        print("wrote", name)
