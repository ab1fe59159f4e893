"""One network on two ranks (two processes sharing cuda:0, gloo exchange) vs one process.

Each rank simulates half of the cells; cell spikes cross ranks once per window as
external spike inputs.  The sharded run must reproduce the single-process run bit
for bit: every soma trace and the whole raster (cells and NetStims).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import mind_b200 as mb
import netcases

pytestmark = pytest.mark.gpu

T_STOP = 40.0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(os.path.dirname(here), "mind.jl_b200"), here]
    import torch.distributed as dist
    import mind_b200 as mbw
    import netcases as nc
    from mind_b200 import sharding

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    layout = mbw.build(nc.recurrent_trees())
    run = sharding.ShardedRun(layout, rank, world, precision="fp64", device="cpu")
    cells = run.shard.cells
    nodes = [layout.voltage_node(int(c) + 1) for c in cells]
    result = run.run_steps(int(round(T_STOP / layout.dt)), run.records(nodes))
    out[rank] = ({int(n): result.traces[f"n{n}"].tolist() for n in nodes}, result.spike_sources.tolist(),
                 result.spike_times.tolist(), run.window, len(run.shard.external_source))
    run.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_reproduce_the_single_gpu_run():
    model = netcases.recurrent_trees()
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    mb.initialize(model)
    whole = mb.run(model, T_STOP, records=[mb.RecordSpec(n, f"n{n}") for n in nodes])
    model.state.close()

    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    traces = {}
    sids, times = [], []
    for r in range(world):
        traces.update(out[r][0])
        sids += out[r][1]
        times += out[r][2]
        assert out[r][4] > 0           # NetCons really cross ranks
        assert 0 < out[r][3] <= 64
    assert sorted(traces) == sorted(nodes)
    for n in nodes:
        np.testing.assert_array_equal(np.asarray(traces[n]), whole.traces[f"n{n}"])
    # NetStims driving synapses on both ranks run on both: merge the rasters as sets
    merged = sorted(set(zip(times, sids)))
    want = sorted(zip(whole.spike_times.tolist(), whole.spike_sources.tolist()))
    assert merged == want
    assert np.sum(whole.spike_sources < layout.n_cells) > 10   # cells fired
