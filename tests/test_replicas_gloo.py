"""The N>1 path on CPU: two gloo ranks, each running its own seeded replica.

Each rank runs the CPU oracle on a replica built with seed 1 + rank (as bench.py
does on GPUs) and the ranks reduce timing as bench.py does: max of the run time,
sum of compartment-steps.  The test checks the reduction and that each rank's
raster equals a single-process run of the same replica.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica_raster(seed):
    import mind_b200 as mb
    import oracle
    from mind_b200 import networks

    model = networks.config1(n_cells=4)
    for chunk in model.connection_chunks:
        chunk.weights = chunk.weights * 40.0
    layout = mb.build(model, seed=seed)
    ref = oracle.run(layout, 1200, [])
    return layout, ref


def _worker(rank, world, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path[:0] = [os.path.join(root, "mind.jl_b200"), os.path.join(root, "oracle")]
    import torch.distributed as dist
    from mind_b200 import replicas

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    layout, ref = _replica_raster(replicas.replica_seed(1, rank))
    units = layout.segment_count * 1200
    max_ms, total = replicas.reduce_timing(ref.run_ms + rank, units)
    out[rank] = (max_ms, total, ref.run_ms + rank, units, ref.spike_times.tolist(), ref.spike_sids.tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_bench():
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    local_ms = [out[r][2] for r in range(world)]
    local_units = [out[r][3] for r in range(world)]
    for r in range(world):
        assert out[r][0] == max(local_ms)
        assert out[r][1] == sum(local_units)
    for r in range(world):
        _, ref = _replica_raster(1 + r)
        np.testing.assert_array_equal(out[r][4], ref.spike_times)
        np.testing.assert_array_equal(out[r][5], ref.spike_sids)
    assert out[0][4] != out[1][4]   # different seeds, different NetStim trains
