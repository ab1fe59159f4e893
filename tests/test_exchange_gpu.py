"""The device-resident spike exchange of a sharded network (mind_attach_exchange).

Two shards of one network run in this process on cuda:0, window by window; after each
window every shard packs its cells' spikes on the device (mind_exchange_pack), the blocks
are concatenated on the device (what ncclAllGather does between GPUs), and every shard
enters the received spikes (mind_exchange_inject).  The traces and rasters must equal the
unsharded run bit for bit.  A one-rank NCCL communicator then runs the exchange inside
mind_run (pack, ncclAllGather, inject on the handle's stream).
"""
import os
import socket

import numpy as np
import pytest
import torch

import mind_b200 as mb
import netcases
from mind_b200 import sharding
from mind_b200.runtime import DeviceState

pytestmark = pytest.mark.gpu

T_STOP = 40.0


def _whole(layout_model):
    model = layout_model
    layout = model.layout
    nodes = netcases.soma_nodes(layout)
    mb.initialize(model)
    whole = mb.run(model, T_STOP, records=[mb.RecordSpec(n, f"n{n}") for n in nodes])
    model.state.close()
    return whole, nodes


def test_device_exchange_kernels_reproduce_the_single_gpu_run():
    model = netcases.recurrent_trees()
    layout = mb.build(model)
    whole, nodes = _whole(model)
    owners = sharding.partition_cells(layout, 2)
    shards = [sharding.shard_layout(layout, np.nonzero(owners == r)[0]) for r in range(2)]
    states = [DeviceState(sh.layout, "fp64") for sh in shards]
    for st in states:
        st.initialize()
    window = min(st.window_steps() for st in states)
    maps = [sharding.exchange_maps(sh) for sh in shards]
    assert all(len(m[2]) > 0 for m in maps)   # NetCons really cross the shards
    width = max(len(m[0]) for m in maps) + 16
    for r, (st, m) in enumerate(zip(states, maps)):
        st.attach_exchange(None, 2, r, window, width, *m)
    send = [torch.zeros(1 + 2 * width, dtype=torch.int64, device="cuda") for _ in range(2)]
    mine = [[n for n in nodes if sh.node_map[n] > 0] for sh in shards]
    recs = [[mb.RecordSpec(int(sh.node_map[n]), f"n{n}") for n in mine[r]] for r, sh in enumerate(shards)]
    traces = {n: [] for n in nodes}
    times, sids = [], []
    steps, done = int(round(T_STOP / layout.dt)), 0
    exchanged = 0
    while done < steps:
        k = min(window, steps - done)
        for r, st in enumerate(states):
            res = st.run_steps(k, recs[r], True)
            for n in mine[r]:
                tr = res.traces[f"n{n}"]
                traces[n].append(tr if not traces[n] else tr[1:])
            ext = np.asarray(sorted(shards[r].external_source), dtype=np.int64)
            keep = ~np.isin(res.spike_sources, ext)
            times += res.spike_times[keep].tolist()
            sids += res.spike_sources[keep].tolist()
            st.exchange_pack(send[r].data_ptr())
        torch.cuda.synchronize()
        recv = torch.cat(send)
        torch.cuda.synchronize()
        exchanged += int(send[0][0].item() + send[1][0].item())
        for st in states:
            st.exchange_inject(recv.data_ptr())
        done += k
    for st in states:
        st.close()
    assert exchanged > 10
    for n in nodes:
        np.testing.assert_array_equal(np.concatenate(traces[n]), whole.traces[f"n{n}"])
    merged = sorted(set(zip(times, sids)))
    want = sorted(zip(whole.spike_times.tolist(), whole.spike_sources.tolist()))
    assert merged == want


def test_nccl_exchange_inside_mind_run_on_one_rank():
    """A communicator of one rank: every window's pack, ncclAllGather and inject run inside
    mind_run on the handle's stream; the run equals the plain one."""
    import torch.distributed as dist

    model = netcases.recurrent_trees()
    layout = mb.build(model)
    whole, nodes = _whole(model)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        run = sharding.ShardedRun(layout, 0, 1, precision="fp64", device="cpu", exchange="device")
        res = run.run_steps(int(round(T_STOP / layout.dt)), run.records(nodes))
        # the ranks share the exchange's window length: regions, which set their own, are refused
        from mind_b200 import abi
        from mind_b200.macro import MacroModel
        lone = MacroModel(dt_macro=0.1, bin_ms=1.0)
        lone.add_region(micro_gain=0.0)
        with pytest.raises(abi.MindError) as err:
            run.state.attach_macro(lone)
        assert err.value.status == abi.MIND_EARG
        run.close()
    finally:
        dist.destroy_process_group()
    for n in nodes:
        np.testing.assert_array_equal(res.traces[f"n{n}"], whole.traces[f"n{n}"])
    np.testing.assert_array_equal(np.sort(res.spike_times), np.sort(whole.spike_times))
