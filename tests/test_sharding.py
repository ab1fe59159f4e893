"""Cells partitioned over ranks (CPU): the shards' layouts and the spike exchange.

A shard keeps its cells' nodes and rows, the NetStims that drive them, its detectors,
and every NetCon into its synapses; a presynaptic cell on another rank becomes an
external spike input there.  The exchange all-gathers variable-length (sid, time)
lists over two gloo ranks.  The GPU test (test_sharded_gpu.py) checks that a
sharded run reproduces the single-GPU raster and traces.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import mind_b200 as mb
import netcases
from mind_b200 import sharding


def _edges(layout):
    """(target point's (group, row) identity, source sid, delay, weight) of every NetCon."""
    fan = np.asarray(layout.fanout_offsets) - 1
    out = []
    for s in range(len(layout.source_ids)):
        for e in range(fan[s], fan[s + 1]):
            p = layout.edge_targets[e] - 1
            g = layout.groups[layout.point_group[p] - 1]
            row = layout.point_row[p] - 1
            out.append((g.mechanism.name, int(g.logical_ids[row]), int(layout.source_ids[s]),
                        float(layout.edge_delays[e]), float(layout.edge_weights[e])))
    return out


def test_shards_partition_cells_rows_and_netcons():
    model = netcases.recurrent_trees(n_cells=24, synapses=12)
    layout = mb.build(model)
    world = 3
    owners = sharding.partition_cells(layout, world)
    assert owners.min() == 0 and owners.max() == world - 1 and np.all(np.diff(owners) >= 0)
    shards = [sharding.shard_layout(layout, np.nonzero(owners == r)[0]) for r in range(world)]
    assert sum(s.layout.n_nodes for s in shards) == layout.n_nodes
    assert sum(s.layout.n_cells for s in shards) == layout.n_cells
    assert sum(s.layout.segment_count for s in shards) == layout.segment_count
    # cell-mechanism rows are partitioned; NetStims may be repeated where they drive synapses
    for gi, g in enumerate(layout.groups):
        if g.mechanism.name == "NetStim":
            continue
        ids = np.concatenate([s.layout.groups[gi].logical_ids for s in shards])
        assert sorted(ids.tolist()) == sorted(np.asarray(g.logical_ids).tolist())
    # every NetCon appears once, on the rank owning its target, with its source sid, delay, weight
    whole = sorted(_edges(layout))
    parts = sorted(e for s in shards for e in _edges(s.layout))
    assert parts == whole
    # remote presynaptic cells enter as external inputs; owned detectors stay detectors
    detector_sids = set(np.asarray(layout.source_ids)[np.asarray(layout.source_nodes) > 0].tolist())
    for r, s in enumerate(shards):
        sub = s.layout
        ext = (sub.source_nodes == 0) & (sub.source_points == 0)
        assert set(sub.source_ids[ext].tolist()) == set(s.external_source)
        assert set(s.external_source) <= detector_sids
        assert not set(s.external_source) & set(s.detector_sids.tolist())
        for sid, local in s.external_source.items():
            assert sub.source_ids[local - 1] == sid
        # parents stay inside the shard and before their children
        parent = np.asarray(sub.parent)
        assert np.all(parent < np.arange(1, sub.n_nodes + 1))
    # voltages, geometry and the node map agree
    s0 = shards[1]
    cell = int(s0.cells[0])
    node = layout.voltage_node(cell + 1)
    local = int(s0.node_map[node])
    assert local > 0
    assert s0.layout.area[local - 1] == layout.area[node - 1]
    assert s0.layout.axial_diagonal[local - 1] == layout.axial_diagonal[node - 1]


def test_external_spike_input_in_layout():
    model = netcases.strong_config1(n_cells=2)
    ext = mb.register_spike_source(model)
    first_syn = 1
    mb.connect(ext, mb.PointProcess(model, first_syn), weight=0.01, delay=1.5)
    layout = mb.build(model)
    k = ext.index - 1
    assert layout.source_nodes[k] == 0 and layout.source_points[k] == 0
    assert layout.fanout_offsets[k + 1] - layout.fanout_offsets[k] == 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(os.path.dirname(here), "mind.jl_b200")]
    import torch.distributed as dist
    from mind_b200 import sharding as sh

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sids = np.arange(rank * 10, rank * 10 + 3 * rank, dtype=np.int64)   # rank 0 sends nothing
    times = sids * 0.5 + 0.1
    all_s, all_t = sh.exchange_spikes(sids, times)
    window = sh.global_window(20 + 5 * rank)
    out[rank] = (all_s.tolist(), all_t.tolist(), window)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_exchange_variable_length_spike_lists():
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    want_s = [10, 11, 12]
    want_t = [s * 0.5 + 0.1 for s in want_s]
    for r in range(world):
        assert out[r][0] == want_s
        assert out[r][1] == want_t
        assert out[r][2] == 20


def test_exchange_maps_pair_every_crossing_netcon_with_a_detector():
    """The maps of the device exchange (mind_attach_exchange): each shard's packed sids are
    its own detectors, every sid it receives is a detector of the other shard, and the
    external source a received sid enters through is the one whose NetCons carry it."""
    layout = mb.build(netcases.recurrent_trees())
    owners = sharding.partition_cells(layout, 2)
    shards = [sharding.shard_layout(layout, np.nonzero(owners == r)[0]) for r in range(2)]
    maps = [sharding.exchange_maps(sh) for sh in shards]
    for r, (sh, (det_src, det_sid, ext_sid, ext_src)) in enumerate(zip(shards, maps)):
        nodes = np.asarray(sh.layout.source_nodes)
        assert np.all(nodes[det_src] > 0)                          # detectors of this shard
        assert set(det_sid.tolist()) == set(np.asarray(sh.detector_sids).tolist())
        other_det = set(maps[1 - r][1].tolist())
        assert len(ext_sid) > 0 and set(ext_sid.tolist()) <= other_det
        ids = np.asarray(sh.layout.source_ids)
        np.testing.assert_array_equal(ids[ext_src], ext_sid)       # the source carries that sid
        assert np.all(np.asarray(sh.layout.source_points)[ext_src] == 0) and np.all(nodes[ext_src] == 0)
        assert np.all(np.diff(ext_sid) > 0)
