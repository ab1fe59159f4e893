"""One network over several GPUs: cells partitioned across ranks, spikes exchanged per window.

Each rank simulates the cells it owns with their synapses and the NetStims that
drive them; a NetCon whose presynaptic cell lives on another rank enters the
rank's layout as an external spike input (a source with neither detector nor
point, as register_spike_source!(model; sid) makes in the reference).  Ranks
advance in windows of at most `mind_window_steps` steps, the shortest NetCon
delay out of a cell expressed in steps, so a spike detected in one window is
delivered in a later one.  After each window every rank all-gathers the
(sid, time) pairs of its cells' spikes (the counts first, then the padded
lists) and injects the ones it has inputs for through `mind_inject_spikes`
(inject_spike!, src/runtime/state.jl:637-659).  Event times are spike time plus
NetCon delay in FP64, and each target cell applies a bin's events in the
canonical (target, time, edge) order, so the sharded run reproduces the
single-GPU run bit for bit.

Two exchanges.  exchange="device" (the GPU path): the library holds an NCCL
communicator (mind_attach_exchange) and, inside mind_run, packs each window's
spikes on the device, all-gathers them on its own stream and enters the received
ones through the external inputs' NetCons; nothing crosses to the host between
windows.  exchange="host": the window's spikes come back with the run and are
all-gathered by torch.distributed (NCCL, or gloo on the CPU for the host-side
tests) and injected with mind_inject_spikes.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, Sequence

import numpy as np

from .layout import GroupLayout, Layout
from .runtime import DeviceState, RecordSpec, SimulationResult


def partition_cells(layout: Layout, world: int) -> np.ndarray:
    """Owner rank of every cell: contiguous blocks with about equal node counts."""
    nodes = np.diff(np.asarray(layout.cell_offsets, dtype=np.int64))
    prefix = np.cumsum(nodes) - nodes  # nodes before each cell
    total = max(int(nodes.sum()), 1)
    return np.minimum((prefix * world) // total, world - 1).astype(np.int64)


@dataclass
class Shard:
    """A rank's sub-layout and the maps between it and the whole network's layout."""

    layout: Layout
    cells: np.ndarray                 # 0-based global cells owned, ascending
    node_map: np.ndarray              # global 1-based node -> local 1-based node (0 = not here)
    detector_sids: np.ndarray         # sids of the owned cells' detectors
    external_source: Dict[int, int] = field(default_factory=dict)  # remote sid -> local 1-based source
    local_sids: np.ndarray = None     # sid of every local source (for the merged raster)


def shard_layout(layout: Layout, cells: Sequence[int]) -> Shard:
    """Sub-layout of `cells` (0-based): their nodes and rows, the NetStims driving them,
    their detectors, remote detectors as external inputs, and the NetCons into them.

    Orders are kept (nodes, rows, sources, edges) so that the device's canonical
    orders, which break ties by these indices, agree with the whole network's.
    """
    cells = np.asarray(sorted(int(c) for c in cells), dtype=np.int64)
    offsets = np.asarray(layout.cell_offsets, dtype=np.int64)
    n_all = layout.n_nodes
    node_map = np.zeros(n_all + 1, dtype=np.int64)
    own_nodes = np.concatenate([np.arange(offsets[c] + 1, offsets[c + 1] + 1) for c in cells]) \
        if len(cells) else np.zeros(0, np.int64)
    node_map[own_nodes] = np.arange(1, len(own_nodes) + 1)
    sel = own_nodes - 1

    parent = np.asarray(layout.parent, dtype=np.int64)[sel]
    parent = np.where(parent > 0, node_map[np.maximum(parent, 0)], 0).astype(np.int32)

    # Points of cell mechanisms on owned nodes are targets here.
    point_group = np.asarray(layout.point_group, dtype=np.int64)
    point_row = np.asarray(layout.point_row, dtype=np.int64)
    n_points = len(point_group)
    group_nodes = [np.asarray(g.nodes, dtype=np.int64) for g in layout.groups]
    artificial = [bool(len(nd)) and bool(np.all(nd == 0)) for nd in group_nodes]
    point_node = np.zeros(n_points, dtype=np.int64)
    for p in range(n_points):
        point_node[p] = group_nodes[point_group[p] - 1][point_row[p] - 1]
    own_target = (point_node > 0) & (node_map[point_node] > 0)

    fan = np.asarray(layout.fanout_offsets, dtype=np.int64) - 1
    targets = np.asarray(layout.edge_targets, dtype=np.int64) - 1   # 0-based points
    edge_here = own_target[targets] if len(targets) else np.zeros(0, bool)
    n_src = len(layout.source_ids)
    src_edges_here = np.array([edge_here[fan[s]:fan[s + 1]].any() for s in range(n_src)], dtype=bool)

    # NetStims (artificial points) are kept where they drive an owned target.
    source_points = np.asarray(layout.source_points, dtype=np.int64)
    source_nodes = np.asarray(layout.source_nodes, dtype=np.int64)
    keep_point = own_target.copy()
    for s in range(n_src):
        p = source_points[s]
        if p > 0 and artificial[point_group[p - 1] - 1] and src_edges_here[s]:
            keep_point[p - 1] = True

    groups = []
    row_maps = []
    for gi, g in enumerate(layout.groups):
        nodes = group_nodes[gi]
        if artificial[gi]:
            keep = np.zeros(len(nodes), dtype=bool)
            pts = np.nonzero((point_group == gi + 1) & keep_point)[0]
            keep[point_row[pts] - 1] = True
        else:
            keep = (nodes > 0) & (node_map[np.maximum(nodes, 0)] > 0)
        rows = np.nonzero(keep)[0]
        row_map = np.zeros(len(nodes) + 1, dtype=np.int64)
        row_map[rows + 1] = np.arange(1, len(rows) + 1)
        row_maps.append(row_map)
        new_nodes = np.where(nodes[rows] > 0, node_map[np.maximum(nodes[rows], 0)], 0).astype(np.int32)
        groups.append(GroupLayout(g.mechanism, np.ascontiguousarray(g.data[rows]), new_nodes,
                                  np.asarray(g.logical_ids)[rows].copy()))

    kept_points = np.nonzero(keep_point)[0]
    point_map = np.zeros(n_points + 1, dtype=np.int64)
    point_map[kept_points + 1] = np.arange(1, len(kept_points) + 1)
    new_point_group = point_group[kept_points].astype(np.int32)
    new_point_row = np.array([row_maps[point_group[p] - 1][point_row[p]] for p in kept_points], dtype=np.int32)

    # Sources: owned detectors, kept NetStims, and remote detectors / external inputs with
    # NetCons into owned targets (as external inputs).
    sids = np.asarray(layout.source_ids, dtype=np.int64)
    src_keep, src_node, src_point, src_thr, external = [], [], [], [], {}
    detector_sids = []
    for s in range(n_src):
        node, point = source_nodes[s], source_points[s]
        if node > 0 and node_map[node] > 0:
            src_keep.append(s); src_node.append(node_map[node]); src_point.append(0)
            detector_sids.append(sids[s])
        elif point > 0:
            if point_map[point] == 0:
                continue
            src_keep.append(s); src_node.append(0); src_point.append(point_map[point])
        elif src_edges_here[s]:
            src_keep.append(s); src_node.append(0); src_point.append(0)
            external[int(sids[s])] = len(src_keep)
        else:
            continue
        src_thr.append(layout.source_thresholds[s])

    edges = [np.nonzero(edge_here[fan[s]:fan[s + 1]])[0] + fan[s] for s in src_keep]
    counts = np.array([len(e) for e in edges], dtype=np.int64)
    fanout = np.ones(len(src_keep) + 1, dtype=np.int64)
    fanout[1:] = 1 + np.cumsum(counts)
    edges = np.concatenate(edges) if edges else np.zeros(0, np.int64)

    own_cells = cells
    new_offsets = np.zeros(len(own_cells) + 1, dtype=np.int64)
    new_offsets[1:] = np.cumsum(offsets[own_cells + 1] - offsets[own_cells])
    cell_morph = np.asarray(layout.cell_morphology)[own_cells]
    seg_per_morph = [sum(len(v) - 1 for v in m.section_nodes.values()) for m in layout.morphologies]
    segments = int(sum(seg_per_morph[int(m)] for m in cell_morph))

    sub = Layout(
        parent=parent, voltage=np.asarray(layout.voltage)[sel].copy(), area=np.asarray(layout.area)[sel].copy(),
        capacitance=np.asarray(layout.capacitance)[sel].copy(), axial=np.asarray(layout.axial)[sel].copy(),
        axial_diagonal=np.asarray(layout.axial_diagonal)[sel].copy(), groups=groups,
        point_group=new_point_group, point_row=new_point_row,
        source_ids=sids[src_keep].copy(), source_nodes=np.array(src_node, dtype=np.int32),
        source_thresholds=np.array(src_thr, dtype=np.float64), source_points=np.array(src_point, dtype=np.int32),
        fanout_offsets=fanout, edge_targets=point_map[targets[edges] + 1].astype(np.int32),
        edge_delays=np.asarray(layout.edge_delays)[edges].copy(),
        edge_weights=np.asarray(layout.edge_weights)[edges].copy(),
        connection_edges=np.zeros(0, np.int64), dt=layout.dt, celsius=layout.celsius, seed=layout.seed,
        event_capacity=layout.event_capacity, spike_capacity=layout.spike_capacity,
        secondorder=layout.secondorder, cell_offsets=new_offsets, cell_morphology=cell_morph,
        morphologies=layout.morphologies, segment_count=segments,
    )
    return Shard(sub, cells, node_map, np.array(detector_sids, dtype=np.int64), external, sids[src_keep].copy())


def local_shard(layout: Layout) -> Shard:
    """A rank's layout built directly for its cells (networks.config2(rank=, world=)): its
    external inputs already stand for the other ranks' cells."""
    sids = np.asarray(layout.source_ids, dtype=np.int64)
    nodes = np.asarray(layout.source_nodes)
    points = np.asarray(layout.source_points)
    external = {int(sids[k]): k + 1 for k in np.nonzero((nodes == 0) & (points == 0))[0]}
    return Shard(layout, np.arange(layout.n_cells), np.arange(layout.n_nodes + 1, dtype=np.int64),
                 sids[nodes > 0].copy(), external, sids.copy())


def exchange_maps(shard: Shard):
    """The maps of mind_attach_exchange: (0-based sources of the shard's detectors, their
    sids, the sids it receives, the 0-based external sources they enter through)."""
    local_sids = np.asarray(shard.local_sids, dtype=np.int64)
    det_src = np.nonzero(np.isin(local_sids, np.asarray(shard.detector_sids, dtype=np.int64)))[0]
    ext_sid = np.array(sorted(shard.external_source), dtype=np.int64)
    ext_src = np.array([shard.external_source[int(s)] - 1 for s in ext_sid], dtype=np.int64)
    return det_src, local_sids[det_src], ext_sid, ext_src


def exchange_spikes(sids: np.ndarray, times: np.ndarray, device="cpu"):
    """All-gather variable-length (sid, time) lists: counts first, then the padded lists."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    count = torch.tensor([len(sids)], dtype=torch.int64, device=device)
    counts = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(counts, count)
    counts = [int(c.item()) for c in counts]
    width = max(max(counts), 1)
    s = torch.zeros(width, dtype=torch.int64, device=device)
    t = torch.zeros(width, dtype=torch.float64, device=device)
    if len(sids):
        s[:len(sids)] = torch.as_tensor(np.asarray(sids, dtype=np.int64))
        t[:len(times)] = torch.as_tensor(np.asarray(times, dtype=np.float64))
    all_s = [torch.zeros(width, dtype=torch.int64, device=device) for _ in range(world)]
    all_t = [torch.zeros(width, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(all_s, s)
    dist.all_gather(all_t, t)
    out_s = np.concatenate([x[:n].cpu().numpy() for x, n in zip(all_s, counts)])
    out_t = np.concatenate([x[:n].cpu().numpy() for x, n in zip(all_t, counts)])
    return out_s, out_t


def global_window(steps: int, device="cpu") -> int:
    """The smallest window over ranks: every rank exchanges after the same steps."""
    import torch
    import torch.distributed as dist

    w = torch.tensor([int(steps)], dtype=torch.int64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.MIN)
    return int(w.item())


class ShardedRun:
    """This rank's part of a network partitioned over the process group's ranks."""

    def __init__(self, layout: Layout, rank: int, world: int, *, precision: str = "fp64", device="cpu",
                 owners: np.ndarray = None, local: bool = False, exchange: str = "host"):
        """`layout` is the whole network, partitioned here (by `owners` or partition_cells), or,
        with local=True, this rank's own part with external inputs for the other ranks' cells.
        exchange: "device" (NCCL inside the library; needs the GPU and libnccl) or "host"."""
        if exchange not in ("device", "host"):
            raise ValueError("exchange is 'device' or 'host'")
        if local:
            self.owners = None
            self.shard = local_shard(layout)
        else:
            self.owners = partition_cells(layout, world) if owners is None else np.asarray(owners)
            self.shard = shard_layout(layout, np.nonzero(self.owners == rank)[0])
        self.device = device
        self.dt = layout.dt
        self.state = DeviceState(self.shard.layout, precision)
        self.state.initialize()
        self.window = global_window(self.state.window_steps(), device)
        self._external_sids = np.array(sorted(self.shard.external_source), dtype=np.int64)
        self.launches = 0
        self.exchange = exchange
        if exchange == "device":
            self._attach_device_exchange(rank, world)

    def _attach_device_exchange(self, rank: int, world: int):
        import ctypes

        import torch
        import torch.distributed as dist

        from . import abi

        det_src, det_sid, ext_sid, ext_src = exchange_maps(self.shard)
        most = torch.tensor([len(det_src)], dtype=torch.int64, device=self.device)
        dist.all_reduce(most, op=dist.ReduceOp.MAX)
        # a cell spikes at most once in a window shorter than its refractory time; the
        # margin covers the rest, and a window with more spikes raises status 3
        width = int(most.item()) + 16
        ident = [None]
        if rank == 0:
            buf = (ctypes.c_uint8 * 128)()
            status = self.state.lib.mind_exchange_id(buf)
            if status != abi.MIND_OK:
                raise abi.MindError(status, "mind_exchange_id: no NCCL")
            ident = [bytes(buf)]
        dist.broadcast_object_list(ident, src=0)
        self.state.attach_exchange(ident[0], world, rank, self.window, width, det_src, det_sid, ext_sid, ext_src)

    def records(self, nodes: Sequence[int]):
        """RecordSpecs for global 1-based nodes of owned cells (named by the global node)."""
        specs = []
        for node in nodes:
            local = int(self.shard.node_map[int(node)])
            if local == 0:
                raise ValueError(f"node {node} is not on this rank")
            specs.append(RecordSpec(local, f"n{int(node)}"))
        return specs

    def run_steps(self, steps: int, records: Sequence[RecordSpec] = (), record_spikes: bool = True):
        """Advance `steps` steps in windows, exchanging cell spikes after each window.

        Returns this rank's result: its traces and the spikes of its own sources (remote
        inputs, which enter the local raster when injected, are left out).
        """
        if self.exchange == "device":   # the library exchanges after every window
            result = self.state.run_steps(steps, records, record_spikes)
            self.launches += self.state.run_stats().launches
            mine = ~np.isin(result.spike_sources, self._external_sids)
            result.spike_times = result.spike_times[mine]
            result.spike_sources = result.spike_sources[mine]
            return result
        traces = {r.name: [] for r in records}
        times, sids = [], []
        start = None
        done = 0
        device_ms = 0.0
        while done < steps:
            k = min(self.window, steps - done)
            result = self.state.run_steps(k, records, True)
            device_ms += result.device_ms
            self.launches += self.state.run_stats().launches
            if start is None:
                start = result.time[0]
            for r in records:
                traces[r.name].append(result.traces[r.name] if not traces[r.name] else result.traces[r.name][1:])
            mine = ~np.isin(result.spike_sources, self._external_sids)
            if record_spikes:
                times.append(result.spike_times[mine])
                sids.append(result.spike_sources[mine])
            cell = np.isin(result.spike_sources, self.shard.detector_sids)
            all_s, all_t = exchange_spikes(result.spike_sources[cell], result.spike_times[cell], self.device)
            local = [self.shard.external_source.get(int(s), 0) for s in all_s]
            want = np.array([x > 0 for x in local], dtype=bool)
            if want.any():
                self.state.inject_spikes(np.asarray(local, dtype=np.int64)[want], all_t[want])
            done += k
        n = steps + 1
        time = (np.arange(n, dtype=np.float64) * self.dt + (start if start is not None else 0.0))
        out = SimulationResult(time, {name: np.concatenate(v) if v else np.zeros(0) for name, v in traces.items()},
                               np.concatenate(times) if times else np.zeros(0),
                               np.concatenate(sids) if sids else np.zeros(0, np.int64), device_ms)
        order = np.lexsort((out.spike_sources, out.spike_times))
        out.spike_times = out.spike_times[order]
        out.spike_sources = out.spike_sources[order]
        return out

    def close(self):
        self.state.close()
