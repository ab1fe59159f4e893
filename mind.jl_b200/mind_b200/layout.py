"""build: pack a micro model into the flat layout the C-ABI receives.

Mirrors `build!`/`pack_micro` (src/model/build.jl:120-220,
src/model/micro/model.jl:420-902) up to the point where the reference starts
its own GPU-specific permutation (DHS planning, micro/model.jl:906-1077): nodes
are numbered cell by cell in discretization order, which already puts every
parent before its children, and the device library derives its own per-cell
layout from this forest.

What is packed, in the reference's terms:
* node geometry (parent, area, capacitance, axial conductance, axial_diagonal,
  initial voltage) — axial_diagonal is the node's own axial conductance plus
  its children's, added in ascending child order (micro/model.jl:857-863);
* mechanism groups in order of first appearance, density bindings first, then
  point processes (micro/model.jl:480-530); rows of a group sorted by node,
  stably, artificial cells in creation order (micro/model.jl:535-550);
  random-stream identities: node for density rows, point index + node count for
  point rows (micro/model.jl:510-530);
* spike sources and the NetCon fanout CSR grouped by source in creation order
  (micro/model.jl:590-671).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import abi
from .mechanisms import Mechanism
from .morphology import MorphologyLayout


@dataclass
class GroupLayout:
    mechanism: Mechanism
    data: np.ndarray          # [rows, fields] float64, column-major semantics
    nodes: np.ndarray         # int32 1-based (0 for artificial)
    logical_ids: np.ndarray   # uint64

    @property
    def rows(self) -> int:
        return len(self.nodes)

    def column(self, name: str) -> np.ndarray:
        return self.data[:, self.mechanism.field_index(name)]


@dataclass
class Layout:
    """The packed micro layout (ModelLayout.micro) plus build settings."""

    parent: np.ndarray
    voltage: np.ndarray
    area: np.ndarray
    capacitance: np.ndarray
    axial: np.ndarray
    axial_diagonal: np.ndarray
    groups: List[GroupLayout]
    point_group: np.ndarray
    point_row: np.ndarray
    source_ids: np.ndarray
    source_nodes: np.ndarray
    source_thresholds: np.ndarray
    source_points: np.ndarray
    fanout_offsets: np.ndarray
    edge_targets: np.ndarray
    edge_delays: np.ndarray
    edge_weights: np.ndarray
    connection_edges: np.ndarray
    dt: float
    celsius: float
    seed: int
    event_capacity: int
    spike_capacity: int
    secondorder: int = 0
    # PatternStim firings sorted by time (stable, point order), micro/model.jl:586-613
    pattern_times: np.ndarray = field(default_factory=lambda: np.zeros(0))
    pattern_points: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    # Host-side maps for references (voltage_ref) and reporting.
    cell_offsets: np.ndarray = None
    cell_morphology: np.ndarray = None
    morphologies: List[MorphologyLayout] = field(default_factory=list)
    segment_count: int = 0
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_nodes(self) -> int:
        return len(self.parent)

    @property
    def n_cells(self) -> int:
        return len(self.cell_offsets) - 1

    def group(self, name: str) -> GroupLayout:
        for g in self.groups:
            if g.mechanism.name == name:
                return g
        raise KeyError(name)

    def voltage_node(self, cell: int, section: str = "soma", x: float = 0.5) -> int:
        """Global 1-based node of (section, x) on a 1-based cell (voltage_ref)."""
        from .morphology import location_node

        morph = self.morphologies[self.cell_morphology[cell - 1]]
        return int(self.cell_offsets[cell - 1]) + location_node(morph, section, x)

    def to_c(self) -> abi.MindLayout:
        """A MindLayout struct pointing into this layout's arrays (kept alive by self)."""
        keep = []

        def ptr(array, ctype):
            array = np.ascontiguousarray(array)
            keep.append(array)
            return array.ctypes.data_as(ctypes.POINTER(ctype))

        mechs = (abi.MindMechanism * max(1, len(self.groups)))()
        for i, g in enumerate(self.groups):
            data = np.asfortranarray(g.data, dtype=np.float64)
            keep.append(data)
            names = (ctypes.c_char_p * len(g.mechanism.fields))(*[f.encode() for f in g.mechanism.fields])
            keep.append(names)
            m = mechs[i]
            m.kind = g.mechanism.code
            m.n_fields = len(g.mechanism.fields)
            m.rows = g.rows
            m.data = data.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            m.field_names = ctypes.cast(names, ctypes.POINTER(ctypes.c_char_p))
            m.nodes = ptr(g.nodes.astype(np.int32), ctypes.c_int32)
            m.logical_ids = ptr(g.logical_ids.astype(np.uint64), ctypes.c_uint64)
            m.digest = g.mechanism.digest
        keep.append(mechs)
        c = abi.MindLayout()
        c.abi_version = abi.MIND_ABI_VERSION
        c.secondorder = self.secondorder
        c.n_nodes = self.n_nodes
        c.parent = ptr(self.parent.astype(np.int32), ctypes.c_int32)
        c.voltage = ptr(self.voltage, ctypes.c_double)
        c.area = ptr(self.area, ctypes.c_double)
        c.capacitance = ptr(self.capacitance, ctypes.c_double)
        c.axial = ptr(self.axial, ctypes.c_double)
        c.axial_diagonal = ptr(self.axial_diagonal, ctypes.c_double)
        c.n_mechanisms = len(self.groups)
        c.mechanisms = ctypes.cast(mechs, ctypes.POINTER(abi.MindMechanism))
        c.n_points = len(self.point_group)
        c.point_group = ptr(self.point_group.astype(np.int32), ctypes.c_int32)
        c.point_row = ptr(self.point_row.astype(np.int32), ctypes.c_int32)
        c.n_sources = len(self.source_ids)
        c.source_ids = ptr(self.source_ids.astype(np.int64), ctypes.c_int64)
        c.source_nodes = ptr(self.source_nodes.astype(np.int32), ctypes.c_int32)
        c.source_thresholds = ptr(self.source_thresholds, ctypes.c_double)
        c.source_points = ptr(self.source_points.astype(np.int32), ctypes.c_int32)
        c.n_edges = len(self.edge_targets)
        c.fanout_offsets = ptr(self.fanout_offsets.astype(np.int64), ctypes.c_int64)
        c.edge_targets = ptr(self.edge_targets.astype(np.int32), ctypes.c_int32)
        c.edge_delays = ptr(self.edge_delays, ctypes.c_double)
        c.edge_weights = ptr(self.edge_weights, ctypes.c_double)
        c.dt = self.dt
        c.celsius = self.celsius
        c.seed = self.seed
        c.event_capacity = self.event_capacity
        c.spike_capacity = self.spike_capacity
        c.n_pattern = len(self.pattern_times)
        c.pattern_times = ptr(np.asarray(self.pattern_times, dtype=np.float64), ctypes.c_double)
        c.pattern_points = ptr(np.asarray(self.pattern_points, dtype=np.int32), ctypes.c_int32)
        self._keep = keep
        return c


def _section_node_lists(morph: MorphologyLayout, names) -> np.ndarray:
    return np.concatenate([morph.section_nodes[n][:-1] for n in names]) if names else np.zeros(0, np.int32)


def build(model, *, dt_micro: float = 0.025, seed: int = 1, event_capacity: Optional[int] = None,
          spike_capacity: Optional[int] = None, secondorder: int = 0) -> Layout:
    """Pack the model (build!). The layout is also stored on model.layout."""
    dt = float(dt_micro)
    if not (math.isfinite(dt) and dt > 0.0):
        raise ValueError("dt_micro must be positive and finite")
    if seed < 0:
        raise ValueError("seed must be nonnegative")
    if secondorder not in (0, 1, 2):
        raise ValueError("secondorder must be 0, 1 or 2")

    # 1. Nodes, cell by cell in discretization order.
    n_cells = len(model.cells)
    morphs = [model.morphology_layout(i) for i in range(len(model.morphologies))]
    counts = np.array([morphs[c.morphology].node_count for c in model.cells], dtype=np.int64)
    offsets = np.zeros(n_cells + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    total = int(offsets[-1])
    if total >= 2**31 - 1:
        raise ValueError("packed node count exceeds Int32 range")
    parent = np.empty(total, dtype=np.int32)
    voltage = np.empty(total)
    area = np.empty(total)
    capacitance = np.empty(total)
    axial = np.empty(total)
    segment_count = 0
    cell_morph = np.array([c.morphology for c in model.cells], dtype=np.int64)
    for ci, cell in enumerate(model.cells):
        m = morphs[cell.morphology]
        lo, hi = offsets[ci], offsets[ci + 1]
        parent[lo:hi] = np.where(m.parent > 0, m.parent + lo, 0)
        area[lo:hi] = m.area
        capacitance[lo:hi] = m.capacitance
        axial[lo:hi] = m.axial
        voltage[lo:hi] = cell.voltage
        for name, value in cell.section_voltages.items():
            voltage[lo + m.section_nodes[name] - 1] = value
            for endpoint in (m.section_starts[name], m.section_nodes[name][-1]):
                if m.parent[endpoint - 1] == 0:
                    voltage[lo + endpoint - 1] = value
        segment_count += sum(len(v) - 1 for v in m.section_nodes.values())
    has_parent = parent > 0
    axial_diagonal = np.where(has_parent, axial, 0.0)
    children = np.nonzero(has_parent)[0]  # ascending child index
    np.add.at(axial_diagonal, parent[children] - 1, axial[children])

    # 2. Mechanism groups: density bindings first, then point processes.
    group_index: Dict[str, int] = {}
    group_mechs: List[Mechanism] = []

    def group_for(mech: Mechanism) -> int:
        if mech.name not in group_index:
            group_index[mech.name] = len(group_mechs)
            group_mechs.append(mech)
        return group_index[mech.name]

    density_rows: Dict[int, list] = {}
    for ci, cell in enumerate(model.cells):
        m = morphs[cell.morphology]
        for binding in cell.bindings:
            g = group_for(binding.mechanism)
            nodes = _section_node_lists(m, binding.sections) + offsets[ci]
            density_rows.setdefault(g, []).append((nodes, binding, ci))
    point_chunks_by_group: Dict[int, list] = {}
    for chunk in model.point_chunks:
        g = group_for(chunk.mechanism)
        point_chunks_by_group.setdefault(g, []).append(chunk)

    groups: List[GroupLayout] = []
    point_group = np.zeros(model.point_count, dtype=np.int32)
    point_row = np.zeros(model.point_count, dtype=np.int32)
    for g, mech in enumerate(group_mechs):
        nf = len(mech.fields)
        if mech.kind == "density":
            parts = density_rows.get(g, [])
            nodes = np.concatenate([p[0] for p in parts]).astype(np.int64)
            data = np.tile(np.asarray(mech.defaults, dtype=np.float64), (len(nodes), 1))
            cursor = 0
            for node_ids, binding, ci in parts:
                n = len(node_ids)
                for name, value in binding.params.items():
                    data[cursor:cursor + n, mech.field_index(name)] = value
                for fld, ion in mech.ion_reads:
                    override = model.cells[ci].ions.get(fld)
                    data[cursor:cursor + n, mech.field_index(fld)] = (
                        override if override is not None else model.ions[ion].reversal_at(model.celsius))
                cursor += n
            order = np.argsort(nodes, kind="stable")
            nodes = nodes[order]
            data = data[order]
            if len(nodes) and np.any(nodes[1:] == nodes[:-1]):
                raise ValueError(f"{mech.name} inserted twice on one node")
            groups.append(GroupLayout(mech, data, nodes.astype(np.int32), nodes.astype(np.uint64)))
        else:
            chunks = point_chunks_by_group[g]
            point_ids = np.concatenate([np.arange(c.first, c.first + c.count) for c in chunks])
            nodes = np.zeros(len(point_ids), dtype=np.int64)
            data = np.tile(np.asarray(mech.defaults, dtype=np.float64), (len(point_ids), 1))
            cursor = 0
            for c in chunks:
                if mech.kind == "point":
                    nodes[cursor:cursor + c.count] = _point_nodes(model, morphs, offsets, c)
                for name, value in c.params.items():
                    data[cursor:cursor + c.count, mech.field_index(name)] = value
                if mech.kind == "point" and mech.ion_reads:
                    # USEION READ e<ion>: the species' reversal, or the owning cell's own value
                    # (the reference loads these from the ion table before BREAKPOINT,
                    # src/runtime/cuda/micro.jl:436-438, so they take precedence over params)
                    cells = np.broadcast_to(np.asarray(c.cells, dtype=np.int64), (c.count,))
                    for fld, ion in mech.ion_reads:
                        col = np.full(c.count, model.ions[ion].reversal_at(model.celsius))
                        for ci in np.unique(cells[cells > 0]):
                            override = model.cells[int(ci) - 1].ions.get(fld)
                            if override is not None:
                                col[cells == ci] = override
                        data[cursor:cursor + c.count, mech.field_index(fld)] = col
                cursor += c.count
            if mech.kind == "point":
                order = np.argsort(nodes, kind="stable")
            else:
                order = np.arange(len(nodes))
            nodes = nodes[order]
            data = data[order]
            point_ids = point_ids[order]
            point_group[point_ids - 1] = g + 1
            point_row[point_ids - 1] = np.arange(1, len(point_ids) + 1)
            groups.append(GroupLayout(mech, data, nodes.astype(np.int32),
                                      (point_ids + total).astype(np.uint64)))

    # 3. Sources.
    n_src = model.source_count
    source_ids = np.zeros(n_src, dtype=np.int64)
    source_nodes = np.zeros(n_src, dtype=np.int32)
    source_points = np.zeros(n_src, dtype=np.int32)
    source_thresholds = np.zeros(n_src)
    for chunk in model.source_chunks:
        lo = chunk.first - 1
        n = len(chunk.sids)
        source_ids[lo:lo + n] = chunk.sids
        source_points[lo:lo + n] = chunk.points
        source_thresholds[lo:lo + n] = chunk.thresholds
        for k in range(n):
            cell = int(chunk.cells[k])
            if cell:
                section = chunk.sections if isinstance(chunk.sections, str) else chunk.sections[k]
                from .morphology import location_node
                m = morphs[model.cells[cell - 1].morphology]
                source_nodes[lo + k] = offsets[cell - 1] + location_node(m, section, float(chunk.xs[k]))

    # 4. NetCon fanout CSR grouped by source, creation order within a source.
    if model.connection_chunks:
        src = np.concatenate([c.sources for c in model.connection_chunks])
        tgt = np.concatenate([c.targets for c in model.connection_chunks])
        wts = np.concatenate([c.weights for c in model.connection_chunks])
        dly = np.concatenate([c.delays for c in model.connection_chunks])
    else:
        src = tgt = np.zeros(0, np.int64)
        wts = dly = np.zeros(0)
    order = np.argsort(src, kind="stable")
    fanout = np.ones(n_src + 1, dtype=np.int64)
    counts_src = np.bincount(src, minlength=n_src + 1)[1:] if len(src) else np.zeros(n_src, np.int64)
    fanout[1:] = 1 + np.cumsum(counts_src)
    connection_edges = np.empty(len(src), dtype=np.int64)
    connection_edges[order] = np.arange(1, len(src) + 1)

    # 5. PatternStim spike times, point order, then stably by time.
    p_times, p_points = [], []
    for chunk in model.point_chunks:
        if chunk.spike_times:
            for k, times in enumerate(chunk.spike_times):
                p_times.append(times)
                p_points.append(np.full(len(times), chunk.first + k, dtype=np.int32))
    pattern_times = np.concatenate(p_times) if p_times else np.zeros(0)
    pattern_points = np.concatenate(p_points) if p_points else np.zeros(0, np.int32)
    by_time = np.argsort(pattern_times, kind="stable")
    pattern_times, pattern_points = pattern_times[by_time], pattern_points[by_time]

    n_events = event_capacity if event_capacity is not None else 0
    n_spikes = spike_capacity if spike_capacity is not None else 0
    layout = Layout(
        parent=parent, voltage=voltage, area=area, capacitance=capacitance, axial=axial,
        axial_diagonal=axial_diagonal, groups=groups, point_group=point_group, point_row=point_row,
        source_ids=source_ids, source_nodes=source_nodes, source_thresholds=source_thresholds,
        source_points=source_points, fanout_offsets=fanout, edge_targets=tgt[order].astype(np.int32),
        edge_delays=dly[order].astype(np.float64), edge_weights=wts[order].astype(np.float64),
        connection_edges=connection_edges, dt=dt, celsius=model.celsius, seed=int(seed),
        event_capacity=int(n_events), spike_capacity=int(n_spikes), secondorder=int(secondorder),
        pattern_times=pattern_times, pattern_points=pattern_points,
        cell_offsets=offsets, cell_morphology=cell_morph, morphologies=morphs,
        segment_count=int(segment_count),
    )
    model.layout = layout
    model.state = None
    return layout


def _point_nodes(model, morphs, offsets, chunk) -> np.ndarray:
    """Global 1-based node of each point of a chunk (location_node per point)."""
    out = np.empty(chunk.count, dtype=np.int64)
    cells = chunk.cells
    xs = chunk.xs
    sections = chunk.sections
    single = isinstance(sections, str)
    boundaries = np.flatnonzero(np.diff(cells)) + 1
    starts = np.concatenate(([0], boundaries))
    ends = np.concatenate((boundaries, [len(cells)]))
    for lo, hi in zip(starts, ends):
        cell = int(cells[lo])
        m = morphs[model.cells[cell - 1].morphology]
        base = offsets[cell - 1]
        if single:
            nodes = m.section_nodes[sections]
            nseg = len(nodes) - 1
            x = xs[lo:hi]
            idx = np.minimum(np.floor(x * nseg).astype(np.int64), nseg - 1)
            local = nodes[idx].astype(np.int64)
            local = np.where(x == 0.0, m.section_starts[sections], local)
            local = np.where(x == 1.0, nodes[-1], local)
            out[lo:hi] = base + local
            continue
        # points on many sections of one cell: the same rule, point by point
        for k in range(lo, hi):
            name = str(sections[k])
            nodes = m.section_nodes[name]
            x = float(xs[k])
            if x == 0.0:
                local = m.section_starts[name]
            elif x == 1.0:
                local = nodes[-1]
            else:
                nseg = len(nodes) - 1
                local = nodes[min(int(math.floor(x * nseg)), nseg - 1)]
            out[k] = base + int(local)
    return out
