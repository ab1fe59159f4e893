"""Sections and their discretization into the cable node tree.

Mirrors MIND.jl's Section/discretize (src/model/micro/morphology.jl:36-79,
406-484; src/model/micro/utils/morphology.jl:1-119).  Discretization produces,
per morphology:

* a root node for every root section (area 100 um2, no capacitance, no axial),
* nseg segment nodes per section whose area, axial conductance to the parent
  and capacitance integrate the section geometry over half segments,
* one zero-capacitance endpoint per section at its x=1 end, which is where
  child sections attach.

Every parent is numbered before its children.  The geometry integration follows
the reference's half-compartment walk over pt3d spans step for step, because
the packed coefficients feed an FP64 solve whose results are compared bit for
bit; sections given by length and diameter are evaluated for all their
half-segments at once with the same floating-point operations.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

HALF_PI = 0.5 * math.pi


@dataclass(frozen=True)
class Point3D:
    """A morphology sample in micrometres."""

    x: float
    y: float
    z: float
    diameter: float

    def __post_init__(self):
        values = (self.x, self.y, self.z, self.diameter)
        if not all(math.isfinite(v) for v in values):
            raise ValueError("non-finite morphology coordinate")
        if self.diameter < 0.0:
            raise ValueError("sample diameter must be nonnegative")


@dataclass
class Section:
    """One unbranched cable section (L, diam in um; Ra in ohm cm; cm in uF/cm2).

    The section's `child_x` end (0 or 1) attaches at `parent_x` of `parent`.
    """

    name: str
    label: str = "dend"
    parent: Optional[str] = None
    parent_x: float = 1.0
    child_x: float = 0.0
    nseg: int = 1
    length: float = 100.0
    diameter: float = 1.0
    points: List[Point3D] = field(default_factory=list)
    Ra: float = 100.0
    cm: float = 1.0

    def __post_init__(self):
        self.name = str(self.name)
        self.label = str(self.label)
        self.parent = None if self.parent is None else str(self.parent)
        if len(self.points) >= 2:
            total = 0.0
            for left, right in zip(self.points[:-1], self.points[1:]):
                dx, dy, dz = right.x - left.x, right.y - left.y, right.z - left.z
                total += math.sqrt(dx * dx + dy * dy + dz * dz)
            self.length = total
            self.diameter = self.points[0].diameter
        if not (isinstance(self.nseg, (int, np.integer)) and self.nseg > 0):
            raise ValueError("nseg must be a positive integer")
        self.nseg = int(self.nseg)
        if not 0.0 <= self.parent_x <= 1.0:
            raise ValueError("parent_x must be in [0, 1]")
        if self.child_x not in (0, 1, 0.0, 1.0):
            raise ValueError("child_x must be 0 or 1")
        values = (self.length, self.diameter, self.Ra, self.cm, self.parent_x)
        if not all(math.isfinite(float(v)) for v in values):
            raise ValueError("non-finite section parameter")
        if not (self.length > 0 and (self.diameter > 0 or (self.points and self.diameter == 0))
                and self.Ra > 0 and self.cm >= 0):
            raise ValueError("invalid section geometry or biophysics")
        self.length = float(self.length)
        self.diameter = float(self.diameter)
        self.Ra = float(self.Ra)
        self.cm = float(self.cm)
        self.parent_x = float(self.parent_x)
        self.child_x = float(self.child_x)


@dataclass
class MorphologyLayout:
    """Discretized node tree of one morphology (1-based node ids, parent 0 = none)."""

    parent: np.ndarray
    area: np.ndarray
    diameter: np.ndarray
    axial: np.ndarray
    capacitance: np.ndarray
    edge_length: np.ndarray
    section_nodes: Dict[str, np.ndarray]  # nseg segment nodes then the x=1 node
    section_starts: Dict[str, int]        # node at logical x=0

    @property
    def node_count(self) -> int:
        return len(self.parent)


def section_order(sections: Sequence[Section]) -> List[int]:
    """Parents before children, resolving each parent chain in input order."""
    names = {s.name: i for i, s in enumerate(sections)}
    if len(names) != len(sections):
        raise ValueError("duplicate section name")
    marks = [0] * len(sections)
    order: List[int] = []
    pending: List[int] = []
    for start in range(len(sections)):
        index = start
        while marks[index] != 2:
            if marks[index] == 1:
                raise ValueError("morphology contains a cycle")
            marks[index] = 1
            pending.append(index)
            parent = sections[index].parent
            if parent is None:
                break
            if parent not in names:
                raise ValueError(f"unknown parent section {parent}")
            index = names[parent]
        while pending:
            index = pending.pop()
            marks[index] = 2
            order.append(index)
    return order


def _integrate_geometry(points, arcs, boundary, Ra, cursor):
    """Area, axial resistance and diameter integral from the cursor to `boundary`."""
    area = 0.0
    resistance = 0.0
    diameter_integral = 0.0
    index, previous_arc, previous_diameter = cursor
    last = len(points) - 1
    while True:
        nxt = index + 1
        at_boundary = arcs[nxt] > boundary or nxt == last
        if at_boundary:
            span = arcs[nxt] - arcs[index]
            fraction = 1.0 if abs(span) < 1.0e-10 else (boundary - arcs[index]) / span
            arc = boundary
            diameter = (1.0 - fraction) * points[index].diameter + fraction * points[nxt].diameter
        else:
            arc, diameter = arcs[nxt], points[nxt].diameter
        delta = arc - previous_arc
        diameter_integral += (previous_diameter + diameter) * delta
        distance = max(delta, 1.0e-15)
        conductance = previous_diameter * diameter / distance
        resistance += 1.0 / (1.0e-15 if conductance == 0.0 else conductance)
        jump = diameter - previous_diameter
        area += (previous_diameter + diameter) * math.sqrt(distance * distance + 0.25 * (jump * jump))
        previous_arc, previous_diameter = arc, diameter
        if at_boundary:
            break
        index = nxt
    return (HALF_PI * area, ((0.04 * Ra) / math.pi) * resistance, 0.5 * diameter_integral,
            (index, previous_arc, previous_diameter))


def _section_points(section: Section):
    if len(section.points) >= 2:
        points = list(section.points)
    else:
        points = [Point3D(0.0, 0.0, 0.0, section.diameter),
                  Point3D(section.length, 0.0, 0.0, section.diameter)]
    arcs = [0.0]
    for left, right in zip(points[:-1], points[1:]):
        dx, dy, dz = right.x - left.x, right.y - left.y, right.z - left.z
        arcs.append(arcs[-1] + math.sqrt(dx * dx + dy * dy + dz * dz))
    if not arcs[-1] > 0.0:
        raise ValueError(f"section {section.name} has zero arc length")
    return points, arcs


def _segment_geometry_pt3d(section: Section):
    """Per-segment (area, diameter, axial, capacitance) and the endpoint axial, scalar walk."""
    points, arcs = _section_points(section)
    nseg = section.nseg
    step = arcs[-1] / nseg
    cursor = (0, arcs[0], points[0].diameter)
    previous_right = 0.0
    area = np.empty(nseg)
    diam = np.empty(nseg)
    axial = np.empty(nseg)
    cap = np.empty(nseg)
    for k in range(1, nseg + 1):
        middle = (k - 0.5) * step
        right = k * step
        al, rl, dl, cursor = _integrate_geometry(points, arcs, middle, section.Ra, cursor)
        ar, rr, dr, cursor = _integrate_geometry(points, arcs, right, section.Ra, cursor)
        node_area = al + ar
        area[k - 1] = node_area
        diam[k - 1] = (dl + dr) / step
        axial[k - 1] = 1.0 / (previous_right + rl)
        cap[k - 1] = section.cm * node_area * 1.0e-5
        previous_right = rr
    return area, diam, axial, cap, 1.0 / previous_right, step


def _segment_geometry_cylinders(lengths, diameters, nsegs, Ras, cms):
    """Vectorized half-segment walk for sections without pt3d samples.

    A two-sample section has one pt3d span, so every half-segment ends inside
    it; the operations are those of `_integrate_geometry` on that span.
    """
    lengths = np.asarray(lengths, dtype=np.float64)
    diameters = np.asarray(diameters, dtype=np.float64)
    nsegs = np.asarray(nsegs, dtype=np.int64)
    Ras = np.asarray(Ras, dtype=np.float64)
    cms = np.asarray(cms, dtype=np.float64)
    arc_end = np.sqrt(lengths * lengths + 0.0 * 0.0 + 0.0 * 0.0)
    step = arc_end / nsegs
    total = int(nsegs.sum())
    sec = np.repeat(np.arange(len(nsegs)), nsegs)
    first = np.concatenate(([0], np.cumsum(nsegs)[:-1]))
    ordinal = (np.arange(total) - np.repeat(first, nsegs) + 1).astype(np.float64)
    s_step = step[sec]
    s_arc = arc_end[sec]
    s_d = diameters[sec]
    s_Ra = Ras[sec]
    middle = (ordinal - 0.5) * s_step
    right = ordinal * s_step
    # Interleave boundaries: b[2j] = middle_j, b[2j+1] = right_j (per section).
    bounds = np.empty(2 * total)
    bounds[0::2] = middle
    bounds[1::2] = right
    b_arc = np.repeat(s_arc, 2)
    b_d = np.repeat(s_d, 2)
    b_Ra = np.repeat(s_Ra, 2)
    small = np.abs(b_arc) < 1.0e-10
    fraction = np.where(small, 1.0, bounds / np.where(small, 1.0, b_arc))
    diameter = (1.0 - fraction) * b_d + fraction * b_d
    # Previous boundary and diameter of each half; the first half of a section
    # starts at arc 0 with the first sample's diameter.
    prev_arc = np.empty_like(bounds)
    prev_arc[1:] = bounds[:-1]
    prev_d = np.empty_like(diameter)
    prev_d[1:] = diameter[:-1]
    starts = 2 * first
    prev_arc[starts] = 0.0
    prev_d[starts] = diameters
    delta = bounds - prev_arc
    diameter_integral = (prev_d + diameter) * delta
    distance = np.maximum(delta, 1.0e-15)
    conductance = prev_d * diameter / distance
    resistance = 1.0 / np.where(conductance == 0.0, 1.0e-15, conductance)
    jump = diameter - prev_d
    area_sum = (prev_d + diameter) * np.sqrt(distance * distance + 0.25 * (jump * jump))
    half_area = HALF_PI * area_sum
    half_res = ((0.04 * b_Ra) / math.pi) * resistance
    half_diam = 0.5 * diameter_integral
    al, ar = half_area[0::2], half_area[1::2]
    rl, rr = half_res[0::2], half_res[1::2]
    dl, dr = half_diam[0::2], half_diam[1::2]
    node_area = al + ar
    node_diam = (dl + dr) / s_step
    previous_right = np.empty(total)
    previous_right[1:] = rr[:-1]
    previous_right[first] = 0.0
    axial = 1.0 / (previous_right + rl)
    cap = cms[sec] * node_area * 1.0e-5
    last = first + nsegs - 1
    endpoint_axial = 1.0 / rr[last]
    return node_area, node_diam, axial, cap, endpoint_axial, step, first


def discretize(sections: Sequence[Section]) -> MorphologyLayout:
    """Discretize sections into the cable node tree (morphology.jl:406-484)."""
    sections = list(sections)
    order = section_order(sections)
    for s in sections:
        if not (s.nseg > 0 and math.isfinite(s.Ra) and s.Ra > 0 and math.isfinite(s.cm) and s.cm >= 0):
            raise ValueError(f"invalid segmentation or biophysics on section {s.name}")
    plain = [i for i in range(len(sections)) if len(sections[i].points) < 2]
    geometry = {}
    if plain:
        area, diam, axial, cap, end_axial, step, first = _segment_geometry_cylinders(
            [sections[i].length for i in plain], [sections[i].diameter for i in plain],
            [sections[i].nseg for i in plain], [sections[i].Ra for i in plain],
            [sections[i].cm for i in plain])
        for j, i in enumerate(plain):
            lo, hi = first[j], first[j] + sections[i].nseg
            geometry[i] = (area[lo:hi], diam[lo:hi], axial[lo:hi], cap[lo:hi], end_axial[j], step[j])
    for i in range(len(sections)):
        if i not in geometry:
            geometry[i] = _segment_geometry_pt3d(sections[i])

    total = sum(s.nseg + 1 for s in sections) + sum(1 for s in sections if s.parent is None)
    parent = np.zeros(total, dtype=np.int32)
    area = np.empty(total)
    diameter = np.empty(total)
    axial_c = np.empty(total)
    capacitance = np.empty(total)
    edge_length = np.empty(total)
    section_nodes: Dict[str, np.ndarray] = {}
    starts: Dict[str, int] = {}
    count = 0

    def add(parent_node, a, d, g, c, span):
        nonlocal count
        parent[count] = parent_node
        area[count] = a
        diameter[count] = d
        axial_c[count] = g
        capacitance[count] = c
        edge_length[count] = span
        count += 1
        return count

    def location(name, x):
        if x == 0.0:
            return starts[name]
        nodes = section_nodes[name]
        if x == 1.0:
            return int(nodes[-1])
        index = min(int(math.floor(x * (len(nodes) - 1))), len(nodes) - 2)
        return int(nodes[index])

    for index in order:
        s = sections[index]
        seg_area, seg_diam, seg_axial, seg_cap, end_axial, step = geometry[index]
        if s.parent is None:
            connection = add(0, 100.0, 0.0, 0.0, 0.0, 0.0)
        else:
            connection = location(s.parent, s.parent_x)
        nodes = np.empty(s.nseg + 1, dtype=np.int32)
        reversed_ = s.child_x == 1.0
        previous = connection
        base = count
        n = s.nseg
        parent[base:base + n] = np.arange(base, base + n, dtype=np.int32)
        parent[base] = previous
        area[base:base + n] = seg_area
        diameter[base:base + n] = seg_diam
        axial_c[base:base + n] = seg_axial
        capacitance[base:base + n] = seg_cap
        edge_length[base:base + n] = step
        edge_length[base] = 0.5 * step
        ids = np.arange(base + 1, base + n + 1, dtype=np.int32)
        count = base + n
        if reversed_:
            nodes[:n] = ids[::-1]
        else:
            nodes[:n] = ids
        endpoint = add(count, 100.0, 0.0, end_axial, 0.0, 0.5 * step)
        starts[s.name] = endpoint if reversed_ else connection
        nodes[n] = connection if reversed_ else endpoint
        section_nodes[s.name] = nodes
    assert count == total
    return MorphologyLayout(parent, area, diameter, axial_c, capacitance, edge_length,
                            section_nodes, starts)


def location_node(layout: MorphologyLayout, section: str, x: float) -> int:
    """1-based local node at (section, x): x=0 the start, x=1 the end, else its segment."""
    name = str(section)
    if name not in layout.section_nodes:
        raise ValueError(f"unknown section {name}")
    if not 0.0 <= x <= 1.0:
        raise ValueError("section location must be in [0, 1]")
    if x == 0.0:
        return int(layout.section_starts[name])
    nodes = layout.section_nodes[name]
    if x == 1.0:
        return int(nodes[-1])
    index = min(int(math.floor(x * (len(nodes) - 1))), len(nodes) - 2)
    return int(nodes[index])


def segment_nodes(layout: MorphologyLayout, section: str) -> np.ndarray:
    """The nseg segment nodes of a section in x order (1-based local ids)."""
    return layout.section_nodes[str(section)][:-1]
