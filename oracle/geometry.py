"""numpy restatement of MIND.jl's discretize -- the checker of the library's mind_discretize.

TEST INFRASTRUCTURE: only tests/ import this module.  The product discretizes sections in
C++ (mind.jl_b200/csrc/planner.cpp, reached through mind_b200.morphology.discretize); this
file restates the same algorithm independently in numpy so the tests can require the two
to agree bit for bit:

* section order: parents first, each parent chain resolved in input order
  (src/model/micro/utils/morphology.jl:77-104);
* the half-compartment geometry walk over pt3d spans (utils/morphology.jl:28-63), and a
  vectorised form of the same operations for sections given by length and diameter;
* node numbering with a root node per root section and an x = 1 node per section
  (src/model/micro/morphology.jl:406-484).
"""
from __future__ import annotations

import math
import os
import sys
from typing import Dict, List, Sequence

import numpy as np

_PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mind.jl_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from mind_b200.morphology import MorphologyLayout, Point3D, Section  # noqa: E402

HALF_PI = 0.5 * math.pi


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
    """Discretize sections into the cable node tree (morphology.jl:406-484), in numpy."""
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
