"""Sections and their discretization into the cable node tree.

Mirrors MIND.jl's Section/discretize (src/model/micro/morphology.jl:36-79,
406-484; src/model/micro/utils/morphology.jl:1-119).  Discretization produces,
per morphology:

* a root node for every root section (area 100 um2, no capacitance, no axial),
* nseg segment nodes per section whose area, axial conductance to the parent
  and capacitance integrate the section geometry over half segments,
* one zero-capacitance endpoint per section at its x=1 end, which is where
  child sections attach.

Every parent is numbered before its children.  The discretization itself runs in
the library's C++ planner (csrc/planner.cpp, mind_discretize), which follows the
reference's half-compartment walk over pt3d spans step for step, because the
packed coefficients feed an FP64 solve whose results are compared bit for bit;
oracle/geometry.py restates it in numpy as the tests' check.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np



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


def discretize(sections: Sequence[Section]) -> MorphologyLayout:
    """Discretize sections into the cable node tree (morphology.jl:406-484).

    The work runs in the library's C++ planner (mind_discretize): sections parents first,
    a root node per root section, nseg segment nodes integrating the geometry over half
    segments (pt3d spans, or one span of constant diameter), and an x = 1 node per section.
    """
    import ctypes

    from . import abi

    sections = list(sections)
    index = {s.name: i for i, s in enumerate(sections)}
    if len(index) != len(sections):
        raise ValueError("duplicate section name")
    specs = (abi.MindSection * max(1, len(sections)))()
    keep = []
    for i, s in enumerate(sections):
        if s.parent is not None and s.parent not in index:
            raise ValueError(f"unknown parent section {s.parent}")
        c = specs[i]
        c.parent = -1 if s.parent is None else index[s.parent]
        c.nseg = int(s.nseg)
        c.parent_x, c.child_x = float(s.parent_x), float(s.child_x)
        c.length, c.diameter, c.Ra, c.cm = float(s.length), float(s.diameter), float(s.Ra), float(s.cm)
        if len(s.points) >= 2:
            pts = np.ascontiguousarray([[p.x, p.y, p.z, p.diameter] for p in s.points], dtype=np.float64)
            keep.append(pts)
            c.n_points = len(s.points)
            c.points = pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        else:
            c.n_points = 0
    total = sum(s.nseg + 1 for s in sections) + sum(1 for s in sections if s.parent is None)
    parent = np.zeros(total, dtype=np.int32)
    arrays = [np.empty(total) for _ in range(5)]
    start, end, first = (np.zeros(max(1, len(sections)), dtype=np.int64) for _ in range(3))
    f64 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    i64 = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    out = abi.MindMorphology(0, parent.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), *[f64(a) for a in arrays],
                             i64(start), i64(end), i64(first))
    message = ctypes.create_string_buffer(256)
    status = abi.load_library().mind_discretize(specs, len(sections), total, ctypes.byref(out), message, 256)
    if status != abi.MIND_OK:
        raise ValueError(message.value.decode() or f"mind_discretize status {status}")
    area, diameter, axial, capacitance, edge_length = arrays
    section_nodes: Dict[str, np.ndarray] = {}
    starts: Dict[str, int] = {}
    for i, s in enumerate(sections):
        ids = np.arange(first[i], first[i] + s.nseg, dtype=np.int32)
        nodes = np.empty(s.nseg + 1, dtype=np.int32)
        nodes[:s.nseg] = ids[::-1] if s.child_x == 1.0 else ids
        nodes[s.nseg] = end[i]
        section_nodes[s.name] = nodes
        starts[s.name] = int(start[i])
    return MorphologyLayout(parent, area, diameter, axial, capacitance, edge_length, section_nodes, starts)


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
