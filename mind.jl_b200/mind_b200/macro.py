"""Cross-scale coupling: neural-mass regions driven by and driving the micro network.

Mirrors MIND.jl's macro side for the neural-mass configuration (advance_macro!,
src/runtime/step.jl:156-204; regions, edges with delays, micro input and output
groups, src/runtime/cuda/macro.jl): regions are Jansen-Rit masses advanced by RK4
every `dt_macro`; edges carry a region's output to another's input after an integer
number of macro steps; each input (an external spike input of the micro layout, with
its NetCons) fires as a Poisson process at `scale * output` Hz of its region; each
output (a cell's detector) adds its spikes to its region's rate bin, which feeds the
region's input one bin later.  The exact rules are stated with mind_attach_macro in
include/mindgpu.h; the library evaluates them on the device, the oracle on the CPU.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import abi

JANSEN_RIT = {"A": 3.25, "B": 22.0, "a": 100.0, "b": 50.0, "e0": 2.5, "r": 0.56, "v0": 6.0, "C": 135.0,
              "p0": 120.0}
PARAM_ORDER = ("A", "B", "a", "b", "e0", "r", "v0", "C", "p0")


@dataclass
class MacroModel:
    """Regions and their coupling to a built micro layout (sources are 1-based layout sources)."""

    dt_macro: float = 0.1
    bin_ms: float = 1.0
    params: List[List[float]] = field(default_factory=list)
    y0: List[List[float]] = field(default_factory=list)
    micro_gain: List[float] = field(default_factory=list)
    edges: List[tuple] = field(default_factory=list)        # (src, dst, gain, delay steps), 1-based
    inputs: List[tuple] = field(default_factory=list)       # (region, source, scale)
    outputs: List[tuple] = field(default_factory=list)      # (region, detector source)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_regions(self) -> int:
        return len(self.params)

    def add_region(self, *, micro_gain: float = 0.0, y0=None, **params) -> int:
        """A Jansen-Rit region (defaults: JANSEN_RIT); returns its 1-based index."""
        values = dict(JANSEN_RIT)
        values.update(params)
        self.params.append([float(values[k]) for k in PARAM_ORDER])
        self.y0.append([0.0] * 6 if y0 is None else [float(x) for x in y0])
        self.micro_gain.append(float(micro_gain))
        return self.n_regions

    def connect(self, src: int, dst: int, gain: float, delay_steps: int = 1) -> None:
        if delay_steps < 1:
            raise ValueError("region edges are delayed by at least one macro step")
        self.edges.append((int(src), int(dst), float(gain), int(delay_steps)))

    def add_inputs(self, region: int, sources, scale: float = 1.0) -> None:
        for s in np.asarray(sources, dtype=np.int64).reshape(-1):
            self.inputs.append((int(region), int(s), float(scale)))

    def add_outputs(self, region: int, sources) -> None:
        for s in np.asarray(sources, dtype=np.int64).reshape(-1):
            self.outputs.append((int(region), int(s)))

    def to_c(self) -> abi.MindMacroLayout:
        keep = []

        def ptr(values, dtype, ctype):
            a = np.ascontiguousarray(np.asarray(values, dtype=dtype).reshape(-1))
            if a.size == 0:
                a = np.zeros(1, dtype=dtype)
            keep.append(a)
            return a.ctypes.data_as(ctypes.POINTER(ctype))

        c = abi.MindMacroLayout()
        c.n_regions = self.n_regions
        c.params = ptr(self.params, np.float64, ctypes.c_double)
        c.y0 = ptr(self.y0, np.float64, ctypes.c_double)
        c.micro_gain = ptr(self.micro_gain, np.float64, ctypes.c_double)
        c.n_edges = len(self.edges)
        c.edge_src = ptr([x[0] for x in self.edges], np.int32, ctypes.c_int32)
        c.edge_dst = ptr([x[1] for x in self.edges], np.int32, ctypes.c_int32)
        c.edge_gain = ptr([x[2] for x in self.edges], np.float64, ctypes.c_double)
        c.edge_delay = ptr([x[3] for x in self.edges], np.int32, ctypes.c_int32)
        c.n_inputs = len(self.inputs)
        c.input_region = ptr([x[0] for x in self.inputs], np.int32, ctypes.c_int32)
        c.input_source = ptr([x[1] for x in self.inputs], np.int64, ctypes.c_int64)
        c.input_scale = ptr([x[2] for x in self.inputs], np.float64, ctypes.c_double)
        c.n_outputs = len(self.outputs)
        c.output_region = ptr([x[0] for x in self.outputs], np.int32, ctypes.c_int32)
        c.output_source = ptr([x[1] for x in self.outputs], np.int64, ctypes.c_int64)
        c.dt_macro = float(self.dt_macro)
        c.bin_ms = float(self.bin_ms)
        self._keep = keep
        return c
