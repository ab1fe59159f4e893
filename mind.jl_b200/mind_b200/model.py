"""Micro model builders: populations, mechanisms, point processes, sources, NetCons.

Mirrors MIND.jl's construction API (src/model/micro/model.jl:91-400,
src/model/micro/utils/model.jl:72-260) with Python names: `add_population!`
becomes `add_population`, `insert!` becomes `insert`, and so on.  Argument
meaning, defaults and validation follow the reference; the builders only record
what the user asked for, and `build` packs it (src/model/build.jl:120-220).

Point processes and connections are stored in columnar chunks so that the
bulk builders used for networks of millions of synapses stay cheap; the
scalar builders append chunks of one.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence, Union

import numpy as np

from .mechanisms import Mechanism, resolve_mechanism
from .morphology import Section, discretize, MorphologyLayout


# Gas constant and Faraday constant, mV/mM units (src/model/micro/utils/biophysics.jl:47-48)
_GAS_CONSTANT = 1.380649e-23 * 6.02214076e23
_FARADAY = 1.602176634e-19 * 6.02214076e23


def _validate_ion_arguments(internal, external, valence, celsius) -> None:
    if not (all(math.isfinite(x) for x in (internal, external, valence, celsius)) and internal >= 0
            and external >= 0 and celsius > -273.15):
        raise ValueError("invalid ion arguments")


def nernst_potential(internal: float, external: float, valence: float, celsius: float) -> float:
    """Reversal potential (mV) of concentrations in mM, with the reference's limits: 0 for
    valence 0, +1e6 for no internal and -1e6 for no external concentration
    (src/model/micro/utils/biophysics.jl:43-51; the same operation order)."""
    if valence == 0.0:
        return 0.0
    if internal <= 0.0:
        return 1.0e6
    if external <= 0.0:
        return -1.0e6
    return (1000.0 * _GAS_CONSTANT * (celsius + 273.15) / _FARADAY) / valence * math.log(external / internal)


def nernst(internal: float, external: float, valence: float, *, celsius: float = 6.3) -> float:
    """nernst (src/model/micro/biophysics.jl:53-61): validated nernst_potential."""
    _validate_ion_arguments(internal, external, valence, celsius)
    return nernst_potential(float(internal), float(external), float(valence), float(celsius))


def ghk(voltage: float, internal: float, external: float, valence: float, *, celsius: float = 6.3) -> float:
    """Goldman-Hodgkin-Katz current factor in NEURON's mV and mM conventions, with its
    small-argument branch (src/model/micro/biophysics.jl:63-74,
    src/model/micro/utils/biophysics.jl:53-70)."""
    _validate_ion_arguments(internal, external, valence, celsius)
    if not math.isfinite(voltage):
        raise ValueError("voltage must be finite")
    thermal_voltage = 1000.0 * _GAS_CONSTANT * (float(celsius) + 273.15) / _FARADAY
    scaled = float(valence) * float(voltage) / thermal_voltage

    def quotient(x):
        return 1.0 - x / 2.0 if abs(x) < 1.0e-4 else x / (math.exp(x) - 1.0)

    return 0.001 * float(valence) * _FARADAY * (float(internal) * quotient(-scaled) - float(external) * quotient(scaled))


@dataclass(frozen=True)
class IonSpecies:
    """Ion species defaults (src/model/micro/utils/biophysics.jl:31-41).  With nernst=True the
    species' reversal potential is the Nernst potential of its concentrations at the model's
    temperature (src/model/micro/model.jl:766-768); concentrations stay at these values,
    since no mechanism here writes them, so that reversal holds for the whole run."""

    name: str
    valence: int
    internal: float
    external: float
    reversal: float = 0.0
    nernst: bool = False

    def __post_init__(self):
        if not math.isfinite(self.valence):
            raise ValueError("ion valence must be finite")
        if not all(math.isfinite(x) for x in (self.internal, self.external, self.reversal)):
            raise ValueError("non-finite ion parameter")
        if self.internal < 0 or self.external < 0:
            raise ValueError("ion concentrations must be nonnegative")

    def reversal_at(self, celsius: float) -> float:
        """The reversal a mechanism's USEION READ e<ion> sees on a node without an override."""
        if self.nernst:
            return nernst_potential(float(self.internal), float(self.external), float(self.valence), float(celsius))
        return self.reversal


def default_ions() -> Dict[str, IonSpecies]:
    return {
        "na": IonSpecies("na", 1, 10.0, 140.0, 50.0),
        "k": IonSpecies("k", 1, 54.4, 2.5, -77.0),
        "ca": IonSpecies("ca", 2, 5.0e-5, 2.0, 132.4579341637009),
    }


@dataclass
class DensityBinding:
    mechanism: Mechanism
    sections: List[str]
    params: Dict[str, Any]


@dataclass
class CellInstance:
    morphology: int
    gid: int
    voltage: float
    section_voltages: Dict[str, float]
    bindings: List[DensityBinding] = field(default_factory=list)
    ions: Dict[str, float] = field(default_factory=dict)  # reversal overrides, e.g. {"ena": 55.0}


@dataclass
class PointChunk:
    """`count` point processes of one mechanism; scalars or per-point arrays."""

    mechanism: Mechanism
    first: int                 # 1-based point index of the first member
    count: int
    cells: np.ndarray          # 1-based cell index, 0 for artificial cells
    sections: Union[str, Sequence[str]]
    xs: np.ndarray
    params: Dict[str, Any]
    spike_times: Optional[List[np.ndarray]] = None   # PatternStim: each member's firing times (ms)


@dataclass
class SourceChunk:
    """Spike sources: voltage detectors (cell > 0) or point net_event sources (point > 0)."""

    first: int                 # 1-based source index of the first member
    sids: np.ndarray
    cells: np.ndarray          # 1-based cell, 0 for point sources
    sections: Union[str, Sequence[str]]
    xs: np.ndarray
    points: np.ndarray         # 1-based point, 0 for detectors
    thresholds: np.ndarray


@dataclass
class ConnectionChunk:
    sources: np.ndarray        # 1-based source index
    targets: np.ndarray        # 1-based point index
    weights: np.ndarray
    delays: np.ndarray


class MicroModel:
    """A micro model: morphologies, cells, point processes, sources and NetCons."""

    def __init__(self, celsius: float = 6.3, ions: Sequence[IonSpecies] = ()):
        if not (math.isfinite(celsius) and celsius > -273.15):
            raise ValueError("invalid temperature")
        self.celsius = float(celsius)
        self.ions = default_ions()
        for ion in ions:
            self.ions[ion.name] = ion
        self.morphologies: List[List[Section]] = []
        self.morphology_layouts: List[Optional[MorphologyLayout]] = []
        self.cells: List[CellInstance] = []
        self.gids: set = set()
        self.point_chunks: List[PointChunk] = []
        self.point_count = 0
        self.source_chunks: List[SourceChunk] = []
        self.source_count = 0
        self.source_ids: Dict[int, int] = {}
        self.point_sources: Dict[int, int] = {}
        self.detector_sources: Dict[tuple, int] = {}
        self.next_source_id = 0
        self.connection_chunks: List[ConnectionChunk] = []
        self.connection_count = 0
        # Set by build/initialize.
        self.layout = None
        self.state = None

    def morphology_layout(self, index: int) -> MorphologyLayout:
        layout = self.morphology_layouts[index]
        if layout is None:
            layout = discretize(self.morphologies[index])
            self.morphology_layouts[index] = layout
        return layout


@dataclass(frozen=True)
class Cell:
    model: MicroModel
    index: int  # 1-based
    gid: int


class Population(list):
    """A fixed range of cells in one model."""


@dataclass(frozen=True)
class PointProcess:
    model: MicroModel
    index: int  # 1-based


@dataclass(frozen=True)
class SpikeSource:
    model: MicroModel
    index: int  # 1-based
    sid: int


def add_population(model: MicroModel, sections: Sequence[Section], count: int, *,
                   first_gid: Optional[int] = None, voltage=-65.0) -> Population:
    """Create `count` cells sharing one morphology (micro/model.jl:217-284)."""
    if count < 0:
        raise ValueError("population size must be nonnegative")
    if count == 0:
        return Population()
    model.morphologies.append([Section(**vars(s)) if isinstance(s, Section) else s for s in sections])
    model.morphology_layouts.append(None)
    morphology = len(model.morphologies) - 1
    names = {s.name: s for s in model.morphologies[morphology]}
    first_gid = len(model.cells) if first_gid is None else int(first_gid)
    population = Population()
    for k in range(count):
        gid = first_gid + k
        if gid in model.gids:
            raise ValueError(f"duplicate cell gid {gid}")
        value = voltage(k + 1) if callable(voltage) else voltage
        section_voltages: Dict[str, float] = {}
        if isinstance(value, dict):
            base = float(value.get("all", -65.0))
            for selector, v in value.items():
                if selector == "all":
                    continue
                if not math.isfinite(v):
                    raise ValueError("non-finite initial voltage")
                for name in _select_sections(model.morphologies[morphology], selector):
                    section_voltages[name] = float(v)
        else:
            base = float(value)
        if not math.isfinite(base):
            raise ValueError("non-finite initial voltage")
        model.cells.append(CellInstance(morphology, gid, base, section_voltages))
        model.gids.add(gid)
        population.append(Cell(model, len(model.cells), gid))
    del names
    return population


def _select_sections(morphology: Sequence[Section], selectors) -> List[str]:
    if isinstance(selectors, str):
        names = [selectors]
    else:
        names = [str(s) for s in selectors]
    if "all" in names:
        return [s.name for s in morphology]
    out = []
    for name in names:
        explicit = any(s.name == name for s in morphology)
        hits = [s.name for s in morphology if (s.name if explicit else s.label) == name]
        if not hits:
            raise ValueError(f"unknown section group {name}")
        for h in hits:
            if h not in out:
                out.append(h)
    return out


def insert(cell: Cell, mechanism, *, sections="all", params: Optional[Dict[str, Any]] = None) -> Cell:
    """Insert a density mechanism where absent (micro/model.jl:153-170)."""
    model = cell.model
    instance = model.cells[cell.index - 1]
    compiled = resolve_mechanism(mechanism)
    if compiled.kind != "density":
        raise ValueError("cell insertion requires a distributed micro mechanism")
    selected = _select_sections(model.morphologies[instance.morphology], sections)
    for binding in instance.bindings:
        if binding.mechanism.name != compiled.name:
            continue
        existing = set(binding.sections)
        selected = [name for name in selected if name not in existing]
        if not selected:
            break
    params = dict(params or {})
    for name in params:
        compiled.field_index(name)
    if selected:
        instance.bindings.append(DensityBinding(compiled, selected, params))
    return cell


def add_pointprocess(target: Union[Cell, MicroModel], mechanism, *, section="soma", x=0.5,
                     params: Optional[Dict[str, Any]] = None, spike_times=()) -> PointProcess:
    """Create one point process on a cell, or one artificial cell on the model
    (add_pointprocess!, src/model/micro/model.jl:178-193); `spike_times` are the firing
    times of a PatternStim."""
    if isinstance(target, Cell):
        model, cell = target.model, target.index
    else:
        model, cell = target, 0
    first = add_pointprocesses(model, mechanism, np.array([cell]), section, np.array([float(x)]),
                               params or {}, spike_times=[spike_times])
    return PointProcess(model, first)


def add_pointprocesses(model: MicroModel, mechanism, cells, sections, xs,
                       params: Optional[Dict[str, Any]] = None, spike_times=None) -> int:
    """Bulk variant: len(cells) point processes; params values may be arrays; `spike_times`,
    one sequence per member, only for PatternStim.  Returns the first index."""
    compiled = resolve_mechanism(mechanism)
    cells = np.asarray(cells, dtype=np.int64).reshape(-1)
    xs = np.asarray(xs, dtype=np.float64).reshape(-1)
    if len(xs) == 1 and len(cells) > 1:
        xs = np.full(len(cells), xs[0])
    if compiled.kind not in ("point", "artificial"):
        raise ValueError("expected micro point process or artificial cell")
    if compiled.kind == "point" and np.any(cells == 0):
        raise ValueError("point process requires a cell")
    if np.any((xs < 0.0) | (xs > 1.0)):
        raise ValueError("point location must be in [0, 1]")
    params = dict(params or {})
    for name, value in params.items():
        compiled.field_index(name)
        arr = np.asarray(value, dtype=np.float64)
        if not np.all(np.isfinite(arr)):
            raise ValueError(f"non-finite value for {name}")
    times = None
    if spike_times is not None and any(len(t) for t in spike_times):
        if compiled.name != "PatternStim":
            raise ValueError("spike_times applies to PatternStim only")
        if len(spike_times) != len(cells):
            raise ValueError("one spike_times sequence per point")
        times = [np.asarray(t, dtype=np.float64).reshape(-1) for t in spike_times]
        if any(np.any(~np.isfinite(t) | (t < 0.0)) for t in times):
            raise ValueError("PatternStim spike times must be finite and >= 0")
    first = model.point_count + 1
    model.point_chunks.append(PointChunk(compiled, first, len(cells), cells, sections, xs, params, times))
    model.point_count += len(cells)
    return first


def _new_sid(model: MicroModel, sid: Optional[int]) -> int:
    identity = model.next_source_id if sid is None else int(sid)
    if identity < 0:
        raise ValueError("spike-source IDs must be nonnegative")
    if identity in model.source_ids:
        raise ValueError(f"duplicate spike-source ID {identity}")
    return identity


def register_spike_source(source: Union[Cell, PointProcess, "MicroModel"], *, sid: Optional[int] = None,
                          section="soma", x=0.5, threshold: Optional[float] = None) -> SpikeSource:
    """Register a cell's voltage detector, a point process's net_event output, or (given the
    model itself) an external spike input that only `inject_spike` drives.

    Defaults follow micro/model.jl:286-371: detectors at soma(0.5) with threshold
    10 mV; a point source reuses one registration for all its connections.
    """
    if isinstance(source, MicroModel):
        identity = _new_sid(source, sid)
        index = _append_sources(source, np.array([identity]), np.array([0]), "none", np.array([0.0]),
                                np.array([0]), np.array([0.0]))
        return SpikeSource(source, index, identity)
    if isinstance(source, PointProcess):
        model = source.model
        existing = model.point_sources.get(source.index)
        if existing:
            return SpikeSource(model, existing, _source_sid(model, existing))
        identity = _new_sid(model, sid)
        index = _append_sources(model, np.array([identity]), np.array([0]), "none",
                                np.array([0.0]), np.array([source.index]),
                                np.array([10.0 if threshold is None else float(threshold)]))
        model.point_sources[source.index] = index
        return SpikeSource(model, index, identity)
    model = source.model
    if not 0.0 <= x <= 1.0:
        raise ValueError("invalid spike detector")
    thr = 10.0 if threshold is None else float(threshold)
    if not math.isfinite(thr):
        raise ValueError("invalid spike detector")
    key = (source.index, str(section), float(x))
    existing = model.detector_sources.get(key)
    if existing:
        return SpikeSource(model, existing, _source_sid(model, existing))
    identity = _new_sid(model, sid)
    index = _append_sources(model, np.array([identity]), np.array([source.index]), str(section),
                            np.array([float(x)]), np.array([0]), np.array([thr]))
    model.detector_sources[key] = index
    return SpikeSource(model, index, identity)


def register_external_sources(model: MicroModel, count: int) -> np.ndarray:
    """Bulk register_spike_source!(model): `count` external spike inputs; returns their indices."""
    ids = np.arange(model.next_source_id, model.next_source_id + int(count), dtype=np.int64)
    first = _append_sources(model, ids, np.zeros(len(ids), np.int64), "none", np.zeros(len(ids)),
                            np.zeros(len(ids), np.int64), np.zeros(len(ids)))
    return np.arange(first, first + len(ids), dtype=np.int64)


def register_point_sources(model: MicroModel, points, sids=None) -> np.ndarray:
    """Bulk: register net_event sources for 1-based point indices; returns source indices.

    `sids` optionally fixes the source ids of newly registered points (they must be unused).
    """
    points = np.asarray(points, dtype=np.int64).reshape(-1)
    out = np.empty(len(points), dtype=np.int64)
    fresh = []
    for j, p in enumerate(points):
        existing = model.point_sources.get(int(p))
        if existing:
            out[j] = existing
        else:
            fresh.append(j)
    if fresh:
        if sids is not None:
            ids = np.asarray(sids, dtype=np.int64).reshape(-1)[fresh]
            if any(int(i) in model.source_ids for i in ids):
                raise ValueError("source id already in use")
        else:
            ids = np.arange(model.next_source_id, model.next_source_id + len(fresh), dtype=np.int64)
        first = _append_sources(model, ids, np.zeros(len(fresh), np.int64), "none",
                                np.zeros(len(fresh)), points[fresh], np.full(len(fresh), 10.0))
        for k, j in enumerate(fresh):
            model.point_sources[int(points[j])] = first + k
            out[j] = first + k
    return out


def _append_sources(model, sids, cells, sections, xs, points, thresholds) -> int:
    first = model.source_count + 1
    model.source_chunks.append(SourceChunk(first, np.asarray(sids, np.int64), np.asarray(cells, np.int64),
                                           sections, np.asarray(xs, np.float64),
                                           np.asarray(points, np.int64), np.asarray(thresholds, np.float64)))
    for k, sid in enumerate(np.asarray(sids).tolist()):
        model.source_ids[int(sid)] = first + k
        model.next_source_id = max(model.next_source_id, int(sid) + 1)
    model.source_count += len(sids)
    return first


def _source_sid(model: MicroModel, index: int) -> int:
    for chunk in model.source_chunks:
        if chunk.first <= index < chunk.first + len(chunk.sids):
            return int(chunk.sids[index - chunk.first])
    raise KeyError(index)


def spike_source(model: MicroModel, sid: int) -> SpikeSource:
    return SpikeSource(model, model.source_ids[int(sid)], int(sid))


def _point_mechanism(model: MicroModel, point: int) -> Mechanism:
    for chunk in model.point_chunks:
        if chunk.first <= point < chunk.first + chunk.count:
            return chunk.mechanism
    raise ValueError(f"unknown point process {point}")


def connect(source: Union[SpikeSource, PointProcess], target: PointProcess, *, weight=1.0,
            delay=0.0) -> int:
    """Connect a source to a point process with NET_RECEIVE (micro/model.jl:379-400)."""
    model = source.model
    if target.model is not model:
        raise ValueError("connection endpoints belong to different micro models")
    mechanism = _point_mechanism(model, target.index)
    if not mechanism.has_net_receive:
        raise ValueError("target has no NET_RECEIVE block")
    if isinstance(source, PointProcess):
        source_index = register_spike_source(source).index
    else:
        source_index = source.index
    return connect_many(model, np.array([source_index]), np.array([target.index]),
                        np.array([weight], dtype=np.float64), np.array([delay], dtype=np.float64))


def connect_many(model: MicroModel, sources, targets, weights, delays) -> int:
    """Bulk NetCons from 1-based source indices to 1-based points. Returns the last index."""
    sources = np.asarray(sources, dtype=np.int64).reshape(-1)
    targets = np.asarray(targets, dtype=np.int64).reshape(-1)
    weights = np.asarray(weights, dtype=np.float64).reshape(-1)
    delays = np.asarray(delays, dtype=np.float64).reshape(-1)
    if not (len(sources) == len(targets) == len(weights) == len(delays)):
        raise ValueError("connection arrays differ in length")
    if not (np.all(np.isfinite(weights)) and np.all(np.isfinite(delays)) and np.all(delays >= 0.0)):
        raise ValueError("invalid connection weight or delay")
    if np.any((sources < 1) | (sources > model.source_count)):
        raise ValueError("unknown spike source")
    if np.any((targets < 1) | (targets > model.point_count)):
        raise ValueError("unknown target point process")
    model.connection_chunks.append(ConnectionChunk(sources, targets, weights, delays))
    model.connection_count += len(sources)
    return model.connection_count
