"""initialize / run / step through libmindgpu.so (the reference's runtime seams).

Mirrors MIND.jl's runtime API (src/runtime/initialize.jl:256-429,
src/runtime/step.jl:4-86, src/runtime/recording.jl:1-295): `initialize`
uploads the built layout and runs INITIAL, `run` advances to an absolute stop
time that must be an integer number of steps away and returns a
SimulationResult with the recorded traces and the spike raster sorted by
(time, sid).  Every call goes through the C-ABI; nothing here computes.
"""
from __future__ import annotations

import ctypes
from collections.abc import Mapping
from dataclasses import dataclass, field
from typing import Dict, List, Sequence

import numpy as np

from . import abi


@dataclass(frozen=True)
class RecordSpec:
    """A recorded or read quantity: RecordSpec / VariableRef (src/model/references.jl:4-80).

    A voltage reference names a 1-based node; a mechanism reference a 1-based group, row and
    field (column of the group's data).  The fields a mechanism reference may name are the
    PARAMETER and STATE fields kept on the device (include/mindgpu.h, MindRecord)."""

    node: int  # voltage: global 1-based node
    name: str
    kind: int = abi.MIND_RECORD_VOLTAGE
    group: int = 0   # mechanism: 1-based group of the layout
    row: int = 0     # mechanism: 1-based row of that group
    field: int = 0   # mechanism: 1-based column of the group's data

    def to_c(self) -> abi.MindRecord:
        return abi.MindRecord(self.kind, self.node, self.group, self.row, self.field)


class TraceMap(Mapping):
    """The traces of a run by record name, each a row view of one [records, samples] array.

    The array is copied out of the device once; the name index is built on the first lookup,
    so a run recording thousands of quantities costs no per-record work until asked."""

    def __init__(self, names: Sequence[str], by_record: np.ndarray):
        self._names = list(names)
        self.by_record = by_record
        self._index = None

    def __getitem__(self, name):
        if self._index is None:
            self._index = {n: i for i, n in enumerate(self._names)}
        return self.by_record[self._index[name]]

    def __iter__(self):
        return iter(self._names)

    def __len__(self):
        return len(self._names)


@dataclass
class SimulationResult:
    time: np.ndarray
    traces: Mapping = field(default_factory=dict)
    spike_times: np.ndarray = field(default_factory=lambda: np.zeros(0))
    spike_sources: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    device_ms: float = 0.0
    macro_trace: np.ndarray = None   # [macro boundaries, regions] region outputs, when regions are attached
    drive: np.ndarray = None         # [bins, cells, 32] synaptic drive, when recording it


class DeviceState:
    """Owns one libmindgpu handle for a built layout."""

    def __init__(self, layout, precision: str = "fp64"):
        self.lib = abi.load_library()
        self.layout = layout
        self.c_layout = layout.to_c()
        handle = ctypes.c_void_p()
        status = self.lib.mind_create(ctypes.byref(self.c_layout), ctypes.byref(handle))
        if status != abi.MIND_OK:
            message = self.lib.mind_last_error(None)
            raise abi.MindError(status, message.decode() if message else "")
        self.handle = handle
        self.set_precision(precision)

    def attach_macro(self, macro) -> None:
        """mind_attach_macro: regions and coupling (mind_b200.macro.MacroModel); before initialize."""
        c = macro.to_c()
        abi.check(self.lib, self.handle, self.lib.mind_attach_macro(self.handle, ctypes.byref(c)))
        self.n_regions = macro.n_regions

    def attach_surrogate(self, mlp, surrogate_cells, drive_scale: float) -> None:
        """mind_attach_surrogate: `mlp` (mind_b200.surrogate.Mlp) stands in for the cells where
        surrogate_cells (one flag per cell) is true; regions must be attached; initialize follows."""
        mask = np.ascontiguousarray(np.asarray(surrogate_cells, dtype=bool).astype(np.uint8))
        if mask.size != self.layout.n_cells:
            raise ValueError("one flag per cell")
        abi.check(self.lib, self.handle, self.lib.mind_attach_surrogate(
            self.handle, mlp.handle, mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), float(drive_scale)))
        self._surrogate = mlp   # the network must outlive the handle's use of it

    def set_surrogate_cells(self, surrogate_cells) -> None:
        """mind_set_surrogate_cells: between runs, the cells (a subset of the attached ones)
        the surrogate stands in for; the others are simulated from their next step."""
        mask = np.ascontiguousarray(np.asarray(surrogate_cells, dtype=bool).astype(np.uint8))
        if mask.size != self.layout.n_cells:
            raise ValueError("one flag per cell")
        abi.check(self.lib, self.handle, self.lib.mind_set_surrogate_cells(
            self.handle, mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    def set_surrogate_offsets(self, offsets) -> None:
        """mind_set_surrogate_offsets: per-cell logit offsets of the surrogate's spike
        probability (calibration)."""
        v = np.ascontiguousarray(np.asarray(offsets, dtype=np.float32))
        if v.size != self.layout.n_cells:
            raise ValueError("one offset per cell")
        abi.check(self.lib, self.handle, self.lib.mind_set_surrogate_offsets(
            self.handle, v.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), v.size))

    def attach_exchange(self, nccl_id, world: int, rank: int, window: int, width: int, detector_sources,
                        detector_sids, external_sids, external_sources) -> None:
        """mind_attach_exchange: this handle's shard of a network over `world` ranks (0-based
        source indices; nccl_id None: the host drives the exchange with exchange_pack /
        exchange_inject)."""
        def i32(a):
            v = np.ascontiguousarray(np.asarray(a, dtype=np.int64))
            if v.size and (v.min() < -(1 << 31) or v.max() >= (1 << 31)):
                raise ValueError("sids and sources must fit in int32")
            return np.ascontiguousarray(v.astype(np.int32))
        ds, dd, es, eo = i32(detector_sources), i32(detector_sids), i32(external_sids), i32(external_sources)
        if ds.size != dd.size or es.size != eo.size:
            raise ValueError("one sid per detector and one source per received sid")
        idbuf = None
        if nccl_id is not None:
            idbuf = (ctypes.c_uint8 * 128).from_buffer_copy(bytes(nccl_id))
        p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        abi.check(self.lib, self.handle, self.lib.mind_attach_exchange(
            self.handle, idbuf, int(world), int(rank), int(window), int(width), p(ds), p(dd), ds.size,
            p(es), p(eo), es.size))

    def exchange_pack(self, send_ptr: int) -> None:
        """mind_exchange_pack into device memory at send_ptr (1 + 2 width int64)."""
        abi.check(self.lib, self.handle, self.lib.mind_exchange_pack(self.handle, ctypes.c_void_p(send_ptr)))

    def exchange_inject(self, recv_ptr: int) -> None:
        """mind_exchange_inject from device memory at recv_ptr (world blocks)."""
        abi.check(self.lib, self.handle, self.lib.mind_exchange_inject(self.handle, ctypes.c_void_p(recv_ptr)))

    def set_drive_recording(self, bin_ms: float) -> None:
        """mind_set_drive_recording: each run also returns the cells' binned synaptic drive."""
        abi.check(self.lib, self.handle, self.lib.mind_set_drive_recording(self.handle, float(bin_ms)))
        self.drive_on = bin_ms > 0

    def set_precision(self, precision: str) -> None:
        mode = {"fp64": abi.MIND_FP64, "mixed": abi.MIND_MIXED}[precision]
        abi.check(self.lib, self.handle, self.lib.mind_set_precision(self.handle, mode))

    def initialize(self) -> None:
        abi.check(self.lib, self.handle, self.lib.mind_initialize(self.handle))

    def time(self):
        step = ctypes.c_int64()
        t = ctypes.c_double()
        abi.check(self.lib, self.handle, self.lib.mind_time(self.handle, ctypes.byref(step), ctypes.byref(t)))
        return step.value, t.value

    def _c_records(self, records: Sequence[RecordSpec]):
        """The MindRecord array of `records`, built once per record list (a host that records
        the same list every call converts it once; the library keeps its tables too)."""
        cached = getattr(self, "_rec_cache", None)
        if cached is not None and cached[0] is records:
            return cached[1]
        table = np.zeros((max(1, len(records)), 5), dtype=np.int32)
        if records:
            table[:len(records)] = [(r.kind, r.node, r.group, r.row, r.field) for r in records]
        self._rec_cache = (records, table)
        return table

    def run_steps(self, steps: int, records: Sequence[RecordSpec], record_spikes: bool = True):
        table = self._c_records(records)
        recs = table.ctypes.data_as(ctypes.POINTER(abi.MindRecord))
        start_step, _ = self.time()
        abi.check(self.lib, self.handle,
                  self.lib.mind_run(self.handle, steps, recs, len(records), 1 if record_spikes else 0))
        samples = steps + 1
        by_record = np.empty((len(records), samples))   # transposed on the device: one copy
        if records:
            abi.check(self.lib, self.handle, self.lib.mind_get_trace_by_record(
                self.handle, by_record.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), by_record.size))
        n = ctypes.c_int64()
        abi.check(self.lib, self.handle, self.lib.mind_get_spikes(self.handle, None, None, 0, ctypes.byref(n)))
        times = np.zeros(n.value)
        sids = np.zeros(n.value, dtype=np.int64)
        if n.value:
            abi.check(self.lib, self.handle, self.lib.mind_get_spikes(
                self.handle, times.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                sids.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n.value, ctypes.byref(n)))
        ms = ctypes.c_double()
        abi.check(self.lib, self.handle, self.lib.mind_last_run_ms(self.handle, ctypes.byref(ms)))
        time = np.arange(start_step, start_step + samples, dtype=np.float64) * self.layout.dt
        result = SimulationResult(time, {}, times, sids, ms.value)
        if getattr(self, "drive_on", False):
            bins = ctypes.c_int64()
            abi.check(self.lib, self.handle, self.lib.mind_get_drive(self.handle, None, 0, ctypes.byref(bins)))
            drive = np.zeros((bins.value, self.layout.n_cells, 32), dtype=np.float32)
            if drive.size:
                abi.check(self.lib, self.handle, self.lib.mind_get_drive(
                    self.handle, drive.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), drive.size, ctypes.byref(bins)))
            result.drive = drive
        if getattr(self, "n_regions", 0):
            samples = ctypes.c_int64()
            abi.check(self.lib, self.handle, self.lib.mind_get_macro_trace(self.handle, None, 0, ctypes.byref(samples)))
            mt = np.zeros((samples.value, self.n_regions))
            if mt.size:
                abi.check(self.lib, self.handle, self.lib.mind_get_macro_trace(
                    self.handle, mt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), mt.size, ctypes.byref(samples)))
            result.macro_trace = mt
        if records:   # each trace is a row view of the one record-major copy
            result.traces = TraceMap([r.name for r in records], by_record)
        return result

    def run_stats(self) -> abi.MindRunStats:
        stats = abi.MindRunStats()
        abi.check(self.lib, self.handle, self.lib.mind_run_stats(self.handle, ctypes.byref(stats)))
        return stats

    def set_profiling(self, enable: bool) -> None:
        abi.check(self.lib, self.handle, self.lib.mind_set_profiling(self.handle, 1 if enable else 0))

    def step(self) -> None:
        abi.check(self.lib, self.handle, self.lib.mind_step(self.handle))

    def read_voltage(self, node: int) -> float:
        value = ctypes.c_double()
        abi.check(self.lib, self.handle, self.lib.mind_read_voltage(self.handle, node, ctypes.byref(value)))
        return value.value

    def read_value(self, ref: RecordSpec) -> float:
        value = ctypes.c_double()
        c = ref.to_c()
        abi.check(self.lib, self.handle, self.lib.mind_read_value(self.handle, ctypes.byref(c), ctypes.byref(value)))
        return value.value

    def inject_event(self, connection: int, t: float) -> None:
        edge = int(self.layout.connection_edges[connection - 1])
        abi.check(self.lib, self.handle, self.lib.mind_inject_event(self.handle, edge, float(t)))

    def inject_spikes(self, sources, times) -> None:
        """inject_spike! for many spikes: 1-based external source indices and absolute times."""
        sources = np.ascontiguousarray(sources, dtype=np.int64)
        times = np.ascontiguousarray(times, dtype=np.float64)
        if sources.shape != times.shape:
            raise ValueError("sources and times differ in length")
        abi.check(self.lib, self.handle, self.lib.mind_inject_spikes(
            self.handle, sources.size, sources.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            times.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def autotune(self, windows: int = 4) -> List[int]:
        """mind_autotune: time the launch shapes of the size bins and keep the fastest; the
        state is initialized again (t = 0).  Returns threads per cell of each bin."""
        abi.check(self.lib, self.handle, self.lib.mind_autotune(self.handle, int(windows)))
        return self.bin_threads()

    def bin_threads(self) -> List[int]:
        n = ctypes.c_int32()
        abi.check(self.lib, self.handle, self.lib.mind_bin_threads(self.handle, None, 0, ctypes.byref(n)))
        out = (ctypes.c_int32 * max(1, n.value))()
        abi.check(self.lib, self.handle, self.lib.mind_bin_threads(self.handle, out, n.value, ctypes.byref(n)))
        return list(out[:n.value])

    def set_bin_threads(self, threads: Sequence[int]) -> None:
        arr = (ctypes.c_int32 * max(1, len(threads)))(*[int(t) for t in threads])
        abi.check(self.lib, self.handle, self.lib.mind_set_bin_threads(self.handle, arr, len(threads)))

    def window_steps(self) -> int:
        steps = ctypes.c_int32()
        abi.check(self.lib, self.handle, self.lib.mind_window_steps(self.handle, ctypes.byref(steps)))
        return steps.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.mind_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def initialize(model, precision: str = "fp64"):
    """initialize!: allocate on the device (first call) and run INITIAL."""
    if model.layout is None:
        raise ValueError("model is not built")
    if model.state is None:
        model.state = DeviceState(model.layout, precision)
        macro = getattr(model, "macro", None)
        if macro is not None:
            model.state.attach_macro(macro)
    else:
        model.state.set_precision(precision)
    model.state.initialize()
    return model


def _steps_to(layout, state: DeviceState, stop_time: float) -> int:
    _, now = state.time()
    duration = float(stop_time) - now
    if not np.isfinite(duration):
        raise ValueError("stop time must be finite")
    count = int(round(duration / layout.dt))
    tolerance = 64.0 * np.spacing(max(abs(stop_time), abs(now), layout.dt))
    if count < 0 or abs(duration - count * layout.dt) > tolerance:
        raise ValueError("stop time must be an integer number of steps after the current time")
    return count


def run(model, stop_time: float, *, records: Sequence[RecordSpec] = (), record_spikes: bool = True):
    """run!: advance to an absolute stop time and return a SimulationResult."""
    if model.state is None:
        raise ValueError("simulation is not initialized")
    steps = _steps_to(model.layout, model.state, stop_time)
    if not isinstance(records, (list, tuple)):
        records = list(records)
    return model.state.run_steps(steps, records, record_spikes)


def step(model):
    if model.state is None:
        raise ValueError("simulation is not initialized")
    model.state.step()
    return model


def inject_spike(model, source, t: float):
    """inject_spike!(state, source, time) (src/runtime/state.jl:637-659): an external input fires at t."""
    if model.state is None:
        raise ValueError("simulation is not initialized")
    model.state.inject_spikes([source.index], [float(t)])
    return model


def voltage_record(model, cell, *, section: str = "soma", x: float = 0.5, name=None) -> RecordSpec:
    node = model.layout.voltage_node(cell.index, section, x)
    return RecordSpec(node, name if name is not None else f"v_{cell.gid}")


def _field_ref(layout, gi: int, row: int, field, name) -> RecordSpec:
    mech = layout.groups[gi].mechanism
    col = mech.field_index(field) if isinstance(field, str) else int(field) - 1
    if not 0 <= col < len(mech.fields):
        raise ValueError("invalid mechanism field")
    if not 1 <= int(row) <= layout.groups[gi].rows:
        raise ValueError("invalid mechanism row")
    label = name if name is not None else f"mechanism.{gi + 1}.{int(row)}.{mech.fields[col]}"
    return RecordSpec(0, label, abi.MIND_RECORD_MECHANISM, gi + 1, int(row), col + 1)


def mechanism_ref(model, target, *args, section: str = "soma", x: float = 0.5, name=None) -> RecordSpec:
    """mechanism_ref (src/model/references.jl:43-146), in its three forms:

    * ``mechanism_ref(model, group, row, field)``: `group` a 1-based group index or a
      mechanism name (its first group), `row` 1-based, `field` a MOD field name or a
      1-based column;
    * ``mechanism_ref(model, point, field)``: a field of a point process;
    * ``mechanism_ref(model, cell, mechanism, field, section=, x=)``: a density
      mechanism's field at (section, x) of a cell.
    """
    from .model import Cell, PointProcess

    layout = model.layout
    if layout is None:
        raise ValueError("model is not built")
    if isinstance(target, PointProcess):
        (field,) = args
        gi = int(layout.point_group[target.index - 1]) - 1
        return _field_ref(layout, gi, int(layout.point_row[target.index - 1]), field, name)
    if isinstance(target, Cell):
        mechanism, field = args
        node = layout.voltage_node(target.index, section, x)
        for gi, g in enumerate(layout.groups):
            if g.mechanism.name != mechanism or g.mechanism.kind != "density":
                continue
            rows = np.flatnonzero(np.asarray(g.nodes) == node)
            if len(rows):
                return _field_ref(layout, gi, int(rows[0]) + 1, field, name)
        raise ValueError(f"no {mechanism} at {section}({x}) of cell {target.index}")
    group = target
    row, field = args
    if isinstance(group, str):
        matches = [i for i, g in enumerate(layout.groups) if g.mechanism.name == group]
        if not matches:
            raise ValueError(f"no {group} group in the layout")
        gi = matches[0]
    else:
        gi = int(group) - 1
        if not 0 <= gi < len(layout.groups):
            raise ValueError("invalid mechanism group")
    return _field_ref(layout, gi, row, field, name)


def mechanism_record(model, target, *args, section: str = "soma", x: float = 0.5, name=None) -> RecordSpec:
    """mechanism_record: a RecordSpec of mechanism_ref's selection (named as given)."""
    return mechanism_ref(model, target, *args, section=section, x=x, name=name)


def voltage_ref(model, cell, *, section: str = "soma", x: float = 0.5) -> RecordSpec:
    """voltage_ref(plan, cell; section, x) (src/model/references.jl:93-99)."""
    node = model.layout.voltage_node(cell.index, section, x)
    return RecordSpec(node, f"voltage.{node}")


def connection_weights(model, connection: int) -> np.ndarray:
    """connection_weights(state, connection) (src/runtime/state.jl:603-616): the NetCon's
    NET_RECEIVE weights.  The builtin synapses never write their weight, so the device
    value is the built one."""
    layout = model.layout
    if not 1 <= int(connection) <= len(layout.connection_edges):
        raise ValueError("invalid connection")
    edge = int(layout.connection_edges[int(connection) - 1])
    return np.array([layout.edge_weights[edge - 1]])


def inject_event(model, connection: int, t: float):
    """inject_event!(state, connection, time) (src/runtime/state.jl:618-635): deliver one
    NetCon event at an absolute time, without its delay."""
    if model.state is None:
        raise ValueError("simulation is not initialized")
    model.state.inject_event(int(connection), float(t))
    return model


def autotune(model, windows: int = 4) -> List[int]:
    """Choose each size bin's CTA size by timing (mind_autotune); leaves the model initialized at t = 0."""
    if model.state is None:
        raise ValueError("simulation is not initialized")
    return model.state.autotune(windows)


def read_value(model, ref: RecordSpec) -> float:
    """read_value(state, selection) (src/runtime/state.jl:585-599)."""
    if model.state is None:
        raise ValueError("simulation is not initialized")
    return model.state.read_value(ref)


def runtime_configuration(model) -> dict:
    """runtime_configuration(state) (src/runtime/state.jl:573-581): the built step settings."""
    layout = model.layout
    if layout is None:
        raise ValueError("model is not built")
    macro = getattr(model, "macro", None)
    return {"dt_micro": float(layout.dt), "dt_macro": float(macro.dt_macro) if macro is not None else None,
            "celsius": float(layout.celsius), "secondorder": int(layout.secondorder)}


def simulation_time(model) -> float:
    return model.state.time()[1]
