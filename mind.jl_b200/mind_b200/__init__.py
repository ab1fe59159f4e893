"""mind_b200 — host-side mirror of MIND.jl's micro model/runtime API over libmindgpu.so.

The Julia names map one to one (`add_population!` -> `add_population`,
`insert!` -> `insert`, `build!` -> `build`, `initialize!` -> `initialize`,
`run!` -> `run`, `step!` -> `step`).  Model construction and packing run on
the host; every simulation step runs in the CUDA library through its C-ABI.
"""
from .mechanisms import (Mechanism, builtin, clear_mod_cache, compile_mod, compiled_mechanisms, emitted, load_mod,
                         mechanism_ir, register_mod)
from .morphology import Point3D, Section, discretize, location_node
from .model import (Cell, IonSpecies, MicroModel, PointProcess, Population, SpikeSource, ghk, nernst,
                    add_pointprocess, add_pointprocesses, add_population, connect, connect_many,
                    insert, register_external_sources, register_point_sources, register_spike_source, spike_source)
from .layout import Layout, build
from .runtime import (RecordSpec, SimulationResult, autotune, connection_weights, initialize, inject_event,
                      inject_spike, mechanism_record, mechanism_ref, read_value, run, runtime_configuration,
                      simulation_time, step, voltage_record, voltage_ref)

__all__ = [
    "Mechanism", "builtin", "clear_mod_cache", "compile_mod", "compiled_mechanisms", "emitted", "load_mod",
    "mechanism_ir", "register_mod", "Point3D", "Section", "discretize", "location_node", "Cell",
    "IonSpecies", "MicroModel", "PointProcess", "Population", "SpikeSource", "ghk", "nernst", "add_pointprocess",
    "add_pointprocesses", "add_population", "connect", "connect_many", "insert",
    "register_external_sources", "register_point_sources", "register_spike_source", "spike_source", "Layout", "build",
    "RecordSpec", "SimulationResult", "autotune", "connection_weights", "initialize", "inject_event",
    "inject_spike", "mechanism_record", "mechanism_ref", "read_value", "run", "runtime_configuration",
    "simulation_time", "step",
    "voltage_record", "voltage_ref",
]
