"""Runtime surface through the C-ABI on the GPU: failure codes, event injection, step!.

Failures are made on the host (a singular cable, a spike record too small, a
NetCon the device path does not support); none of them faults or hangs the
GPU: each run returns the reference's status code and the handle is usable
again after initialize.
"""
import math

import numpy as np
import pytest

import mind_b200 as mb
import netcases
from mind_b200 import abi
from mind_b200 import model as M

pytestmark = pytest.mark.gpu


def passive_cell(mech=True):
    model = M.MicroModel()
    soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=3)
    cell = M.add_population(model, [soma], 1)[0]
    if mech:
        M.insert(cell, mb.builtin("pas"), params={"g": 1e-4, "e": -65.0})
    return model, cell


def test_singular_cable_reports_status_6_and_recovers():
    model, _ = passive_cell(mech=False)
    layout = mb.build(model)
    layout.capacitance[:] = 0.0
    layout.axial[:] = 0.0
    layout.axial_diagonal[:] = 0.0
    mb.initialize(model)
    with pytest.raises(abi.MindError) as err:
        mb.run(model, 1.0)
    assert err.value.status in (abi.MIND_ESINGULAR, abi.MIND_ENONFINITE)
    with pytest.raises(abi.MindError) as again:       # uninitialized after an error, as run! leaves it
        mb.run(model, 1.0)
    assert again.value.status == abi.MIND_EARG
    model2, cell2 = passive_cell()
    mb.build(model2)
    mb.initialize(model2)
    assert mb.run(model2, 1.0).time[-1] == pytest.approx(1.0)


def test_spike_record_overflow_reports_status_3():
    model = netcases.strong_config1(n_cells=4)
    mb.build(model, spike_capacity=2)
    mb.initialize(model)
    with pytest.raises(abi.MindError) as err:
        mb.run(model, 50.0)
    assert err.value.status == abi.MIND_ECAPACITY
    mb.initialize(model)                                # the same handle runs again after initialize
    result = mb.run(model, 1.0, record_spikes=False)
    assert len(result.time) == 41


def test_netcon_onto_netstim_is_rejected():
    model = M.MicroModel()
    a = M.add_pointprocess(model, mb.builtin("NetStim"), params={"number": 1, "start": 1.0})
    b = M.add_pointprocess(model, mb.builtin("NetStim"), params={"number": 1, "start": 1.0})
    M.connect(a, b, weight=1.0, delay=1.0)
    mb.build(model)
    with pytest.raises(abi.MindError) as err:
        mb.initialize(model)
    assert err.value.status == abi.MIND_ELAYOUT


def test_injected_event_equals_a_netstim_spike():
    """inject_event!(connection, 5.0) drives the synapse exactly like a NetStim spike at 5.0."""
    def build(with_stim):
        model, cell = passive_cell()
        syn = M.add_pointprocess(cell, mb.builtin("ExpSyn"), section="soma", x=0.5, params={"tau": 2.0})
        stim = M.add_pointprocess(model, mb.builtin("NetStim"),
                                  params={"interval": 10.0, "number": 1 if with_stim else 0, "start": 5.0})
        conn = M.connect(stim, syn, weight=0.002, delay=0.0)
        layout = mb.build(model)
        return model, conn, layout

    model_a, conn_a, layout_a = build(with_stim=True)
    model_b, conn_b, layout_b = build(with_stim=False)
    node = layout_a.voltage_node(1)
    rec = [mb.RecordSpec(node, "v")]
    mb.initialize(model_a)
    want = mb.run(model_a, 20.0, records=rec).traces["v"]
    mb.initialize(model_b)
    model_b.state.inject_event(conn_b, 5.0)
    got = mb.run(model_b, 20.0, records=rec).traces["v"]
    np.testing.assert_array_equal(got, want)
    assert np.max(np.abs(want - want[0])) > 1e-3


def test_injected_spike_equals_a_netstim_spike():
    """inject_spike!(external input, 4.0) through a 1 ms NetCon drives the synapse exactly like a
    NetStim spike at 4.0 through the same NetCon, and enters the raster under its sid."""
    def build(external):
        model, cell = passive_cell()
        syn = M.add_pointprocess(cell, mb.builtin("ExpSyn"), section="soma", x=0.5, params={"tau": 2.0})
        stim = M.add_pointprocess(model, mb.builtin("NetStim"),
                                  params={"interval": 10.0, "number": 0 if external else 1, "start": 4.0})
        M.connect(stim, syn, weight=0.002, delay=1.0)
        source = M.register_spike_source(model, sid=900) if external else None
        if external:
            M.connect(source, syn, weight=0.002, delay=1.0)
        return model, source, mb.build(model)

    model_a, _, layout_a = build(external=False)
    model_b, source, layout_b = build(external=True)
    rec = [mb.RecordSpec(layout_a.voltage_node(1), "v")]
    mb.initialize(model_a)
    want = mb.run(model_a, 20.0, records=rec)
    mb.initialize(model_b)
    mb.inject_spike(model_b, source, 4.0)
    got = mb.run(model_b, 20.0, records=rec)
    np.testing.assert_array_equal(got.traces["v"], want.traces["v"])
    assert np.max(np.abs(want.traces["v"] - want.traces["v"][0])) > 1e-3
    assert got.spike_sources.tolist() == [900] and got.spike_times.tolist() == [4.0]
    # only external inputs accept injected spikes, and never in the past
    with pytest.raises(abi.MindError) as info:
        model_b.state.inject_spikes([1], [30.0])
    assert info.value.status == abi.MIND_EARG
    with pytest.raises(abi.MindError):
        mb.inject_spike(model_b, source, 1.0)


def test_step_matches_run_and_read_voltage():
    model = netcases.recurrent_trees(n_cells=6, synapses=8)
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    mb.initialize(model)
    ref = mb.run(model, 2.0, records=[mb.RecordSpec(n, str(n)) for n in nodes])
    mb.initialize(model)
    for _ in range(80):
        mb.step(model)
    assert mb.simulation_time(model) == pytest.approx(2.0)
    for n in nodes:
        assert model.state.read_voltage(n) == ref.traces[str(n)][-1]
