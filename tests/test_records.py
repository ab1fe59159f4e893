"""Mechanism references (MindRecord kind MIND_RECORD_MECHANISM) in the CPU oracle.

A reference names a layout column of one row (mechanism_ref, src/model/references.jl:43-73);
the kept columns are PARAMETER and STATE fields.  These checks run the oracle alone: a
recorded parameter stays at its layout value, a synaptic state decays by the cnexp factor
between events, hh's gates start at their steady state, and an ASSIGNED field is refused.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import abi


def _model():
    model = netcases.recurrent_trees(n_cells=4, synapses=6)
    mb.build(model)
    return model


def test_parameter_and_state_records():
    model = _model()
    layout = model.layout
    steps = 2000
    syn = [g for g in layout.groups if g.mechanism.name == "Exp2Syn"][0]
    pas = mb.mechanism_ref(model, "pas", 3, "g")
    amp = mb.mechanism_ref(model, "IClamp", 1, "amp")
    m = mb.mechanism_ref(model, "hh", 1, "m")
    soma = mb.RecordSpec(layout.voltage_node(1), "v1")
    a = [mb.mechanism_ref(model, "Exp2Syn", r, "A") for r in range(1, syn.rows + 1)]
    b = [mb.mechanism_ref(model, "Exp2Syn", r, "B") for r in range(1, syn.rows + 1)]
    ref = oracle.run(layout, steps, records=[soma, pas, amp, m] + a + b)
    assert ref.status == 0, ref.message
    g_pas = [g for g in layout.groups if g.mechanism.name == "pas"][0]
    np.testing.assert_array_equal(ref.trace[:, 1], g_pas.column("g")[2])
    assert np.all(ref.trace[:, 2] == 0.3)
    # hh m starts at minf(v0) in (0, 1) and moves with the voltage
    assert 0.0 < ref.trace[0, 3] < 1.0 and np.ptp(ref.trace[:, 3]) > 0.0
    # A and B decay by exp(-dt/tau) per step wherever no event arrived
    A = ref.trace[:, 4:4 + syn.rows]
    B = ref.trace[:, 4 + syn.rows:]
    assert np.all(A >= 0.0) and np.count_nonzero(A.max(axis=0)) >= syn.rows // 2
    for X, tau in ((A, syn.column("tau1")), (B, syn.column("tau2"))):
        prev, nxt = X[:-1], X[1:]
        quiet = (prev > 0.0) & (nxt < prev)
        assert quiet.sum() > 1000
        ratio = nxt[quiet] / prev[quiet]
        want = np.exp(-layout.dt / np.broadcast_to(tau, X.shape)[1:][quiet])
        np.testing.assert_allclose(ratio, want, rtol=1e-12)


def test_assigned_field_is_refused():
    model = _model()
    ref = oracle.run(model.layout, 10, records=[mb.mechanism_ref(model, "hh", 1, "ina")])
    assert ref.status == abi.MIND_EARG


def test_mechanism_ref_validates_indices():
    model = _model()
    for args in (("hh", 0, "m"), ("hh", 10**6, "m"), ("hh", 1, "nope"), (99, 1, 1)):
        try:
            mb.mechanism_ref(model, *args)
        except ValueError:
            continue
        raise AssertionError(f"accepted {args}")


def test_reference_forms_of_mechanism_ref():
    """The point-process and cell/density forms of mechanism_ref (references.jl:101-146)
    select the same rows as the group/row form; voltage_ref, mechanism_record and
    connection_weights follow the layout."""
    from mind_b200 import model as M

    model = netcases.strong_config1(n_cells=3, synapses=4)
    layout = mb.build(model)
    # a point process of the model: the first ExpSyn's PointProcess handle
    point = M.PointProcess(model, 1)
    ref_point = mb.mechanism_ref(model, point, "g")
    gi = int(layout.point_group[0]) - 1
    assert ref_point.group == gi + 1 and ref_point.row == int(layout.point_row[0])
    assert layout.groups[gi].mechanism.fields[ref_point.field - 1] == "g"
    # the cell form: hh at the soma of cell 2 is the hh row on that node
    cell2 = M.Cell(model, 2, 2)
    ref_cell = mb.mechanism_ref(model, cell2, "hh", "m")
    hh = layout.groups[ref_cell.group - 1]
    assert hh.mechanism.name == "hh"
    assert int(hh.nodes[ref_cell.row - 1]) == layout.voltage_node(2)
    with pytest.raises(ValueError):
        mb.mechanism_ref(model, cell2, "hh", "m", section="dend")   # hh only at the soma
    # the same selection records the same trace
    a = oracle.run(layout, 200, records=[ref_cell, mb.mechanism_ref(model, ref_cell.group, ref_cell.row, "m")])
    assert a.status == 0 and np.array_equal(a.trace[:, 0], a.trace[:, 1])
    assert mb.voltage_ref(model, cell2).node == layout.voltage_node(2)
    assert mb.mechanism_record(model, point, "g", name="g1").name == "g1"
    edge = int(layout.connection_edges[0])
    np.testing.assert_array_equal(mb.connection_weights(model, 1), [layout.edge_weights[edge - 1]])
    with pytest.raises(ValueError):
        mb.connection_weights(model, 10 ** 6)


def test_runtime_configuration_reports_the_build():
    model = _model()
    cfg = mb.runtime_configuration(model)
    assert cfg == {"dt_micro": 0.025, "dt_macro": None, "celsius": 6.3, "secondorder": 0}
    coupled, macro = netcases.coupled_regions()
    assert mb.runtime_configuration(coupled)["dt_macro"] == macro.dt_macro
