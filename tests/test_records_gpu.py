"""Mechanism references on the device: recorded fields and read_value, against the oracle.

FP64 mode records the same bits as the CPU oracle for voltages, hh gates, Exp2Syn A/B
(staged state in shared memory), pas and IClamp parameters (read from HBM); read_value
after a run returns the last recorded sample; NetStim fields are readable but not
recordable; ASSIGNED fields are refused with MIND_EARG; mind_run_noalloc records the same.
"""
import ctypes

import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import abi

pytestmark = pytest.mark.gpu


def _model():
    model = netcases.recurrent_trees(n_cells=6, synapses=6)
    mb.build(model)
    return model


def _records(model):
    layout = model.layout
    syn = [g for g in layout.groups if g.mechanism.name == "Exp2Syn"][0]
    hh = [g for g in layout.groups if g.mechanism.name == "hh"][0]
    recs = [mb.RecordSpec(layout.voltage_node(c), f"v{c}") for c in (1, 4)]
    recs += [mb.mechanism_ref(model, "hh", r, f) for r in (1, hh.rows) for f in ("m", "h", "n")]
    recs += [mb.mechanism_ref(model, "Exp2Syn", r, f) for r in range(1, syn.rows + 1) for f in ("A", "B")]
    recs += [mb.mechanism_ref(model, "pas", 5, "g"), mb.mechanism_ref(model, "IClamp", 1, "amp"),
             mb.mechanism_ref(model, "Exp2Syn", 3, "tau2"), mb.mechanism_ref(model, "hh", 2, "gnabar")]
    return recs


def test_recorded_fields_match_oracle_fp64():
    model = _model()
    recs = _records(model)
    steps = 1200
    ref = oracle.run(model.layout, steps, records=recs)
    assert ref.status == 0, ref.message
    mb.initialize(model, precision="fp64")
    result = mb.run(model, steps * model.layout.dt, records=recs)
    got = np.stack([result.traces[r.name] for r in recs], axis=1)
    assert np.array_equal(got, ref.trace)
    assert np.count_nonzero(got[:, 2 + 6:2 + 6 + 12].max(axis=0)) > 0   # synapses received events
    for k, r in enumerate(recs):
        assert mb.read_value(model, r) == got[-1, k]


def test_read_value_kinds_and_refusals():
    model = _model()
    mb.initialize(model)
    mb.run(model, 5.0)
    stim = mb.mechanism_ref(model, "NetStim", 1, "interval")
    assert mb.read_value(model, stim) == 50.0
    with pytest.raises(abi.MindError) as err:
        mb.read_value(model, mb.mechanism_ref(model, "hh", 1, "ina"))
    assert err.value.status == abi.MIND_EARG
    with pytest.raises(abi.MindError) as err:
        mb.run(model, 10.0, records=[stim])
    assert err.value.status == abi.MIND_EARG
    # a refused reference leaves the simulation usable
    mb.run(model, 10.0, records=[mb.mechanism_ref(model, "hh", 1, "m")])


def test_noalloc_records_mechanism_fields():
    model = _model()
    recs = _records(model)
    steps = 200
    mb.initialize(model)
    want = mb.run(model, steps * model.layout.dt, records=recs)
    want = np.stack([want.traces[r.name] for r in recs], axis=1)
    mb.initialize(model)
    c = (abi.MindRecord * len(recs))(*[r.to_c() for r in recs])
    out = np.zeros((steps + 1, len(recs)))
    status = model.state.lib.mind_run_noalloc(model.state.handle, steps, c, len(recs),
                                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert status == 0
    assert np.array_equal(out, want)
