"""mind_run_noalloc: run! for callers that must not allocate device memory.

Some hosts own all device memory through their own allocator and size it up
front, or step a model inside a loop that must not call into the CUDA
allocator.  For them libmindgpu.so offers mind_run_noalloc, whose per-run
scratch is a static 16 MiB device array instead of cudaMalloc'd buffers.  This
file checks, through the C-ABI, that two calls in a row give the same voltage
traces as the ordinary mind_run (FP64: bit for bit), and that a run too large
for the static array is refused with a clear message.  It is collected last so
that a failure here leaves every other test already run; it also passes alone
in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import mind_b200 as mb
import netcases
from mind_b200 import abi

pytestmark = pytest.mark.gpu


def _noalloc(state, steps, nodes):
    recs = (abi.MindRecord * len(nodes))()
    for i, node in enumerate(nodes):
        recs[i].kind = abi.MIND_RECORD_VOLTAGE
        recs[i].node = int(node)
    trace = np.zeros((steps + 1, len(nodes)))
    status = state.lib.mind_run_noalloc(state.handle, steps, recs, len(nodes),
                                        trace.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return status, trace


def test_noalloc_matches_mind_run_on_two_calls():
    model = netcases.recurrent_trees(n_cells=12, synapses=16)
    layout = mb.build(model)
    nodes = netcases.soma_nodes(layout)
    records = [mb.RecordSpec(n, f"n{n}") for n in nodes]

    mb.initialize(model)
    first = mb.run(model, 20.0, records=records)
    second = mb.run(model, 40.0, records=records)
    want1 = np.stack([first.traces[r.name] for r in records], axis=1)
    want2 = np.stack([second.traces[r.name] for r in records], axis=1)

    mb.initialize(model)
    steps = int(round(20.0 / layout.dt))
    status, got1 = _noalloc(model.state, steps, nodes)
    assert status == abi.MIND_OK, model.state.lib.mind_last_error(model.state.handle)
    status, got2 = _noalloc(model.state, steps, nodes)
    assert status == abi.MIND_OK, model.state.lib.mind_last_error(model.state.handle)

    assert np.max(np.abs(got1 - want1)) <= 1e-9
    assert np.max(np.abs(got2 - want2)) <= 1e-9
    np.testing.assert_array_equal(got1, want1)
    np.testing.assert_array_equal(got2, want2)
    assert np.any(got2 > -10.0)   # cells fired during the compared runs


def test_noalloc_refuses_runs_beyond_its_scratch():
    model = netcases.strong_config1(n_cells=2)
    layout = mb.build(model)
    mb.initialize(model)
    nodes = netcases.soma_nodes(layout)
    steps = abi.MIND_NOALLOC_SCRATCH_BYTES // (8 * len(nodes)) + 10
    recs = (abi.MindRecord * len(nodes))()
    for i, node in enumerate(nodes):
        recs[i].kind = abi.MIND_RECORD_VOLTAGE
        recs[i].node = int(node)
    dummy = (ctypes.c_double * 1)()
    status = model.state.lib.mind_run_noalloc(model.state.handle, steps, recs, len(nodes), dummy)
    assert status == abi.MIND_ECAPACITY
    assert b"scratch" in model.state.lib.mind_last_error(model.state.handle)
