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


def test_noalloc_refuses_step_counts_whose_size_would_wrap():
    """Step counts whose trace size overflows 64 bits (steps + 1 == 2^63, or (steps+1) * 8 *
    records past 2^64) are refused with status 3 before any launch; the clock does not move
    and the state stays usable."""
    model = netcases.strong_config1(n_cells=8)
    layout = mb.build(model)
    mb.initialize(model)
    nodes = netcases.soma_nodes(layout)
    recs = (abi.MindRecord * len(nodes))()
    for i, node in enumerate(nodes):
        recs[i].kind = abi.MIND_RECORD_VOLTAGE
        recs[i].node = int(node)
    dummy = (ctypes.c_double * 1)()
    lib, handle = model.state.lib, model.state.handle
    for steps in ((1 << 63) - 1, 1 << 61, (1 << 64) // (8 * len(nodes)) - 1):
        assert lib.mind_run_noalloc(handle, steps, recs, len(nodes), dummy) == abi.MIND_ECAPACITY
        assert model.state.time()[0] == 0
    assert lib.mind_run_noalloc(handle, (1 << 63) - 1, recs, 0, dummy) == abi.MIND_ECAPACITY
    status, trace = _noalloc(model.state, 40, nodes)
    assert status == abi.MIND_OK
    assert model.state.time()[0] == 40 and np.all(np.isfinite(trace))


def test_noalloc_runs_a_handle_with_surrogate_cells():
    """Surrogate inference uses the buffers reserved when the network was attached (its
    products are this library's own kernels): a noalloc run of a handle with surrogate cells
    gives the voltages of an ordinary run, bit for bit, over several surrogate bins."""
    from mind_b200 import surrogate

    model, _ = netcases.coupled_regions(n_regions=2, cells_per_region=8, synapses=8, seed=3)
    net = surrogate.Mlp(seed=1)
    params = net.params
    params[-1] = -1.0                       # output bias: surrogate cells fire now and then
    net.params = params
    mask = np.arange(model.layout.n_cells) % 2 == 0
    nodes = np.asarray(netcases.soma_nodes(model.layout))[~mask]
    steps = int(round(30.0 / model.layout.dt))
    traces = []
    for use_noalloc in (False, True):
        state = mb.runtime.DeviceState(model.layout)
        state.attach_macro(model.macro)
        state.attach_surrogate(net, mask, 1.0)
        state.initialize()
        if use_noalloc:
            status, trace = _noalloc(state, steps, nodes)
            assert status == abi.MIND_OK, state.lib.mind_last_error(state.handle)
        else:
            result = state.run_steps(steps, [mb.RecordSpec(int(n), f"n{n}") for n in nodes], False)
            trace = np.stack([result.traces[f"n{n}"] for n in nodes], axis=1)
        assert state.time()[0] == steps
        traces.append(trace)
        state.close()
    np.testing.assert_array_equal(traces[1], traces[0])
    net.close()
