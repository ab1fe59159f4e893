"""Regions coupled to the micro network on the GPU vs the CPU oracle (FP64, bit for bit).

Jansen-Rit regions drive every synapse through external spike inputs (Poisson, from the
regions' outputs), cells feed the regions' 1 ms rate bins, regions are coupled with
delayed edges, and cells are coupled by NetCons: the soma traces, the raster and the
regions' outputs must equal the oracle's exactly.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import abi
from mind_b200.macro import MacroModel

pytestmark = pytest.mark.gpu


def test_coupled_regions_match_the_oracle_exactly():
    model, macro = netcases.coupled_regions()
    layout = model.layout
    nodes = netcases.soma_nodes(layout)
    steps = 1600
    ref = oracle.run(layout, steps, nodes, macro=macro)
    assert ref.status == 0, ref.message
    mb.initialize(model)
    got = mb.run(model, steps * layout.dt, records=[mb.RecordSpec(n, f"n{n}") for n in nodes])
    trace = np.stack([got.traces[f"n{n}"] for n in nodes], axis=1)
    np.testing.assert_array_equal(trace, ref.trace)
    np.testing.assert_array_equal(got.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(got.spike_times, ref.spike_times)
    np.testing.assert_array_equal(got.macro_trace, ref.macro_trace)
    assert np.sum(ref.spike_sids <= layout.n_cells) > 5        # cells fired and fed the regions
    assert np.ptp(ref.macro_trace) > 0.5


def test_unequal_windows_within_a_bin_match_the_oracle():
    """Cell NetCons from 0.45 ms allow windows of 16 to 19 steps: the library runs 16-step
    windows and ends one at every 40-step rate bin (16, 16, 8 per bin), and the run must
    still equal the oracle's step-by-step restatement bit for bit."""
    model, macro = netcases.coupled_regions(seed=12, min_cell_delay=0.45)
    layout = model.layout
    nodes = netcases.soma_nodes(layout)
    steps = 1000
    ref = oracle.run(layout, steps, nodes, macro=macro)
    assert ref.status == 0, ref.message
    mb.initialize(model)
    assert model.state.window_steps() == 16
    got = mb.run(model, steps * layout.dt, records=[mb.RecordSpec(n, f"n{n}") for n in nodes])
    trace = np.stack([got.traces[f"n{n}"] for n in nodes], axis=1)
    np.testing.assert_array_equal(trace, ref.trace)
    np.testing.assert_array_equal(got.spike_sources, ref.spike_sids)
    np.testing.assert_array_equal(got.spike_times, ref.spike_times)
    np.testing.assert_array_equal(got.macro_trace, ref.macro_trace)
    assert np.sum(ref.spike_sids <= layout.n_cells) > 3


def test_split_runs_continue_the_regions():
    model, macro = netcases.coupled_regions(n_regions=2, cells_per_region=3)
    layout = model.layout
    mb.initialize(model)
    whole = mb.run(model, 30.0)
    mb.initialize(model)
    first = mb.run(model, 401 * layout.dt)   # ends inside a macro step
    second = mb.run(model, 30.0)
    assert first.macro_trace.shape[0] == 101 and second.macro_trace.shape[0] == 200
    joined = np.concatenate([first.macro_trace, second.macro_trace])
    np.testing.assert_array_equal(joined, whole.macro_trace)
    np.testing.assert_array_equal(np.concatenate([first.spike_times, second.spike_times]), whole.spike_times)


def test_attach_rejects_inconsistent_regions():
    model, _ = netcases.coupled_regions(n_regions=2, cells_per_region=2)
    layout = model.layout
    bad = MacroModel(dt_macro=0.1, bin_ms=1.0)
    bad.add_region()
    bad.add_inputs(1, [1])          # source 1 is a cell detector, not an external input
    state = mb.runtime.DeviceState(layout)
    with pytest.raises(abi.MindError) as info:
        state.attach_macro(bad)
    assert info.value.status == abi.MIND_ELAYOUT
    odd = MacroModel(dt_macro=0.03, bin_ms=1.0)   # not a multiple of dt
    odd.add_region()
    with pytest.raises(abi.MindError):
        state.attach_macro(odd)
    state.close()
