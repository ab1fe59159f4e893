"""PatternStim (add_pointprocess!(model, PatternStim; spike_times), src/model/micro/model.jl:
586-613; replayed at every reset, src/runtime/utils/events.jl:92-110): the oracle fires each
prescribed time as a spike of the PatternStim's source -- in the raster, through its NetCons."""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle


def test_oracle_fires_the_prescribed_times_through_netcons():
    model, trains = netcases.pattern_driven()
    layout = mb.build(model)
    assert len(layout.pattern_times) == sum(len(t) for t in trains.values())
    assert np.all(np.diff(layout.pattern_times) >= 0)
    ref = oracle.run(layout, 1400, netcases.soma_nodes(layout))
    assert ref.status == 0, ref.message
    for sid, times in trains.items():
        np.testing.assert_array_equal(ref.spike_times[ref.spike_sids == sid], np.sort(times))
    assert np.sum(ref.spike_sids < layout.n_cells) > 0          # the trains drove the cells to fire
    quiet = mb.build(netcases.pattern_driven()[0])
    quiet.pattern_times, quiet.pattern_points = quiet.pattern_times[:0], quiet.pattern_points[:0]
    assert np.sum(oracle.run(quiet, 1400, ()).spike_sids < layout.n_cells) == 0


def test_spike_times_apply_to_patternstim_only():
    model, _ = netcases.pattern_driven()
    with pytest.raises(ValueError, match="PatternStim only"):
        mb.model.add_pointprocess(model, mb.builtin("NetStim"), spike_times=[1.0])
    with pytest.raises(ValueError, match=">= 0"):
        mb.model.add_pointprocess(model, mb.builtin("PatternStim"), spike_times=[-1.0])
