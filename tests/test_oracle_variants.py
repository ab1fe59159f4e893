"""How much a run depends on the two choices where this build's arithmetic can differ from
MIND.jl's (CPU only).

1. The math library.  The CUDA path and the oracle share the project's exp, log and pow
   (mind_math.h), which is what makes their FP64 runs bit-identical; MIND.jl computes with
   CUDA.jl's device math.  Both are faithfully rounded implementations of the same
   functions, and so is the C library's: liboracle_other.so is the oracle built on it.
2. The order of sums MIND.jl leaves to FP64 atomics (several mechanism rows into one node,
   sibling branches into one parent), which varies from run to run there and is fixed
   here: liboracle_rev.so sums every such term in the opposite order.

Each variant runs the same networks as the oracle, and the tests require what the FP64
mode is specified to meet against the reference: max |dV| <= 1e-9 mV on every recorded
soma, and the same raster (cell ids and step indices).  Spike times may differ in the last
bits (a NetStim interval is -log(u)), never in their step.
"""
import numpy as np
import pytest

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import networks

DV_BOUND_MV = 1e-9
VARIANTS = [pytest.param({"libm": True}, id="libm"), pytest.param({"reversed_order": True}, id="reversed_sums")]


def _compare(layout, steps, variant, macro=None):
    nodes = netcases.soma_nodes(layout)
    own = oracle.run(layout, steps, nodes, macro=macro)
    other = oracle.run(layout, steps, nodes, macro=macro, **variant)
    assert own.status == 0 and other.status == 0, (own.message, other.message)
    assert float(np.max(np.abs(own.trace - other.trace))) <= DV_BOUND_MV
    np.testing.assert_array_equal(own.spike_sids, other.spike_sids)
    step = lambda r: np.floor(r.spike_times / layout.dt + 1e-9).astype(np.int64)
    np.testing.assert_array_equal(step(own), step(other))
    np.testing.assert_allclose(own.spike_times, other.spike_times, rtol=0, atol=1e-12)
    if macro is not None:
        np.testing.assert_allclose(own.macro_trace, other.macro_trace, rtol=1e-12, atol=1e-12)
    return own


@pytest.mark.parametrize("variant", VARIANTS)
def test_config1_full_100ms(variant):
    layout = mb.build(networks.config1())
    ref = _compare(layout, 4000, variant)
    assert len(ref.spike_sids) > 500          # NetStim-driven: each interval draws a log


@pytest.mark.parametrize("variant", VARIANTS)
def test_recurrent_trees_40ms(variant):
    layout = mb.build(netcases.recurrent_trees())
    ref = _compare(layout, 1600, variant)
    assert np.sum(ref.spike_sids <= layout.n_cells) > 20   # recurrent cell spikes


@pytest.mark.parametrize("variant", VARIANTS)
def test_coupled_regions_40ms(variant):
    model, macro = netcases.coupled_regions()
    ref = _compare(model.layout, 1600, variant, macro=macro)
    assert np.sum(ref.spike_sids <= model.layout.n_cells) > 5


@pytest.mark.parametrize("variant", VARIANTS)
def test_config3_150_pyramidal_cells_30ms(variant):
    layout = mb.build(networks.config3(n_cells=150))
    _compare(layout, 1200, variant)
