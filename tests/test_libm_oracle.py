"""How much a run depends on the math library (CPU only).

The CUDA path and the oracle share the project's exp, log and pow (mind_math.h), which is
what makes their FP64 runs bit-identical; MIND.jl computes with CUDA.jl's device math.
Both are faithfully rounded implementations of the same functions, and so is the C
library's.  liboracle_libm.so is the oracle built on the C library's exp, log and pow;
these tests run the same networks through both oracles and require what the FP64 mode is
specified to meet against the reference: max |dV| <= 1e-9 mV on every recorded soma, and
the same raster (cell ids and step indices).  So the choice of a faithful math library,
one of the two places where the arithmetic here can differ from MIND.jl's (the other is
the order of the sums MIND.jl leaves to FP64 atomics), stays inside that bound on these
networks.  Spike times may differ in the last bits (a NetStim interval is -log(u)), never
in their step.
"""
import numpy as np

import mind_b200 as mb
import netcases
import oracle
from mind_b200 import networks

DV_BOUND_MV = 1e-9


def _compare(layout, steps, macro=None):
    nodes = netcases.soma_nodes(layout)
    own = oracle.run(layout, steps, nodes, macro=macro)
    libm = oracle.run(layout, steps, nodes, macro=macro, libm=True)
    assert own.status == 0 and libm.status == 0, (own.message, libm.message)
    assert float(np.max(np.abs(own.trace - libm.trace))) <= DV_BOUND_MV
    np.testing.assert_array_equal(own.spike_sids, libm.spike_sids)
    step = lambda r: np.floor(r.spike_times / layout.dt + 1e-9).astype(np.int64)
    np.testing.assert_array_equal(step(own), step(libm))
    np.testing.assert_allclose(own.spike_times, libm.spike_times, rtol=0, atol=1e-12)
    if macro is not None:
        np.testing.assert_allclose(own.macro_trace, libm.macro_trace, rtol=1e-12, atol=1e-12)
    return own


def test_config1_full_100ms_does_not_depend_on_the_math_library():
    layout = mb.build(networks.config1())
    ref = _compare(layout, 4000)
    assert len(ref.spike_sids) > 500          # NetStim-driven: every interval drew a log


def test_recurrent_trees_40ms_do_not_depend_on_the_math_library():
    layout = mb.build(netcases.recurrent_trees())
    ref = _compare(layout, 1600)
    assert np.sum(ref.spike_sids <= layout.n_cells) > 20   # recurrent cell spikes


def test_coupled_regions_40ms_do_not_depend_on_the_math_library():
    model, macro = netcases.coupled_regions()
    ref = _compare(model.layout, 1600, macro=macro)
    assert np.sum(ref.spike_sids <= model.layout.n_cells) > 5


def test_config3_150_pyramidal_cells_30ms_do_not_depend_on_the_math_library():
    layout = mb.build(networks.config3(n_cells=150))
    _compare(layout, 1200)
