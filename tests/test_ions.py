"""Ion species at build time (CPU): nernst and ghk (src/model/micro/biophysics.jl:53-74), and
IonSpecies(nernst=True), whose reversal is the Nernst potential of its concentrations at the
model's temperature (src/model/micro/model.jl:766-768) and is what USEION READ e<ion> sees."""
import math

import numpy as np
import pytest

import mind_b200 as mb
import oracle
from mind_b200 import model as M

R = 1.380649e-23 * 6.02214076e23      # J / (mol K), exact SI
F = 1.602176634e-19 * 6.02214076e23   # C / mol, exact SI


def test_nernst_is_rt_over_zf_log_of_the_concentration_ratio():
    for ci, co, z, celsius in [(10.0, 140.0, 1, 6.3), (54.4, 2.5, 1, 36.0), (5e-5, 2.0, 2, 6.3), (12.0, 120.0, -1, 20.0)]:
        expect = 1000.0 * R * (celsius + 273.15) / (z * F) * math.log(co / ci)
        assert mb.nernst(ci, co, z, celsius=celsius) == pytest.approx(expect, rel=1e-14)
    assert mb.nernst(10.0, 140.0, 1) == pytest.approx(63.5515, abs=1e-4)   # na at 6.3 degC


def test_nernst_limits_and_invalid_arguments():
    assert mb.nernst(1.0, 2.0, 0) == 0.0
    assert mb.nernst(0.0, 2.0, 1) == 1.0e6
    assert mb.nernst(1.0, 0.0, 1) == -1.0e6
    for args in [(-1.0, 2.0, 1), (1.0, -2.0, 1), (math.nan, 2.0, 1), (1.0, 2.0, math.inf)]:
        with pytest.raises(ValueError):
            mb.nernst(*args)
    with pytest.raises(ValueError):
        mb.nernst(1.0, 2.0, 1, celsius=-274.0)


def test_ghk_matches_its_formula_and_joins_its_small_argument_branch():
    def direct(v, ci, co, z, celsius):
        x = z * v / (1000.0 * R * (celsius + 273.15) / F)
        q = lambda y: y / math.expm1(y) if y != 0.0 else 1.0
        return 0.001 * z * F * (ci * q(-x) - co * q(x))

    for v in (-80.0, -65.0, -1.0, 10.0, 40.0):
        assert mb.ghk(v, 5e-5, 2.0, 2) == pytest.approx(direct(v, 5e-5, 2.0, 2, 6.3), rel=1e-9)
    assert mb.ghk(0.0, 1.0, 1.0, 1) == 0.0          # equal concentrations at 0 mV: no current
    # below |x| = 1e-4 the factor is 1 - x/2, within x^2/12 of x/(e^x - 1)
    vt = 1000.0 * R * (6.3 + 273.15) / F
    for frac in (0.5e-4, 0.99e-4, 1.01e-4):
        assert mb.ghk(frac * vt, 1.0, 2.0, 1) == pytest.approx(direct(frac * vt, 1.0, 2.0, 1, 6.3), rel=1e-8)
    with pytest.raises(ValueError):
        mb.ghk(math.nan, 1.0, 2.0, 1)


def _hh_cells(ions=(), celsius=6.3, override=None):
    model = M.MicroModel(celsius=celsius, ions=ions)
    soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
    cells = M.add_population(model, [soma], 2, voltage=-65.0)
    for cell in cells:
        M.insert(cell, mb.builtin("hh"), sections="soma")
    if override:
        model.cells[cells[1].index - 1].ions.update(override)   # the cell's own reversal values
    return model


def _hh_column(layout, name):
    group = next(g for g in layout.groups if g.mechanism.name == "hh")
    return group.data[:, group.mechanism.field_index(name)]


def test_nernst_species_set_the_reversal_that_hh_reads():
    na = mb.IonSpecies("na", 1, 15.0, 145.0, nernst=True)
    layout = mb.build(_hh_cells([na], celsius=18.5))
    np.testing.assert_array_equal(_hh_column(layout, "ena"), mb.nernst(15.0, 145.0, 1, celsius=18.5))
    np.testing.assert_array_equal(_hh_column(layout, "ek"), -77.0)      # the default species keeps its constant
    # a fixed reversal is used as given; a cell's own override still wins
    layout = mb.build(_hh_cells([mb.IonSpecies("na", 1, 15.0, 145.0, 52.0)], override={"ena": 45.0}))
    np.testing.assert_array_equal(_hh_column(layout, "ena"), [52.0, 45.0])


def test_species_values_are_validated():
    with pytest.raises(ValueError):
        mb.IonSpecies("na", 1, -1.0, 140.0)
    with pytest.raises(ValueError):
        mb.IonSpecies("na", 1, 10.0, math.inf)


def test_a_nernst_species_runs_as_its_fixed_equivalent():
    """The reversal is fixed at build time, so the run equals one with that value as the
    species' constant reversal (CPU oracle, bit for bit)."""
    e = mb.nernst(12.0, 130.0, 1)
    a = mb.build(_hh_cells([mb.IonSpecies("na", 1, 12.0, 130.0, nernst=True)]))
    b = mb.build(_hh_cells([mb.IonSpecies("na", 1, 12.0, 130.0, e)]))
    ra, rb = oracle.run(a, 400, [1, 2]), oracle.run(b, 400, [1, 2])
    assert ra.status == 0 and rb.status == 0
    np.testing.assert_array_equal(ra.trace, rb.trace)


def test_point_processes_read_their_ion_reversal_too():
    """A point mechanism with USEION na READ ena (a descriptor such as compile_mod returns)
    gets the species' reversal, or its cell's own value, whatever its parameters say."""
    from mind_b200.mechanisms import Mechanism

    probe = Mechanism("NaProbe", "point", 99, ("gmax", "ena", "i"), (0.001, 0.0, 0.0), 1, 0, (("ena", "na"),))
    model = M.MicroModel(ions=[mb.IonSpecies("na", 1, 15.0, 145.0, nernst=True)])
    soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
    cells = M.add_population(model, [soma], 2, voltage=-65.0)
    model.cells[cells[1].index - 1].ions["ena"] = 45.0
    for cell in (cells[0], cells[1], cells[1]):
        M.add_pointprocess(cell, probe, params={"ena": -1.0})
    layout = mb.build(model)
    group = next(g for g in layout.groups if g.mechanism.name == "NaProbe")
    by_node = dict(zip(group.nodes.tolist(), group.data[:, 1].tolist()))
    assert len(group.nodes) == 3
    np.testing.assert_array_equal(sorted(group.data[:, 1]), sorted([mb.nernst(15.0, 145.0, 1), 45.0, 45.0]))
    assert by_node[min(by_node)] == mb.nernst(15.0, 145.0, 1)      # cell 1's node comes first
