"""The C++ build planner (mind_discretize) against the numpy restatement of MIND.jl's
discretize (oracle/geometry.py): node parents, areas, diameters, axial conductances,
capacitances, edge lengths and section node maps equal bit for bit on seeded random
morphologies -- cylinders and pt3d sections, sections attached by either end, at
interior, 0 and 1 positions of their parent -- and invalid morphologies are refused."""
import numpy as np
import pytest

import geometry
import mind_b200 as mb
from mind_b200 import networks


def random_morphology(rng, n_sections=40, pt3d=0.5):
    sections = [mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)]
    for k in range(1, n_sections):
        parent = sections[int(rng.integers(0, k))].name
        px = float(rng.choice([0.0, 1.0, rng.uniform(0.0, 1.0)]))
        cx = float(rng.choice([0.0, 1.0], p=[0.8, 0.2]))
        nseg = int(rng.integers(1, 12))
        if rng.uniform() < pt3d:
            m = int(rng.integers(2, 8))
            xyz = np.cumsum(rng.normal(0.0, 8.0, (m, 3)), axis=0)
            diam = rng.uniform(0.3, 4.0, m)
            if m >= 3 and rng.uniform() < 0.3:
                xyz[1] = xyz[0]                           # a zero-length span
            points = [mb.Point3D(*xyz[j], float(diam[j])) for j in range(m)]
            sections.append(mb.Section(f"s{k}", parent=parent, parent_x=px, child_x=cx, nseg=nseg, points=points,
                                       Ra=float(rng.uniform(50, 200)), cm=float(rng.uniform(0.5, 2.0))))
        else:
            sections.append(mb.Section(f"s{k}", parent=parent, parent_x=px, child_x=cx, nseg=nseg,
                                       length=float(rng.lognormal(3.5, 0.7)), diameter=float(rng.uniform(0.2, 5.0)),
                                       Ra=float(rng.uniform(50, 200)), cm=float(rng.uniform(0.5, 2.0))))
    order = rng.permutation(len(sections))              # input order need not put parents first
    return [sections[i] for i in order]


def assert_same(a, b):
    for name in ("parent", "area", "diameter", "axial", "capacitance", "edge_length"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape and np.array_equal(x, y), name
    assert a.section_starts == b.section_starts
    assert a.section_nodes.keys() == b.section_nodes.keys()
    for k in a.section_nodes:
        np.testing.assert_array_equal(a.section_nodes[k], b.section_nodes[k])


@pytest.mark.parametrize("seed", range(12))
def test_cpp_planner_equals_the_numpy_restatement(seed):
    rng = np.random.default_rng(seed)
    sections = random_morphology(rng, pt3d=[0.0, 0.5, 1.0][seed % 3])
    assert_same(mb.discretize(sections), geometry.discretize(sections))


def test_benchmark_binary_trees_plan_identically():
    rng = np.random.default_rng(3)
    for size in (100, 400, 1000):
        soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
        secs = networks._binary_tree(rng, size, soma)
        assert_same(mb.discretize(secs), geometry.discretize(secs))


@pytest.mark.parametrize("mutate, message", [
    (lambda s: setattr(s[1], "parent", "nowhere"), "unknown parent"),
    (lambda s: (setattr(s[0], "parent", "s1"), setattr(s[1], "parent", "soma")), "cycle"),
])
def test_invalid_morphologies_are_refused(mutate, message):
    sections = [mb.Section("soma", length=20.0, diameter=20.0), mb.Section("s1", parent="soma", length=50.0)]
    mutate(sections)
    with pytest.raises(ValueError, match=message):
        mb.discretize(sections)
