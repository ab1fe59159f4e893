"""Regions coupled to the micro network (CPU): the oracle's Jansen-Rit mass against an
independent ODE solve, and the Poisson counts of the region inputs.

The GPU parity of the coupled network (cells, NetCons, regions, inputs and rate bins)
is in test_macro_gpu.py.
"""
import math

import numpy as np
from scipy.integrate import solve_ivp

import mind_b200 as mb
import oracle
from mind_b200 import model as M
from mind_b200.macro import JANSEN_RIT, MacroModel


def _one_passive_cell():
    model = M.MicroModel(celsius=6.3)
    soma = mb.Section("soma", label="soma", length=20.0, diameter=20.0, nseg=1)
    cell = M.add_population(model, [soma], 1, voltage=-65.0)[0]
    M.insert(cell, mb.builtin("pas"), sections="soma", params={"g": 1e-4, "e": -65.0})
    return model


def _jansen_rit(t, y, p):
    A, B, a, b, e0, r, v0, C = (JANSEN_RIT[k] for k in ("A", "B", "a", "b", "e0", "r", "v0", "C"))
    S = lambda v: 2.0 * e0 / (1.0 + math.exp(r * (v0 - v)))
    return [y[3], y[4], y[5],
            A * a * S(y[1] - y[2]) - 2 * a * y[3] - a * a * y[0],
            A * a * (p + 0.8 * C * S(C * y[0])) - 2 * a * y[4] - a * a * y[1],
            B * b * 0.25 * C * S(0.25 * C * y[0]) - 2 * b * y[5] - b * b * y[2]]


def test_jansen_rit_region_matches_an_independent_ode_solve():
    """RK4 at dt_macro = 0.1 ms reproduces the Jansen-Rit trajectory (p = p0, no coupling)."""
    model = _one_passive_cell()
    layout = mb.build(model)
    macro = MacroModel(dt_macro=0.1, bin_ms=1.0)
    y0 = [0.01, 2.0, 1.0, 0.0, 0.0, 0.0]
    macro.add_region(y0=y0, p0=200.0)
    steps = 4000  # 100 ms
    result = oracle.run(layout, steps, [], macro=macro)
    assert result.status == 0, result.message
    t = np.arange(result.macro_trace.shape[0]) * 1e-4
    sol = solve_ivp(_jansen_rit, (0.0, t[-1]), y0, t_eval=t, args=(200.0,), rtol=1e-11, atol=1e-12, method="DOP853")
    e0, r, v0 = JANSEN_RIT["e0"], JANSEN_RIT["r"], JANSEN_RIT["v0"]
    want = 2.0 * e0 / (1.0 + np.exp(r * (v0 - (sol.y[1] - sol.y[2]))))
    got = result.macro_trace[:, 0]
    assert np.max(np.abs(got - want)) < 1e-6 * max(1.0, np.max(np.abs(want)))
    assert np.ptp(got) > 0.1   # the mass moved


def test_region_input_counts_follow_the_poisson_law():
    for mu in (0.02, 0.3, 1.5):
        counts = np.array([oracle.region_input_count(1, 7, k, mu) for k in range(100_000)])
        assert abs(counts.mean() - mu) < 5 * math.sqrt(mu / counts.size) + (mu ** 4 / 24 if mu > 1 else 0.0) * 3
        assert abs(np.mean(counts == 0) - math.exp(-mu)) < 5 * math.sqrt(math.exp(-mu) / counts.size) + 1e-3
        assert counts.max() <= 3
    # streams are keyed by input and step
    a = [oracle.region_input_count(1, 0, k, 0.5) for k in range(200)]
    b = [oracle.region_input_count(1, 1, k, 0.5) for k in range(200)]
    assert a != b
