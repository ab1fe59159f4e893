"""Known-answer tests of the oracle's physics (CPU).

The reference ships no tests or fixtures, so the FP64 oracle is pinned here
against closed forms and an independent ODE integration:
* a passive compartment decays as backward Euler predicts,
  v_n = e + (v0 - e) / (1 + dt * 1000 g / cm)^n (units: mV, ms, S/cm2, uF/cm2);
* discretization of a cylinder gives pi d L / nseg per segment and
  pi d^2 / (0.04 Ra step) uS between segments;
* a Hodgkin-Huxley soma driven by IClamp fires where scipy's tight
  integration of the same ODE fires (within the method's O(dt) error);
* NetStim with noise 0 fires at start, start + interval, ...; an event at
  time t enters the first step whose mid-step cutoff m dt + dt/2 is >= t.
"""
import math

import numpy as np
import pytest

import mind_b200 as mb
import oracle
from mind_b200 import model as M


def single_section(nseg=1, mech="pas", params=None, L=20.0, diam=20.0):
    model = M.MicroModel(celsius=6.3)
    soma = mb.Section("soma", label="soma", length=L, diameter=diam, nseg=nseg, Ra=100.0, cm=1.0)
    cell = M.add_population(model, [soma], 1, voltage=-65.0)[0]
    M.insert(cell, mb.builtin(mech), sections="soma", params=params or {})
    return model, cell


def test_secondorder_is_crank_nicolson():
    """secondorder 1 and 2 (C/(dt/2) in the matrix, v += 2 x) step a passive compartment by
    the trapezoidal rule, v_n = e + (v0 - e) ((1 - k/2)/(1 + k/2))^n with k = dt 1000 g / cm,
    and its error against the exact exponential shrinks as dt^2 where backward Euler's
    shrinks as dt."""
    g, e, T = 1.0e-3, -70.0, 10.0
    errors = {}
    for order in (0, 1, 2):
        for dt in (0.1, 0.05):
            model, cell = single_section(params={"g": g, "e": e})
            layout = mb.build(model, dt_micro=dt, secondorder=order)
            steps = int(round(T / dt))
            ref = oracle.run(layout, steps, [layout.voltage_node(1)])
            assert ref.status == 0
            k = dt * 1000.0 * g / 1.0
            if order:
                n = np.arange(steps + 1)
                np.testing.assert_allclose(ref.trace[:, 0], e + (-65.0 - e) * ((1 - k / 2) / (1 + k / 2)) ** n,
                                           rtol=0, atol=1e-9)
            errors[order, dt] = abs(ref.trace[-1, 0] - (e + (-65.0 - e) * math.exp(-T * 1000.0 * g / 1.0)))
    assert 1.8 < errors[0, 0.1] / errors[0, 0.05] < 2.2
    assert 3.6 < errors[1, 0.1] / errors[1, 0.05] < 4.4
    assert errors[1, 0.05] < 0.05 * errors[0, 0.05] and errors[2, 0.05] == errors[1, 0.05]


def test_passive_decay_matches_backward_euler():
    g, e, dt, steps = 1.0e-3, -70.0, 0.025, 400
    model, cell = single_section(params={"g": g, "e": e})
    layout = mb.build(model, dt_micro=dt)
    node = layout.voltage_node(1)
    ref = oracle.run(layout, steps, [node])
    assert ref.status == 0
    n = np.arange(steps + 1)
    want = e + (-65.0 - e) / (1.0 + dt * 1000.0 * g / 1.0) ** n
    assert np.max(np.abs(ref.trace[:, 0] - want)) < 1e-9


def test_cylinder_discretization_closed_form():
    sec = mb.Section("dend", length=500.0, diameter=2.0, nseg=50, Ra=100.0, cm=1.0)
    m = mb.discretize([sec])
    seg = m.section_nodes["dend"][:-1] - 1
    step = 10.0
    np.testing.assert_allclose(m.area[seg], math.pi * 2.0 * step, rtol=1e-13)
    np.testing.assert_allclose(m.axial[seg[1:]], math.pi * 4.0 / (0.04 * 100.0 * step), rtol=1e-13)
    assert m.axial[seg[0]] == pytest.approx(2.0 * math.pi * 4.0 / (0.04 * 100.0 * step), rel=1e-13)
    np.testing.assert_allclose(m.capacitance[seg], 1.0 * m.area[seg] * 1e-5, rtol=0)
    assert np.all(m.parent[1:] < np.arange(2, len(m.parent) + 1))   # parents first


def test_vectorized_and_pt3d_geometry_agree_exactly():
    plain = mb.Section("a", length=123.0, diameter=1.7, nseg=7, Ra=80.0, cm=0.9)
    pts = mb.Section("a", points=[mb.Point3D(0, 0, 0, 1.7), mb.Point3D(123.0, 0, 0, 1.7)], nseg=7, Ra=80.0, cm=0.9)
    a, b = mb.discretize([plain]), mb.discretize([pts])
    for field in ("area", "axial", "capacitance", "diameter"):
        np.testing.assert_array_equal(getattr(a, field), getattr(b, field))


def hh_ode_spikes(amp_nA, delay, duration, t_stop, area_um2):
    from scipy.integrate import solve_ivp

    cm, ena, ek, gna, gk, gl, el = 1.0, 50.0, -77.0, 0.12, 0.036, 0.0003, -54.3
    area_cm2 = area_um2 * 1e-8
    i_density = amp_nA * 1e-6 / area_cm2  # mA/cm2

    def vtrap(x, y):
        return y * (1 - x / y / 2) if abs(x / y) < 1e-6 else x / (math.exp(x / y) - 1)

    def rates(v):
        am, bm = 0.1 * vtrap(-(v + 40), 10), 4 * math.exp(-(v + 65) / 18)
        ah, bh = 0.07 * math.exp(-(v + 65) / 20), 1 / (math.exp(-(v + 35) / 10) + 1)
        an, bn = 0.01 * vtrap(-(v + 55), 10), 0.125 * math.exp(-(v + 65) / 80)
        return am, bm, ah, bh, an, bn

    def f(t, y):
        v, m, h, n = y
        am, bm, ah, bh, an, bn = rates(v)
        i_ion = gna * m ** 3 * h * (v - ena) + gk * n ** 4 * (v - ek) + gl * (v - el)
        i_inj = i_density if delay <= t < delay + duration else 0.0
        return [1000.0 * (i_inj - i_ion) / cm, am * (1 - m) - bm * m, ah * (1 - h) - bh * h, an * (1 - n) - bn * n]

    am, bm, ah, bh, an, bn = rates(-65.0)
    y0 = [-65.0, am / (am + bm), ah / (ah + bh), an / (an + bn)]
    sol = solve_ivp(f, (0, t_stop), y0, method="LSODA", rtol=1e-9, atol=1e-11, max_step=0.01, dense_output=True)
    t = np.arange(0, t_stop, 0.001)
    v = sol.sol(t)[0]
    up = np.nonzero((v[1:] > -10.0) & (v[:-1] <= -10.0))[0]
    return t[up + 1]


def hh_soma_spikes(dt):
    model, cell = single_section(mech="hh")
    M.add_pointprocess(cell, mb.builtin("IClamp"), section="soma", x=0.5,
                       params={"del": 5.0, "dur": 40.0, "amp": 0.1})
    M.register_spike_source(cell, threshold=-10.0)
    layout = mb.build(model, dt_micro=dt)
    ref = oracle.run(layout, int(round(50.0 / dt)), [layout.voltage_node(1)])
    assert ref.status == 0
    return ref.spike_times, layout.area[layout.voltage_node(1) - 1]


def test_hh_soma_spike_times_match_ode():
    """Same spike count as the ODE, first spike within 0.05 ms, ISIs within 1%, O(dt) convergence."""
    got, area = hh_soma_spikes(0.025)
    finer, _ = hh_soma_spikes(0.0125)
    want = hh_ode_spikes(0.1, 5.0, 40.0, 50.0, area)
    assert len(want) >= 2 and len(got) == len(want) == len(finer)
    assert abs(got[0] - want[0]) < 0.05
    np.testing.assert_allclose(np.diff(got), np.diff(want), rtol=0.01)
    assert np.max(np.abs(finer - want)) < 0.65 * np.max(np.abs(got - want))


def test_netstim_regular_train_and_delivery_bin():
    model, cell = single_section(mech="pas", params={"g": 1e-4, "e": -65.0})
    syn = M.add_pointprocess(cell, mb.builtin("ExpSyn"), section="soma", x=0.5, params={"tau": 2.0, "e": 0.0})
    stim = M.add_pointprocess(model, mb.builtin("NetStim"),
                              params={"interval": 10.0, "number": 3, "start": 5.0, "noise": 0.0})
    M.connect(stim, syn, weight=0.001, delay=0.0)
    layout = mb.build(model)
    ref = oracle.run(layout, 1200, [layout.voltage_node(1)])
    np.testing.assert_array_equal(ref.spike_times, [5.0, 15.0, 25.0])
    v = ref.trace[:, 0]
    # The event at t = 5.0 joins step 200 (200*dt + dt/2 >= 5.0 > 199*dt + dt/2): the
    # first sample that moves is the boundary after step 200.
    moved = np.nonzero(np.abs(v - v[0]) > 1e-12)[0]
    assert moved[0] == 201


def test_config1_poisson_counts():
    from mind_b200 import networks

    layout = mb.build(networks.config1())
    ref = oracle.run(layout, 4000, [])
    assert ref.status == 0
    stims = ref.spike_sids >= 64
    assert abs(int(stims.sum()) - 640) < 4 * math.sqrt(640)   # 640 NetStims at 10 Hz for 0.1 s


def test_alpha_synapse_matches_linearized_backward_euler():
    """AlphaSynapse (mod/AlphaSynapse.mod) on an isopotential soma with pas: the oracle's
    voltage equals the one-compartment update v += -I(v) / (C/dt + G) with the synaptic
    conductance gmax alpha((t + dt/2 - onset)/tau) of each step."""
    dt, steps = 0.025, 600
    gp, ep = 2.0e-4, -65.0
    onset, tau, gmax, es = 2.0, 1.5, 0.004, 0.0
    model, cell = single_section(params={"g": gp, "e": ep})
    M.add_pointprocess(cell, mb.builtin("AlphaSynapse"), section="soma", x=0.5,
                       params={"onset": onset, "tau": tau, "gmax": gmax, "e": es})
    layout = mb.build(model, dt_micro=dt)
    node = layout.voltage_node(1)
    ref = oracle.run(layout, steps, [node])
    assert ref.status == 0, ref.message
    area = layout.area[node - 1]
    cap = layout.capacitance[node - 1]
    g_pas = gp * area * 0.01
    v = np.empty(steps + 1)
    v[0] = -65.0
    for n in range(steps):
        x = (n * dt + 0.5 * dt - onset) / tau
        gs = gmax * (x * math.exp(1.0 - x) if 0.0 <= x <= 10.0 else 0.0)
        current = g_pas * (v[n] - ep) + gs * (v[n] - es)
        v[n + 1] = v[n] - current / (cap / dt + g_pas + gs)
    assert np.max(np.abs(ref.trace[:, 0] - v)) < 1e-9
    assert np.max(v) > -60.0        # the synapse depolarised the soma
