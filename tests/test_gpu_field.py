"""GPU: time-dependent Hamiltonian (the e_field pre-evaluate action):
H(t) = H - E(t) D- - conj(E(t)) D+ built on the device before every
derivative evaluation.  The oracle runs the classical RK4 with the same H(t)
set at every stage time; populations must agree to 1e-10 and one derivative
(heom_solve at time + step_size) to 1e-13."""
import numpy as np
import pytest

import heom_b200 as hb
from parity import assert_pops
import heom_oracle as ho

pytestmark = pytest.mark.gpu

INVCM = 1.986456217327470903861498336971e-23


def field(t, pulses):
    e = 0j
    for p in pulses:
        e += p["efield"] * np.exp(-(t - p["time_center"]) ** 2 / (2 * p["time_width"] ** 2)) * \
            np.exp(1j * (p["phase"] + p["frequency"] * t))
    return e


def setup(n, m, depth, seed):
    h = ho.synthetic_hamiltonian(n, seed)
    prob = ho.build_problem(ho.drude_system(n, depth, m, seed, h_invcm=h))
    rng = np.random.default_rng(seed + 7)
    dm = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) * 40.0 * INVCM  # J per unit field
    dp = dm.conj().T
    pulses = [dict(efield=1.0, time_center=15e-15, time_width=8e-15, frequency=2.0e14, phase=0.3),
              dict(efield=0.6, time_center=30e-15, time_width=5e-15, frequency=1.5e14, phase=-1.1)]
    return prob, dp, dm, pulses


def h_at(prob, h0, dp, dm, pulses, t):
    n = prob.states
    E = field(t, pulses)
    H = h0 - E * dm - np.conj(E) * dp
    flat = np.empty(n * n * 2)
    flat[0::2] = H.reshape(-1).real
    flat[1::2] = H.reshape(-1).imag
    prob.hamiltonian[:] = flat


def oracle_rk4_field(prob, dp, dm, pulses, y, t0, dt, steps, every):
    n = prob.states
    h0 = (prob.hamiltonian[0::2] + 1j * prob.hamiltonian[1::2]).reshape(n, n).copy()
    pops = [ho.populations(prob, y)]
    t = t0
    for s in range(steps):
        h_at(prob, h0, dp, dm, pulses, t)
        k1 = ho.derivative(prob, y)
        h_at(prob, h0, dp, dm, pulses, t + dt / 2)
        k2 = ho.derivative(prob, y + dt / 2 * k1)
        k3 = ho.derivative(prob, y + dt / 2 * k2)
        h_at(prob, h0, dp, dm, pulses, t + dt)
        k4 = ho.derivative(prob, y + dt * k3)
        y = y + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        t += dt
        if (s + 1) % every == 0:
            pops.append(ho.populations(prob, y))
    return np.array(pops), y


@pytest.mark.parametrize("n,m,depth", [(4, 2, 3), (7, 1, 3), (9, 1, 2)])
def test_field_propagation_matches_oracle(n, m, depth):
    prob, dp, dm, pulses = setup(n, m, depth, 11 + n)
    dt, steps, every, t0 = 1e-15, 60, 10, -5e-15
    y0 = prob.initial_state()
    ref, _ = oracle_rk4_field(prob, dp, dm, pulses, y0.copy(), t0, dt, steps, every)
    prob2 = ho.build_problem(ho.drude_system(n, depth, m, 11 + n, h_invcm=ho.synthetic_hamiltonian(n, 11 + n)))
    with hb.Heom.from_problem(prob2) as H:
        H.set_state(y0)
        H.set_field(dp, dm, pulses[0], pulses[1])
        H.set_time(t0)
        pops = H.populations_from_tops(H.propagate(dt, steps, every))
        assert abs(H.time() - (t0 + steps * dt)) <= 1e-28
    assert_pops(pops, ref)
    assert np.max(np.abs(pops[-1] - ref[0])) > 1e-3  # the field did something


def test_zero_field_is_the_time_independent_rk4():
    prob, dp, dm, pulses = setup(5, 2, 3, 3)
    for p in pulses:
        p["efield"] = 0.0
    y0 = prob.initial_state()
    with hb.Heom.from_problem(prob) as H:
        H.set_state(y0)
        ref = H.propagate(1e-15, 40, 10)
        H.set_state(y0)
        H.set_field(dp, dm, pulses[0], pulses[1])
        got = H.propagate(1e-15, 40, 10)
        H.clear_field()
        H.set_state(y0)
        again = H.propagate(1e-15, 40, 10)
    assert np.max(np.abs(got - ref)) <= 1e-13
    assert np.array_equal(again, ref)


def test_solve_evaluates_at_time_plus_step_size():
    prob, dp, dm, pulses = setup(6, 1, 2, 5)
    y = np.random.default_rng(2).normal(size=prob.state_len)
    n = prob.states
    h0 = (prob.hamiltonian[0::2] + 1j * prob.hamiltonian[1::2]).reshape(n, n).copy()
    time, step = 10e-15, 0.5e-15
    with hb.Heom.from_problem(prob) as H:
        H.set_field(dp, dm, pulses[0], pulses[1])
        bi, bo = H.buffer(), H.buffer()
        bi.write(y)
        H.solve(bi, bo, hb.SOLVE_PURE, time=time, step_size=step)
        out = bo.read()
        bi.close(), bo.close()
    h_at(prob, h0, dp, dm, pulses, time + step)
    ref = ho.derivative(prob, y)
    assert np.max(np.abs(out - ref)) <= 1e-13 * np.max(np.abs(ref))
