"""GPU: adjoint gradients (heom_adjoint_gradient) of a time-integrated
observable, J = sum_n w_n Re(sum_ij conj(O_ij) rho_n(i,j)).

Checked against
  * an FP64 reference gradient built independently of the adjoint code: the
    oracle's derivative applied to unit vectors gives L as a dense matrix,
    the RK4 polynomial R of dt L propagates y and its tangent
    dy_{n+1} = R dy_n + dR y_n; dL/dH from two oracle operators (L is affine
    in H), dL/dlambda and dL/dgamma by central differences of oracle
    operators.  Tolerances: 1e-9 (H, rho0; relative to the largest entry),
    1e-6 (lambda, gamma: the reference's own central-difference error).
  * central finite differences of GPU forward solves (h = 1e-4 cm^-1 for H
    and lambda, relative 1e-5 for gamma): 1e-5 relative.
  * torch.autograd through heom_torch.HeomObservableLoss.
"""
import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho

pytestmark = pytest.mark.gpu

INVCM = 1.986456217327470903861498336971e-23  # J per cm^-1


def dense_L(prob):
    n = prob.state_len // 2
    Lm = np.zeros((n, n), complex)
    for k in range(n):
        y = np.zeros(2 * n)
        y[2 * k] = 1.0
        out = ho.derivative(prob, y, threads=1)
        Lm[:, k] = out[0::2] + 1j * out[1::2]
    return Lm


def problem(h_cm, lam, inv, m, depth, omega=0.0):
    n = h_cm.shape[0]
    return ho.build_problem(ho.make_system(h_cm, [lam] * n, [inv] * n, [omega] * n, m, 300.0, depth))


def rk4_parts(A):
    I = np.eye(A.shape[0])
    return I + A + A @ A / 2 + A @ A @ A / 6 + A @ A @ A @ A / 24


def rk4_tangent_apply(A, dA, y):
    """dR y for R = I + A + A^2/2 + A^3/6 + A^4/24, by matrix-vector products."""
    Ay = A @ y
    A2y = A @ Ay
    A3y = A @ A2y
    d0 = dA @ y
    d1 = dA @ Ay
    d2 = dA @ A2y
    d3 = dA @ A3y
    return (d0 + (d1 + A @ d0) / 2 + (d2 + A @ d1 + A @ (A @ d0)) / 6 +
            (d3 + A @ d2 + A @ (A @ d1) + A @ (A @ (A @ d0))) / 24)


def reference_gradients(h_cm, lam, inv, m, depth, dt_fs, steps, rho0, obs, w, omega=0.0, entries=None):
    n = h_cm.shape[0]
    base = problem(h_cm, lam, inv, m, depth, omega)
    L = dense_L(base)
    dt = dt_fs * 1e-15
    A = dt * L
    R = rk4_parts(A)
    y0 = np.zeros(L.shape[0], complex)
    y0[: n * n] = rho0.reshape(-1)
    c = np.zeros_like(y0)
    c[: n * n] = obs.reshape(-1)
    ys = [y0]
    for k in range(steps):
        ys.append(R @ ys[-1])
    J = sum(w[k] * np.real(np.vdot(c, ys[k])) for k in range(steps + 1))

    def tangent(dL):
        dA = dt * dL
        dy = np.zeros_like(y0)
        dJ = 0.0
        for k in range(steps + 1):
            dJ += w[k] * np.real(np.vdot(c, dy))
            if k < steps:
                dy = R @ dy + rk4_tangent_apply(A, dA, ys[k])
        return dJ

    if entries is None:
        entries = [(a, b) for a in range(n) for b in range(n)]
    gh = {}
    for (a, b) in entries:
        v = 0.0
        for part in (1.0, 1j):
            hp = h_cm.astype(complex).copy()
            hp[a, b] += part * 1.0
            dL = dense_L(problem(hp, lam, inv, m, depth, omega)) - L  # affine in H: exact
            v += part * tangent(dL)
        gh[(a, b)] = v
    dl = 1e-4 * lam
    gl = tangent((dense_L(problem(h_cm, lam + dl, inv, m, depth, omega)) -
                  dense_L(problem(h_cm, lam - dl, inv, m, depth, omega))) / (2 * dl))
    g = 1.0 / inv
    dg = 1e-5 * g
    gg = tangent((dense_L(problem(h_cm, lam, 1.0 / (g + dg), m, depth, omega)) -
                  dense_L(problem(h_cm, lam, 1.0 / (g - dg), m, depth, omega))) / (2 * dg))
    # dJ/dy0 = sum_n w_n (R^H)^n c
    adj = np.zeros_like(y0)
    v = c.copy()
    RH = R.conj().T
    for k in range(steps + 1):
        adj += w[k] * v
        v = RH @ v
    return J, gh, gl, gg, adj[: n * n].reshape(n, n)


def complex_h(n, seed):
    h = ho.synthetic_hamiltonian(n, seed).astype(complex)
    rng = np.random.default_rng(seed + 100)
    iu = np.triu_indices(n, 1)
    im = rng.normal(0.0, 20.0, size=len(iu[0]))
    h[iu] += 1j * im
    h[(iu[1], iu[0])] -= 1j * im
    return h


CASES = {
    # name: (H, lambda, invnu, matsubaras, depth, omega)
    "n3_m2_d2": (ho.synthetic_hamiltonian(3, 1), 35.0, 50.0, 2, 2, 0.0),
    "n4_m1_d3": (ho.synthetic_hamiltonian(4, 2), 35.0, 50.0, 1, 3, 0.0),
    "n3_complex_omega": (complex_h(3, 3), 20.0, 80.0, 2, 2, 15.0),
    "n9_m1_d1": (ho.synthetic_hamiltonian(9, 4), 35.0, 50.0, 1, 1, 0.0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_adjoint_matches_dense_fp64_reference(case):
    h, lam, inv, m, depth, omega = CASES[case]
    n = h.shape[0]
    steps, dt_fs = 30, 1.0
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[min(2, n - 1), min(2, n - 1)] = 1.0
    w = hb.trapezoid_weights(steps, dt_fs)
    entries = None if n <= 4 else [(0, 0), (2, 2), (8, 8), (0, 1), (1, 0), (3, 7), (2, 6)]
    J, gh, gl, gg, g0 = reference_gradients(h, lam, inv, m, depth, dt_fs, steps, rho0, obs, w, omega, entries)
    system = hb.System(h, [lam] * n, [inv] * n, [omega] * n, m, 300.0, depth)
    with hb.Adjoint(system) as A:
        out = A.gradient(rho0, obs, w, dt_fs * 1e-15, steps)
    assert abs(out["loss"] - J) <= 1e-12 * max(1.0, abs(J))
    scale = max(abs(v) for v in gh.values())
    for (a, b), v in gh.items():
        assert abs(out["h"][a, b] - v) <= 1e-9 * scale, (a, b, out["h"][a, b], v)
    assert abs(out["lambda"] - gl) <= 1e-6 * abs(gl)
    assert abs(out["gamma"] - gg) <= 1e-6 * abs(gg)
    assert np.max(np.abs(out["rho0"] - g0)) <= 1e-9 * np.max(np.abs(g0))


def loss_gpu(h, lam, inv, m, depth, dt_fs, steps, rho0_top, obs_idx, w):
    n = h.shape[0]
    system = hb.System(h, [lam] * n, [inv] * n, [0.0] * n, m, 300.0, depth)
    with hb.from_system(system, scheme="product") as H:
        H.set_top(rho0_top)
        tops = H.propagate(dt_fs * 1e-15, steps, 1)
    return float(np.dot(w, tops[:, 2 * obs_idx]))


def test_adjoint_matches_gpu_central_differences():
    n, m, depth, steps, dt_fs = 7, 1, 3, 200, 1.0
    h = ho.synthetic_hamiltonian(n, 12)
    lam, inv = 35.0, 50.0
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[2, 2] = 1.0
    w = hb.trapezoid_weights(steps, dt_fs)
    system = hb.System(h, [lam] * n, [inv] * n, [0.0] * n, m, 300.0, depth)
    with hb.Adjoint(system) as A:
        out = A.gradient(rho0, obs, w, dt_fs * 1e-15, steps)
    top0 = rho0.reshape(-1).view(np.float64).copy()
    idx = 2 * n + 2
    f = lambda hh, ll=lam, ii=inv: loss_gpu(hh, ll, ii, m, depth, dt_fs, steps, top0, idx, w)
    assert abs(f(h) - out["loss"]) <= 1e-12 * abs(out["loss"])
    hstep = 1e-4
    for (a, b) in [(0, 0), (2, 2), (5, 5), (0, 1), (2, 4)]:
        e = np.zeros((n, n))
        e[a, b] = e[b, a] = 1.0  # symmetric perturbation (a site energy or a coupling)
        fd = (f(h + hstep * e) - f(h - hstep * e)) / (2 * hstep)
        ad = out["h"][a, b].real + (out["h"][b, a].real if a != b else 0.0)
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.max(np.abs(out["h"].real))), (a, b, ad, fd)
    fd_l = (f(h, lam + hstep) - f(h, lam - hstep)) / (2 * hstep)
    assert abs(out["lambda"] - fd_l) <= 1e-5 * abs(fd_l)
    g = 1.0 / inv
    dg = 1e-5 * g
    fd_g = (f(h, lam, 1.0 / (g + dg)) - f(h, lam, 1.0 / (g - dg))) / (2 * dg)
    assert abs(out["gamma"] - fd_g) <= 1e-5 * abs(fd_g)


def test_adjoint_through_torch_autograd():
    import torch
    from heom_torch import HeomObservableLoss
    n, steps, dt_fs = 4, 60, 1.0
    h0 = ho.synthetic_hamiltonian(n, 21)
    e = torch.tensor(np.diag(h0).copy(), dtype=torch.float64, requires_grad=True)
    iu = np.triu_indices(n, 1)
    cpl = torch.tensor(h0[iu].copy(), dtype=torch.float64, requires_grad=True)
    lam = torch.tensor(35.0, dtype=torch.float64, requires_grad=True)
    gam = torch.tensor(1.0 / 50.0, dtype=torch.float64, requires_grad=True)
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[2, 2] = 1.0
    spec = dict(depth=3, matsubaras=2, temperature=300.0, dt_fs=dt_fs, steps=steps, rho0=rho0,
                observable=obs, weights=hb.trapezoid_weights(steps, dt_fs))

    def build(e_, c_):
        H = torch.diag(e_)
        U = torch.zeros(n, n, dtype=torch.float64)
        U[iu] = c_
        return H + U + U.T

    J = HeomObservableLoss.apply(build(e, cpl), lam, gam, spec)
    J.backward()
    # chain rule by hand: symmetric couplings gather both entries
    system = hb.System(h0, [35.0] * n, [50.0] * n, [0.0] * n, 2, 300.0, 3)
    with hb.Adjoint(system) as A:
        out = A.gradient(rho0, obs, spec["weights"], dt_fs * 1e-15, steps)
    gr = out["h"].real
    assert np.allclose(e.grad.numpy(), np.diag(gr), rtol=1e-13, atol=0)
    assert np.allclose(cpl.grad.numpy(), gr[iu] + gr.T[iu], rtol=1e-13, atol=0)
    assert abs(float(lam.grad) - out["lambda"]) <= 1e-13 * abs(out["lambda"])
    assert abs(float(gam.grad) - out["gamma"]) <= 1e-13 * abs(out["gamma"])


def test_batched_adjoint_matches_single_instance_sweeps():
    # static-disorder realisations (different H, two depths) in one sweep
    n, m, steps, dt_fs = 5, 2, 40, 1.0
    base = ho.synthetic_hamiltonian(n, 31)
    rng = np.random.default_rng(5)
    systems = []
    for k in range(3):
        h = base.copy()
        h[np.diag_indices(n)] += rng.normal(0.0, 100.0, size=n)
        systems.append(hb.System(h, [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, 2 + k % 2))
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((3, n, n), complex)
    for k in range(3):
        obs[k, k, k] = 1.0  # a different site population per instance
    w = hb.trapezoid_weights(steps, dt_fs)
    with hb.Adjoint(systems) as A:
        out = A.gradient(rho0, obs, w, dt_fs * 1e-15, steps)
    for k in range(3):
        with hb.Adjoint(systems[k]) as A1:
            ref = A1.gradient(rho0, obs[k], w, dt_fs * 1e-15, steps)
        assert abs(out["loss"][k] - ref["loss"]) <= 1e-14 * abs(ref["loss"])
        assert np.max(np.abs(out["h"][k] - ref["h"])) <= 1e-12 * np.max(np.abs(ref["h"]))
        assert abs(out["lambda"][k] - ref["lambda"]) <= 1e-12 * abs(ref["lambda"])
        assert abs(out["gamma"][k] - ref["gamma"]) <= 1e-12 * abs(ref["gamma"])
        assert np.max(np.abs(out["rho0"][k] - ref["rho0"])) <= 1e-13 * np.max(np.abs(ref["rho0"]))


def test_adjoint_graphs_equal_eager_launches_and_survive_regrowth():
    # the captured per-segment graphs and eager launches run the same kernels in
    # the same order; a longer second call reallocates and recaptures
    n, steps = 4, 50
    system = hb.System(ho.synthetic_hamiltonian(n, 8), [35.0] * n, [50.0] * n, [0.0] * n, 2, 300.0, 3)
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[1, 1] = 1.0
    outs = []
    for graphs in (True, False):
        with hb.Adjoint(system, graphs=graphs) as A:
            A.gradient(rho0, obs, hb.trapezoid_weights(10, 1.0), 1e-15, 10)
            outs.append(A.gradient(rho0, obs, hb.trapezoid_weights(steps, 1.0), 1e-15, steps))
    a, b = outs
    assert a["loss"] == b["loss"]
    assert np.array_equal(a["h"], b["h"]) and np.array_equal(a["rho0"], b["rho0"])
    assert a["lambda"] == b["lambda"] and a["gamma"] == b["gamma"]


@pytest.mark.parametrize("limit_states,free_slots", [(8, 0), (11, 3), (20, 12)])
def test_recursive_checkpointing_is_bit_identical_to_sqrt_layout(limit_states, free_slots):
    # a memory limit below the sqrt layout's states switches the sweep to
    # recursive checkpointing: the same kernels in the same backward order
    n, steps = 5, 47
    systems = [hb.System(ho.synthetic_hamiltonian(n, 60 + k), [35.0] * n, [50.0] * n, [0.0] * n, 2, 300.0, 2 + k)
               for k in range(2)]
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((2, n, n), complex)
    obs[0, 1, 1] = obs[1, 2, 2] = 1.0
    w = hb.trapezoid_weights(steps, 1.0)
    with hb.Adjoint(systems) as A:
        ref = A.gradient(rho0, obs, w, 1e-15, steps)
        assert A.recursive_slots() == 0
        pairs = n * (n - 1) // 2 + (n + 1) // 2
        st = sum(int(hb.build_tables(s)["matrices"]) for s in systems) * pairs * 32  # bytes per state
        A.set_memory_limit(limit_states * st)
        out = A.gradient(rho0, obs, w, 1e-15, steps)
        assert A.recursive_slots() == free_slots + 1
        A.set_memory_limit(0)
        again = A.gradient(rho0, obs, w, 1e-15, steps)
        assert A.recursive_slots() == 0
    for o in (out, again):
        assert np.array_equal(o["loss"], ref["loss"])
        assert np.array_equal(o["h"], ref["h"]) and np.array_equal(o["rho0"], ref["rho0"])
        assert np.array_equal(o["lambda"], ref["lambda"]) and np.array_equal(o["gamma"], ref["gamma"])


def test_gradient_subset_skips_work_and_keeps_bits():
    # NULL outputs skip their accumulation; the others are bit-identical
    n, steps = 9, 30
    system = hb.System(ho.synthetic_hamiltonian(n, 17), [35.0] * n, [50.0] * n, [0.0] * n, 2, 300.0, 2)
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[2, 2] = 1.0
    w = hb.trapezoid_weights(steps, 1.0)
    with hb.Adjoint(system) as A:
        full = A.gradient(rho0, obs, w, 1e-15, steps)
        only_h = A.gradient(rho0, obs, w, 1e-15, steps, outputs=("h",))
        only_bath = A.gradient(rho0, obs, w, 1e-15, steps, outputs=("lambda", "gamma"))
    assert only_h["lambda"] is None and only_h["rho0"] is None and only_bath["h"] is None
    assert np.array_equal(only_h["h"], full["h"]) and only_h["loss"] == full["loss"]
    assert only_bath["lambda"] == full["lambda"] and only_bath["gamma"] == full["gamma"]


def test_adjoint_at_full_size_matches_oracle_tangents():
    """The adjoint of the 7-site, depth-8 hierarchy (6435 ADOs; the size of the
    adjoint benchmark) against an FP64 reference gradient that shares no code
    with it: forward-mode tangents of the oracle's RK4 steps,
      dk1 = L dy + L' y, ..., dy_{n+1} = dy + dt/6 (dk1 + 2 dk2 + 2 dk3 + dk4),
    with L' the derivative of the operator along the parameter.  For an H
    entry L' is exact (L is affine in H: L' v = i/hbar (v E - E v) on every
    ADO; checked against a difference of two oracle operators); for lambda
    and gamma it is a central difference of oracle operators (steps 1e-4
    relative), whose O(step^2) error bounds the comparison at 1e-6.
    50 RK4 steps of 1 fs; loss = trapezoid integral of the site-3 population;
    gradients w.r.t. the 7 site energies, 3 couplings (symmetric), lambda and
    gamma."""
    n, depth, steps, dt_fs = 7, 8, 50, 1.0
    dt = dt_fs * 1e-15
    h = ho.synthetic_hamiltonian(n, 44)
    lam, inv = 35.0, 50.0
    w = hb.trapezoid_weights(steps, dt_fs)
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[2, 2] = 1.0

    with hb.Adjoint(hb.System(h, [lam] * n, [inv] * n, [0.0] * n, 1, 300.0, depth)) as A:
        gpu = A.gradient(rho0, obs, w, dt, steps)

    base = problem(h, lam, inv, 1, depth)
    L = lambda prob, v: ho.derivative(prob, v)
    y = base.initial_state()
    j_idx = 2 * (2 * n + 2)  # Re rho(2, 2) of the top ADO
    stages = []  # stage inputs of every step, for the tangents
    J = w[0] * y[j_idx]
    for k in range(steps):
        k1 = L(base, y)
        s2 = y + 0.5 * dt * k1
        k2 = L(base, s2)
        s3 = y + 0.5 * dt * k2
        k3 = L(base, s3)
        s4 = y + dt * k3
        k4 = L(base, s4)
        stages.append((y, s2, s3, s4))
        y = y + dt / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        J += w[k + 1] * y[j_idx]
    assert abs(J - gpu["loss"]) <= 1e-12 * abs(J)

    def tangent(dL):
        dy = np.zeros_like(y)
        dJ = 0.0
        for k in range(steps):
            dJ += w[k] * dy[j_idx]
            y0, s2, s3, s4 = stages[k]
            dk1 = L(base, dy) + dL(y0)
            dk2 = L(base, dy + 0.5 * dt * dk1) + dL(s2)
            dk3 = L(base, dy + 0.5 * dt * dk2) + dL(s3)
            dk4 = L(base, dy + dt * dk3) + dL(s4)
            dy = dy + dt / 6.0 * (dk1 + 2.0 * dk2 + 2.0 * dk3 + dk4)
        return dJ + w[steps] * dy[j_idx]

    hbar = 1.05457148e-34  # the reference's value (common.cl, constants.hpp)

    def comm_dir(E_cm):
        E = E_cm * INVCM

        def apply(v):
            s = v.view(np.complex128).reshape(-1, n, n)
            return (1j / hbar * (s @ E - E @ s)).reshape(-1).view(np.float64)
        return apply

    # the exact H direction against a difference of two oracle operators
    v = np.random.default_rng(5).normal(size=base.state_len)
    E = np.zeros((n, n))
    E[1, 4] = E[4, 1] = 1.0
    diff = L(problem(h + E, lam, inv, 1, depth), v) - L(base, v)
    assert np.max(np.abs(comm_dir(E)(v) - diff)) <= 1e-9 * np.max(np.abs(diff))

    g_h = gpu["h"].real
    entries = [(a, a) for a in range(n)] + [(0, 1), (1, 4), (2, 6)]
    for (a, b) in entries:
        E = np.zeros((n, n))
        E[a, b] = E[b, a] = 1.0
        ref = tangent(comm_dir(E))
        got = g_h[a, b] + (g_h[b, a] if a != b else 0.0)
        assert abs(got - ref) <= 1e-9 * max(abs(ref), 1e-3 * np.max(np.abs(g_h))), (a, b, got, ref)

    dl = 1e-4 * lam
    pl, ml = problem(h, lam + dl, inv, 1, depth), problem(h, lam - dl, inv, 1, depth)
    ref_l = tangent(lambda v: (L(pl, v) - L(ml, v)) / (2 * dl))
    assert abs(gpu["lambda"] - ref_l) <= 1e-6 * abs(ref_l), (gpu["lambda"], ref_l)
    g = 1.0 / inv
    dg = 1e-4 * g
    pg, mg = problem(h, lam, 1.0 / (g + dg), 1, depth), problem(h, lam, 1.0 / (g - dg), 1, depth)
    ref_g = tangent(lambda v: (L(pg, v) - L(mg, v)) / (2 * dg))
    assert abs(gpu["gamma"] - ref_g) <= 1e-6 * abs(ref_g), (gpu["gamma"], ref_g)
