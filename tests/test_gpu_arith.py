"""GPU: hierarchy arithmetic (hierarchy_arithmetic_*.cl) and host
pre-evaluate actions (ode::add_pre_evaluate_action).

The arithmetic follows the reference kernels' operation order (complex
products a.x*b.x - a.y*b.y, sums in k order, no contraction), so results are
compared bit for bit with numpy doing the same operations."""
import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho

pytestmark = pytest.mark.gpu


def cplx(y):
    return y[0::2] + 1j * y[1::2]


def cmul(x, y):
    """Complex product as the reference kernels form it, in plain float64
    operations (numpy's own complex multiply may order or fuse them)."""
    x, y = np.asarray(x, complex), np.asarray(y, complex)
    return (x.real * y.real - x.imag * y.imag) + 1j * (x.real * y.imag + x.imag * y.real)


def real(z):
    out = np.empty(z.size * 2)
    out[0::2] = z.real
    out[1::2] = z.imag
    return out


@pytest.mark.parametrize("n,m,depth", [(4, 2, 2), (5, 1, 3), (9, 1, 2)])
def test_hierarchy_arithmetic_bit_exact(n, m, depth):
    sysd = hb.System(ho.synthetic_hamiltonian(n, n), [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, depth)
    rng = np.random.default_rng(n)
    with hb.from_system(sysd) as H:
        nodes = H.matrices
        a, b = rng.normal(size=H.state_len), rng.normal(size=H.state_len)
        M = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        f = 0.3 - 1.7j
        ba, bb, bo = H.buffer(), H.buffer(), H.buffer()
        za, zb = cplx(a), cplx(b)

        def run(op, **kw):
            ba.write(a)
            bb.write(b)
            H.hierarchy_op(op, ba, bb, bo, **kw)
            return cplx(bo.read())

        assert np.array_equal(run("add"), za + zb)
        assert np.array_equal(run("subtract"), za - zb)
        assert np.array_equal(run("dot_product"), cmul(za, np.conj(zb)))
        assert np.array_equal(run("scale", factor=f), cmul(f, za))
        A = za.reshape(nodes, n, n)
        left = np.zeros_like(A)
        right = np.zeros_like(A)
        for i in range(n):
            for j in range(n):
                vl = np.zeros(nodes, complex)
                vr = np.zeros(nodes, complex)
                for k in range(n):
                    vl = vl + cmul(M[i, k], A[:, k, j])
                    vr = vr + cmul(A[:, i, k], M[k, j])
                left[:, i, j] = vl
                right[:, i, j] = vr
        assert np.array_equal(run("mmult_left", matrix=M), left.reshape(-1))
        assert np.array_equal(run("mmult_right", matrix=M), right.reshape(-1))
        # in place: out aliases the input
        ba.write(a)
        H.hierarchy_op("mmult_left", ba, None, ba, matrix=M)
        assert np.array_equal(cplx(ba.read()), left.reshape(-1))
        for x in (ba, bb, bo):
            x.close()


def test_host_pre_evaluate_action_sets_h_before_every_solve():
    n = 4
    h0 = ho.synthetic_hamiltonian(n, 5)
    prob = ho.build_problem(ho.drude_system(n, 3, 2, 5, h_invcm=h0))
    y = np.random.default_rng(1).normal(size=prob.state_len)
    seen = []

    def action(H, t, dt):
        seen.append((t, dt))
        hk = prob.hamiltonian.copy()
        hk[0] += 1e-23 * (t + dt) * 1e15  # the site-0 energy drifts with time (J)
        H.set_hamiltonian(hk)
        return 0

    with hb.Heom.from_problem(prob) as H:
        H.add_pre_evaluate_action(action)
        bi, bo = H.buffer(), H.buffer()
        bi.write(y)
        H.solve(bi, bo, hb.SOLVE_PURE, time=3e-15, step_size=1e-15)
        out = bo.read()
        with pytest.raises(hb.HeomError) as e:
            H.rk4_steps(1e-15, 1)
        assert "heom error -5" in str(e.value)
        H.clear_pre_evaluate_actions()
        H.rk4_steps(1e-15, 1)
        bi.close(), bo.close()
    assert seen == [(3e-15, 1e-15)]
    prob.hamiltonian[0] += 1e-23 * 4.0
    ref = ho.derivative(prob, y)
    assert np.max(np.abs(out - ref)) <= 1e-13 * np.max(np.abs(ref))
