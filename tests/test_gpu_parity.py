"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Tolerances (floating point; the CUDA kernels contract products into FMAs and
combine the per-neighbour coefficients on the host, so results differ from
the reference's operation order by rounding only):
  * one derivative evaluation: max |gpu - ref| <= 1e-13 * max |ref|
  * propagated populations:   |gpu - ref| <= 1e-10 * max(|ref|, 1e-3) (parity.py),
    the accuracy the path must keep
"""
import numpy as np
import pytest

import heom_b200 as hb
from parity import assert_pops
import heom_oracle as ho
import make_golden as mg

pytestmark = pytest.mark.gpu

DERIV_TOL = 1e-13


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def derivative_gpu(prob, y, mask=None, **kw):
    with hb.Heom.from_problem(prob, **kw) as H:
        if mask is not None:
            H.set_mask(mask)
        bi, bo = H.buffer(), H.buffer()
        bi.write(y)
        H.solve(bi, bo, hb.SOLVE_PURE)
        out = bo.read()
        bi.close(), bo.close()
    return out


def complex_problem():
    return ho.build_problem(mg.complex_system())


def complex_hermitian(n, seed, scale=20.0):
    rng = np.random.default_rng(seed)
    im = np.zeros((n, n))
    iu = np.triu_indices(n, 1)
    im[iu] = rng.normal(0.0, scale, size=len(iu[0]))
    return ho.synthetic_hamiltonian(n, seed) + 1j * (im - im.T)


def ring_shared_problem(n, m, depth, seed):
    """Every site coupled to its own bath and its neighbour's (two baths per site)."""
    coupling = np.array([[i, (i + 1) % n] for i in range(n)], np.int32)
    lam = [35.0 + 2.0 * i for i in range(n)]
    invnu = [50.0 + 3.0 * i for i in range(n)]
    return ho.build_problem(ho.make_system(ho.synthetic_hamiltonian(n, seed), lam, invnu, [0.0] * n, m,
                                           300.0, depth, coupling=coupling))


CASES = {
    "cfg1_real_m1": lambda: ho.build_problem(ho.drude_system(7, 4, 1, seed=11)),
    "cfg2_small_m2": lambda: ho.build_problem(ho.drude_system(8, 3, 2, seed=22)),
    "complex_m2": complex_problem,
    "shared_baths": lambda: ho.build_problem(mg.shared_system()),
    "n12_m1": lambda: ho.build_problem(ho.drude_system(12, 2, 1, seed=5)),
    "n1": lambda: ho.build_problem(ho.drude_system(1, 5, 2, seed=6)),
    "n16_m1": lambda: ho.build_problem(ho.drude_system(16, 1, 1, seed=7)),
    "n10_m2": lambda: ho.build_problem(ho.drude_system(10, 2, 2, seed=8)),
    "n13_m1": lambda: ho.build_problem(ho.drude_system(13, 2, 1, seed=9)),
    "n11_m2_complex": lambda: ho.build_problem(ho.make_system(complex_hermitian(11, 10), [35.0] * 11,
                                                              [50.0] * 11, [0.0] * 11, 2, 300.0, 2)),
    "n15_m1_complex": lambda: ho.build_problem(ho.make_system(complex_hermitian(15, 12), [35.0] * 15,
                                                              [50.0] * 15, [0.0] * 15, 1, 300.0, 2)),
    "n9_ring_shared_m2": lambda: ring_shared_problem(9, 2, 2, 13),
    "m3_t77": lambda: ho.build_problem(ho.make_system(ho.synthetic_hamiltonian(4, 9), [35] * 4,
                                                      [50] * 4, [0] * 4, 3, 77.0, 3)),
}


@pytest.mark.parametrize("order", ["lex", "reference"])
@pytest.mark.parametrize("case", sorted(CASES))
def test_derivative_matches_oracle(case, order):
    prob = CASES[case]()
    y = np.random.default_rng(1).normal(size=prob.state_len)
    out = derivative_gpu(prob, y, order=order)
    ref = ho.derivative(prob, y)
    assert rel_err(out, ref) <= DERIV_TOL


def test_derivative_modes_match_reference_kernels(golden):
    """pure / ACCUMULATE / SUBDIAGONAL against outputs of heom_ode.cl itself."""
    prob = complex_problem()
    y = golden["d_complex_y"]
    acc0 = golden["d_complex_acc0"]
    with hb.Heom.from_problem(prob) as H:
        bi, bo, ba = H.buffer(), H.buffer(), H.buffer()
        bi.write(y)
        H.solve(bi, bo, hb.SOLVE_PURE)
        assert rel_err(bo.read(), golden["d_complex_pure"]) <= DERIV_TOL
        ba.write(acc0)
        H.solve(bi, bo, hb.SOLVE_ACCUMULATE, acc=ba, acc_coeff=0.25, acc_init=False)
        assert rel_err(bo.read(), golden["d_complex_acc_out"]) <= DERIV_TOL
        assert rel_err(ba.read(), golden["d_complex_acc_acc"]) <= DERIV_TOL
        ba.write(acc0)
        H.solve(bi, bo, hb.SOLVE_ACCUMULATE, acc=ba, acc_coeff=0.5, acc_init=True)
        assert rel_err(ba.read(), golden["d_complex_accinit_acc"]) <= DERIV_TOL
        ba.write(acc0)
        H.solve(bi, None, hb.SOLVE_SUBDIAGONAL, out_coeff=0.5e-15, acc=ba)
        assert rel_err(ba.read(), golden["d_complex_subdiag_acc"]) <= DERIV_TOL
        for b in (bi, bo, ba):
            b.close()


def test_masked_and_shared_match_reference_kernels(golden):
    prob = complex_problem()
    out = derivative_gpu(prob, golden["d_masked_y"], mask=golden["d_masked_mask"])
    assert rel_err(out, golden["d_masked_pure"]) <= DERIV_TOL
    ps = ho.build_problem(mg.shared_system())
    out = derivative_gpu(ps, golden["d_shared_y"])
    assert rel_err(out, golden["d_shared_pure"]) <= DERIV_TOL


def test_weighted_add_matches_reference_order():
    prob = ho.build_problem(ho.drude_system(5, 2, 1, seed=3))
    rng = np.random.default_rng(4)
    y = rng.normal(size=prob.state_len)
    ks = [rng.normal(size=prob.state_len) for _ in range(4)]
    c = [1.0 / 6, 0.0, 1.0 / 3, 1.0 / 6]
    with hb.Heom.from_problem(prob) as H:
        bufs = [H.buffer() for _ in range(6)]
        bufs[0].write(y)
        for b, k in zip(bufs[1:5], ks):
            b.write(k)
        H.weighted_add(1e-15, bufs[5], bufs[0], c, bufs[1:5])
        out = bufs[5].read()
        for b in bufs:
            b.close()
    # rk_weighted_add.cl order: acc = sum c_l k_l (zero c skipped), acc *= h, acc += y
    acc = np.zeros_like(y)
    for cl, k in zip(c, ks):
        if cl != 0.0:
            acc = acc + cl * k
    ref = acc * 1e-15 + y
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("scheme", ["product", "horner", "reference"])
def test_cfg1_populations_match_reference_run(golden, scheme):
    """7 sites, depth 4, RK4 dt = 1 fs, 1000 steps vs the reference kernels' run."""
    prob = ho.build_problem(ho.drude_system(7, 4, 1, seed=11))
    with hb.Heom.from_problem(prob, scheme=scheme) as H:
        H.set_state(prob.initial_state())
        tops = H.propagate(1.0e-15, 1000, 1)
        pops = H.populations_from_tops(tops)
        final = H.get_state()
    assert_pops(pops, golden["cfg1_pops"])
    assert rel_err(final, golden["cfg1_final"]) <= 1e-9


@pytest.mark.parametrize("scheme", ["product", "horner", "reference"])
def test_cfg2_shape_reduced_depth(scheme):
    """8 sites, 16 modes (M=2), depth 4, dt = 0.5 fs, 200 steps vs the oracle."""
    prob = ho.build_problem(ho.drude_system(8, 4, 2, seed=22))
    _, ref = ho.propagate(prob, 0.5e-15, 200, 10)
    with hb.Heom.from_problem(prob, scheme=scheme) as H:
        H.set_state(prob.initial_state())
        pops = H.populations_from_tops(H.propagate(0.5e-15, 200, 10))
    assert_pops(pops, ref)


def test_complex_hamiltonian_masked_propagation(golden):
    prob = ho.build_problem(mg.complex_system(), mask=golden["d_masked_mask"])
    _, ref = ho.propagate(prob, 1e-15, 100, 10)
    with hb.Heom.from_problem(prob) as H:
        H.set_mask(golden["d_masked_mask"])
        H.set_state(prob.initial_state())
        pops = H.populations_from_tops(H.propagate(1e-15, 100, 10))
    assert_pops(pops, ref)


def test_state_roundtrip_and_top():
    prob = ho.build_problem(ho.drude_system(6, 3, 2, seed=2))
    y = np.random.default_rng(3).normal(size=prob.state_len)
    with hb.Heom.from_problem(prob) as H:
        H.set_state(y)
        assert np.array_equal(H.get_state(), y)
        assert np.array_equal(H.get_top(), y[: 6 * 6 * 2])
        top = np.arange(72, dtype=np.float64)
        H.set_top(top)
        y2 = y.copy()
        y2[:72] = top
        assert np.array_equal(H.get_state(), y2)


def test_set_hamiltonian_switches_variant():
    prob = complex_problem()
    y = np.random.default_rng(8).normal(size=prob.state_len)
    real_prob = ho.build_problem(ho.make_system(ho.synthetic_hamiltonian(4, 404), [35.0, 40.0, 30.0, 45.0],
                                                [50.0, 60.0, 40.0, 55.0], [0.0] * 4, 2, 300.0, 3))
    with hb.Heom.from_problem(real_prob) as H:
        bi, bo = H.buffer(), H.buffer()
        bi.write(y)
        H.solve(bi, bo)
        assert rel_err(bo.read(), ho.derivative(real_prob, y)) <= DERIV_TOL
        H.set_hamiltonian(prob.hamiltonian)
        H.solve(bi, bo)
        assert rel_err(bo.read(), ho.derivative(prob, y)) <= DERIV_TOL
        bi.close(), bo.close()


def test_library_built_tables_drive_the_gpu():
    """heom_create_from_system path (tables from the library's own host code)."""
    h = ho.synthetic_hamiltonian(7, 11)
    with hb.from_system(hb.System(h, [35.0] * 7, [50.0] * 7, [0.0] * 7, 1, 300.0, 4)) as H:
        y0 = np.zeros(H.state_len)
        y0[0] = 1.0
        H.set_state(y0)
        pops = H.populations_from_tops(H.propagate(1e-15, 100, 100))
    prob = ho.build_problem(ho.drude_system(7, 4, 1, seed=11))
    _, ref = ho.propagate(prob, 1e-15, 100, 100)
    assert_pops(pops, ref)


def test_nonfinite_state_is_reported():
    prob = ho.build_problem(ho.drude_system(3, 2, 1, seed=1))
    y = np.zeros(prob.state_len)
    y[5] = np.nan
    with hb.Heom.from_problem(prob) as H:
        H.set_state(y)
        with pytest.raises(hb.HeomError) as e:
            H.propagate(1e-15, 2, 1)
        assert "heom error -6" in str(e.value)


@pytest.mark.parametrize("n,m,depth,layer", [(4, 2, 4, 1), (7, 1, 4, 2), (9, 1, 3, 1)])
def test_compacted_mask_is_bit_identical_on_active_ados(n, m, depth, layer):
    """heom_set_mask_compact sweeps only the active ADOs; they (and every top)
    evolve exactly as under heom_set_mask, masked entries keep their values."""
    sysd = hb.System(ho.synthetic_hamiltonian(n, 40 + n), [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, depth)
    mask = hb.tables_mask(sysd, "single_excitation", layer)
    assert 0 < mask.sum() < mask.size
    y0 = np.zeros(hb.build_tables(sysd)["matrices"] * n * n * 2)
    y0[0] = 1.0
    y0[-2] = 0.25  # an entry of the last ADO (masked for these systems)
    runs = []
    for compact in (False, True):
        with hb.from_system(sysd) as H:
            H.set_state(y0)
            H.set_mask(mask, compact=compact)
            assert H.active_matrices() == (mask.sum() if compact else mask.size)
            tops = H.propagate(1e-15, 60, 10)
            runs.append((tops, H.get_state()))
    (t1, s1), (t2, s2) = runs
    assert np.array_equal(t1, t2)
    act = np.repeat(mask.astype(bool), n * n * 2)
    assert np.array_equal(s1[act], s2[act])
    assert np.array_equal(s2[~act], y0[~act])


def test_compaction_switches_back_and_keeps_the_state():
    n = 4
    sysd = hb.System(ho.synthetic_hamiltonian(n, 3), [35.0] * n, [50.0] * n, [0.0] * n, 2, 300.0, 3)
    mask = hb.tables_mask(sysd, "single_excitation", 1)
    with hb.from_system(sysd) as H:
        y = np.random.default_rng(0).normal(size=H.state_len)
        H.set_state(y)
        H.set_mask(mask, compact=True)
        assert np.array_equal(H.get_state(), y)  # reordering keeps every entry
        H.set_mask(mask)
        assert H.active_matrices() == mask.size
        assert np.array_equal(H.get_state(), y)


@pytest.mark.parametrize("case", ["complex_m2", "n12_m1", "cfg1_real_m1"])
def test_flow_buffers_match_reference_kernel_terms(case):
    """heom_set_flow_buffers: each heom_solve adds acc_coeff x the plus term and
    acc_coeff x the minus term (heom_ode.cl:436-441); the terms are taken from
    the reference's own kernel built with HEOM_ODE_DISABLE_PLUS / _MINUS."""
    prob = CASES[case]()
    y = np.random.default_rng(4).normal(size=prob.state_len)
    full, _ = ho.ref_derivative(prob, y)
    plus = full - ho.ref_derivative(prob, y, mode=3)[0]
    minus = full - ho.ref_derivative(prob, y, mode=4)[0]
    with hb.Heom.from_problem(prob) as H:
        bi, bo, fa, fb = H.buffer(), H.buffer(), H.buffer(), H.buffer()
        bi.write(y)
        H.set_flow_buffers(fa, fb)
        H.solve(bi, bo, hb.SOLVE_PURE, acc_coeff=0.7)
        H.solve(bi, bo, hb.SOLVE_PURE, acc_coeff=0.3)
        above, below, out = fa.read(), fb.read(), bo.read()
        H.set_flow_buffers(None, None)
        H.solve(bi, bo, hb.SOLVE_PURE, acc_coeff=5.0)
        assert np.array_equal(fa.read(), above)  # tracking off
        for b in (bi, bo, fa, fb):
            b.close()
    assert rel_err(out, full) <= DERIV_TOL
    assert np.max(np.abs(above - plus)) <= 1e-12 * np.max(np.abs(plus))
    assert np.max(np.abs(below - minus)) <= 1e-12 * np.max(np.abs(minus))
