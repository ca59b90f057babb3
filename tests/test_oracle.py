"""CPU: the oracle restatement pinned against the reference.

* bit-for-bit against the reference's own kernel sources compiled for the
  host (oracle/_ref, when built) and its integer_partition.cpp
* against the committed golden fixtures (generated from those kernels)
* graph invariants of hierarchy_graph.cpp:30-181
"""
import os
import re

import numpy as np
import pytest

import heom_oracle as ho

REF = os.environ.get("HEOM_REFERENCE_ROOT", "/root/reference")


def test_graph_invariants():
    for (w, d) in [(1, 1), (3, 2), (7, 4), (16, 3), (14, 5)]:
        g = ho.build_graph(w, d)
        assert g.nodes == ho.lib().ho_binomial(w + d, w)
        assert g.first_non_plus == ho.lib().ho_binomial(w + d - 1, w)
        sums = g.tuples.sum(axis=1)
        assert (np.diff(sums) >= 0).all()          # layer order
        assert (sums[: g.first_non_plus] < d).all() and (sums[g.first_non_plus:] == d).all()
        assert len({tuple(t) for t in g.tuples}) == g.nodes
        assert (g.tuples[0] == 0).all()
        for u in range(g.nodes):
            for j in range(w):
                p, m = g.plus[u, j], g.minus[u, j]
                if sums[u] < d:
                    assert g.minus[p, j] == u
                    t = g.tuples[u].copy(); t[j] += 1
                    assert (g.tuples[p] == t).all()
                else:
                    assert p == ho.INVALID_UID
                if g.tuples[u, j] > 0:
                    assert g.plus[m, j] == u
                else:
                    assert m == ho.INVALID_UID


def test_graph_sizes_of_benchmark_configs():
    # nodes = C(W+D, W), first_non_plus = C(W+D-1, W)
    for (w, d, nodes, fnp) in [(7, 4, 330, 120), (16, 8, 735471, 245157), (7, 6, 1716, 792),
                               (7, 8, 6435, 3432)]:
        assert ho.lib().ho_binomial(w + d, w) == nodes
        assert ho.lib().ho_binomial(w + d - 1, w) == fnp
    g = ho.build_graph(7, 6)
    assert g.nodes == 1716 and g.first_non_plus == 792


def test_partitions_match_reference_source():
    R = ho.ref_ip_lib()
    if R is None:
        pytest.skip("oracle/_ref not built")
    for n in range(1, 13):
        for s in range(1, 18):
            mine = ho.integer_partitions(n, s)
            out = np.zeros(200000 * s, np.int64)
            cnt = R.refip_integer_partitions(n, s, out, 200000)
            assert cnt == mine.shape[0]
            assert (out[: cnt * s].reshape(cnt, s) == mine).all()


def _system_complex():
    rng = np.random.default_rng(3)
    h = ho.synthetic_hamiltonian(5, 3)
    im = np.triu(rng.normal(0, 15.0, size=(5, 5)), 1)
    return ho.make_system(h + 1j * (im - im.T), [35, 20, 50, 35, 10], [50, 30, 80, 50, 20],
                          [0, 0, 0, 0, 0], 2, 250.0, 3)


@pytest.mark.parametrize("case", ["real_m1", "complex_m2", "shared", "masked"])
def test_oracle_bitwise_equal_reference_kernels(case):
    if ho.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    mask = None
    if case == "real_m1":
        s = ho.drude_system(7, 4, 1, seed=1)
    elif case == "complex_m2":
        s = _system_complex()
    elif case == "shared":
        s = ho.make_system(ho.synthetic_hamiltonian(3, 4), [35, 25, 45], [50, 45, 65], [0, 0, 0], 2,
                           280.0, 3, coupling=np.array([[0, 1], [1, 2], [2, -1]], np.int32))
    else:
        s = _system_complex()
        g = ho.build_graph(s.width, s.depth)
        mask = (np.random.default_rng(5).random(g.nodes) > 0.3).astype(np.uint8)
    p = ho.build_problem(s, mask=mask)
    y = np.random.default_rng(0).normal(size=p.state_len)
    a = ho.derivative(p, y)
    b, _ = ho.ref_derivative(p, y)
    assert np.array_equal(a, b)
    r1 = ho.rk4_step(p, 1e-15, y)
    r2 = ho.ref_rk4_step(p, 1e-15, y)
    assert np.array_equal(r1, r2)


def test_oracle_reproduces_golden(golden):
    # cfg1: 1000 RK4 steps of the reference kernels
    h = golden["cfg1_h_invcm"]
    s = ho.drude_system(7, 4, 1, seed=11)
    assert np.array_equal(ho.synthetic_hamiltonian(7, 11), h)
    p = ho.build_problem(s)
    y, pops = ho.propagate(p, 1.0e-15, 1000, 1)
    assert np.array_equal(pops, golden["cfg1_pops"])
    assert np.array_equal(y, golden["cfg1_final"])


def test_oracle_modes_against_golden(golden):
    import make_golden as mg
    pc = ho.build_problem(mg.complex_system())
    y = golden["d_complex_y"]
    assert np.array_equal(ho.derivative(pc, y), golden["d_complex_pure"])
    pm = ho.build_problem(mg.complex_system(), mask=golden["d_masked_mask"])
    assert np.array_equal(ho.derivative(pm, golden["d_masked_y"]), golden["d_masked_pure"])
    ps = ho.build_problem(mg.shared_system())
    assert np.array_equal(ho.derivative(ps, golden["d_shared_y"]), golden["d_shared_pure"])


def test_long_double_oracle_close():
    s = ho.drude_system(7, 3, 1, seed=2)
    p = ho.build_problem(s)
    y1, pops1 = ho.propagate(p, 1e-15, 50, 10)
    y2, pops2 = ho.propagate(p, 1e-15, 50, 10, long_double=True)
    assert np.max(np.abs(pops1 - pops2)) < 1e-13


def _parse_pade(path, name):
    import mpmath as mp
    mp.mp.dps = 50
    src = open(path).read()
    body = src.split(name + "[")[1].split("{", 1)[1].split("};")[0]
    return [mp.mpf(v.rstrip("L")) for v in re.findall(r"[0-9][0-9.eE+-]*L?", body)]


def test_pade_tables_from_mathematics_match_reference(root):
    import mpmath as mp
    gen = [os.path.join(root, "oracle", "pade_tables.inc"),
           os.path.join(root, "dm-heom_b200", "csrc", "pade_tables.inc")]
    ref = os.path.join(REF, "dm-heom", "src", "heom", "constants.cpp")
    if not os.path.exists(ref):
        pytest.skip("reference sources not present")
    for name in ("eta_pade", "xi_pade"):
        r = _parse_pade(ref, name)
        assert len(r) == 100
        for g in gen:
            v = _parse_pade(g, name)
            assert len(v) == 100
            for a, b in zip(v, r):
                # the reference literals carry ~32 correct digits; long double needs ~20
                assert abs(a - b) <= mp.mpf("1e-28") * max(abs(b), 1)


def test_pade_tables_reproduce_bose_function():
    # sum_j 2 eta_j x/(x^2 + xi_j^2) approximates coth(x/2)/2 - 1/x
    import heom_oracle as o
    src = open(os.path.join(o.HERE, "pade_tables.inc")).read()
    import mpmath as mp
    eta = _parse_pade(os.path.join(o.HERE, "pade_tables.inc"), "eta_pade")
    xi = _parse_pade(os.path.join(o.HERE, "pade_tables.inc"), "xi_pade")
    assert src
    for n in (3, 6, 10):
        for x in (0.1, 1.0, 5.0):
            approx = sum(2 * eta[(n - 1) * 10 + j] * x / (x * x + xi[(n - 1) * 10 + j] ** 2) for j in range(n))
            exact = mp.coth(x / 2) / 2 - 1 / mp.mpf(x)
            assert abs(approx - exact) < 1e-6 * abs(exact)
