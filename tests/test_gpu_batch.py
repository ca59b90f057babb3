"""GPU: batches (several instances in one handle) and ensembles (instances of
any sizes, grouped into classes that run as concurrent graph branches).

Every instance of a batch goes through the same per-ADO arithmetic as when it
is propagated alone, so batch and single-instance results must agree bit for
bit; against the oracle the populations agree to 1e-10 (the bar of the
single-instance parity tests)."""
import numpy as np
import pytest

import heom_b200 as hb
from parity import assert_pops
import heom_oracle as ho

pytestmark = pytest.mark.gpu

DT = 1e-15


def top0(n):
    t = np.zeros(n * n * 2)
    t[0] = 1.0
    return t


def alone(prob, steps, every, **kw):
    with hb.Heom.from_problem(prob, **kw) as H:
        H.set_top(top0(prob.states))
        return H.propagate(DT, steps, every)


def disorder_problems(count, n, depths, m, seed, complex_h=False):
    rng = np.random.default_rng(seed)
    base = ho.synthetic_hamiltonian(n, seed)
    if complex_h:  # Hermitian with an imaginary antisymmetric part
        im = np.triu(rng.normal(0.0, 20.0, size=(n, n)), 1)
        base = base + 1j * (im - im.T)
    out = []
    for k in range(count):
        h = base.copy()
        h[np.diag_indices(n)] += rng.normal(0.0, 100.0, size=n)
        prob = ho.build_problem(ho.drude_system(n, depths[k % len(depths)], m, seed, h_invcm=h))
        prob.h_invcm = h
        out.append(prob)
    return out


@pytest.mark.parametrize("n,m,depths,complex_h", [(7, 1, [3, 4], False), (5, 2, [2, 3], False),
                                                 (10, 1, [2, 3], False), (6, 2, [2, 3], True),
                                                 (9, 2, [1, 2], True), (13, 1, [1, 2], False)])
@pytest.mark.parametrize("scheme", ["product", "reference"])
def test_batch_bitwise_equal_to_single_instances(n, m, depths, complex_h, scheme):
    probs = disorder_problems(3, n, depths, m, seed=40 + n, complex_h=complex_h)
    with hb.Heom.batch([hb.Heom.tables_of(p) for p in probs], scheme=scheme) as H:
        assert H.instances == 3
        for k, p in enumerate(probs):
            H.set_instance_top(k, top0(n))
        tops = H.propagate(DT, 40, 10)  # [rows, inst, n*n*2]
    for k, p in enumerate(probs):
        ref = alone(p, 40, 10, scheme=scheme)
        assert np.array_equal(tops[:, k, :], ref), f"instance {k}"


def test_batch_populations_match_oracle():
    probs = disorder_problems(4, 7, [3, 4], 1, seed=3)
    with hb.Heom.batch([hb.Heom.tables_of(p) for p in probs]) as H:
        for k in range(4):
            H.set_instance_top(k, top0(7))
        pops = H.populations_from_tops(H.propagate(DT, 200, 20))
    for k, p in enumerate(probs):
        _, ref = ho.propagate(p, DT, 200, 20)
        assert_pops(pops[:, k, :], ref)


def test_batch_state_and_top_round_trip():
    probs = disorder_problems(3, 6, [2, 3], 2, seed=9)
    with hb.Heom.batch([hb.Heom.tables_of(p) for p in probs]) as H:
        y = np.random.default_rng(2).normal(size=H.state_len)
        H.set_state(y)
        assert np.array_equal(H.get_state(), y)
        tops = H.get_top().reshape(3, -1)
        for k in range(3):
            off = H.instance_offset(k) * 6 * 6 * 2
            assert np.array_equal(tops[k], y[off:off + 72])
            assert np.array_equal(H.get_instance_top(k), tops[k])
        # one instance's Hamiltonian changed (+200 cm^-1 on site 0): only that instance follows it
        h_cm = probs[1].h_invcm.copy()
        h_cm[0, 0] += 200.0
        p1 = ho.build_problem(ho.drude_system(6, 3, 2, seed=9, h_invcm=h_cm))
        H.set_instance_hamiltonian(1, p1.hamiltonian)
        H.set_state(np.zeros(H.state_len))
        for k in range(3):
            H.set_instance_top(k, top0(6))
        tops = H.propagate(DT, 20, 20)
    ref_changed = alone(p1, 20, 20)
    assert np.max(np.abs(tops[:, 1, :] - ref_changed)) <= 1e-12
    assert np.array_equal(tops[:, 0, :], alone(probs[0], 20, 20))


def uneven_problems():
    # (5, 2, 1) last: same kernel function as the (5, *, 2) class with a smaller shared-memory
    # footprint, resolved after it (the per-function limit must only grow)
    spec = [(3, 3, 1, 1), (5, 2, 2, 2), (9, 2, 1, 3), (5, 3, 2, 4), (3, 4, 1, 5), (8, 2, 2, 6), (4, 3, 1, 7),
            (5, 2, 1, 8)]
    return [ho.build_problem(ho.drude_system(n, d, m, seed=s)) for n, d, m, s in spec]


def test_ensemble_uneven_sizes_bitwise_and_oracle():
    probs = uneven_problems()
    with hb.Ensemble([hb.Heom.tables_of(p) for p in probs]) as E:
        assert E.classes() == 6  # (3,M1) (5,M2) (9,M1) (8,M2) (4,M1) (5,M1)
        assert E.locate(4) == (0, 1) and E.locate(3) == (1, 1)
        for k, p in enumerate(probs):
            E.set_top(k, top0(p.states))
        us = E.autotune()
        assert us > 0.0
        launches = E.kernel_launches()
        tops = E.propagate(DT, 60, 20)
        assert E.kernel_launches() - launches >= 3 * 4 * 6  # 4 stage launches per class and step
        assert np.array_equal(E.get_top(2), tops[2][-1])
    for k, p in enumerate(probs):
        assert np.array_equal(tops[k], alone(p, 60, 20)), f"instance {k}"
        _, ref = ho.propagate(p, DT, 60, 20)
        pops = tops[k][:, [(p.states + 1) * 2 * i for i in range(p.states)]]
        assert_pops(pops, ref)


def test_ensemble_rejects_footprint_beyond_device_memory():
    # 4 sites, 12 modes (M = 3), depth 6: 18564 ADOs; the footprint scales with
    # the count, so 10^6 copies ask for far more than any device holds
    p = ho.build_problem(ho.drude_system(4, 6, 3, seed=1))
    t = hb.Heom.tables_of(p)
    per = hb.Ensemble.footprint([t])
    assert per > 18564 * 10 * 32 * 3
    assert per * 20000 > 300e9
    with pytest.raises(hb.HeomError) as e:
        hb.Ensemble([t] * 20000)  # rejected at admission, before any allocation
    assert "heom error -3" in str(e.value) and "GB of device memory" in str(e.value)


@pytest.mark.parametrize("n,m,depth,count,complex_h", [(7, 1, 4, 40, False), (8, 2, 3, 33, False),
                                                       (6, 2, 3, 12, True), (4, 1, 5, 64, False),
                                                       (5, 3, 2, 9, False), (3, 4, 2, 8, True)])
def test_ensemble_lockstep_class_bitwise_equal_to_single_instances(n, m, depth, count, complex_h):
    """An ensemble class of 8 or more instances of one depth (the realisations
    of a static-disorder ensemble) runs in the lockstep layout (instance-minor
    state, one warp per sector with a lane per instance): every instance bit
    for bit as when propagated alone, and the oracle's populations; instance
    counts that are not a multiple of 32 leave padding lanes idle."""
    probs = disorder_problems(count, n, [depth], m, seed=60 + n, complex_h=complex_h)
    with hb.Ensemble([hb.Heom.tables_of(p) for p in probs]) as E:
        assert E.classes() == 1
        E.clear()
        for k in range(count):
            E.set_top(k, top0(n))
        tops = E.propagate(DT, 40, 10)
        assert np.array_equal(E.get_top(count - 1), tops[count - 1][-1])
        # a lockstep class refuses the calls that read or write its state in another layout
        cls = hb.lib().heom_ensemble_class(E.h, 0)
        y = np.zeros(sum(int(hb.Heom.tables_of(p)["matrices"]) for p in probs) * n * n * 2)
        assert hb.lib().heom_set_state(cls, y.ctypes.data) == -5
    for k in sorted({0, 1, count // 2, count - 1}):
        assert np.array_equal(tops[k], alone(probs[k], 40, 10)), f"instance {k}"
    for k in (0, count - 1):
        _, ref = ho.propagate(probs[k], DT, 40, 10)
        assert_pops(tops[k][:, [(n + 1) * 2 * i for i in range(n)]], ref)


def test_ensemble_splits_a_class_into_lockstep_and_mixed_depths():
    """Ten instances of depth 3 form a lockstep class; three of depth 4 of the
    same states and baths stay one batch handle."""
    probs = disorder_problems(10, 7, [3], 1, seed=71) + disorder_problems(3, 7, [4], 1, seed=72)
    with hb.Ensemble([hb.Heom.tables_of(p) for p in probs]) as E:
        assert E.classes() == 2
        E.clear()
        for k in range(13):
            E.set_top(k, top0(7))
        tops = E.propagate(DT, 30, 10)
    for k in (0, 9, 10, 12):
        assert np.array_equal(tops[k], alone(probs[k], 30, 10)), f"instance {k}"
