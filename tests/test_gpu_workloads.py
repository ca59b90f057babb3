"""GPU: the benchmark's own batched workloads against the oracle, and the
ensemble adjoint (heom_ensemble_adjoint_*) against single-instance sweeps.

  * the static-disorder draw (256 realisations of 7 sites, depth 6, seed 33):
    the whole ensemble propagated in one ensemble handle (one lockstep class),
    a sample of 8 realisations checked against the oracle after 100 steps and
    the first and last bit for bit against their single-instance solves;
  * the uneven draw (64 instances, seed 5): one instance per class (the
    smallest of each of its 18 classes, 4..12 sites, 0 or 1 Matsubara term)
    propagated together, each checked against the oracle (20 steps; 4 for
    the 376,740-ADO instance, whose oracle run would otherwise take minutes);
  * the ensemble adjoint over systems of three and more classes: every
    instance's loss and gradients against its own single-instance adjoint,
    bit for bit when each instance is swept alone and to rounding when a
    class is packed into one batch.
Population tolerance: parity.py (1e-10 relative, floor 1e-3)."""
import numpy as np
import pytest

import bench
import heom_b200 as hb
import heom_oracle as ho
from parity import assert_pops

pytestmark = pytest.mark.gpu

DT = 1e-15


def oracle_pops(system, steps, every):
    n = system.sites
    h = (system.h[0::2] + 1j * system.h[1::2]).reshape(n, n)
    prob = ho.build_problem(ho.make_system(h.real if not np.any(h.imag) else h, list(system.lambda_),
                                           list(system.invnu), list(system.omega), system.matsubaras,
                                           system.temperature, system.depth))
    _, pops = ho.propagate(prob, DT, steps, every)
    return pops


def top0(n):
    t = np.zeros(n * n * 2)
    t[0] = 1.0
    return t


def test_static_disorder_draw_sample_matches_oracle():
    systems = bench.ensemble_systems(256)
    tables = [hb.build_tables(s) for s in systems]
    with hb.Ensemble(tables) as E:
        assert E.classes() == 1
        E.clear()
        for k, s in enumerate(systems):
            E.set_top(k, top0(s.sites))
        tops = E.propagate(DT, 100, 50)
        for k in range(0, 256, 32):
            assert_pops(E.populations(tops[k], k), oracle_pops(systems[k], 100, 50),
                        what=f"realisation {k} of the 256-member draw")
    # the draw runs as one lockstep class; its first and last realisations equal their own solves
    for k in (0, 255):
        with hb.Heom(**tables[k]) as H:
            H.set_top(top0(systems[k].sites))
            assert np.array_equal(tops[k], H.propagate(DT, 100, 50)), f"realisation {k}"


def test_uneven_draw_one_instance_per_class_matches_oracle():
    from math import comb
    systems = bench.uneven_systems(64)
    smallest = {}
    for k, s in enumerate(systems):
        a = comb(s.sites * s.matsubaras + s.depth, s.depth)
        key = (s.sites, s.matsubaras)
        if key not in smallest or a < smallest[key][0]:
            smallest[key] = (a, k)
    picks = sorted(k for _, k in smallest.values())
    assert len(picks) == 18
    sel = [systems[k] for k in picks]
    with hb.Ensemble([hb.build_tables(s) for s in sel]) as E:
        assert E.classes() >= 18
        E.clear()
        for q, s in enumerate(sel):
            E.set_top(q, top0(s.sites))
        tops = E.propagate(DT, 20, 4)
        for q, s in enumerate(sel):
            ados = comb(s.sites * s.matsubaras + s.depth, s.depth)
            steps = 20 if ados <= 100_000 else 4
            got = E.populations(tops[q], q)[: steps // 4 + 1]
            assert_pops(got, oracle_pops(s, steps, 4),
                        what=f"instance {picks[q]} ({s.sites} sites, M={s.matsubaras}, depth {s.depth}, {ados} ADOs)")


def make_systems(spec):
    return [hb.System(ho.synthetic_hamiltonian(n, seed), [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, d)
            for n, m, d, seed in spec]


# four classes, one instance each (every group holds one instance)
DISTINCT = [(3, 1, 3, 1), (4, 2, 2, 2), (9, 1, 2, 4), (5, 1, 2, 8)]
# three classes (3 sites M=1; 4 sites M=2; 9 sites M=1), several depths each (packed into batches)
MIXED = [(3, 1, 3, 1), (4, 2, 2, 2), (3, 1, 4, 3), (9, 1, 2, 4), (4, 2, 3, 5), (3, 1, 2, 6), (9, 1, 1, 7)]


def single(system, rho0, obs, w, steps):
    with hb.Adjoint(system) as A:
        return A.gradient(rho0, obs, w, DT, steps)


@pytest.mark.parametrize("alone", [True, False])
def test_ensemble_adjoint_matches_single_instance_sweeps(alone):
    systems = make_systems(DISTINCT if alone else MIXED)
    steps = 30
    w = hb.trapezoid_weights(steps, 1.0)
    rho0, obs = [], []
    for k, s in enumerate(systems):
        r = np.zeros((s.sites, s.sites), complex)
        r[0, 0] = 1.0
        o = np.zeros((s.sites, s.sites), complex)
        o[k % s.sites, k % s.sites] = 1.0
        rho0.append(r)
        obs.append(o)
    with hb.EnsembleAdjoint(systems) as E:
        out = E.gradient(rho0, obs, w, DT, steps)
        groups = E.groups()
    by_group = {}
    for k, (g, _) in enumerate(groups):
        by_group.setdefault(g, []).append(k)
    for members in by_group.values():  # a group never mixes classes
        assert len({(systems[k].sites, systems[k].matsubaras) for k in members}) == 1
    assert len(by_group) == (len(systems) if alone else 3)
    for k, s in enumerate(systems):
        ref = single(s, rho0[k], obs[k], w, steps)
        if alone:
            assert out["loss"][k] == ref["loss"]
            assert np.array_equal(out["h"][k], ref["h"]) and np.array_equal(out["rho0"][k], ref["rho0"])
            assert out["lambda"][k] == ref["lambda"] and out["gamma"][k] == ref["gamma"]
        else:
            assert abs(out["loss"][k] - ref["loss"]) <= 1e-14 * abs(ref["loss"])
            assert np.max(np.abs(out["h"][k] - ref["h"])) <= 1e-12 * np.max(np.abs(ref["h"]))
            assert abs(out["lambda"][k] - ref["lambda"]) <= 1e-12 * abs(ref["lambda"])
            assert abs(out["gamma"][k] - ref["gamma"]) <= 1e-12 * abs(ref["gamma"])
            assert np.max(np.abs(out["rho0"][k] - ref["rho0"])) <= 1e-13 * np.max(np.abs(ref["rho0"]))
