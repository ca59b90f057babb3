#!/usr/bin/env python3
"""Generate tests/golden/golden_small.npz from the reference's own kernels.

The reference (noma/dm-heom) ships no golden vectors.  These fixtures are
outputs of its own OpenCL kernel sources, dm-heom/cl/heom/heom_ode.cl and
rk_weighted_add.cl, compiled unmodified for the host by oracle/Makefile
(oracle/_ref/libheom_refcl.so), driven by the classical RK4 tableau.  The
hierarchy tables come from the oracle's restatement of hierarchy_graph.cpp /
instance.cpp (the reference's host code needs Boost and the un-vendored
noma submodules).

Cases (all inputs are seeded and stored next to the outputs):
  cfg1_pops      7 sites, 1 bath/site, M=1, depth 4 (330 ADOs), T=300 K,
                 lambda=35 cm^-1, invnu=50 fs, RK4 dt=1 fs, 1000 steps,
                 populations after every step
  d_complex_*    4 sites, M=2, depth 3 (165 ADOs), Hermitian complex H,
                 random state: heom_ode in pure, ACCUMULATE and SUBDIAGONAL mode
  d_masked_*     same system with a single_excitation mask from layer 1
  d_shared_*     3 sites, 2 baths per site with a shared bath, M=2, depth 2

Run:  python tests/golden/make_golden.py   (needs oracle/_ref built)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import heom_oracle as ho  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_small.npz")


def complex_system():
    rng = np.random.default_rng(404)
    n = 4
    h = ho.synthetic_hamiltonian(n, 404)
    iu = np.triu_indices(n, 1)
    im = np.zeros((n, n))
    im[iu] = rng.normal(0.0, 20.0, size=len(iu[0]))
    h = h + 1j * (im - im.T)
    return ho.make_system(h, [35.0, 40.0, 30.0, 45.0], [50.0, 60.0, 40.0, 55.0],
                          [0.0, 0.0, 0.0, 0.0], 2, 300.0, 3)


def shared_system():
    h = ho.synthetic_hamiltonian(3, 505)
    coupling = np.array([[0, 1], [1, 2], [2, -1]], np.int32)
    return ho.make_system(h, [35.0, 25.0, 45.0], [50.0, 45.0, 65.0], [0.0, 0.0, 0.0], 2, 280.0, 2,
                          coupling=coupling)


def single_excitation_mask(graph, matsubaras, first_layer):
    # hierarchy_mask.cpp:48-110
    w = graph.width
    baths = w // matsubaras
    mask = np.ones(graph.nodes, np.uint8)
    for u in range(graph.nodes):
        t = graph.tuples[u]
        s = int(t.sum())
        if s < first_layer:
            continue
        found = any(int(t[b * matsubaras:(b + 1) * matsubaras].sum()) == s for b in range(baths))
        mask[u] = 1 if found else 0
    return mask


def modes(prob, y, tag, out):
    rng = np.random.default_rng(7)
    acc0 = rng.normal(size=y.size)
    pure, _ = ho.ref_derivative(prob, y, mode=0)
    acc_o, acc_a = ho.ref_derivative(prob, y, mode=1, acc=acc0, acc_coeff=0.25, acc_init=False)
    acc_o2, acc_a2 = ho.ref_derivative(prob, y, mode=1, acc=acc0, acc_coeff=0.5, acc_init=True)
    _, sub = ho.ref_derivative(prob, y, mode=2, out_coeff=0.5e-15, acc=acc0)
    out[f"{tag}_y"] = y
    out[f"{tag}_acc0"] = acc0
    out[f"{tag}_pure"] = pure
    out[f"{tag}_acc_out"] = acc_o
    out[f"{tag}_acc_acc"] = acc_a
    out[f"{tag}_accinit_acc"] = acc_a2
    out[f"{tag}_subdiag_acc"] = sub


def main():
    if ho.ref_lib() is None:
        sys.exit("oracle/_ref/libheom_refcl.so missing: build the oracle first")
    out = {}
    # cfg1
    s1 = ho.drude_system(7, 4, 1, seed=11)
    p1 = ho.build_problem(s1)
    y = p1.initial_state()
    pops = [ho.populations(p1, y)]
    for _ in range(1000):
        y = ho.ref_rk4_step(p1, 1.0e-15, y)
        pops.append(ho.populations(p1, y))
    out["cfg1_h_invcm"] = ho.synthetic_hamiltonian(7, 11)
    out["cfg1_pops"] = np.array(pops)
    out["cfg1_final"] = y
    # complex H, all write modes
    sc = complex_system()
    pc = ho.build_problem(sc)
    yc = np.random.default_rng(9).normal(size=pc.state_len) * 1e-2
    out["complex_h_joule"] = pc.hamiltonian
    modes(pc, yc, "d_complex", out)
    # masked
    mask = single_excitation_mask(pc.graph, 2, 1)
    pm = ho.build_problem(sc, mask=mask)
    out["d_masked_mask"] = mask
    out["d_masked_y"] = yc
    out["d_masked_pure"], _ = ho.ref_derivative(pm, yc, mode=0)
    # shared bath coupling
    ss = shared_system()
    ps = ho.build_problem(ss)
    ys = np.random.default_rng(10).normal(size=ps.state_len)
    out["d_shared_y"] = ys
    out["d_shared_pure"], _ = ho.ref_derivative(ps, ys, mode=0)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
