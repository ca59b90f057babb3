"""GPU: the population-dynamics and linear-absorption applications end to end
(reference command line and config files, all five population observers, the
dipole pseudo pathway) and the hierarchy norm."""
import os
import subprocess

import numpy as np
import pytest

import heom_b200 as hb
from parity import assert_pops
import heom_oracle as ho
from test_host import FMO_CFG, LA_CFG

pytestmark = pytest.mark.gpu

APP = os.path.join(os.path.dirname(hb.__file__), "bin", "heom_population_dynamics")
LA_APP = os.path.join(os.path.dirname(hb.__file__), "bin", "heom_linear_absorption")
CD_APP = os.path.join(os.path.dirname(hb.__file__), "bin", "heom_circular_dichroism")


def read_dat(path):
    lines = open(path).read().strip().split("\n")
    return lines[0].split("\t"), np.array([[float(x) for x in l.split("\t")] for l in lines[1:]])


def test_app_observers_match_oracle(tmp_path):
    cfg = FMO_CFG.replace(
        "observations={(matrix_complete, m.dat), (matrix_diagonal, d.dat), (matrix_trace_id, t.dat)}",
        "observations={(matrix_complete, m.dat), (matrix_diagonal, d.dat), (matrix_trace_id, t.dat), "
        "(hierarchy_norm, n.dat), (hierarchy_complete, c.dat)}")
    (tmp_path / "heom.cfg").write_text(cfg)
    (tmp_path / "rt.cfg").write_text("[opencl]\nplatform_index=0\n[cuda]\ndevice_index=0\nrk4_scheme=product\n")
    r = subprocess.run([APP, "rt.cfg", "heom.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    h = np.array([[12410.0, -87.7, 5.5], [-87.7, 12530.0, 30.8], [5.5, 30.8, 12210.0]])
    prob = ho.build_problem(ho.make_system(h, [35] * 3, [50] * 3, [0] * 3, 2, 77.0, 3))
    _, ref = ho.propagate(prob, 1e-15, 20, 5)
    hd, d = read_dat(tmp_path / "d.dat")
    assert hd == ["time", "site_0", "site_1", "site_2"]
    assert_pops(d[:, 1:], ref)
    assert np.allclose(d[:, 0], np.arange(5) * 5e-15, rtol=1e-15, atol=0)
    _, t = read_dat(tmp_path / "t.dat")
    assert np.max(np.abs(t[:, 1] - 1.0)) <= 1e-12
    # hierarchy_complete: the whole state in uid order; hierarchy_norm: sum |sigma_ij|^2 per ADO
    hc, c = read_dat(tmp_path / "c.dat")
    nodes = prob.graph.nodes
    assert len(hc) == 1 + nodes * 9 * 2 and hc[1] == "mat_0_elem_0_0_real"
    hn, nrm = read_dat(tmp_path / "n.dat")
    assert len(hn) == 1 + nodes and hn[1] == "{0, 0, 0, 0, 0, 0}"
    states = c[:, 1:].reshape(len(c), nodes, 18)
    assert np.max(np.abs(nrm[:, 1:] - (states ** 2).sum(axis=2))) <= 1e-14 * max(1.0, nrm[:, 1:].max())
    # the top of the last complete state is the last matrix_complete line
    _, m = read_dat(tmp_path / "m.dat")
    assert np.array_equal(m[-1, 1:], states[-1, 0])


def test_hierarchy_norm_and_threshold_filter():
    n = 4
    sysd = hb.System(ho.synthetic_hamiltonian(n, 2), [35.0] * n, [50.0] * n, [0.0] * n, 2, 300.0, 3)
    with hb.from_system(sysd) as H:
        top = np.zeros(n * n * 2)
        top[0] = 1.0
        H.set_top(top)
        H.rk4_steps(1e-15, 30)
        y = H.get_state().reshape(H.matrices, n * n * 2)
        norms = H.hierarchy_norm()
        assert np.max(np.abs(norms - (y ** 2).sum(axis=1))) <= 1e-15 * norms.max()
        # filter: protect two ADOs, switch off every other at or below the median
        mask = np.ones(H.matrices, np.uint8)
        low = np.argsort(norms)[:3]
        mask[low[:2]] = 2
        H.set_mask(mask)
        thr = float(np.median(norms))
        H.hierarchy_norm(thr)
        got = H.get_mask()
        want = mask.copy()
        want[(norms <= thr) & (mask != 2)] = 0
        assert np.array_equal(got, want)


@pytest.mark.parametrize("scheme,filtering", [("product", None), ("reference", None),
                                              ("product", ("single_excitation", 1))])
def test_linear_absorption_app_matches_oracle(tmp_path, scheme, filtering):
    """tr(D- rho_top(t)) after D+ |g><g|, averaged over the three tensor
    components, against the oracle propagating the ground-state system."""
    cfg = LA_CFG
    if filtering:
        cfg = cfg.replace("strategy=none", f"strategy={filtering[0]}").replace(
            "first_layer=-1", f"first_layer={filtering[1]}")
    (tmp_path / "heom.cfg").write_text(cfg)
    (tmp_path / "rt.cfg").write_text(f"[cuda]\ndevice_index=0\nrk4_scheme={scheme}\n")
    r = subprocess.run([LA_APP, "rt.cfg", "heom.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    hdr, got = read_dat(tmp_path / "la.dat")
    assert hdr == ["time", "trace_real", "trace_imag"]
    assert np.allclose(got[:, 0], np.arange(5) * 5e-15, rtol=1e-15, atol=0)
    # the state system: ground state 0 with zero H row/column and no bath, sites 1..3
    h = np.array([[12410.0, -87.7, 5.5], [-87.7, 12530.0, 30.8], [5.5, 30.8, 12210.0]])
    hs = np.zeros((4, 4))
    hs[1:, 1:] = h
    coupling = np.array([[-1], [0], [1], [2]], np.int32)
    sysd = ho.make_system(hs, [35] * 3, [50] * 3, [0] * 3, 2, 77.0, 3, coupling=coupling)
    mask = None
    if filtering:
        import make_golden as mg
        mask = mg.single_excitation_mask(ho.build_graph(6, 3), 2, filtering[1])
    prob = ho.build_problem(sysd, mask=mask)
    dirs = np.array([[-0.741, -0.561, -0.370], [-0.857, 0.504, -0.107], [-0.197, 0.957, -0.211]])
    strengths = np.array([4, 3.5, 4.2])
    want = np.zeros(5, complex)
    for comp in range(3):  # tensor_components {{0, 0}, {1, 1}, {2, 2}}, prefactors 1
        v = dirs[:, comp] * strengths
        dm = np.zeros((4, 4))
        dm[0, 1:] = v
        dp = dm.T
        top = np.zeros((4, 4))
        top[:, 0] = dp[:, 0]
        y = np.zeros(prob.state_len)
        y[0:32:2] = top.reshape(-1)
        for row in range(5):
            if row:
                y, _ = ho.propagate(prob, 1e-15, 5, 5, y=y)
            rho = (y[0:32:2] + 1j * y[1:32:2]).reshape(4, 4)
            want[row] += np.trace(dm @ rho)
    want /= 3
    scale = np.max(np.abs(want))
    assert np.max(np.abs(got[:, 1] - want.real)) <= 1e-10 * scale
    assert np.max(np.abs(got[:, 2] - want.imag)) <= 1e-10 * scale
    # at t = 0 the trace is the mean squared dipole length over the components
    assert abs(want[0] - sum(np.sum((dirs[:, c] * strengths) ** 2) for c in range(3)) / 3) <= 1e-12 * scale


def test_circular_dichroism_app_matches_oracle(tmp_path):
    """As linear absorption with the magnetic dipole (center x direction) in
    D- and no filtering mask (the configured filter is not applied)."""
    cfg = LA_CFG.replace("task=linear_absorption", "task=circular_dichroism").replace(
        "strategy=none", "strategy=single_excitation").replace("first_layer=-1", "first_layer=1")
    (tmp_path / "heom.cfg").write_text(cfg)
    (tmp_path / "rt.cfg").write_text("[cuda]\ndevice_index=0\n")
    r = subprocess.run([CD_APP, "rt.cfg", "heom.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    hdr, got = read_dat(tmp_path / "la.dat")
    assert hdr == ["time", "trace_real", "trace_imag"]
    h = np.array([[12410.0, -87.7, 5.5], [-87.7, 12530.0, 30.8], [5.5, 30.8, 12210.0]])
    hs = np.zeros((4, 4))
    hs[1:, 1:] = h
    coupling = np.array([[-1], [0], [1], [2]], np.int32)
    prob = ho.build_problem(ho.make_system(hs, [35] * 3, [50] * 3, [0] * 3, 2, 77.0, 3, coupling=coupling))
    dirs = np.array([[-0.741, -0.561, -0.370], [-0.857, 0.504, -0.107], [-0.197, 0.957, -0.211]])
    ctrs = np.array([[2.651, 0.260, -1.135], [1.561, -0.152, -1.725], [0.339, -1.361, -1.385]])
    strengths = np.array([4, 3.5, 4.2])
    mag = np.cross(ctrs, dirs)
    want = np.zeros(5, complex)
    for comp in range(3):
        dm = np.zeros((4, 4))
        dm[0, 1:] = mag[:, comp] * strengths
        dp = np.zeros((4, 4))
        dp[1:, 0] = dirs[:, comp] * strengths
        y = np.zeros(prob.state_len)
        y[0:32:2] = (dp @ np.diag([1.0, 0, 0, 0])).reshape(-1)
        for row in range(5):
            if row:
                y, _ = ho.propagate(prob, 1e-15, 5, 5, y=y)
            rho = (y[0:32:2] + 1j * y[1:32:2]).reshape(4, 4)
            want[row] += np.trace(dm @ rho)
    want /= 3
    scale = np.max(np.abs(want))
    assert np.max(np.abs(got[:, 1] - want.real)) <= 1e-10 * scale
    assert np.max(np.abs(got[:, 2] - want.imag)) <= 1e-10 * scale


def test_app_tracks_flows_like_the_reference_solver(tmp_path):
    """solver.track_flows = true (population_dynamics_solver.hpp:141-150,
    236-263): the application hands two flow buffers to the derivative, the
    stepping zeroes them at every step and accumulates dt b_i x the plus and
    minus terms of every evaluation; the flow file holds, at every
    observation, the sum over ADOs of each buffer's hierarchy norm after the
    last step.  Checked against the reference's own kernel terms (the kernel
    built with HEOM_ODE_DISABLE_PLUS / _MINUS) over the classical RK4 stage
    inputs of the oracle; the populations are those of the untracked run."""
    cfg = FMO_CFG.replace("track_flows=false", "track_flows=true").replace("flow_filename=", "flow_filename=f.dat")
    (tmp_path / "heom.cfg").write_text(cfg)
    (tmp_path / "rt.cfg").write_text("[cuda]\ndevice_index=0\n")
    r = subprocess.run([APP, "rt.cfg", "heom.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    h = np.array([[12410.0, -87.7, 5.5], [-87.7, 12530.0, 30.8], [5.5, 30.8, 12210.0]])
    prob = ho.build_problem(ho.make_system(h, [35] * 3, [50] * 3, [0] * 3, 2, 77.0, 3))
    dt = 1e-15
    _, ref = ho.propagate(prob, dt, 20, 5)
    _, d = read_dat(tmp_path / "d.dat")
    assert_pops(d[:, 1:], ref)
    hf, f = read_dat(tmp_path / "f.dat")
    assert hf == ["time", "flow_from_above_norm", "flow_from_below_norm"]
    assert f.shape == (4, 3)  # one row per observation after t = 0

    def terms(v):
        full, _ = ho.ref_derivative(prob, v)
        return full - ho.ref_derivative(prob, v, mode=3)[0], full - ho.ref_derivative(prob, v, mode=4)[0]

    y = prob.initial_state()
    for obs_row in range(4):
        for step in range(5):
            k1, _ = ho.ref_derivative(prob, y)
            s2 = y + 0.5 * dt * k1
            k2, _ = ho.ref_derivative(prob, s2)
            s3 = y + 0.5 * dt * k2
            k3, _ = ho.ref_derivative(prob, s3)
            s4 = y + dt * k3
            k4, _ = ho.ref_derivative(prob, s4)
            above = np.zeros_like(y)
            below = np.zeros_like(y)
            for s, b in zip((y, s2, s3, s4), (1 / 6, 1 / 3, 1 / 3, 1 / 6)):
                p, m = terms(s)
                above += dt * b * p
                below += dt * b * m
            y = y + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        want = [float(np.sum(x ** 2)) for x in (above, below)]
        assert f[obs_row, 0] == pytest.approx((obs_row + 1) * 5 * dt, rel=1e-14)
        for c in range(2):
            assert abs(f[obs_row, 1 + c] - want[c]) <= 1e-10 * want[c], (obs_row, c, f[obs_row, 1 + c], want[c])
