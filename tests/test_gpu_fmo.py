"""GPU: the applications on the reference's own example configurations
(tests/golden/fmo/: data/examples_fmo/ of noma/dm-heom with solver.steps
reduced by tests/golden/make_fmo_fixtures.py, nothing else changed), run with
the reference command line, against the oracle.

  * fmo_population_dynamics_77K.cfg: 7 sites, depth 3, M = 2, 77 K, the three
    observers it configures (matrix_complete, matrix_diagonal,
    matrix_trace_id), 100 steps observed every 5;
  * fmo_linear_absorption_77K.cfg and fmo_circular_dichroism_77K.cfg: the
    dipole pseudo pathway on the ground-state state system, trace observer,
    50 steps of 1 fs and 5 fs.
Tolerances: populations 1e-10 relative (parity.py); traces 1e-10 of the
largest trace."""
import ctypes as C
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho
from parity import assert_pops

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(hb.__file__), "bin")
FMO = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fmo")


def read_dat(path):
    lines = open(path).read().strip().split("\n")
    return lines[0].split("\t"), np.array([[float(x) for x in l.split("\t")] for l in lines[1:]])


def config_system(path):
    """(H cm^-1 [n, n], lambda, invnu, omega, matsubaras, temperature, depth) of a config."""
    c = hb.Config(path)
    d = c.system_desc()
    n, b = d.sites, d.baths
    arr = lambda p, k: np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(k,)).copy()
    h = arr(d.hamiltonian, 2 * n * n)
    h = (h[0::2] + 1j * h[1::2]).reshape(n, n)
    return (h.real if not np.any(h.imag) else h, arr(d.lambda_, b), arr(d.invnu, b), arr(d.omega, b),
            d.matsubaras, d.temperature, d.ado_depth, c)


def run_app(app, cfg_name, tmp_path):
    shutil.copy(os.path.join(FMO, cfg_name), tmp_path / cfg_name)
    (tmp_path / "runtime.cfg").write_text("[cuda]\ndevice_index=0\n")
    r = subprocess.run([os.path.join(BIN, app), "runtime.cfg", cfg_name], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_fmo_population_dynamics_example(tmp_path):
    name = "fmo_population_dynamics_77K.cfg"
    run_app("heom_population_dynamics", name, tmp_path)
    h, lam, inv, om, m, temp, depth, c = config_system(os.path.join(FMO, name))
    n = h.shape[0]
    steps, every, dt = int(c.get("solver.steps")), int(c.get("program.observe_steps")), float(c.get("solver.step_size"))
    prob = ho.build_problem(ho.make_system(h, lam, inv, om, m, temp, depth))
    _, ref = ho.propagate(prob, dt, steps, every)
    hd, d = read_dat(tmp_path / "fmo_population_dynamics_77K_diagonal.dat")
    assert hd == ["time"] + [f"site_{i}" for i in range(n)]
    assert d.shape == (steps // every + 1, n + 1)
    assert np.allclose(d[:, 0], np.arange(steps // every + 1) * every * dt, rtol=1e-14, atol=0)
    assert_pops(d[:, 1:], ref, what="FMO 77 K site populations")
    _, t = read_dat(tmp_path / "fmo_population_dynamics_77K_trace.dat")
    assert np.max(np.abs(t[:, 1] - 1.0)) <= 1e-12
    _, mc = read_dat(tmp_path / "fmo_population_dynamics_77K_matrix.dat")
    assert np.array_equal(mc[:, 1:][:, [(n + 1) * 2 * i for i in range(n)]], d[:, 1:])
    assert np.max(np.abs(ref[-1] - ref[0])) > 1e-2  # energy transfer happened


def parse_matrix(text):
    return np.array([[float(x) for x in row.split(",")] for row in re.findall(r"\{([^{}]*)\}", text)])


@pytest.mark.parametrize("kind", ["linear_absorption", "circular_dichroism"])
def test_fmo_spectroscopy_examples(tmp_path, kind):
    name = f"fmo_{kind}_77K.cfg"
    run_app(f"heom_{kind}", name, tmp_path)
    h, lam, inv, om, m, temp, depth, c = config_system(os.path.join(FMO, name))
    n = h.shape[0]
    steps, every, dt = int(c.get("solver.steps")), int(c.get("program.observe_steps")), float(c.get("solver.step_size"))
    dirs = parse_matrix(c.get("dipole.directions"))
    ctrs = parse_matrix(c.get("dipole.centers"))
    strengths = np.array([float(x) for x in re.findall(r"[-+0-9.eE]+", c.get("dipole.strengths"))])
    comps = parse_matrix(c.get("dipole.tensor_components")).astype(int)
    pref = [float(x) for x in re.findall(r"[-+0-9.eE]+", c.get("dipole.tensor_prefactors"))]
    assert c.get("filtering.strategy") == "none"
    # the state system: ground state 0 with zero H row and column and no bath, sites 1..n
    hs = np.zeros((n + 1, n + 1), dtype=h.dtype)
    hs[1:, 1:] = h
    coupling = np.array([[-1]] + [[i] for i in range(n)], np.int32)
    prob = ho.build_problem(ho.make_system(hs, lam, inv, om, m, temp, depth, coupling=coupling))
    minus_vec = np.cross(ctrs, dirs) if kind == "circular_dichroism" else dirs
    rows = steps // every + 1
    want = np.zeros(rows, complex)
    N = n + 1
    for (cm, cp), p in zip(comps, pref):  # tensor component: (minus, plus) indices of the pathway
        dm = np.zeros((N, N))
        dm[0, 1:] = minus_vec[:, cm] * strengths * p
        dp = np.zeros((N, N))
        dp[1:, 0] = dirs[:, cp] * strengths
        y = np.zeros(prob.state_len)
        y[0:2 * N * N:2] = (dp @ np.diag([1.0] + [0.0] * n)).reshape(-1)
        for row in range(rows):
            if row:
                y, _ = ho.propagate(prob, dt, every, every, y=y)
            rho = (y[0:2 * N * N:2] + 1j * y[1:2 * N * N:2]).reshape(N, N)
            want[row] += np.trace(dm @ rho)
    want /= len(comps)
    hdr, got = read_dat(tmp_path / f"fmo_{kind}_77K.dat")
    assert hdr == ["time", "trace_real", "trace_imag"]
    assert got.shape == (rows, 3)
    scale = np.max(np.abs(want))
    err = max(np.max(np.abs(got[:, 1] - want.real)), np.max(np.abs(got[:, 2] - want.imag))) / scale
    print(f"{kind}: max trace error {err:.3e} of the largest trace")
    assert err <= 1e-10
