"""GPU at the benchmark's full size: 8 sites, one Drude-Lorentz bath per site
with one Matsubara term (16 modes), depth 8 (735,471 ADOs of 8 x 8), RK4
dt = 0.5 fs.

Checked here: two full RK4 steps against the oracle (whole state), and over a
longer run the size-independent properties of the propagator: conservation
of the trace of the top, Hermiticity of the top, agreement of the three RK4
evaluation orders.
"""
import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho

pytestmark = pytest.mark.gpu

N, DEPTH, M, SEED, DT = 8, 8, 2, 22, 0.5e-15


@pytest.fixture(scope="module")
def system():
    h = ho.synthetic_hamiltonian(N, SEED)
    return h, hb.System(h, [35.0] * N, [50.0] * N, [0.0] * N, M, 300.0, DEPTH)


def initial(n_states, length):
    y = np.zeros(length)
    y[0] = 1.0
    return y


def test_two_steps_match_oracle_full_state(system):
    h, sysd = system
    prob = ho.build_problem(ho.drude_system(N, DEPTH, M, seed=SEED))
    y0 = prob.initial_state()
    ref = ho.rk4_step(prob, DT, ho.rk4_step(prob, DT, y0))
    with hb.from_system(sysd) as H:
        assert H.matrices == 735471
        H.set_state(y0)
        H.rk4_steps(DT, 2)
        out = H.get_state()
    err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    assert err <= 1e-12, err


def test_properties_over_long_run(system):
    _, sysd = system
    res = {}
    for scheme in ("product", "horner", "reference"):
        with hb.from_system(sysd, scheme=scheme) as H:
            H.set_state(initial(N, H.state_len))
            tops = H.propagate(DT, 200, 10)
            res[scheme] = tops
    for scheme, tops in res.items():
        for row in tops:
            rho = (row[0::2] + 1j * row[1::2]).reshape(N, N)
            assert abs(np.trace(rho) - 1.0) <= 1e-12, scheme
            assert np.max(np.abs(rho - rho.conj().T)) <= 1e-12, scheme
            assert np.all(np.diag(rho).real >= -1e-9), scheme
    for scheme in ("horner", "reference"):
        assert np.max(np.abs(res[scheme] - res["product"])) <= 1e-11
