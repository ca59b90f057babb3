"""GPU: heom_rk4_steps_noalloc, the entry point for callers that cannot call
cudaMalloc while they step (code inside another runtime's device-memory
arena, or a latency-critical loop that must not take cudaMalloc's implicit
device synchronisation).  Its stage buffers live in a static device array in
the library; the test owns the state buffer (allocated here, not by the
library) and compares two consecutive calls with the ordinary entry point
heom_rk4_steps on the same system.  Collected last on purpose, and
self-contained so that it also passes alone in a fresh process."""
import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho

pytestmark = pytest.mark.gpu

TOL = 1e-12  # same kernels in the same order: agreement to rounding


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_noalloc_matches_rk4_steps_on_two_calls():
    import torch
    sysd = hb.System(ho.synthetic_hamiltonian(7, 11), [35.0] * 7, [50.0] * 7, [0.0] * 7, 1, 300.0, 4)
    with hb.from_system(sysd, scheme="product") as H:
        y0 = np.zeros(H.state_len)
        y0[0] = 1.0
        H.set_state(y0)
        H.rk4_steps(1e-15, 40)
        ref1 = H.get_state()
        H.rk4_steps(1e-15, 40)
        ref2 = H.get_state()

        d = torch.tensor(y0, dtype=torch.float64, device="cuda")  # caller-owned device memory
        out1_host = torch.empty_like(d, device="cpu")
        torch.cuda.synchronize()  # the call's stream does not wait for torch's: finish the writes first
        free_before = torch.cuda.mem_get_info()[0]
        H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 40)
        free_after_first = torch.cuda.mem_get_info()[0]
        out1_host.copy_(d)
        H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 40)
        free_after_second = torch.cuda.mem_get_info()[0]
        out1 = out1_host.numpy()
        out2 = d.cpu().numpy()
    assert rel_err(out1, ref1) <= TOL
    assert rel_err(out2, ref2) <= TOL
    # neither call allocated device memory (device-wide free memory, read with
    # no allocation of this process in between)
    assert free_after_first == free_before
    assert free_after_second == free_before
    pops = [out2[(7 + 1) * 2 * i] for i in range(7)]
    assert abs(sum(pops) - 1.0) <= 1e-12


def test_noalloc_rejects_hierarchies_beyond_the_scratch():
    import torch
    # 8 sites, 16 modes, depth 5: 20349 ADOs x 1 KB > 16 MiB per buffer
    sysd = hb.System(ho.synthetic_hamiltonian(8, 22), [35.0] * 8, [50.0] * 8, [0.0] * 8, 2, 300.0, 5)
    with hb.from_system(sysd) as H:
        d = torch.zeros(H.state_len, dtype=torch.float64, device="cuda")
        with pytest.raises(hb.HeomError) as e:
            H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 1)
    assert "heom error -5" in str(e.value) and "static scratch" in str(e.value)


def test_noalloc_refuses_handle_state_it_cannot_honour():
    """A time-dependent field, host pre-evaluate actions and flow buffers need
    buffers that the static scratch does not hold: the call is refused with
    HEOM_E_UNSUPPORTED (-5) before anything is launched."""
    import torch
    n = 4
    sysd = hb.System(ho.synthetic_hamiltonian(n, 3), [35.0] * n, [50.0] * n, [0.0] * n, 1, 300.0, 2)
    pulse = {"efield": 1e8, "time_center": 0.0, "time_width": 5e-15, "frequency": 0.0, "phase": 0.0}
    dp = np.eye(n, k=1)
    with hb.from_system(sysd) as H:
        d = torch.zeros(H.state_len, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        H.set_field(dp, dp.T, pulse, pulse)
        with pytest.raises(hb.HeomError) as e:
            H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 1)
        assert "heom error -5" in str(e.value) and "field" in str(e.value)
        H.clear_field()
        H.add_pre_evaluate_action(lambda h, t, dt: 0)
        with pytest.raises(hb.HeomError) as e:
            H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 1)
        assert "heom error -5" in str(e.value) and "pre-evaluate" in str(e.value)
        H.clear_pre_evaluate_actions()
        above, below = H.buffer(), H.buffer()
        H.set_flow_buffers(above, below)
        with pytest.raises(hb.HeomError) as e:
            H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 1)
        assert "heom error -5" in str(e.value) and "flow" in str(e.value)
        H.set_flow_buffers(None, None)
        H.rk4_steps_noalloc(d.data_ptr(), 1e-15, 1)  # plain handle again: accepted
