"""torch.autograd.Function over the adjoint C ABI (heom_adjoint_gradient).

The loss is J = sum_n weights[n] Re(sum_ij conj(O_ij) rho_n(i,j)) of an RK4
propagation from rho0; its inputs are the Hamiltonian H (states x states,
real, cm^-1), lambda (cm^-1) and gamma = 1/invnu (fs^-1), both shared by all
baths.  backward() returns dJ/dH (every entry independent), dJ/dlambda and
dJ/dgamma from one adjoint sweep on the GPU, so any torch parametrisation of
H (site energies, symmetric couplings) gets its gradient by the chain rule.
"""
from __future__ import annotations

import numpy as np
import torch

import heom_b200 as hb


class HeomObservableLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, H, lam, gamma, spec):
        """spec: dict with depth, matsubaras, temperature, omega, dt_fs, steps,
        rho0, observable, weights, device."""
        n = H.shape[0]
        h = H.detach().cpu().numpy().astype(np.float64)
        lam_v = float(lam.detach().cpu())
        gam_v = float(gamma.detach().cpu())
        system = hb.System(h, [lam_v] * n, [1.0 / gam_v] * n, [spec.get("omega", 0.0)] * n,
                           spec["matsubaras"], spec["temperature"], spec["depth"])
        with hb.Adjoint(system, device=spec.get("device", 0)) as A:
            out = A.gradient(spec["rho0"], spec["observable"], spec["weights"], spec["dt_fs"] * 1e-15,
                             spec["steps"])
        ctx.save_for_backward(torch.as_tensor(out["h"].real, dtype=H.dtype),
                              torch.tensor(out["lambda"], dtype=lam.dtype),
                              torch.tensor(out["gamma"], dtype=gamma.dtype))
        return torch.tensor(out["loss"], dtype=H.dtype)

    @staticmethod
    def backward(ctx, g):
        gh, gl, gg = ctx.saved_tensors
        return g * gh, g * gl, g * gg, None
