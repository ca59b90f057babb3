"""Population tolerance shared by the parity tests.

The bar is relative: |p_gpu - p_ref| <= 1e-10 * max(|p_ref|, floor).  The
floor keeps the relative measure meaningful for populations that are still
(near) zero, which are then held to 1e-10 * floor absolute.  Every check
prints the worst relative error it saw (visible with pytest -s or on failure).
"""
import numpy as np

POP_REL = 1e-10   # relative error allowed in populations
POP_FLOOR = 1e-3  # populations below this are held to POP_REL * POP_FLOOR absolute


def pop_rel_err(got, ref, floor=POP_FLOOR):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), floor)))


def assert_pops(got, ref, rel=POP_REL, floor=POP_FLOOR, what="populations"):
    err = pop_rel_err(got, ref, floor)
    print(f"{what}: max relative error {err:.3e} (bar {rel:g}, floor {floor:g})")
    assert err <= rel, f"{what}: max relative error {err:.3e} > {rel:g}"
    return err
