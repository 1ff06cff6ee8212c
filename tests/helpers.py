"""Shared helpers for the parity tests."""
import numpy as np

FIELDS = ("rho", "rhotheta", "rhoKE", "rhoQKE", "rhoscalar", "rhoqv", "rhoqc", "rhoqr")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    if den == 0.0:
        return num
    return num / den


def compare_states(got, ref):
    """Per-field relative L2 of (cons comps..., u, v, w, theta)."""
    cg, ug, vg, wg = got
    cr, ur, vr, wr = ref
    out = {}
    for n in range(cr.shape[0]):
        if not np.any(cr[n]) and not np.any(cg[n]):
            continue
        out[FIELDS[n]] = rel_l2(cg[n], cr[n])
    out["u"] = rel_l2(ug, ur)
    out["v"] = rel_l2(vg, vr)
    out["w"] = rel_l2(wg, wr)
    out["theta"] = rel_l2(cg[1] / cg[0], cr[1] / cr[0])
    return out
