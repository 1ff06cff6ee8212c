"""GPU: the FP32-bulk mixed form against the FP64 oracle.

The mixed form keeps the prognostic state, the base state and the equation of
state in FP64 and runs advection, diffusion and the acoustic substeps in FP32.
Its error budget: relative L2 <= 1e-2 in u, v, w and theta after 100 full RK3
steps against the FP64 oracle on the same seeded inputs.  The errors of the
other outputs (qv, qc, qr, surface pressure) are computed and printed.
"""
import json

import numpy as np
import pytest

import oracle
from erf_b200 import cases, config as C
from helpers import rel_l2

pytestmark = pytest.mark.gpu
TOL_MIXED = 1e-2


def output_errors(got, ref, moist):
    """Relative L2 of the output fields (u, v, w, theta, water species, surface pressure)."""
    cg, ug, vg, wg = got
    cr, ur, vr, wr = ref
    err = {"u": rel_l2(ug, ur), "v": rel_l2(vg, vr), "w": rel_l2(wg, wr),
           "theta": rel_l2(cg[1] / cg[0], cr[1] / cr[0])}
    if moist:
        for n, nm in ((5, "qv"), (6, "qc"), (7, "qr")):
            if n < cr.shape[0]:
                err[nm] = rel_l2(cg[n] / cg[0], cr[n] / cr[0])

    def psfc(c):
        qv = c[5, 0] / c[0, 0] if moist else 0.0
        return 1.0e5 * (287.0 * c[1, 0] * (1.0 + 461.505 / 287.0 * qv) / 1.0e5) ** 1.4
    err["p_sfc"] = rel_l2(psfc(cg), psfc(cr))
    return err


def run_mixed_vs_oracle(case, nsteps):
    from erf_b200 import Dycore
    case.cfg.precision = C.PREC_MIXED
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    got = dy.advance_host(cons, u, v, w, nsteps)
    st = dy.status()
    dy.close()
    case.cfg.precision = C.PREC_FP64
    ref = oracle.advance(case.cfg, base, cons, u, v, w, nsteps)
    return output_errors(got, ref, case.cfg.moisture != C.MOIST_NONE), st


def test_mixed_moist_bubble_100_steps():
    case = cases.moist_bubble(nx=32, ny=32, nz=40)
    case.pert["bubble_rh"] = 8000.0
    err, st = run_mixed_vs_oracle(case, 100)
    print("mixed moist_bubble 32x32x40, 100 steps:", json.dumps(err))
    assert st == 0
    for f in ("u", "v", "w", "theta"):
        assert err[f] <= TOL_MIXED, err


def test_mixed_abl_dry_100_steps():
    case = cases.abl_dry(nx=24, ny=20, nz=16)
    err, st = run_mixed_vs_oracle(case, 100)
    print("mixed abl_dry 24x20x16, 100 steps:", json.dumps(err))
    assert st == 0
    for f in ("u", "v", "w", "theta"):
        assert err[f] <= TOL_MIXED, err


def test_mixed_is_not_the_plain_form():
    """The mixed form really computes in FP32: it differs from the FP64 oracle
    by more than FP64 round-off after one step, yet stays within budget."""
    case = cases.moist_bubble(nx=24, ny=20, nz=40)
    case.pert["bubble_rh"] = 6000.0
    err, st = run_mixed_vs_oracle(case, 1)
    assert st == 0
    assert max(err["u"], err["theta"]) > 1e-12, err
    assert max(err[f] for f in ("u", "v", "w", "theta")) <= TOL_MIXED, err
