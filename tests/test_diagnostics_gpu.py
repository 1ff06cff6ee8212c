"""GPU: the step diagnostics (erf_b200_diagnostics, the integrated
quantities of ERF's sum_integrated_quantities) and the per-step JSON lines
built on them (erf_b200.metrics.run_logged).

  * the device reduction equals the same sums formed on the host from the
    stored state (mass and rho-theta integrals to 1e-13 relative, max |w|
    exactly), flat and over static terrain;
  * the mass line is a conservation check: periodic sides and walls keep the
    mass to round-off, flat, over static terrain and over moving terrain
    (with and without acoustic substeps);
  * every line parses as JSON with the documented keys.
"""
import io
import json

import numpy as np
import pytest

from erf_b200 import cases, metrics
from erf_b200 import terrain as T

pytestmark = pytest.mark.gpu


def _host_sums(cfg, cons, w, detJ=None):
    vol = cfg.dx * cfg.dy * cfg.dz
    J = 1.0 if detJ is None else detJ
    return float(np.sum(cons[0] * J) * vol), float(np.sum(cons[1] * J) * vol), float(np.max(np.abs(w)))


def _detj(cfg, z):
    return 0.25 / cfg.dz * (z[1:, :-1, :-1] + z[1:, :-1, 1:] + z[1:, 1:, :-1] + z[1:, 1:, 1:]
                            - z[:-1, :-1, :-1] - z[:-1, :-1, 1:] - z[:-1, 1:, :-1] - z[:-1, 1:, 1:])


def _logged(dy, state, nsteps, every=1):
    buf = io.StringIO()
    recs = metrics.run_logged(dy, *state, nsteps, every=every, out=buf)
    lines = [json.loads(ln) for ln in buf.getvalue().splitlines()]
    assert lines == json.loads(json.dumps(recs))
    for rec in lines:
        assert {"step", "time", "mass", "rhotheta", "max_w", "wall_s", "cell_steps_per_s"} <= set(rec)
    return recs


def test_flat_diagnostics_match_host_and_conserve_mass():
    from erf_b200 import Dycore
    case = cases.abl_dry(nx=24, ny=20, nz=16)
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    recs = _logged(dy, init, 6, every=2)
    assert [r["step"] for r in recs] == [0, 2, 4, 6]
    cons, u, v, w = dy.store_state(*init)
    m, rt, wm = _host_sums(case.cfg, cons, w)
    d = dy.diagnostics()
    dy.close()
    assert abs(d["mass"] - m) <= 1e-13 * abs(m)
    assert abs(d["rhotheta"] - rt) <= 1e-13 * abs(rt)
    assert d["max_w"] == wm
    print("flat ABL 24x20x16, mass drift per logged step:", [r.get("mass_drift") for r in recs])
    assert all(abs(r["mass_drift"]) <= 1e-13 for r in recs[1:])


def test_static_terrain_diagnostics_weight_by_detj():
    from erf_b200 import Dycore
    case = T.abl_terrain(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0, r0=100.0, amp=5.0)
    dy = Dycore(case.cfg)
    dy.set_terrain(case.z_nd)
    base = dy.make_base_state_terrain(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    recs = _logged(dy, init, 4)
    cons, u, v, w = dy.store_state(*init)
    m, rt, wm = _host_sums(case.cfg, cons, w, _detj(case.cfg, case.z_nd))
    d = dy.diagnostics()
    dy.close()
    assert abs(d["mass"] - m) <= 1e-13 * abs(m)
    assert abs(d["rhotheta"] - rt) <= 1e-13 * abs(rt)
    assert d["max_w"] == wm
    print("terrain 16x12x16, mass drift:", [r.get("mass_drift") for r in recs])
    assert all(abs(r["mass_drift"]) <= 1e-13 for r in recs[1:])


@pytest.mark.parametrize("substeps", [False, True])
def test_moving_terrain_conserves_physical_mass(substeps):
    """Over the moving grid the integral of rho detJ stays put while detJ
    itself changes under every column."""
    from erf_b200 import Dycore
    case = T.moving_terrain(nx=24, ny=4, nz=30, Lx=120.0, Ly=20.0, H=150.0, ampl=0.5, wavelength=60.0,
                            substeps=substeps, dt=0.05 if substeps else 0.005, steps=8)
    if substeps:
        case.cfg.mri_ratio = 6
    dy = Dycore(case.cfg)
    dy.set_base_state(case.base)
    recs = _logged(dy, case.build_state(), case.steps)
    t, z, _, _ = dy.moving_terrain_state()
    cons, u, v, w = dy.store_state(*case.build_state())
    m, _, _ = _host_sums(case.cfg, cons, w, _detj(case.cfg, z))
    d = dy.diagnostics()
    dy.close()
    assert abs(d["mass"] - m) <= 1e-13 * abs(m)
    print("moving terrain, substeps", substeps, "mass drift:", [r.get("mass_drift") for r in recs])
    assert all(abs(r["mass_drift"]) <= 1e-13 for r in recs[1:])
    assert recs[-1]["time"] == pytest.approx(case.steps * case.cfg.dt)
