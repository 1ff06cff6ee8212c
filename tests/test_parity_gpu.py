"""GPU parity: the CUDA dycore (through the C-ABI) against the CPU FP64 oracle.

Bar: relative L2 <= 1e-10 per field after 10 full RK3 steps (the FP64 plain
form's parity target), on seeded synthetic inputs small enough for the oracle.
"""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from helpers import compare_states

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _dycore(cfg):
    from erf_b200 import Dycore
    return Dycore(cfg)


def run_both(case, nsteps):
    dy = _dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    got = dy.advance_host(cons, u, v, w, nsteps)
    st = dy.status()
    ref = oracle.advance(case.cfg, base, cons, u, v, w, nsteps)
    dy.close()
    return compare_states(got, ref), st


def test_base_state_matches_oracle():
    case = cases.moist_bubble(nx=16, ny=16, nz=80)
    dy = _dycore(case.cfg)
    got = dy.make_base_state(case)
    ref = oracle.make_base_state(case.cfg, case)
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r) / np.abs(r)) < 1e-13


@pytest.mark.parametrize("nsteps", [1, 10])
def test_abl_dry_smagorinsky(nsteps):
    case = cases.abl_dry(nx=24, ny=20, nz=16)
    errs, st = run_both(case, nsteps)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


@pytest.mark.parametrize("nsteps", [1, 10])
def test_moist_bubble_kessler_weno5(nsteps):
    case = cases.moist_bubble(nx=24, ny=20, nz=40)
    case.pert["bubble_rh"] = 6000.0
    errs, st = run_both(case, nsteps)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


@pytest.mark.parametrize("diffusing", [False, True])
def test_gpu_reproduces_taylor_green_gold(diffusing):
    """The CUDA path against the reference's gold plotfile directly."""
    import os
    from golden.reference_cases import plot_variables, taylor_green
    name, cfg, base, state, nsteps = taylor_green(diffusing)
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}_gold.npz"))
    dy = _dycore(cfg)
    dy.set_base_state(base)
    out = dy.advance_host(*state, nsteps)
    assert dy.status() == 0
    dy.close()
    for nm, a, b in zip(gold["names"], plot_variables(out), gold["data"]):
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err <= 2e-10, (str(nm), err)


@pytest.mark.parametrize("nsteps", [1, 10])
def test_abl_deardorff(nsteps):
    """Deardorff TKE closure: rho*KE as a slow variable with its buoyancy,
    shear-production and dissipation sources, Theta_v for theta's vertical
    diffusion (neutral and stratified mixing lengths both occur)."""
    case = cases.abl_deardorff(nx=24, ny=20, nz=16)
    errs, st = run_both(case, nsteps)
    assert st == 0
    assert "rhoKE" in errs
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


def _moist_deardorff():
    from erf_b200 import config as C
    case = cases.moist_bubble(nx=20, ny=16, nz=40)
    case.pert["bubble_rh"] = 6000.0
    c = case.cfg
    c.les_type = C.LES_DEARDORFF
    c.Ck, c.Ce, c.Ce_wall, c.sigma_k, c.theta_ref = 0.1, 0.93, 0.0, 0.5, 300.0
    case.pert["tke0"] = 0.5
    case.pert["tke0_zmax"] = 2000.0
    return case


def test_moist_bubble_deardorff_kessler():
    """Deardorff with three moisture species: five slow variables per cell."""
    errs, st = run_both(_moist_deardorff(), 3)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


def test_deardorff_stationary_shear_known_answer():
    """The CUDA path keeps e = Ck/Ce (S Delta)^2 in uniform shear u = S z with
    neutral theta, where shear production balances dissipation."""
    from erf_b200 import config as C
    case = cases.abl_deardorff(nx=8, ny=8, nz=32)
    cfg = case.cfg
    cfg.use_coriolis = 0
    cfg.abl_geo_forcing[0] = cfg.abl_geo_forcing[1] = 0.0
    cfg.zlo_bc = cfg.zhi_bc = C.BC_SLIP_WALL
    case.theta_cc = np.full(cfg.nz, 300.0)
    case.pert = {}
    dy = _dycore(cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    S = 0.01
    z = (np.arange(cfg.nz) + 0.5) * cfg.dz
    u[:] = (S * z)[:, None, None]
    delta = (cfg.dx * cfg.dy * cfg.dz) ** (1.0 / 3.0)
    e_eq = cfg.Ck / cfg.Ce * (S * delta) ** 2
    cons[2] = cons[0] * e_eq
    c2, *_ = dy.advance_host(cons, u, v, w, 1)
    assert dy.status() == 0
    dy.close()
    e = c2[2] / c2[0]
    assert np.max(np.abs(e[12:20] / e_eq - 1.0)) < 1e-10
