"""Checks of the oracle's static-terrain path (test infrastructure).

The reference's terrain kernels cannot be run here (no AMReX), so the
terrain restatement is pinned by properties instead of golden vectors:
  * on flat terrain the terrain path reproduces the flat path to round-off;
  * sum(detJ * rho) is conserved (flux form, Omega = 0 at the ground);
  * an atmosphere at rest in the discrete hydrostatic base state over a hill
    stays at rest to round-off (no spurious metric or boundary terms).
"""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from erf_b200 import terrain as T


def _small_hill(**kw):
    args = dict(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0, r0=100.0, amp=5.0)
    args.update(kw)
    return T.abl_terrain(**args)


@pytest.mark.parametrize("mk", [cases.abl_dry, cases.abl_deardorff])
def test_flat_terrain_reduces_to_flat_path(mk):
    case = mk(nx=12, ny=10, nz=12)
    cfg = case.cfg
    base = oracle.make_base_state(cfg, case)
    cons, u, v, w = case.build_state(base[0])
    ref = oracle.advance(cfg, base, cons, u, v, w, 3)
    znd = T.btf_nodes(T.zlevels(cfg.nz, cfg.dz), np.zeros((cfg.ny + 1, cfg.nx + 1)))
    base3 = [np.repeat(b[:, None], cfg.ny * cfg.nx, axis=1).ravel() for b in base]
    tc = cfg.copy()
    tc.use_terrain = 1
    got = oracle.advance_terrain(tc, znd, base3, cons, u, v, w, 3)
    scale = [np.abs(ref[0]).max(), 10.0, 10.0, 1.0]
    for a, b, s in zip(got, ref, scale):
        assert np.max(np.abs(a - b)) <= 1e-11 * s


def test_terrain_metrics_of_btf_grid():
    case = _small_hill()
    detJ, zcc, ax, ay = oracle.terrain_metrics(case.cfg, case.z_nd)
    assert detJ.min() > 0.0
    # the column heights sum to the domain height
    assert np.allclose((detJ * case.cfg.dz).sum(axis=0), case.z_nd[-1, :-1, :-1] * 0 + (
        0.25 * (case.z_nd[-1, :-1, :-1] + case.z_nd[-1, 1:, :-1] + case.z_nd[-1, :-1, 1:] + case.z_nd[-1, 1:, 1:]
                - case.z_nd[0, :-1, :-1] - case.z_nd[0, 1:, :-1] - case.z_nd[0, :-1, 1:] - case.z_nd[0, 1:, 1:])),
        rtol=1e-12)
    assert np.allclose(zcc, T.cell_heights(case.z_nd), rtol=1e-14)


def test_terrain_conserves_mass():
    case = _small_hill()
    cfg = case.cfg
    base = oracle.make_base_state_terrain(case)
    cons, u, v, w = case.build_state(base[0])
    detJ, *_ = oracle.terrain_metrics(cfg, case.z_nd)
    got = oracle.advance_terrain(cfg, case.z_nd, base, cons, u, v, w, 3)
    m0, m1 = (cons[0] * detJ).sum(), (got[0][0] * detJ).sum()
    assert abs(m1 - m0) <= 1e-14 * m0
    assert all(np.isfinite(a).all() for a in got)
    assert np.abs(got[3]).max() > 0.1          # flow over the hill lifts


def test_resting_atmosphere_over_terrain_stays_at_rest():
    case = _small_hill(u0=0.0)
    cfg = case.cfg
    cfg.use_coriolis = 0
    cfg.abl_geo_forcing[0] = 0.0
    case.pert = {"tke0": 1e-3}
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    base = oracle.make_base_state_terrain(case)
    r0, _, _, th0 = [b.reshape(nz + 2, ny, nx) for b in base]
    cons, u, v, w = case.build_state(base[0])
    cons[1] = r0[1:nz + 1] * th0[1:nz + 1]
    got = oracle.advance_terrain(cfg, case.z_nd, base, cons, u, v, w, 3)
    for a in got[1:]:
        assert np.abs(a).max() < 1e-5
