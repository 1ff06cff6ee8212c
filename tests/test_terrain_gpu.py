"""GPU parity over static terrain: the CUDA terrain passes (through the C-ABI)
against the CPU FP64 oracle's terrain restatement.

Bar: relative L2 <= 1e-10 per field after 1 and 10 full RK3 steps (plain
FP64), on a small periodic hill with stretched levels.
"""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from erf_b200 import config as C
from erf_b200 import terrain as T
from helpers import compare_states

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _hill(**kw):
    args = dict(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0, r0=100.0, amp=5.0)
    args.update(kw)
    return T.abl_terrain(**args)


def _gpu_run(case, nsteps, precision=C.PREC_FP64):
    from erf_b200 import Dycore
    cfg = case.cfg.copy()
    cfg.precision = precision
    dy = Dycore(cfg)
    dy.set_terrain(case.z_nd)
    base = dy.make_base_state_terrain(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    got = dy.advance_host(cons, u, v, w, nsteps)
    st = dy.status()
    dy.close()
    return base, (cons, u, v, w), got, st


def test_terrain_base_state_matches_oracle():
    case = _hill()
    from erf_b200 import Dycore
    dy = Dycore(case.cfg)
    dy.set_terrain(case.z_nd)
    got = dy.make_base_state_terrain(case)
    dy.close()
    ref = oracle.make_base_state_terrain(case)
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r) / np.abs(r)) < 1e-13


@pytest.mark.parametrize("les", ["deardorff", "smagorinsky"])
@pytest.mark.parametrize("nsteps", [1, 10])
def test_terrain_parity(les, nsteps):
    case = _hill(les=les)
    base, init, got, st = _gpu_run(case, nsteps)
    assert st == 0
    ref = oracle.advance_terrain(case.cfg, case.z_nd, base, *init, nsteps)
    errs = compare_states(got, ref)
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


def test_terrain_parity_slip_ground_upwind3():
    """Slip ground (the GradWz-extrapolated strain planes) and Upwind_3rd."""
    case = _hill()
    c = case.cfg
    c.zlo_bc = C.BC_SLIP_WALL
    for f in ("dycore_horiz_adv", "dycore_vert_adv", "dryscal_horiz_adv", "dryscal_vert_adv"):
        setattr(c, f, C.UPWIND_3RD)
    base, init, got, st = _gpu_run(case, 5)
    assert st == 0
    ref = oracle.advance_terrain(case.cfg, case.z_nd, base, *init, 5)
    errs = compare_states(got, ref)
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


def test_terrain_mixed_form_error():
    """FP32 bulk over terrain stays close to the FP64 oracle (10 steps)."""
    case = _hill()
    base, init, got, st = _gpu_run(case, 10, precision=C.PREC_MIXED)
    assert st == 0
    ref = oracle.advance_terrain(case.cfg, case.z_nd, base, *init, 10)
    errs = compare_states(got, ref)
    assert errs["rho"] < 1e-6 and errs["u"] < 1e-3 and errs["w"] < 1e-2, errs


def test_flat_terrain_matches_flat_grid():
    """The terrain passes on a flat grid reproduce the flat-grid passes."""
    from erf_b200 import Dycore
    case = cases.abl_deardorff(nx=16, ny=12, nz=16)
    cfg = case.cfg
    dy = Dycore(cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    ref = dy.advance_host(cons, u, v, w, 3)
    dy.close()
    tc = cfg.copy()
    tc.use_terrain = 1
    dt = Dycore(tc)
    dt.set_terrain(T.btf_nodes(T.zlevels(cfg.nz, cfg.dz), np.zeros((cfg.ny + 1, cfg.nx + 1))))
    dt.set_base_state([np.repeat(b[:, None], cfg.ny * cfg.nx, axis=1).ravel() for b in base])
    got = dt.advance_host(cons, u, v, w, 3)
    assert dt.status() == 0
    dt.close()
    errs = compare_states(got, ref)
    assert all(v < 1e-9 for v in errs.values()), errs


def test_set_terrain_rejects_non_periodic_grid():
    from erf_b200 import Dycore
    from erf_b200.dycore import ErfError
    case = _hill()
    z = case.z_nd.copy()
    z[:, :, -1] += 1.0
    dy = Dycore(case.cfg)
    with pytest.raises(ErfError):
        dy.set_terrain(z)
    dy.close()


@pytest.mark.parametrize("nosub", [False, True])
def test_moist_terrain_parity(nosub):
    """Kessler with rain over terrain (moist_hill: a supersaturated, rainy warm
    bubble over a 1 km hill, WENO5 moisture, buoyancy type 1): condensation,
    evaporation and the sedimentation over detJ (ERF_Kessler.cpp:82-97), the
    moist pressure-gradient factors of the terrain slow and fast passes and
    the total-density buoyancy against the 3-D base state, 10 steps, with
    and without acoustic substepping."""
    case = T.moist_hill()
    if nosub:
        case.cfg.substepping_type = C.SUBSTEP_NONE
        case.cfg.dt = 0.25
    base, init, got, st = _gpu_run(case, 10)
    assert st == 0
    ref = oracle.advance_terrain(case.cfg, case.z_nd, base, *init, 10)
    errs = compare_states(got, ref)
    print("moist hill", nosub, errs)
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs
    # the condensate changed: the bubble condensed and the rain fell
    assert np.max(got[0][6]) > 0.0 and not np.allclose(got[0][7], init[0][7])


def test_moist_terrain_kessler_entry():
    """erf_b200_kessler_advance in a terrain context (sedimentation over
    detJ) matches the oracle's Kessler over the same grid."""
    import ctypes
    import torch
    from erf_b200 import Dycore
    from erf_b200.dycore import dense_fab
    case = T.moist_hill()
    cfg = case.cfg
    dy = Dycore(cfg)
    dy.set_terrain(case.z_nd)
    base = dy.make_base_state_terrain(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    t = torch.from_numpy(np.ascontiguousarray(cons)).cuda()
    f = dense_fab(t, 0, cfg.nx, cfg.ny, cfg.nz, cfg.ncomp)
    dy.lib.erf_b200_kessler_advance.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    torch.cuda.synchronize()
    assert dy.lib.erf_b200_kessler_advance(dy.ctx, ctypes.byref(f), cfg.dt) == 0
    torch.cuda.synchronize()
    got = t.cpu().numpy()
    dy.close()
    ref = oracle.kessler_terrain(cfg, case.z_nd, cons, cfg.dt)
    for n in range(cfg.ncomp):
        den = np.linalg.norm(ref[n])
        if den > 0:
            assert np.linalg.norm(got[n] - ref[n]) / den <= 1e-12, n
