"""The oracle's restatement of the hot path's leaf operators against the
reference's own operator code.

oracle/_ref/libref_ops.so holds ERF's source files for these operators,
compiled unmodified from the reference tree against a single-box AMReX
stand-in (oracle/ref/); the oracle exposes the same operators through
operator hooks.  Each test feeds both the same seeded random inputs, ghost
cells included, and compares every output value:

  * the face interpolants Upwind_3rd/5th, Centered_2nd/4th/6th, WENO3, WENO5
    (Utils/ERF_Interpolation_UPW.H, ERF_Interpolation_WENO.H);
  * AdvectionSrcForScalars with each scheme pair
    (Advection/ERF_AdvectionSrcForState.cpp:119-395);
  * AdvectionSrcForMom with each scheme pair, the vertical w fluxes reduced
    in order next to the walls (Advection/ERF_AdvectionSrcForMom.cpp:41-204,
    ERF_AdvectionSrcForMom_N.H);
  * ComputeStrain_N with slip and no-slip walls, including the one-sided
    wall stencils (Diffusion/ERF_ComputeStrain_N.cpp:28-229);
  * ComputeStrain_T over a terrain-following grid
    (Diffusion/ERF_ComputeStrain_T.cpp);
  * the eddy viscosity of the step prologue: Smagorinsky and Deardorff
    (ERF_advance_dycore.cpp:114-223, Diffusion/ERF_ComputeTurbulentViscosity.cpp);
  * Kessler microphysics with and without rain
    (Microphysics/Kessler/ERF_Kessler.cpp, ERF_Init_Kessler.cpp, ERF_Update_Kessler.cpp);
  * the Flatau saturation mixing ratio (Utils/ERF_Microphysics_Utils.H).

Bar: bit for bit.  Both sides are compiled with -ffp-contract=off and no
value-changing optimisation, and the restatement keeps the reference's
operation order, so every output value is identical (the interpolants are
checked to 1e-14 of the stencil's scale, and are identical too).
"""
import ctypes

import numpy as np
import pytest

import oracle
from oracle import refops
from erf_b200 import cases
from erf_b200 import config as C

pytestmark = pytest.mark.skipif(not refops.available(), reason="reference operators not built and no reference tree")
TOL = 0.0
SCHEMES = [C.CENTERED_2ND, C.UPWIND_3RD, C.CENTERED_4TH, C.UPWIND_5TH, C.CENTERED_6TH, C.WENO_3, C.WENO_5]


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))


def _ocall(name, *args):
    """Call an oracle operator hook; numpy arrays pass as pointers."""
    L = oracle.lib()
    f = getattr(L, name)
    f.restype = ctypes.c_int
    conv = []
    for a in args:
        if isinstance(a, np.ndarray):
            assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
            conv.append(ctypes.c_void_p(a.ctypes.data))
        elif isinstance(a, float):
            conv.append(ctypes.c_double(a))
        else:
            conv.append(a)
    assert f(*conv) == 0


def _cfg(nx=12, ny=10, nz=9, zlo=C.BC_SLIP_WALL, zhi=C.BC_SLIP_WALL):
    c = C.defaults()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dx, c.dy, c.dz = 50.0, 40.0, 20.0
    c.zlo_bc, c.zhi_bc = zlo, zhi
    return c


def test_interpolants_match_reference():
    rng = np.random.default_rng(5)
    L = refops.lib()
    worst = 0.0
    for t in SCHEMES:
        for _ in range(300):
            s = np.ascontiguousarray(rng.normal(size=6) * 10.0 ** rng.uniform(-3, 3))
            upw = float(rng.choice([rng.normal(), 0.0, 1e-14, -1e-14, -abs(rng.normal())]))
            frac = float(rng.choice([1.0, 0.3, 0.0]))
            a = oracle.interp(t, s, upw, frac)
            b = L.ref_interp(t, refops.ptr(s), upw, frac)
            scale = max(np.max(np.abs(s)), 1e-300)
            worst = max(worst, abs(a - b) / scale)
            assert abs(a - b) <= 1e-14 * scale, (t, s, upw, frac, a, b)
    print("interpolants: worst", worst)


@pytest.mark.parametrize("h,v", [(C.UPWIND_5TH, C.UPWIND_5TH), (C.WENO_5, C.WENO_5), (C.UPWIND_3RD, C.UPWIND_3RD),
                                 (C.CENTERED_2ND, C.CENTERED_2ND), (C.CENTERED_4TH, C.CENTERED_6TH),
                                 (C.WENO_3, C.WENO_3), (C.UPWIND_5TH, C.CENTERED_2ND)])
def test_advect_scalars_matches_reference(h, v):
    cfg = _cfg()
    cfg.ncomp = 8
    rng = np.random.default_rng(h * 7 + v)
    ncons, nprim = 8, 7
    av = [np.ascontiguousarray(rng.normal(size=refops.shape(cfg, t, 0))[0]) for t in (1, 2, 3)]
    prim = np.ascontiguousarray(1.0 + 0.1 * rng.normal(size=refops.shape(cfg, 0, 3, nprim)))
    hf, vf = 1.0, 0.7
    out = []
    for side in ("oracle", "ref"):
        rhs = np.zeros(refops.shape(cfg, 0, 0, ncons))
        if side == "oracle":
            _ocall("oracle_op_advect_scalars", ctypes.byref(cfg), 4, 4, h, v, ctypes.c_double(hf), ctypes.c_double(vf),
                   *av, prim, nprim, rhs, ncons)
        else:
            refops.lib().ref_advect_scalars(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, 4, 4, h, v, hf, vf,
                                            *[refops.ptr(a) for a in av], refops.ptr(prim), nprim,
                                            refops.ptr(rhs), ncons)
        out.append(rhs)
    assert np.any(out[1][4:8])
    for n in range(4, 8):
        assert rel(out[0][n], out[1][n]) <= TOL, (n, rel(out[0][n], out[1][n]))


@pytest.mark.parametrize("h,v", [(C.UPWIND_5TH, C.UPWIND_5TH), (C.UPWIND_3RD, C.UPWIND_3RD),
                                 (C.CENTERED_4TH, C.CENTERED_6TH), (C.CENTERED_2ND, C.CENTERED_2ND),
                                 (C.UPWIND_5TH, C.CENTERED_2ND)])
def test_advect_mom_matches_reference(h, v):
    """AdvectionSrcForMom: the three momentum flux divergences, including the
    order reduction of the vertical w fluxes next to the walls."""
    cfg = _cfg(nz=11)
    cfg.dycore_horiz_adv, cfg.dycore_vert_adv = h, v
    cfg.dycore_horiz_upw_frac, cfg.dycore_vert_upw_frac = 1.0, 0.6
    rng = np.random.default_rng(h + 3 * v)
    mom = [np.ascontiguousarray(rng.normal(size=refops.shape(cfg, t, 3))[0]) for t in (1, 2, 3)]
    vel = [np.ascontiguousarray(rng.normal(size=refops.shape(cfg, t, 3))[0]) for t in (1, 2, 3)]
    res = []
    for side in ("oracle", "ref"):
        outs = [np.zeros(refops.shape(cfg, t, 0)[1:]) for t in (1, 2, 3)]
        if side == "oracle":
            _ocall("oracle_op_advect_mom", ctypes.byref(cfg), *mom, *vel, *outs)
        else:
            assert refops.lib().ref_advect_mom(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, h, v,
                                               cfg.dycore_horiz_upw_frac, cfg.dycore_vert_upw_frac,
                                               *[refops.ptr(a) for a in mom + vel + outs]) == 0
        res.append(outs)
    for q, (a, b) in enumerate(zip(*res)):
        if q == 2:   # z-momentum on the interior faces only
            a, b = a[1:-1], b[1:-1]
        assert np.any(b), q
        assert rel(a, b) <= TOL, (q, rel(a, b))


def _vel(cfg, rng, g=2):
    return [np.ascontiguousarray(rng.normal(size=refops.shape(cfg, t, g))[0]) for t in (1, 2, 3)]


@pytest.mark.parametrize("zlo,zhi", [(C.BC_NO_SLIP_WALL, C.BC_SLIP_WALL), (C.BC_SLIP_WALL, C.BC_SLIP_WALL),
                                     (C.BC_NO_SLIP_WALL, C.BC_NO_SLIP_WALL)])
def test_strain_N_matches_reference(zlo, zhi):
    cfg = _cfg(zlo=zlo, zhi=zhi)
    rng = np.random.default_rng(zlo * 10 + zhi)
    u, v, w = _vel(cfg, rng)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    res = []
    for side in ("oracle", "ref"):
        outs = [np.zeros((nz + 2, ny + 2, nx + 2)) for _ in range(3)] + [np.zeros((nz + 3, ny + 3, nx + 3)) for _ in range(3)]
        if side == "oracle":
            _ocall("oracle_op_strain", ctypes.byref(cfg), u, v, w, *outs)
        else:
            refops.lib().ref_strain_N(nx, ny, nz, cfg.dx, cfg.dy, cfg.dz, int(zlo == C.BC_NO_SLIP_WALL),
                                      int(zhi == C.BC_NO_SLIP_WALL), refops.ptr(u), refops.ptr(v), refops.ptr(w),
                                      *[refops.ptr(o) for o in outs])
        res.append(outs)
    for q, (a, b) in enumerate(zip(*res)):
        assert np.any(b), q
        assert rel(a, b) <= TOL, (q, rel(a, b))


def test_strain_T_matches_reference():
    from erf_b200 import terrain as T
    case = T.abl_terrain(nx=12, ny=10, nz=9, dx=25.0, dz0=10.0, h0=60.0, r0=80.0, amp=4.0)
    cfg = case.cfg
    rng = np.random.default_rng(3)
    u, v, w = _vel(cfg, rng)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    z = np.ascontiguousarray(case.z_nd, dtype=np.float64)
    zg = np.zeros((nz + 3, ny + 7, nx + 7))
    dj = np.zeros((nz + 2, ny + 4, nx + 4))
    res = []
    for side in ("oracle", "ref"):
        outs = [np.zeros((nz + 2, ny + 2, nx + 2)) for _ in range(3)] + [np.zeros((nz + 3, ny + 3, nx + 3)) for _ in range(6)]
        if side == "oracle":
            _ocall("oracle_op_strain_T", ctypes.byref(cfg), z, u, v, w, zg, dj, *outs)
        else:
            refops.lib().ref_strain_T(nx, ny, nz, cfg.dx, cfg.dy, cfg.dz, int(cfg.zlo_bc == C.BC_NO_SLIP_WALL),
                                      int(cfg.zhi_bc == C.BC_NO_SLIP_WALL), refops.ptr(u), refops.ptr(v),
                                      refops.ptr(w), refops.ptr(zg), refops.ptr(dj), *[refops.ptr(o) for o in outs])
        res.append(outs)
    for q, (a, b) in enumerate(zip(*res)):
        assert np.any(b), q
        assert rel(a, b) <= TOL, (q, rel(a, b))


@pytest.mark.parametrize("les", [C.LES_SMAGORINSKY, C.LES_DEARDORFF])
@pytest.mark.parametrize("zlo", [C.BC_NO_SLIP_WALL, C.BC_SLIP_WALL])
def test_eddy_viscosity_matches_reference(les, zlo):
    cfg = _cfg(zlo=zlo)
    cfg.les_type = les
    cfg.Cs, cfg.Ck, cfg.Ce, cfg.Ce_wall, cfg.theta_ref, cfg.sigma_k = 0.1, 0.1, 0.93, 0.0, 300.0, 0.5
    cfg.gravity = 9.81
    cfg.ncomp = 5
    rng = np.random.default_rng(les * 3 + zlo)
    u, v, w = _vel(cfg, rng)
    cons = np.zeros(refops.shape(cfg, 0, 1, 5))
    cons[0] = 1.1 + 0.05 * rng.random(cons[0].shape)
    nz = cfg.nz
    zc = (np.arange(-1, nz + 1) + 0.5)[:, None, None]
    cons[1] = cons[0] * (300.0 + 0.02 * zc + 0.3 * rng.random(cons[0].shape))
    cons[2] = cons[0] * 0.4 * rng.random(cons[0].shape)
    cons = np.ascontiguousarray(cons)
    res = []
    for side in ("oracle", "ref"):
        outs = [np.zeros(refops.shape(cfg, 0, 1)[1:]) for _ in range(3)]
        if side == "oracle":
            _ocall("oracle_op_eddy_viscosity", ctypes.byref(cfg), u, v, w, cons, *outs)
        else:
            refops.lib().ref_eddy_viscosity(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz,
                                            int(zlo == C.BC_NO_SLIP_WALL), 0, les, cfg.Cs, cfg.Pr_t, cfg.Sc_t,
                                            cfg.Ck, cfg.Ce, cfg.Ce_wall, cfg.theta_ref, cfg.sigma_k, cfg.gravity,
                                            refops.ptr(u), refops.ptr(v), refops.ptr(w), refops.ptr(cons), 5,
                                            *[refops.ptr(o) for o in outs])
        res.append(outs)
    n = 1 if les == C.LES_SMAGORINSKY else 3
    for q in range(n):
        a, b = res[0][q], res[1][q]
        assert np.any(b), q
        assert rel(a, b) <= TOL, (q, rel(a, b))


@pytest.mark.parametrize("rain", [True, False])
def test_kessler_matches_reference(rain):
    case = cases.moist_bubble(nx=10, ny=8, nz=24)
    cfg = case.cfg
    if not rain:
        cfg.moisture, cfg.ncomp, cfg.buoyancy_type = C.MOIST_KESSLER_NORAIN, 7, 1
    base = oracle.make_base_state(cfg, case)
    cons, _, _, _ = case.build_state(base[0])
    cons = np.ascontiguousarray(cons[:cfg.ncomp])
    rng = np.random.default_rng(9)
    cons[5] *= 1.0 + 0.3 * rng.random(cons[5].shape)
    cons[6] = cons[0] * 2.0e-3 * rng.random(cons[0].shape)
    if rain:
        cons[7] = cons[0] * 1.0e-3 * rng.random(cons[0].shape)
    got = oracle.kessler(cfg, cons, cfg.dt)
    # the reference's state always holds three moisture species (its Kessler
    # copies all three, with or without rain): a zero rain component pads it
    ref = np.zeros((8,) + cons.shape[1:])
    ref[:cfg.ncomp] = cons
    assert refops.lib().ref_kessler(cfg.nx, cfg.ny, cfg.nz, cfg.dx, cfg.dy, cfg.dz, int(rain), cfg.c_p, cfg.dt,
                                    refops.ptr(ref), 8) == 0
    ref = ref[:cfg.ncomp]
    assert not np.array_equal(ref, cons)
    for n in range(cfg.ncomp):
        assert rel(got[n], ref[n]) <= TOL, (n, rel(got[n], ref[n]))


def test_saturation_mixing_ratio_matches_reference():
    L = refops.lib()
    for t in np.linspace(230.0, 320.0, 41):
        for p in (1000.0, 850.0, 500.0, 200.0):
            assert oracle.qsatw(t, p) == L.ref_qsatw(t, p), (t, p)
