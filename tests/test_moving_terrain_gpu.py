"""GPU: moving terrain (terrain_type Moving) without acoustic substepping,
through the C-ABI, against the CPU oracle and the reference's gold
MovingTerrain_nosub (per-box min / max of the final plotfile).

Bars: relative L2 <= 1e-10 per field after 20 steps against the oracle
(v, which is round-off around zero in this 2-D wave, by its absolute
difference), the evolved base state and the final grid likewise; the gold
as the oracle meets it (z_velocity 3e-9, the rest 2e-10, as
|got - gold| / max(1, |gold|)); a run split over
two calls equal to one call (the device clock carries the time); the mixed
form within 1e-3 of FP64.
"""
import math
import os

import numpy as np
import pytest

import oracle
from erf_b200 import config as C
from erf_b200 import terrain as T
from helpers import rel_l2
from test_moving_terrain import gold_box_errors, plot_fields_mt

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10


def _gpu(case, nsteps, precision=C.PREC_FP64, split=None):
    from erf_b200 import Dycore
    cfg = case.cfg.copy()
    cfg.precision = precision
    dy = Dycore(cfg)
    dy.set_base_state(case.base)
    st = case.build_state()
    if split is None:
        out = dy.advance_host(*st, nsteps)
    else:
        out = dy.advance_host(*st, split)
        out = dy.advance_host(*out, nsteps - split)
    t, z, r0, p0 = dy.moving_terrain_state()
    status = dy.status()
    dy.close()
    return out, t, z, r0, p0, status


def _errors(got, ref):
    cg, ug, vg, wg = got
    cr, ur, vr, wr = ref
    e = {"rho": rel_l2(cg[0], cr[0]), "rhotheta": rel_l2(cg[1], cr[1]), "u": rel_l2(ug, ur), "w": rel_l2(wg, wr),
         "theta": rel_l2(cg[1] / cg[0], cr[1] / cr[0])}
    if np.any(cr[4]) or np.any(cg[4]):
        e["rhoscalar"] = rel_l2(cg[4], cr[4])
    return e


def test_moving_terrain_matches_oracle_and_gold():
    case = T.moving_terrain()
    cfg = case.cfg
    got, t, z, r0, p0, status = _gpu(case, case.steps)
    assert status == 0
    assert abs(t - case.steps * cfg.dt) < 1e-15
    st = case.build_state()
    ref = oracle.advance_moving_terrain(cfg, 0.0, case.base, *st, case.steps)
    errs = _errors(got, ref[:4])
    errs["rho0"] = rel_l2(r0, ref[5])
    errs["p0"] = rel_l2(p0, ref[6])
    errs["z_nd"] = rel_l2(z, ref[4])
    vdiff = float(np.max(np.abs(got[2] - ref[2])))
    print("moving terrain 40x8x79, 20 steps, GPU vs oracle:", errs, "max |dv|", vdiff)
    bad = {k: e for k, e in errs.items() if not e <= TOL}
    assert not bad, errs
    assert vdiff <= 1e-15
    # the gold, through the GPU's own final grid and base state
    gold = np.load(os.path.join(HERE, "golden", "MovingTerrain_nosub_minmax.npz"))
    f = plot_fields_mt(cfg, *got, z, r0, p0)
    worst = {}
    for (b, nm, tag), e in gold_box_errors(gold, f).items():
        worst[nm] = max(worst.get(nm, 0.0), e)
    print("vs gold:", worst)
    for nm, e in worst.items():
        assert e <= (3e-9 if nm == "z_velocity" else 2e-10), (nm, e)


def test_moving_terrain_split_run_equals_one_run():
    case = T.moving_terrain(nx=24, ny=4, nz=30, Lx=120.0, Ly=20.0, H=150.0, ampl=0.5, wavelength=60.0, steps=12)
    a = _gpu(case, case.steps)
    b = _gpu(case, case.steps, split=5)
    assert a[5] == 0 and b[5] == 0
    for x, y in zip(a[0], b[0]):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a[3], b[3])
    np.testing.assert_array_equal(a[4], b[4])
    assert a[1] == b[1]


def test_moving_terrain_steeper_wave_matches_oracle():
    """A steeper, shorter wave on a coarser column (slopes ~0.05)."""
    case = T.moving_terrain(nx=24, ny=4, nz=30, Lx=120.0, Ly=20.0, H=150.0, ampl=0.5, wavelength=60.0, steps=12)
    cfg = case.cfg
    got, t, z, r0, p0, status = _gpu(case, case.steps)
    assert status == 0
    ref = oracle.advance_moving_terrain(cfg, 0.0, case.base, *case.build_state(), case.steps)
    errs = _errors(got, ref[:4])
    errs["rho0"] = rel_l2(r0, ref[5])
    errs["p0"] = rel_l2(p0, ref[6])
    print("moving terrain 24x4x30, 12 steps:", errs)
    bad = {k: e for k, e in errs.items() if not e <= TOL}
    assert not bad, errs
    # the ground moved with the wave and w follows it
    assert np.max(np.abs(got[3][0])) > 0.01


def test_moving_terrain_mixed_within_budget():
    case = T.moving_terrain()
    fp64 = _gpu(case, case.steps)
    mixed = _gpu(case, case.steps, precision=C.PREC_MIXED)
    assert mixed[5] == 0
    errs = _errors(mixed[0], fp64[0])
    print("moving terrain mixed vs FP64 after 20 steps:", errs)
    assert all(e <= 1e-3 for e in errs.values()), errs


def test_moving_terrain_entry_points_refuse_other_contexts():
    from erf_b200 import Dycore
    from erf_b200.dycore import ErfError
    case = T.moving_terrain(nx=8, ny=4, nz=10)
    dy = Dycore(case.cfg)
    with pytest.raises(ErfError):
        dy.set_terrain(case.z_nd)       # the grid is generated, not installed
    dy.set_time(0.25)
    t, z, _, _ = dy.moving_terrain_state()
    assert t == 0.25
    kp = 2 * math.pi / 100.0
    x = np.arange(case.cfg.nx + 1) * case.cfg.dx
    np.testing.assert_allclose(z[0, 0], 0.16 * np.sin(kp * x - math.sqrt(9.81 * kp) * 0.25), rtol=0, atol=1e-15)
    dy.close()
    flat = T.abl_terrain(nx=8, ny=8, nz=8)
    dy = Dycore(flat.cfg)
    with pytest.raises(ErfError):
        dy.set_time(1.0)
    dy.close()


def test_moving_terrain_substeps_match_oracle_and_gold():
    """MovingTerrain_sub: 10 steps of 0.1 s with 20 acoustic substeps over
    the moving grid (erf_fast_rhs_MT), use_lagged_delta_rt = false."""
    case = T.moving_terrain(substeps=True)
    cfg = case.cfg
    got, t, z, r0, p0, status = _gpu(case, case.steps)
    assert status == 0
    ref = oracle.advance_moving_terrain(cfg, 0.0, case.base, *case.build_state(), case.steps)
    errs = _errors(got, ref[:4])
    errs["rho0"] = rel_l2(r0, ref[5])
    errs["p0"] = rel_l2(p0, ref[6])
    vdiff = float(np.max(np.abs(got[2] - ref[2])))
    print("moving terrain, substeps, 40x8x79, 10 steps, GPU vs oracle:", errs, "max |dv|", vdiff)
    bad = {k: e for k, e in errs.items() if not e <= TOL}
    assert not bad, errs
    assert vdiff <= 1e-15
    gold = np.load(os.path.join(HERE, "golden", "MovingTerrain_sub_minmax.npz"))
    worst = {}
    for (b, nm, tag), e in gold_box_errors(gold, plot_fields_mt(cfg, *got, z, r0, p0)).items():
        worst[nm] = max(worst.get(nm, 0.0), e)
    print("vs gold:", worst)
    for nm, e in worst.items():
        assert e <= 2e-10, (nm, e)


@pytest.mark.parametrize("lagged", [True, False])
def test_moving_terrain_substeps_steeper_wave(lagged):
    """A steeper, shorter wave, 6 substeps per step, with and without the
    lagged d(rho theta) correction; and the mixed form against FP64."""
    case = T.moving_terrain(nx=24, ny=4, nz=30, Lx=120.0, Ly=20.0, H=150.0, ampl=0.5, wavelength=60.0,
                            substeps=True, dt=0.05, steps=8)
    case.cfg.mri_ratio = 6
    case.cfg.no_lagged_delta_rt = 0 if lagged else 1
    got, t, z, r0, p0, status = _gpu(case, case.steps)
    assert status == 0
    ref = oracle.advance_moving_terrain(case.cfg, 0.0, case.base, *case.build_state(), case.steps)
    errs = _errors(got, ref[:4])
    errs["rho0"] = rel_l2(r0, ref[5])
    print("substeps, 24x4x30, lagged", lagged, errs)
    bad = {k: e for k, e in errs.items() if not e <= TOL}
    assert not bad, errs
    mixed = _gpu(case, case.steps, precision=C.PREC_MIXED)
    assert mixed[5] == 0
    em = _errors(mixed[0], got)
    print("  mixed vs FP64:", em)
    assert all(e <= 1e-3 for e in em.values()), em


def test_moving_terrain_plotfile_matches_gold_header(tmp_path):
    """End to end: the GPU's MovingTerrain_sub result written as an AMReX
    plotfile by the library's writer (with the evolved base state and the
    final grid) carries, for every variable of the gold, the same range as
    the reference's own gold plotfile header (its four boxes taken
    together), within the fcompare-style bound."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from plotfile import read_plotfile_minmax
    from erf_b200.plotfile import write_plotfile
    case = T.moving_terrain(substeps=True)
    cfg = case.cfg
    got, t, z, r0, p0, status = _gpu(case, case.steps)
    assert status == 0
    path = str(tmp_path / "plt00010")
    base = [r0, p0, case.base[2], case.base[3]]
    write_plotfile(cfg, path, *got, base=base, z_nd=z, time=t, step=case.steps)
    ours = read_plotfile_minmax(path)
    gold = np.load(os.path.join(HERE, "golden", "MovingTerrain_sub_minmax.npz"))
    assert abs(ours["time"] - float(gold["time"])) < 1e-12
    names = list(ours["names"])
    worst = {}
    for q, nm in enumerate(gold["names"]):
        nm = str(nm)
        a = names.index(nm)
        lo, hi = gold["vmin"][:, q].min(), gold["vmax"][:, q].max()
        e = max(abs(ours["min"][a] - lo) / max(1.0, abs(lo)), abs(ours["max"][a] - hi) / max(1.0, abs(hi)))
        worst[nm] = e
    print("plotfile vs gold header:", worst)
    assert all(e <= 2e-10 for e in worst.values()), worst
