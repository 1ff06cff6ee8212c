"""The native plotfile writer (host code, no GPU): written files read back by
the independent reader of tests/golden/plotfile.py, checked against the
reference's own gold plotfile (TaylorGreenAdvecting, written by ERF) for the
Header layout and the derived temp / pressure fields, and against numpy for
the rest."""
import os
import sys

import numpy as np
import pytest

from erf_b200 import cases
from erf_b200 import config as C
from erf_b200 import terrain as T
from erf_b200.plotfile import write_plotfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from plotfile import read_plotfile  # noqa: E402


def _taylor_green_state():
    """Cell state of the reference's TaylorGreenAdvecting gold plotfile
    (face velocities set to the cell values)."""
    g = np.load(os.path.join(HERE, "golden", "TaylorGreenAdvecting_gold.npz"))
    names = list(g["names"])
    F = {n: g["data"][names.index(n)] for n in names}
    cfg = C.defaults()
    cfg.nx = cfg.ny = cfg.nz = 16
    cfg.dx = cfg.dy = cfg.dz = 2 * np.pi / 16
    N = 16 ** 3
    cons = np.zeros((cfg.ncomp, N))
    cons[0] = F["density"].ravel()
    cons[1] = (F["density"] * F["theta"]).ravel()
    cons[4] = (F["density"] * F["scalar"]).ravel()
    u = np.concatenate([F["x_velocity"], F["x_velocity"][:, :, :1]], axis=2)
    v = np.concatenate([F["y_velocity"], F["y_velocity"][:, :1, :]], axis=1)
    w = np.concatenate([F["z_velocity"], F["z_velocity"][:1]], axis=0)
    return cfg, g, F, cons, u, v, w


def test_plotfile_matches_reference_gold_layout(tmp_path):
    cfg, g, F, cons, u, v, w = _taylor_green_state()
    out = str(tmp_path / "plt00010")
    write_plotfile(cfg, out, cons, u, v, w, time=float(g["time"]), step=10)
    pf = read_plotfile(out)
    assert pf["names"] == list(g["names"])
    gold_hdr = list(g["header"])
    # identical up to the grid list (the reference run had 4 grids, we write 1)
    assert pf["header"][:21] == gold_hdr[:21]
    assert gold_hdr[21:23] == ["0 4 1.5999999999999999", "10"]
    assert pf["header"][21:] == ["0 1 1.5999999999999999", "10", "0 6.2831853071795862", "0 6.2831853071795862",
                                 "0 6.2831853071795862", "Level_0/Cell"]
    names = pf["names"]
    D = pf["data"]
    for n in ("density", "theta", "scalar"):
        assert np.allclose(D[names.index(n)], F[n], rtol=1e-15, atol=0)
    # derived fields against the reference's own values
    for n in ("temp", "pressure"):
        assert np.max(np.abs(D[names.index(n)] / F[n] - 1)) < 1e-14, n
    # face -> cell averages
    xv = 0.5 * (u[:, :, :-1] + u[:, :, 1:])
    assert np.array_equal(D[names.index("x_velocity")], xv)
    assert np.array_equal(D[names.index("z_velocity")], 0.5 * (w[:-1] + w[1:]))


def test_plotfile_cell_h_min_max(tmp_path):
    cfg, g, F, cons, u, v, w = _taylor_green_state()
    out = str(tmp_path / "plt")
    write_plotfile(cfg, out, cons, u, v, w)
    lines = open(os.path.join(out, "Level_0", "Cell_H")).read().split("\n")
    assert lines[:4] == ["1", "1", "8", "0"]
    assert lines[4:9] == ["(1 0", "((0,0,0) (15,15,15) (0,0,0))", ")", "1", "FabOnDisk: Cell_D_00000 0"]
    D = read_plotfile(out)["data"]
    assert lines[10] == "1,8" and lines[13] == "1,8"
    mins = [float(x) for x in lines[11].rstrip(",").split(",")]
    maxs = [float(x) for x in lines[14].rstrip(",").split(",")]
    assert np.allclose(mins, D.reshape(8, -1).min(1), rtol=1e-15)
    assert np.allclose(maxs, D.reshape(8, -1).max(1), rtol=1e-15)


def test_plotfile_moist_deardorff_base_state(tmp_path):
    case = cases.moist_bubble(nx=8, ny=6, nz=10)
    cfg = case.cfg
    cfg.les_type = C.LES_DEARDORFF
    rng = np.random.default_rng(3)
    N = cfg.nx * cfg.ny * cfg.nz
    cons = np.abs(rng.standard_normal((cfg.ncomp, N))) + 1.0
    cons[1] *= 300.0
    cons[C.RHOQ1_COMP:] *= 1e-3
    u = rng.standard_normal((cfg.nz, cfg.ny, cfg.nx + 1))
    v = rng.standard_normal((cfg.nz, cfg.ny + 1, cfg.nx))
    w = rng.standard_normal((cfg.nz + 1, cfg.ny, cfg.nx))
    base = [rng.random(cfg.nz + 2) + 1.0 for _ in range(4)]
    out = str(tmp_path / "plt")
    write_plotfile(cfg, out, cons, u, v, w, base=base, time=2.5, step=7)
    pf = read_plotfile(out)
    names = pf["names"]
    assert names == ["density", "x_velocity", "y_velocity", "z_velocity", "temp", "theta", "KE", "scalar",
                     "pres_hse", "dens_hse", "pressure", "qv", "qc", "qrain"]
    D = {n: pf["data"][c].ravel() for c, n in enumerate(names)}
    rho = cons[0]
    qv = cons[C.RHOQ1_COMP] / rho
    p = 1e5 * (287.0 * cons[1] * (1 + 461.505 / 287.0 * qv) / 1e5) ** 1.4
    assert np.allclose(D["pressure"], p, rtol=1e-14)
    assert np.allclose(D["temp"], p / (287.0 * rho * (1 + 461.505 / 287.0 * qv)), rtol=1e-14)
    assert np.allclose(D["KE"], cons[C.RHOKE_COMP] / rho, rtol=1e-15)
    assert np.allclose(D["qrain"], cons[C.RHOQ1_COMP + 2] / rho, rtol=1e-15)
    kk = np.repeat(np.arange(cfg.nz), cfg.nx * cfg.ny)
    assert np.array_equal(D["pres_hse"], base[1][kk + 1])
    assert np.array_equal(D["dens_hse"], base[0][kk + 1])
    assert pf["time"] == 2.5


def test_plotfile_terrain_nodal(tmp_path):
    case = T.abl_terrain(nx=8, ny=6, nz=8, dx=25.0, dz0=20.0, h0=100.0, r0=60.0, amp=5.0)
    cfg = case.cfg
    N = cfg.nx * cfg.ny * cfg.nz
    cons = np.ones((cfg.ncomp, N))
    cons[1] = 300.0
    u = np.zeros((cfg.nz, cfg.ny, cfg.nx + 1))
    v = np.zeros((cfg.nz, cfg.ny + 1, cfg.nx))
    w = np.zeros((cfg.nz + 1, cfg.ny, cfg.nx))
    out = str(tmp_path / "plt")
    write_plotfile(cfg, out, cons, u, v, w, z_nd=case.z_nd)
    pf = read_plotfile(out)
    names = pf["names"]
    assert names[-2:] == ["z_phys", "detJ"]
    assert np.allclose(pf["data"][names.index("z_phys")], T.cell_heights(case.z_nd), rtol=1e-14)
    z = case.z_nd
    dz_col = 0.25 * ((z[1:, :-1, :-1] - z[:-1, :-1, :-1]) + (z[1:, :-1, 1:] - z[:-1, :-1, 1:])
                     + (z[1:, 1:, :-1] - z[:-1, 1:, :-1]) + (z[1:, 1:, 1:] - z[:-1, 1:, 1:]))
    assert np.allclose(pf["data"][names.index("detJ")], dz_col / cfg.dz, rtol=1e-14)
    assert pf["nodal_names"] == ["amrexvec_nu_x", "amrexvec_nu_y", "amrexvec_nu_z"]
    nd = pf["nodal"]
    assert nd.shape == (3, cfg.nz + 1, cfg.ny + 1, cfg.nx + 1)
    assert not nd[0].any() and not nd[1].any()
    kz = np.arange(cfg.nz + 1)[:, None, None] * cfg.dz
    assert np.allclose(nd[2], z - kz, rtol=0, atol=1e-12)


def test_plotfile_rejects_bad_arguments(tmp_path):
    from erf_b200.dycore import ErfError
    cfg, g, F, cons, u, v, w = _taylor_green_state()
    cfg.nx = 0
    with pytest.raises(ErfError):
        write_plotfile(cfg, str(tmp_path / "p"), cons, u, v, w)
