"""Checkpoint / restart files (host code, no GPU): round trips through the
native writer and reader, the Header and MultiFab layout of
ERF::WriteCheckpointFile (Source/IO/ERF_Checkpoint.cpp:25-262), and reading
multi-grid, ghost-carrying MultiFabs as the reference writes them."""
import os
import sys

import numpy as np
import pytest

from erf_b200 import cases
from erf_b200 import terrain as T
from erf_b200.checkpoint import read_checkpoint, write_checkpoint
from erf_b200.dycore import ErfError

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from plotfile import _read_multifab  # noqa: E402


def _state(cfg, seed=0):
    rng = np.random.default_rng(seed)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    cons = rng.random((cfg.ncomp, nx * ny * nz)) + 0.5
    u = rng.standard_normal((nz, ny, nx + 1))
    v = rng.standard_normal((nz, ny + 1, nx))
    w = rng.standard_normal((nz + 1, ny, nx))
    nb = (nz + 2) * (nx * ny if cfg.use_terrain else 1)
    base = [rng.random(nb) + 1.0 for _ in range(4)]
    return cons, u, v, w, base


def test_checkpoint_round_trip_moist(tmp_path):
    case = cases.moist_bubble(nx=8, ny=6, nz=10)
    cfg = case.cfg
    cons, u, v, w, base = _state(cfg)
    out = str(tmp_path / "chk00042")
    write_checkpoint(cfg, out, cons, u, v, w, base, step=42, dt=0.5, time=21.0)
    r = read_checkpoint(cfg, out)
    for k, a in zip(("cons", "u", "v", "w"), (cons, u, v, w)):
        assert np.array_equal(r[k].reshape(a.shape), a), k
    for a, b in zip(r["base"], base):
        assert np.array_equal(a, b)
    assert (r["step"], r["dt"], r["time"]) == (42, 0.5, 21.0)
    assert r["z_nd"] is None


def test_checkpoint_header_and_multifabs(tmp_path):
    case = cases.abl_dry(nx=8, ny=6, nz=10)
    cfg = case.cfg
    cons, u, v, w, base = _state(cfg, 1)
    out = str(tmp_path / "chk")
    write_checkpoint(cfg, out, cons, u, v, w, base, step=7, dt=0.1, time=0.7000000000000001)
    hdr = open(os.path.join(out, "Header")).read().split("\n")
    assert hdr[:12] == ["Checkpoint file for ERF", "0", str(cfg.ncomp), "1", "1", "1", "7 ", "0.10000000000000001 ",
                        "0.70000000000000007 ", "(1 0", "((0,0,0) (7,5,9) (0,0,0))", ")"]
    lev = os.path.join(out, "Level_0")
    names = sorted(f for f in os.listdir(lev) if f.endswith("_H"))
    assert names == ["BaseState_H", "Cell_H", "MapFactor_m_H", "MapFactor_u_H", "MapFactor_v_H", "XFace_H",
                     "YFace_H", "ZFace_H"]
    # base state: 3 ghost cells, levels beyond k = -1 .. nz held at the nearest level
    bs = _read_multifab(os.path.join(lev, "BaseState"), 0)
    assert bs.shape == (4, 10 + 6, 6 + 6, 8 + 6)
    for q in range(4):
        col = np.concatenate([[base[q][0]] * 2, base[q], [base[q][-1]] * 2])
        assert np.array_equal(bs[q], np.broadcast_to(col[:, None, None], bs[q].shape))
    assert open(os.path.join(lev, "BaseState_H")).read().split("\n")[3] == "3"
    mf = open(os.path.join(lev, "MapFactor_u_H")).read().split("\n")
    assert mf[5] == "((0,0,0) (8,5,0) (1,0,0))"


def test_checkpoint_round_trip_terrain(tmp_path):
    case = T.abl_terrain(nx=8, ny=6, nz=8, dx=25.0, dz0=20.0, h0=100.0, r0=60.0, amp=5.0)
    cfg = case.cfg
    cons, u, v, w, base = _state(cfg, 2)
    out = str(tmp_path / "chk")
    write_checkpoint(cfg, out, cons, u, v, w, base, z_nd=case.z_nd, step=3, dt=0.1, time=0.3)
    r = read_checkpoint(cfg, out)
    assert np.array_equal(r["z_nd"], case.z_nd)
    for a, b in zip(r["base"], base):
        assert np.array_equal(a, b)
    assert np.array_equal(r["cons"].reshape(cons.shape), cons)
    # Z_Phys_nd carries the reference's ghost width for Upwind_5th / WENO: 3 + 2
    zh = open(os.path.join(out, "Level_0", "Z_Phys_nd_H")).read().split("\n")
    assert zh[3] == "5" and zh[5] == "((0,0,0) (8,6,8) (1,1,1))"
    z = _read_multifab(os.path.join(out, "Level_0", "Z_Phys_nd"), 1)
    assert z.shape == (1, 8 + 11, 6 + 11, 8 + 11)
    # periodic images laterally, linear extrapolation below the ground
    zg = z[0]
    assert np.array_equal(zg[5:5 + 9, 5:5 + 7, 5:5 + 9], case.z_nd)
    assert np.array_equal(zg[5:5 + 9, 5:5 + 7, 0], case.z_nd[:, :, 3])   # i = -5 -> node 3
    assert np.allclose(zg[4, 5:5 + 7, 5:5 + 9], 2 * case.z_nd[0] - case.z_nd[1], rtol=1e-15)


def _write_multigrid_cell(prefix, full, ncomp, split_j, ng):
    """Cell MultiFab of two FABs (j < split_j and j >= split_j) with ng ghost
    cells of junk, in one data file at byte offsets, as VisMF writes it."""
    nz, ny, nx = full.shape[1:]
    boxes = [((0, 0, 0), (nx - 1, split_j - 1, nz - 1)), ((0, split_j, 0), (nx - 1, ny - 1, nz - 1))]
    dname = os.path.basename(prefix) + "_D_00000"
    offs = []
    with open(prefix + "_D_00000", "wb") as fh:
        for lo, hi in boxes:
            glo = [x - ng for x in lo]
            ghi = [x + ng for x in hi]
            offs.append(fh.tell())
            fh.write(("FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))((%d,%d,%d) (%d,%d,%d) (0,0,0)) %d\n"
                      % (*glo, *ghi, ncomp)).encode())
            shape = (ncomp, ghi[2] - glo[2] + 1, ghi[1] - glo[1] + 1, ghi[0] - glo[0] + 1)
            a = np.full(shape, -999.0)
            a[:, ng:ng + hi[2] - lo[2] + 1, ng:ng + hi[1] - lo[1] + 1, ng:ng + hi[0] - lo[0] + 1] = \
                full[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
            fh.write(a.astype("<f8").tobytes())
    with open(prefix + "_H", "w") as fh:
        fh.write("1\n1\n%d\n(%d,%d,%d)\n(2 0\n" % (ncomp, ng, ng, ng))
        for lo, hi in boxes:
            fh.write("((%d,%d,%d) (%d,%d,%d) (0,0,0))\n" % (*lo, *hi))
        fh.write(")\n2\n")
        for o in offs:
            fh.write("FabOnDisk: %s %d\n" % (dname, o))


def test_checkpoint_reads_multigrid_multifab_with_ghosts(tmp_path):
    case = cases.abl_dry(nx=8, ny=6, nz=10)
    cfg = case.cfg
    cons, u, v, w, base = _state(cfg, 3)
    out = str(tmp_path / "chk")
    write_checkpoint(cfg, out, cons, u, v, w, base)
    _write_multigrid_cell(os.path.join(out, "Level_0", "Cell"), cons.reshape(cfg.ncomp, 10, 6, 8), cfg.ncomp, 2, 2)
    r = read_checkpoint(cfg, out)
    assert np.array_equal(r["cons"].reshape(cons.shape), cons)


def test_checkpoint_rejects_mismatch(tmp_path):
    case = cases.abl_dry(nx=8, ny=6, nz=10)
    cfg = case.cfg
    cons, u, v, w, base = _state(cfg, 4)
    out = str(tmp_path / "chk")
    write_checkpoint(cfg, out, cons, u, v, w, base)
    other = cfg.copy()
    other.ncomp = cfg.ncomp + 3
    with pytest.raises(ErfError):
        read_checkpoint(other, out)
    bigger = cfg.copy()
    bigger.nx = 16
    with pytest.raises(ErfError):
        read_checkpoint(bigger, out)
    with pytest.raises(ErfError):
        read_checkpoint(cfg, str(tmp_path / "missing"))
    tc = cfg.copy()
    tc.use_terrain = 1
    with pytest.raises(ErfError):      # terrain needs z_nd
        write_checkpoint(tc, str(tmp_path / "t"), cons, u, v, w, base)
