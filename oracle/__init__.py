"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU FP64 oracle.

The oracle (oracle/erf_oracle.cpp) restates the reference's dycore step on the
CPU.  Only tests/, the smoke check and bench.py's CPU-baseline leg may load it;
the product (erf_b200/) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liberf_oracle.so")
_lib = None


def build(quiet: bool = True) -> str:
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.oracle_advance.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_int]
        L.oracle_advance.restype = ctypes.c_int
        L.oracle_make_base_state.argtypes = [ctypes.c_void_p, dp, dp, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, dp, dp, dp, dp]
        L.oracle_make_base_state.restype = ctypes.c_int
        L.oracle_interp.argtypes = [ctypes.c_int, dp, ctypes.c_double, ctypes.c_double]
        L.oracle_interp.restype = ctypes.c_double
        L.oracle_qsatw.argtypes = [ctypes.c_double, ctypes.c_double]
        L.oracle_qsatw.restype = ctypes.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_base_state(cfg, case):
    nz = cfg.nz
    out = [np.zeros(nz + 2) for _ in range(4)]
    th = np.ascontiguousarray(case.theta_cc, dtype=np.float64)
    qv = np.ascontiguousarray(case.qv_cc, dtype=np.float64)
    lib().oracle_make_base_state(ctypes.byref(cfg), _p(th), _p(qv), case.theta_sfc, case.qv_sfc,
                                 case.p_sfc, *[_p(a) for a in out])
    return out


def advance(cfg, base, cons, u, v, w, nsteps):
    """Advance copies of the dense state arrays by nsteps; returns new arrays."""
    cons, u, v, w = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in (cons, u, v, w))
    r0, p0, pi0, th0 = (np.ascontiguousarray(a, dtype=np.float64) for a in base)
    rc = lib().oracle_advance(ctypes.byref(cfg), _p(r0), _p(p0), _p(pi0), _p(th0),
                              _p(cons), _p(u), _p(v), _p(w), int(nsteps))
    if rc != 0:
        raise RuntimeError("oracle_advance failed: %d" % rc)
    return cons, u, v, w


def kessler(cfg, cons, dt):
    """Kessler microphysics alone on a copy of a dense cons array."""
    L = lib()
    L.oracle_kessler.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_double]
    L.oracle_kessler.restype = ctypes.c_int
    out = np.ascontiguousarray(cons, dtype=np.float64).copy()
    rc = L.oracle_kessler(ctypes.byref(cfg), _p(out), float(dt))
    if rc != 0:
        raise RuntimeError("oracle_kessler failed: %d" % rc)
    return out


def kessler_terrain(cfg, z_nd, cons, dt):
    """Kessler alone over a terrain grid (sedimentation over detJ)."""
    L = lib()
    L.oracle_kessler_terrain.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double), ctypes.c_double]
    L.oracle_kessler_terrain.restype = ctypes.c_int
    out = np.ascontiguousarray(cons, dtype=np.float64).copy()
    z = np.ascontiguousarray(z_nd, dtype=np.float64)
    rc = L.oracle_kessler_terrain(ctypes.byref(cfg), _p(z), _p(out), float(dt))
    if rc != 0:
        raise RuntimeError("oracle_kessler_terrain failed: %d" % rc)
    return out


PASSES = ("closure", "slow_rhs_pre", "fast", "slow_rhs_post", "kessler", "other")


def advance_timed(cfg, base, cons, u, v, w, nsteps):
    """advance() plus the wall seconds spent in each pass (dict over PASSES)."""
    L = lib()
    dp = ctypes.POINTER(ctypes.c_double)
    L.oracle_advance_timed.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_int, dp]
    L.oracle_advance_timed.restype = ctypes.c_int
    cons, u, v, w = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in (cons, u, v, w))
    r0, p0, pi0, th0 = (np.ascontiguousarray(a, dtype=np.float64) for a in base)
    sec = np.zeros(6)
    rc = L.oracle_advance_timed(ctypes.byref(cfg), _p(r0), _p(p0), _p(pi0), _p(th0),
                                _p(cons), _p(u), _p(v), _p(w), int(nsteps), _p(sec))
    if rc != 0:
        raise RuntimeError("oracle_advance_timed failed: %d" % rc)
    return (cons, u, v, w), dict(zip(PASSES, (float(x) for x in sec)))


def interp(kind: int, s6, upw: float, frac: float = 1.0) -> float:
    s = np.ascontiguousarray(s6, dtype=np.float64)
    return lib().oracle_interp(int(kind), _p(s), float(upw), float(frac))


def qsatw(t: float, p_hpa: float) -> float:
    return lib().oracle_qsatw(float(t), float(p_hpa))


def _setup_terrain(L):
    if getattr(L, "_terrain_ready", False):
        return
    dp = ctypes.POINTER(ctypes.c_double)
    L.oracle_make_base_state_terrain.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_double, dp, dp, dp, dp]
    L.oracle_make_base_state_terrain.restype = ctypes.c_int
    L.oracle_terrain_metrics.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp]
    L.oracle_terrain_metrics.restype = ctypes.c_int
    L.oracle_advance_terrain.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_int]
    L.oracle_advance_terrain.restype = ctypes.c_int
    L._terrain_ready = True


def make_base_state_terrain(case):
    """Base state over the terrain: four arrays of (nz+2)*ny*nx values."""
    cfg = case.cfg
    L = lib()
    _setup_terrain(L)
    n = (cfg.nz + 2) * cfg.ny * cfg.nx
    out = [np.zeros(n) for _ in range(4)]
    z = np.ascontiguousarray(case.z_nd, dtype=np.float64)
    th = np.ascontiguousarray(case.theta3, dtype=np.float64)
    qv = np.ascontiguousarray(case.qv3, dtype=np.float64)
    L.oracle_make_base_state_terrain(ctypes.byref(cfg), _p(z), _p(th), _p(qv), case.theta_sfc, case.qv_sfc,
                                     case.p_sfc, *[_p(a) for a in out])
    return out


def terrain_metrics(cfg, z_nd):
    """detJ, z_cc [nz][ny][nx], ax [nz][ny][nx+1], ay [nz][ny+1][nx]."""
    L = lib()
    _setup_terrain(L)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    detJ = np.zeros((nz, ny, nx)); zcc = np.zeros((nz, ny, nx))
    ax = np.zeros((nz, ny, nx + 1)); ay = np.zeros((nz, ny + 1, nx))
    z = np.ascontiguousarray(z_nd, dtype=np.float64)
    L.oracle_terrain_metrics(ctypes.byref(cfg), _p(z), _p(detJ), _p(zcc), _p(ax), _p(ay))
    return detJ, zcc, ax, ay


def advance_moving_terrain(cfg, time0, base, cons, u, v, w, nsteps):
    """Advance copies of the dense state over moving terrain (no acoustic
    substepping) by nsteps from time0.  Returns (cons, u, v, w, z_nd, rho0,
    p0): the state, the grid at the final time and the evolved base state."""
    L = lib()
    dp = ctypes.POINTER(ctypes.c_double)
    L.oracle_advance_moving_terrain.argtypes = [ctypes.c_void_p, ctypes.c_double, dp, dp, dp, dp, dp, dp, dp, dp,
                                                ctypes.c_int, dp, dp, dp]
    L.oracle_advance_moving_terrain.restype = ctypes.c_int
    cons, u, v, w = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in (cons, u, v, w))
    r0, p0, pi0, th0 = (np.ascontiguousarray(a, dtype=np.float64) for a in base)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    z = np.zeros((nz + 1, ny + 1, nx + 1))
    r0o = np.zeros((nz + 2) * ny * nx)
    p0o = np.zeros((nz + 2) * ny * nx)
    rc = L.oracle_advance_moving_terrain(ctypes.byref(cfg), float(time0), _p(r0), _p(p0), _p(pi0), _p(th0),
                                         _p(cons), _p(u), _p(v), _p(w), int(nsteps), _p(z), _p(r0o), _p(p0o))
    if rc != 0:
        raise RuntimeError("oracle_advance_moving_terrain failed: %d" % rc)
    return cons, u, v, w, z, r0o, p0o


def advance_terrain(cfg, z_nd, base, cons, u, v, w, nsteps):
    """Advance copies of the dense state over terrain by nsteps."""
    L = lib()
    _setup_terrain(L)
    cons, u, v, w = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in (cons, u, v, w))
    r0, p0, pi0, th0 = (np.ascontiguousarray(a, dtype=np.float64) for a in base)
    z = np.ascontiguousarray(z_nd, dtype=np.float64)
    rc = L.oracle_advance_terrain(ctypes.byref(cfg), _p(z), _p(r0), _p(p0), _p(pi0), _p(th0),
                                  _p(cons), _p(u), _p(v), _p(w), int(nsteps))
    if rc != 0:
        raise RuntimeError("oracle_advance_terrain failed: %d" % rc)
    return cons, u, v, w
