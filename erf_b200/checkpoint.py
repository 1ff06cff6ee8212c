"""Checkpoint / restart of a host state in ERF's native checkpoint layout.

`write_checkpoint` / `read_checkpoint` call erf_b200_write_checkpoint /
erf_b200_read_checkpoint (native library), which follow
ERF::WriteCheckpointFile / ReadCheckpointFile (Source/IO/ERF_Checkpoint.cpp).
No GPU is needed; restart a context with Dycore.set_base_state (and
set_terrain) plus advance_host or load_state on what read_checkpoint returns.
"""
import ctypes
import os

import numpy as np

from . import config as C
from .dycore import _check, load_library


def _shapes(cfg: C.ErfConfig):
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    nb = (nz + 2) * (nx * ny if cfg.use_terrain else 1)
    return dict(cons=(cfg.ncomp, nz, ny, nx), u=(nz, ny, nx + 1), v=(nz, ny + 1, nx), w=(nz + 1, ny, nx),
                base=nb, z_nd=(nz + 1, ny + 1, nx + 1))


def write_checkpoint(cfg: C.ErfConfig, path: str, cons, u, v, w, base, z_nd=None, step: int = 0, dt: float = 0.0,
                     time: float = 0.0):
    """base: (r0, p0, pi0, th0) as given to Dycore.set_base_state."""
    L = load_library()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (cons, u, v, w)]
    bs = [np.ascontiguousarray(b, dtype=np.float64) for b in base]
    z = np.ascontiguousarray(z_nd, dtype=np.float64) if z_nd is not None else None
    _check(L.erf_b200_write_checkpoint(ctypes.byref(cfg), os.fsencode(path), *[a.ctypes.data for a in arrs + bs],
                                       z.ctypes.data if z is not None else None, int(step), float(dt), float(time)),
           "write_checkpoint")


def read_checkpoint(cfg: C.ErfConfig, path: str):
    """Returns dict(cons, u, v, w, base=[r0, p0, pi0, th0], z_nd (terrain) or None, step, dt, time)."""
    L = load_library()
    s = _shapes(cfg)
    out = {k: np.empty(s[k]) for k in ("cons", "u", "v", "w")}
    base = [np.empty(s["base"]) for _ in range(4)]
    z = np.empty(s["z_nd"]) if cfg.use_terrain else None
    step, dt, t = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
    _check(L.erf_b200_read_checkpoint(ctypes.byref(cfg), os.fsencode(path),
                                      *[out[k].ctypes.data for k in ("cons", "u", "v", "w")],
                                      *[b.ctypes.data for b in base], z.ctypes.data if z is not None else None,
                                      ctypes.byref(step), ctypes.byref(dt), ctypes.byref(t)), "read_checkpoint")
    out.update(base=base, z_nd=z, step=step.value, dt=dt.value, time=t.value)
    return out
