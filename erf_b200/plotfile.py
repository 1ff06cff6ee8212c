"""AMReX plotfiles of a host state.

`write_plotfile` calls erf_b200_write_plotfile (native library), which lays
the state out as ERF::WritePlotFile does (Source/IO/ERF_Plotfile.cpp): Header,
Level_0/Cell_H and Level_0/Cell_D_00000, plus Level_0/Nu_nd over terrain.  It
needs no GPU; AMReX tools (fcompare, amrvis, yt) read the result.
"""
import ctypes
import os

import numpy as np

from . import config as C
from .dycore import _check, load_library


def write_plotfile(cfg: C.ErfConfig, path: str, cons, u, v, w, base=None, z_nd=None, time: float = 0.0,
                   step: int = 0):
    """Write `path` from host arrays in the erf_b200_advance_host layout.

    base: the 4 base-state arrays (rho0, p0, pi0, theta0) as given to
    set_base_state, for pres_hse / dens_hse; z_nd: terrain node heights."""
    L = load_library()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (cons, u, v, w)]
    r0 = p0 = None
    if base is not None:
        r0, p0 = (np.ascontiguousarray(b, dtype=np.float64) for b in base[:2])
    z = np.ascontiguousarray(z_nd, dtype=np.float64) if z_nd is not None else None
    ptr = lambda a: a.ctypes.data if a is not None else None
    _check(L.erf_b200_write_plotfile(ctypes.byref(cfg), os.fsencode(path), *[a.ctypes.data for a in arrs], ptr(r0),
                                     ptr(p0), ptr(z), float(time), int(step)), "write_plotfile")
