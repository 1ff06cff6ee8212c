"""TEST INFRASTRUCTURE ONLY: ctypes binding of oracle/_ref/libref_ops.so, the
reference's own hot-path leaf operators compiled unmodified from its Source/
tree against the single-box AMReX stand-in of oracle/ref/ (recipe:
oracle/ref/Makefile).  The tests use it to pin the oracle's restatement of
each operator; nothing else loads it.

Array convention (shared with the oracle's operator hooks): the valid box of
the array's index type (cells; x-, y-, z-faces nodal in their direction)
grown by a ghost width g on every side, i fastest, components slowest; numpy
shape (ncomp, nz', ny', nx')."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_ops.so")
REF_TREE = os.environ.get("ERF_REFERENCE_TREE", "/root/reference")
_lib = None


def build() -> str | None:
    """Compile the reference operators where the reference tree exists; the
    built library travels with the repository snapshot elsewhere."""
    if not os.path.isdir(os.path.join(REF_TREE, "Source")):
        return LIB if os.path.exists(LIB) else None
    out = subprocess.run(["make", "-C", os.path.join(HERE, "ref"), f"REF={REF_TREE}", "-j8"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("reference operator build failed:\n" + out.stdout[-3000:] + out.stderr[-3000:])
    return LIB


def available() -> bool:
    return os.path.exists(LIB) or os.path.isdir(os.path.join(REF_TREE, "Source"))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        L.ref_interp.argtypes = [i, p, d, d]
        L.ref_interp.restype = d
        L.ref_qsatw.argtypes = [d, d]
        L.ref_qsatw.restype = d
        L.ref_advect_scalars.restype = i
        L.ref_advect_scalars.argtypes = [i, i, i, d, d, d, i, i, i, i, d, d, p, p, p, p, i, p, i]
        L.ref_advect_mom.argtypes = [i, i, i, d, d, d, i, i, d, d] + [p] * 9
        L.ref_advect_mom.restype = i
        L.ref_strain_N.argtypes = [i, i, i, d, d, d, i, i] + [p] * 9
        L.ref_strain_T.argtypes = [i, i, i, d, d, d, i, i] + [p] * 14
        L.ref_eddy_viscosity.argtypes = [i, i, i, d, d, d, i, i, i] + [d] * 9 + [p, p, p, p, i, p, p, p]
        L.ref_kessler.argtypes = [i, i, i, d, d, d, i, d, d, p, i]
        L.ref_kessler.restype = i
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def shape(cfg, t: int, g: int, nc: int = 1):
    """numpy shape of an array of index type t (0 cell, 1-3 x/y/z face) with
    ghost width g and nc components."""
    nx, ny, nz = cfg.nx + (t == 1), cfg.ny + (t == 2), cfg.nz + (t == 3)
    return (nc, nz + 2 * g, ny + 2 * g, nx + 2 * g)
