"""Minimal reader for AMReX plotfiles (single level): the text Header, the
Level_0/Cell_H box list and the Cell_D_* FAB blocks (a text FAB header
followed by raw little-endian float64, Fortran order per component)."""
import os
import re

import numpy as np


def read_plotfile(path):
    with open(os.path.join(path, "Header")) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    nvar = int(lines[1])
    names = lines[2:2 + nvar]
    p = 2 + nvar
    ndim = int(lines[p]); p += 1
    time = float(lines[p]); p += 1
    domain = re.findall(r"-?\d+", lines[p + 4])
    lo = list(map(int, domain[0:3])); hi = list(map(int, domain[3:6]))
    shape = [hi[d] - lo[d] + 1 for d in range(3)]
    data = np.zeros((nvar, shape[2], shape[1], shape[0]))
    lvl = os.path.join(path, "Level_0")
    with open(os.path.join(lvl, "Cell_H")) as fh:
        ch = fh.read()
    files = re.findall(r"FabOnDisk:\s+(\S+)\s+(\d+)", ch)
    for fname, off in files:
        with open(os.path.join(lvl, fname), "rb") as fh:
            fh.seek(int(off))
            head = b""
            while not head.endswith(b"\n"):
                head += fh.read(1)
            txt = head.decode()
            nums = re.findall(r"\(\((-?\d+),(-?\d+),(-?\d+)\) \((-?\d+),(-?\d+),(-?\d+)\)", txt)
            blo = list(map(int, nums[0][0:3])); bhi = list(map(int, nums[0][3:6]))
            nc = int(txt.strip().split()[-1])
            bshape = [bhi[d] - blo[d] + 1 for d in range(3)]
            n = bshape[0] * bshape[1] * bshape[2]
            raw = np.frombuffer(fh.read(8 * n * nc), dtype="<f8").reshape(nc, bshape[2], bshape[1], bshape[0])
            data[:, blo[2]:bhi[2] + 1, blo[1]:bhi[1] + 1, blo[0]:bhi[0] + 1] = raw
    return {"names": names, "time": time, "data": data}
