"""Minimal reader for AMReX plotfiles (single level): the text Header, the
Level_0/Cell_H box list and the Cell_D_* FAB blocks (a text FAB header
followed by raw little-endian float64, Fortran order per component), and the
nodal MultiFab that terrain plotfiles list after the cell one."""
import os
import re

import numpy as np


def _read_multifab(prefix, nodal):
    """Assemble the FABs listed in <prefix>_H over the union of their stored
    (grown) boxes; returns [ncomp, nz, ny, nx] starting at the lowest corner."""
    d = os.path.dirname(prefix)
    with open(prefix + "_H") as fh:
        ch = fh.read()
    files = re.findall(r"FabOnDisk:\s+(\S+)\s+(\d+)", ch)
    boxes = []
    for fname, off in files:
        with open(os.path.join(d, fname), "rb") as fh:
            fh.seek(int(off))
            head = b""
            while not head.endswith(b"\n"):
                head += fh.read(1)
            txt = head.decode()
            assert txt.startswith("FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))"), txt
            nums = re.findall(r"\(\((-?\d+),(-?\d+),(-?\d+)\) \((-?\d+),(-?\d+),(-?\d+)\) \((\d),(\d),(\d)\)", txt)
            blo = list(map(int, nums[0][0:3])); bhi = list(map(int, nums[0][3:6]))
            assert all(int(t) == nodal for t in nums[0][6:9]), txt
            nc = int(txt.strip().split()[-1])
            bshape = [bhi[q] - blo[q] + 1 for q in range(3)]
            n = bshape[0] * bshape[1] * bshape[2]
            raw = np.frombuffer(fh.read(8 * n * nc), dtype="<f8").reshape(nc, bshape[2], bshape[1], bshape[0])
            boxes.append((blo, bhi, raw))
    lo = np.min([b[0] for b in boxes], axis=0)
    hi = np.max([b[1] for b in boxes], axis=0) - lo
    data = np.zeros((boxes[0][2].shape[0], hi[2] + 1, hi[1] + 1, hi[0] + 1))
    for blo, bhi, raw in boxes:
        a, b = np.array(blo) - lo, np.array(bhi) - lo
        data[:, a[2]:b[2] + 1, a[1]:b[1] + 1, a[0]:b[0] + 1] = raw
    return data


def read_plotfile(path):
    with open(os.path.join(path, "Header")) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    nvar = int(lines[1])
    names = lines[2:2 + nvar]
    p = 2 + nvar
    time = float(lines[p + 1])
    ngrids = int(lines[p + 11].split()[1])
    q = p + 13 + 3 * ngrids
    data = _read_multifab(os.path.join(path, lines[q]), 0)
    out = {"names": names, "time": time, "data": data, "header": lines}
    if len(lines) > q + 5 and lines[q + 1] == "1":
        nn = int(lines[q + 2])
        out["nodal_names"] = lines[q + 3:q + 3 + nn]
        out["nodal"] = _read_multifab(os.path.join(path, lines[q + 3 + nn]), 1)
    return out


def read_plotfile_minmax(path):
    """Names, time and the per-component min / max of a single-box plotfile
    whose FAB data is not stored: the two value lines that follow the FAB
    list in Level_0/Cell_H (the MultiFab header's per-FAB minima, then
    maxima)."""
    with open(os.path.join(path, "Header")) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    nvar = int(lines[1])
    names = lines[2:2 + nvar]
    time = float(lines[2 + nvar + 1])
    with open(os.path.join(path, "Level_0", "Cell_H")) as fh:
        ch = [ln.strip() for ln in fh]
    rows = [ln for ln in ch if ln.count(",") >= nvar and not ln.startswith("FabOnDisk")]
    vals = [np.array([float(x) for x in r.split(",") if x], dtype=np.float64) for r in rows]
    assert len(vals) == 2 and all(v.size == nvar for v in vals), rows
    return {"names": names, "time": time, "min": vals[0], "max": vals[1]}


def read_plotfile_minmax_boxes(path):
    """Names, time, the boxes and the per-FAB, per-component min / max of a
    plotfile whose FAB data is not stored: Level_0/Cell_H lists the boxes
    ((lo) (hi) (type)), then nfab rows of minima and nfab rows of maxima."""
    import re
    with open(os.path.join(path, "Header")) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    nvar = int(lines[1])
    names = lines[2:2 + nvar]
    time = float(lines[2 + nvar + 1])
    with open(os.path.join(path, "Level_0", "Cell_H")) as fh:
        text = fh.read()
    boxes = [[[int(a) for a in lo.split(",")], [int(a) for a in hi.split(",")]]
             for lo, hi in re.findall(r"\(\(([-\d,]+)\) \(([-\d,]+)\) \([-\d,]+\)\)", text)]
    ch = [ln.strip() for ln in text.splitlines()]
    rows = [ln for ln in ch if ln.count(",") >= nvar and not ln.startswith("FabOnDisk")]
    vals = np.array([[float(x) for x in r.split(",") if x] for r in rows], dtype=np.float64)
    nfab = len(boxes)
    assert vals.shape == (2 * nfab, nvar), (vals.shape, nfab)
    return {"names": names, "time": time, "boxes": np.array(boxes), "min": vals[:nfab], "max": vals[nfab:]}
