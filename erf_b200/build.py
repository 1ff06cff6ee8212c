"""Build the sm_100a shared library liberf_b200.so in-tree with nvcc.

    python -m erf_b200.build            # incremental
    python -m erf_b200.build --force    # rebuild everything
    python -m erf_b200.build --bounds   # the bounds-checked variant

The bounds-checked variant liberf_b200_bounds.so is the same code compiled
with -DERF_B200_BOUNDS=1: every global index formed by cidx is checked
against its array and a stray one sets ERF_B200_EBOUNDS instead of
touching memory outside the array (the stand-in for a memory checker).
Select it for a process with ERF_B200_LIB=<path>.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liberf_b200.so")
OBJ_BOUNDS = os.path.join(HERE, "_build_bounds")
LIB_BOUNDS = os.path.join(HERE, "liberf_b200_bounds.so")
# the two terrain halves take longest, so they start first
SOURCES = ["terrain.cu", "terrain_f32.cu", "kernels.cu", "api.cu", "noalloc.cu", "mlp.cu", "closure.cu", "plotfile.cu",
           "checkpoint.cu"]
# sources a translation unit includes besides the headers
INCLUDED = {"terrain_f32.cu": ["terrain.cu"]}
HEADERS = ["common.cuh", "kernels.cuh", "tiles.cuh", "tcgen05.cuh", "mlp.cuh", "amrex_io.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-v"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, bounds: bool = False) -> str:
    OBJ = OBJ_BOUNDS if bounds else globals()["OBJ"]
    LIB = LIB_BOUNDS if bounds else globals()["LIB"]
    flags = FLAGS + (["-DERF_B200_BOUNDS=1"] if bounds else [])
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "erf_b200.h")]
    objs = [os.path.join(OBJ, s.replace(".cu", ".o")) for s in SOURCES]
    todo = [(s, o) for s, o in zip(SOURCES, objs) if force or _stale(o, [os.path.join(CSRC, d) for d in [s] + INCLUDED.get(s, [])] + hdrs)]

    def compile_one(job):
        s, obj = job
        cmd = [NVCC, *ARCH, *flags, "-c", os.path.join(CSRC, s), "-o", obj]
        out = subprocess.run(cmd, capture_output=True, text=True)
        with open(os.path.join(OBJ, s + ".log"), "w") as fh:
            fh.write(" ".join(cmd) + "\n" + out.stdout + out.stderr)
        return s, out

    # the translation units are independent: compile them concurrently
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        for s, out in ex.map(compile_one, todo):
            if out.returncode != 0:
                raise RuntimeError(f"nvcc failed for {s}:\n{out.stderr[-4000:]}")
            if verbose:
                sys.stderr.write(out.stderr)
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        out = subprocess.run(cmd, capture_output=True, text=True)
        if out.returncode != 0:
            raise RuntimeError("link failed:\n" + out.stderr[-4000:])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, bounds="--bounds" in sys.argv))
