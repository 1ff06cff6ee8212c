"""Per-step JSON metrics lines: the integrated quantities ERF prints every
`erf.sum_interval` steps (sum_integrated_quantities,
IO/ERF_WriteScalarProfiles.cpp:14-60: the mass and the rho-theta integral
over the physical volume), plus max |w|, the wall time of the steps and
their rate, one JSON object per line.  The mass line doubles as a
conservation check: with periodic sides and walls top and bottom the flux
form keeps it to round-off, over static or moving terrain.
"""
from __future__ import annotations

import json
import sys
import time


def run_logged(dycore, cons, u, v, w, nsteps: int, every: int = 1, out=None, t0: float = 0.0):
    """Advance a state on the device `nsteps` steps (it is made resident
    first), writing a JSON line to `out` (default stdout) for the initial
    state and after every `every` steps.  Returns the list of records."""
    out = sys.stdout if out is None else out
    cfg = dycore.cfg
    cells = cfg.nx * cfg.ny * cfg.nz
    dycore.load_state(cons, u, v, w)
    recs = []

    def emit(step, wall, nadv):
        d = dycore.diagnostics()
        rec = {"step": step, "time": t0 + step * cfg.dt, "mass": d["mass"], "rhotheta": d["rhotheta"],
               "max_w": d["max_w"], "wall_s": wall,
               "cell_steps_per_s": (cells * nadv / wall) if wall > 0 else None}
        if recs:
            rec["mass_drift"] = (d["mass"] - recs[0]["mass"]) / recs[0]["mass"]
        recs.append(rec)
        out.write(json.dumps(rec) + "\n")
        out.flush()

    emit(0, 0.0, 0)
    step = 0
    while step < nsteps:
        n = min(every, nsteps - step)
        tic = time.perf_counter()
        dycore.advance_resident(n)
        status = dycore.status()   # synchronises the stream
        wall = time.perf_counter() - tic
        if status != 0:
            raise RuntimeError(f"device status {status} after step {step + n}")
        step += n
        emit(step, wall, n)
    return recs
