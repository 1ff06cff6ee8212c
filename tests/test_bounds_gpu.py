"""GPU: the bounds-checked build (liberf_b200_bounds.so, the library compiled
with -DERF_B200_BOUNDS=1; `python -m erf_b200.build --bounds`).  Every
global index its kernels form through cidx is checked against the array;
a stray one sets ERF_B200_EBOUNDS and is redirected to element 0, so it
shows as a status code and a parity break, never as a fault.  This is the
memory check of the path (a memory-checking tool is not available on the
GPUs this library is tested on).

The cases run in a child process with ERF_B200_LIB pointing at that
library: small grids of every path (flat dry and moist, the closures, the
MOST ground, no substepping, static and moving terrain with and without
substeps, the mixed form), each with status OK and the fields within 1e-10
of the oracle (the mixed form within its 1e-2 budget).
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BOUNDS_LIB = os.path.join(ROOT, "erf_b200", "liberf_b200_bounds.so")


def _cases():
    """(name, runner) pairs; each runner returns (status, errors dict, bound)."""
    import oracle
    from erf_b200 import Dycore, cases
    from erf_b200 import config as C
    from erf_b200 import terrain as T
    from helpers import compare_states, rel_l2

    def flat(case, steps, precision=C.PREC_FP64, bound=1e-10):
        def run():
            cfg = case.cfg.copy()
            cfg.precision = precision
            dy = Dycore(cfg)
            base = dy.make_base_state(case)
            dy.set_base_state(base)
            init = case.build_state(base[0])
            got = dy.advance_host(*init, steps)
            st = dy.status()
            dy.close()
            ref = oracle.advance(case.cfg, base, *init, steps)
            errs = compare_states(got, ref)
            errs.pop("v", None) if precision != C.PREC_FP64 else None
            return st, errs, bound
        return run

    def static_terrain(case, steps):
        def run():
            dy = Dycore(case.cfg)
            dy.set_terrain(case.z_nd)
            base = dy.make_base_state_terrain(case)
            dy.set_base_state(base)
            init = case.build_state(base[0])
            got = dy.advance_host(*init, steps)
            st = dy.status()
            dy.close()
            ref = oracle.advance_terrain(case.cfg, case.z_nd, base, *init, steps)
            return st, compare_states(got, ref), 1e-10
        return run

    def moving(case):
        def run():
            dy = Dycore(case.cfg)
            dy.set_base_state(case.base)
            st0 = case.build_state()
            got = dy.advance_host(*st0, case.steps)
            st = dy.status()
            dy.close()
            ref = oracle.advance_moving_terrain(case.cfg, 0.0, case.base, *st0, case.steps)
            errs = {"rho": rel_l2(got[0][0], ref[0][0]), "rhotheta": rel_l2(got[0][1], ref[0][1]),
                    "u": rel_l2(got[1], ref[1]), "w": rel_l2(got[3], ref[3])}
            return st, errs, 1e-10
        return run

    nosub = cases.abl_dry(nx=16, ny=12, nz=10)
    nosub.cfg.substepping_type = C.SUBSTEP_NONE
    nosub.cfg.dt = 0.05
    mt_sub = T.moving_terrain(nx=12, ny=4, nz=12, Lx=60.0, Ly=20.0, H=60.0, ampl=0.3, wavelength=30.0,
                              substeps=True, dt=0.02, steps=2)
    mt_sub.cfg.mri_ratio = 4
    return [
        ("moist_bubble", flat(cases.moist_bubble(nx=16, ny=16, nz=24), 2)),
        ("moist_bubble_mixed", flat(cases.moist_bubble(nx=16, ny=16, nz=24), 2, C.PREC_MIXED, 1e-2)),
        ("abl_smagorinsky", flat(cases.abl_dry(nx=16, ny=12, nz=10), 2)),
        ("abl_deardorff", flat(cases.abl_deardorff(nx=16, ny=12, nz=10), 2)),
        ("abl_most", flat(cases.abl_most(nx=16, ny=12, nz=10), 2)),
        ("no_substep", flat(nosub, 2)),
        ("terrain_hill", static_terrain(T.abl_terrain(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0,
                                                      r0=100.0, amp=5.0), 1)),
        ("terrain_moist_hill", static_terrain(T.moist_hill(nx=12, ny=10, nz=12), 1)),
        ("moving_terrain", moving(T.moving_terrain(nx=12, ny=4, nz=12, Lx=60.0, Ly=20.0, H=60.0, ampl=0.3,
                                                   wavelength=30.0, steps=3))),
        ("moving_terrain_substeps", moving(mt_sub)),
    ]


def _child():
    sys.path.insert(0, HERE)
    sys.path.insert(0, ROOT)
    from erf_b200 import dycore
    assert dycore.LIB_PATH == os.environ["ERF_B200_LIB"]
    out = {}
    for name, run in _cases():
        st, errs, bound = run()
        out[name] = {"status": st, "errors": {k: float(v) for k, v in errs.items()}, "bound": bound}
    print("RESULT " + json.dumps(out))


def test_bounds_checked_build_runs_clean_and_matches_oracle():
    if not os.path.exists(BOUNDS_LIB):
        pytest.skip("liberf_b200_bounds.so not built (python -m erf_b200.build --bounds)")
    env = dict(os.environ, ERF_B200_LIB=BOUNDS_LIB)
    p = subprocess.run([sys.executable, os.path.abspath(__file__)], env=env, capture_output=True, text=True,
                       timeout=1200, cwd=ROOT)
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("RESULT ")]
    assert p.returncode == 0 and line, p.stdout[-3000:] + p.stderr[-3000:]
    res = json.loads(line[0][len("RESULT "):])
    for name, r in res.items():
        print(name, "status", r["status"], "worst", max(r["errors"].values()))
    bad = {n: r for n, r in res.items()
           if r["status"] != 0 or not all(np.isfinite(v) and v <= r["bound"] for v in r["errors"].values())}
    assert not bad, bad


if __name__ == "__main__":
    _child()
