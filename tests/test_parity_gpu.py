"""GPU parity: the CUDA dycore (through the C-ABI) against the CPU FP64 oracle.

Bar: relative L2 <= 1e-10 per field after 10 full RK3 steps (the FP64 plain
form's parity target), on seeded synthetic inputs small enough for the oracle.
"""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from helpers import compare_states

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _dycore(cfg):
    from erf_b200 import Dycore
    return Dycore(cfg)


def run_both(case, nsteps):
    dy = _dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    got = dy.advance_host(cons, u, v, w, nsteps)
    st = dy.status()
    ref = oracle.advance(case.cfg, base, cons, u, v, w, nsteps)
    dy.close()
    return compare_states(got, ref), st


def test_base_state_matches_oracle():
    case = cases.moist_bubble(nx=16, ny=16, nz=80)
    dy = _dycore(case.cfg)
    got = dy.make_base_state(case)
    ref = oracle.make_base_state(case.cfg, case)
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r) / np.abs(r)) < 1e-13


@pytest.mark.parametrize("nsteps", [1, 10])
def test_abl_dry_smagorinsky(nsteps):
    case = cases.abl_dry(nx=24, ny=20, nz=16)
    errs, st = run_both(case, nsteps)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


@pytest.mark.parametrize("nsteps", [1, 10])
def test_moist_bubble_kessler_weno5(nsteps):
    case = cases.moist_bubble(nx=24, ny=20, nz=40)
    case.pert["bubble_rh"] = 6000.0
    errs, st = run_both(case, nsteps)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


@pytest.mark.parametrize("diffusing", [False, True])
def test_gpu_reproduces_taylor_green_gold(diffusing):
    """The CUDA path against the reference's gold plotfile directly."""
    import os
    from golden.reference_cases import plot_variables, taylor_green
    name, cfg, base, state, nsteps = taylor_green(diffusing)
    gold = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"{name}_gold.npz"))
    dy = _dycore(cfg)
    dy.set_base_state(base)
    out = dy.advance_host(*state, nsteps)
    assert dy.status() == 0
    dy.close()
    for nm, a, b in zip(gold["names"], plot_variables(out), gold["data"]):
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err <= 2e-10, (str(nm), err)
