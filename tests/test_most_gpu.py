"""GPU: the MOST ground (Monin-Obukhov surface layer with the Moeng stress,
adiabatic, implicit MOST: BoundaryConditions/ERF_ABLMost.cpp:11-142 and
:289-489, ERF_MOSTStress.H:89-124 and :1395-1555).

  * the reference's gold ABL_MOST (only its header is kept upstream, so the
    per-variable min / max; fcompare tolerance 2e-10, Tests/CMakeLists.txt:3-4)
    reproduced by the fused step;
  * the fused step against the CPU oracle, relative L2 <= 1e-10 per field
    after 10 steps, on a noisy ABL over the MOST ground (Smagorinsky with the
    reference height at the first cell centre, Deardorff with it at the
    second; with and without acoustic substepping);
  * the mixed form over the MOST ground within its budget (1e-2 after 100
    steps), as the other mixed-form cases;
  * a moist (Kessler, buoyancy type 2) ABL over the MOST ground against the
    oracle, Smagorinsky and Deardorff.
"""
import os

import numpy as np
import pytest

import oracle
from erf_b200 import cases, config as C
from helpers import compare_states

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10


def test_gpu_reproduces_abl_most_gold():
    from erf_b200 import Dycore
    from golden.reference_cases import abl_most, plot_fields
    name, cfg, base, state, nsteps = abl_most()
    gold = np.load(os.path.join(HERE, "golden", f"{name}_minmax.npz"))
    dy = Dycore(cfg)
    dy.set_base_state(base)
    out = dy.advance_host(*state, nsteps)
    assert dy.status() == 0
    dy.close()
    f = plot_fields(out)
    f["rhoadv_0"] = out[0][4]
    for nm, lo, hi in zip(gold["names"], gold["vmin"], gold["vmax"]):
        a = f[str(nm)]
        print(nm, a.min(), lo, a.max(), hi)
        assert a.min() == pytest.approx(lo, rel=2e-10, abs=2e-10), str(nm)
        assert a.max() == pytest.approx(hi, rel=2e-10, abs=2e-10), str(nm)
    assert f["x_velocity"].min() < 9.95


def _run_both(case, nsteps):
    from erf_b200 import Dycore
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, nsteps)
    st = dy.status()
    dy.close()
    ref = oracle.advance(case.cfg, base, *init, nsteps)
    return compare_states(got, ref), st, got, init


@pytest.mark.parametrize("les,zref,nosub", [("smagorinsky", 0.0, False), ("deardorff", 80.0, False),
                                            ("smagorinsky", 0.0, True)])
def test_most_matches_oracle(les, zref, nosub):
    case = cases.abl_most(nx=24, ny=20, nz=16, les=les, zref=zref)
    if nosub:
        case.cfg.substepping_type = C.SUBSTEP_NONE
        case.cfg.dt = 0.05
    errs, st, got, init = _run_both(case, 10)
    print(les, zref, nosub, errs)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs
    # the ground stress decelerated the lowest level
    assert got[1][0].mean() < init[1][0].mean()


def test_most_mixed_within_budget():
    from erf_b200 import Dycore
    from helpers import rel_l2
    case = cases.abl_most(nx=24, ny=20, nz=16)
    case.cfg.precision = C.PREC_MIXED
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, 100)
    st = dy.status()
    dy.close()
    case.cfg.precision = C.PREC_FP64
    ref = oracle.advance(case.cfg, base, *init, 100)
    err = {"u": rel_l2(got[1], ref[1]), "v": rel_l2(got[2], ref[2]), "w": rel_l2(got[3], ref[3]),
           "theta": rel_l2(got[0][1] / got[0][0], ref[0][1] / ref[0][0])}
    print("mixed abl_most 24x20x16, 100 steps:", err)
    assert st == 0
    assert all(e <= 1e-2 for e in err.values()), err


@pytest.mark.parametrize("les,zref", [("smagorinsky", 0.0), ("deardorff", 80.0)])
def test_moist_most_matches_oracle(les, zref):
    """The MOST ground under a moist (Kessler) ABL with buoyancy type 2: the
    adiabatic ground adds no moisture flux, so the moist dycore runs over the
    dry MOST rule; 10 steps, every field <= 1e-10 against the oracle."""
    case = cases.abl_most_moist(nx=24, ny=20, nz=16, les=les, zref=zref)
    errs, st, got, init = _run_both(case, 10)
    print("moist MOST", les, zref, errs)
    assert st == 0
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs
    assert got[1][0].mean() < init[1][0].mean()
