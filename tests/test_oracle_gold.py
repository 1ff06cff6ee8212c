"""The oracle against the reference's own gold plotfiles.

The fixtures were extracted from Tests/ERFGoldFiles by
tests/golden/extract_gold.py; the reference compares with fcompare at
rtol = atol = 2e-10 (Tests/CMakeLists.txt:3-4).  Here: relative L2 per plot
variable <= 2e-10.
"""
import os

import numpy as np
import pytest

import oracle
from golden.reference_cases import plot_variables, taylor_green

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("diffusing", [False, True])
def test_oracle_reproduces_taylor_green_gold(diffusing):
    name, cfg, base, state, nsteps = taylor_green(diffusing)
    gold = np.load(os.path.join(HERE, "golden", f"{name}_gold.npz"))
    assert gold["time"] == pytest.approx(nsteps * cfg.dt, rel=1e-14)
    out = oracle.advance(cfg, base, *state, nsteps)
    for nm, a, b in zip(gold["names"], plot_variables(out), gold["data"]):
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err <= 2e-10, (str(nm), err)


@pytest.mark.parametrize("case", ["EkmanSpiral", "IsentropicVortexAdvecting"])
def test_oracle_reproduces_no_substep_gold(case):
    """Two gold files run without acoustic substepping (substepping_type
    None, MRISplitIntegrator's no_substep hook):
      * EkmanSpiral: a 400-level column with a no-slip ground (the one-sided
        wall strain / stress stencils), constant molecular viscosity,
        Coriolis and geostrophic forcing;
      * IsentropicVortexAdvecting: a 2-D isentropic vortex advected at Mach
        1.2 with the Upwind_3rd dycore and scalar schemes.
    Every plot variable this path derives (vorticity is not) passes the
    reference's fcompare tolerance; they are in fact within ~1e-15."""
    from golden.reference_cases import ekman_spiral, gold_errors, isentropic_vortex_advecting
    mk = {"EkmanSpiral": ekman_spiral, "IsentropicVortexAdvecting": isentropic_vortex_advecting}[case]
    name, cfg, base, state, nsteps = mk()
    gold = np.load(os.path.join(HERE, "golden", f"{name}_gold.npz"))
    assert gold["time"] == pytest.approx(nsteps * cfg.dt, rel=1e-14)
    out = oracle.advance(cfg, base, *state, nsteps)
    errs = gold_errors(gold, out)
    assert len(errs) >= 6
    bad = {k: v for k, v in errs.items() if not v[2]}
    assert not bad, errs
    # tighter than fcompare: every non-trivial field to 1e-14
    assert all(v[0] <= 1e-14 or v[1] <= 1e-14 for v in errs.values()), errs


def abl_most_minmax(state):
    """Min / max of the ABL_MOST plot variables (ERF_Plotfile.cpp's
    density, rhoadv_0, velocities, temp, theta, pressure) of a dense state."""
    from golden.reference_cases import plot_fields
    f = plot_fields(state)
    f["rhoadv_0"] = state[0][4]
    return f


def test_oracle_reproduces_abl_most_gold():
    """Tests/ERFGoldFiles/ABL_MOST (a MOST ground with Moeng stress under
    Deardorff, 10 steps of 0.1 s on 64^3): the reference keeps only the
    header of this plotfile, so the per-variable min / max are compared.  The
    ground stress slows the lowest level from 10 m/s to 9.9456 m/s; the
    oracle reproduces every min / max to the last digit printed (fcompare's
    tolerance is 2e-10)."""
    from golden.reference_cases import abl_most
    name, cfg, base, state, nsteps = abl_most()
    gold = np.load(os.path.join(HERE, "golden", f"{name}_minmax.npz"))
    assert gold["time"] == pytest.approx(nsteps * cfg.dt, rel=1e-14)
    out = oracle.advance(cfg, base, *state, nsteps)
    f = abl_most_minmax(out)
    for nm, lo, hi in zip(gold["names"], gold["vmin"], gold["vmax"]):
        a = f[str(nm)]
        assert a.min() == pytest.approx(lo, rel=1e-15, abs=1e-300), (str(nm), a.min(), lo)
        assert a.max() == pytest.approx(hi, rel=1e-15, abs=1e-300), (str(nm), a.max(), hi)
    assert f["x_velocity"].min() < 9.95   # the surface stress acted
