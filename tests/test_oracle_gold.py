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
