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
