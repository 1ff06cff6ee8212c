"""Failure detection on the GPU, with no fault and no hang: each check makes
a failure on the host side or through a wait that nothing can complete, and
checks that the library reports it as a status code and stays usable.

  * a bounded mbarrier wait that cannot complete ends by its poll limit and
    reports (the path the tensor-core kernels take before ERF_B200_ETIMEOUT);
  * a non-positive rho*theta in the input state is reported as
    ERF_B200_EBADSTATE, a NaN velocity as ERF_B200_ENAN;
  * the status word is cleared on read, and the same context then advances a
    good state to the same result as a fresh context.
"""
import ctypes

import numpy as np
import pytest

from erf_b200 import cases

pytestmark = pytest.mark.gpu

EBADSTATE, ENAN = 4, 5


def _context(case):
    from erf_b200 import Dycore
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    return dy, base


def test_bounded_wait_ends_and_reports():
    from erf_b200 import load_library
    L = load_library()
    out = ctypes.c_int(-1)
    assert L.erf_b200_selftest_bounded_wait(1000, ctypes.byref(out)) == 0
    assert out.value == 1
    assert L.erf_b200_selftest_bounded_wait(0, ctypes.byref(out)) != 0   # bad argument
    # the device is still usable
    case = cases.abl_dry(nx=8, ny=8, nz=8)
    dy, base = _context(case)
    dy.advance_host(*case.build_state(base[0]), 1)
    assert dy.status() == 0
    dy.close()


@pytest.mark.parametrize("what", ["rhotheta", "velocity"])
def test_bad_input_is_reported_and_context_recovers(what):
    case = cases.abl_dry(nx=16, ny=12, nz=10)
    dy, base = _context(case)
    cons, u, v, w = case.build_state(base[0])
    bad = [a.copy() for a in (cons, u, v, w)]
    if what == "rhotheta":
        bad[0][1, 3, 4, 5] = -1.0
        want = EBADSTATE
    else:
        bad[1][2, 5, 7] = np.nan
        want = ENAN
    dy.advance_host(*bad, 1)
    assert dy.status() == want
    assert dy.status() == 0            # cleared on read
    got = dy.advance_host(cons, u, v, w, 2)
    assert dy.status() == 0
    dy.close()
    fresh, _ = _context(case)
    ref = fresh.advance_host(cons, u, v, w, 2)
    fresh.close()
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
