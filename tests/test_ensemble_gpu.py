"""GPU: resident states, the autotuner and the ensemble graph.

* an ensemble of members of different sizes advanced by one graph launch
  per step gives bit-identical states to advancing each member alone (the
  members are created tallest first, which once left the tallest member's
  vertical kernels without enough shared memory);
* autotuning (which re-times candidate launch shapes on the resident state)
  leaves the resident state unchanged and the tuned step bit-identical;
* the abort word: set before a run, no step starts and the states are
  unchanged; set while a long run is in flight, the device loop stops
  between steps, every member holds a whole number of steps, equal to the
  members advanced alone by that many steps; cleared, the run continues.
"""
import threading
import time

import numpy as np
import pytest

from erf_b200 import cases, config as C

pytestmark = pytest.mark.gpu


def _member(nx, ny, nz, ug, seed, precision=C.PREC_FP64):
    from erf_b200 import Dycore
    case = cases.abl_dry(nx=nx, ny=ny, nz=nz, seed=seed)
    C.set_coriolis(case.cfg, rotational_time_period=4.0 * np.pi / 1.0e-4, latitude_deg=90.0, geo_wind=(ug, 0.0, 0.0))
    case.cfg.precision = precision
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    return dy, case.build_state(base[0])


def test_ensemble_matches_members_alone():
    from erf_b200.dycore import Ensemble
    # the tallest member first: its vertical kernels need the most shared
    # memory, and creating the shorter members after it must not lower the
    # kernels' shared-memory opt-in below its need
    specs = [(32, 32, 48, 6.0, 1), (48, 40, 24, 12.0, 2), (24, 24, 30, 9.0, 3)]
    alone = []
    for s in specs:
        dy, st = _member(*s)
        alone.append(dy.advance_host(*st, 3))
        dy.close()
    members = [_member(*s) for s in specs]
    for dy, st in members:
        dy.load_state(*st)
    ens = Ensemble([dy for dy, _ in members])
    ens.advance(3)
    assert ens.sync()
    assert ens.steps() == 3
    for (dy, st), ref in zip(members, alone):
        got = dy.store_state(*st)
        assert dy.status() == 0
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    ens.close()
    for dy, _ in members:
        dy.close()


@pytest.mark.parametrize("precision", [C.PREC_FP64, C.PREC_MIXED])
def test_autotune_keeps_results(precision):
    dy, st = _member(64, 48, 32, 10.0, 4, precision)
    ref = dy.advance_host(*st, 2)
    dy.load_state(*st)
    ms = dy.autotune(3)
    assert ms > 0
    dy.advance_resident(2)
    got = dy.store_state(*st)
    assert dy.status() == 0
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    dy.close()


def test_ensemble_abort_word():
    from erf_b200.dycore import Ensemble
    specs = [(32, 32, 24, 6.0, 1), (24, 40, 16, 12.0, 2)]
    members = [_member(*s) for s in specs]
    for dy, st in members:
        dy.load_state(*st)
    ens = Ensemble([dy for dy, _ in members])
    # set before the run: nothing starts, the states are untouched
    ens.abort(True)
    ens.advance(5)
    assert not ens.sync()
    assert ens.steps() == 0
    for dy, st in members:
        got = dy.store_state(*st)
        for a, b in zip(got, st):
            assert np.array_equal(a, b)
    # cleared: 4 steps run
    ens.abort(False)
    ens.advance(4)
    assert ens.sync()
    assert ens.steps() == 4
    # set from another thread while a long run is in flight
    ens.advance(400)
    threading.Thread(target=lambda: (time.sleep(0.05), ens.abort(True))).start()
    stopped = not ens.sync()
    n = ens.steps()
    print("abort stopped the loop:", stopped, "after", n, "steps")
    assert 4 <= n <= 404
    if stopped:
        assert n < 404 and n % 2 == 0   # the loop stops between pairs of steps
    outs = [dy.store_state(*st) for dy, st in members]
    for dy, _ in members:
        assert dy.status() == 0
    ens.close()
    # every member is exactly n steps old
    for (dy, st), got, s in zip(members, outs, specs):
        dy.close()
        ref_dy, ref_st = _member(*s)
        ref = ref_dy.advance_host(*ref_st, n)
        ref_dy.close()
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
