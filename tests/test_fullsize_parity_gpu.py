"""GPU-vs-oracle field parity at the workloads' full sizes.

The three single-GPU workloads, at the sizes and settings the benchmark
quotes, advanced through the C-ABI on the device and by the CPU FP64 oracle
from the same seeded inputs; every field is compared at relative L2 <= 1e-10
(the reference's own regression tolerance is 2e-10, Tests/CMakeLists.txt:3-4):

  * dry neutral ABL 64x64x64, Smagorinsky, no-slip ground, Coriolis and
    geostrophic forcing, dt 0.5 s with 6 acoustic substeps: 10 steps;
  * moist bubble 128x128x80, Kessler, WENO5 moisture, buoyancy type 2: 10 steps;
  * terrain ABL 256x256x96 (stretched levels, Deardorff, static terrain):
    2 steps (the oracle's terrain path takes about 20-40 s per step there).
"""
import numpy as np
import pytest

import oracle
from erf_b200 import cases
from erf_b200 import terrain as T
from helpers import compare_states

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _check(errs):
    bad = {k: v for k, v in errs.items() if not v <= TOL}
    assert not bad, errs


def test_abl_dry_64cubed_10_steps():
    from erf_b200 import Dycore
    case = cases.abl_dry()
    c = case.cfg
    assert (c.nx, c.ny, c.nz, c.dt, c.mri_ratio) == (64, 64, 64, 0.5, 6)
    dy = Dycore(c)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, 10)
    st = dy.status()
    dy.close()
    ref = oracle.advance(c, base, *init, 10)
    assert st == 0
    errs = compare_states(got, ref)
    print("abl_dry 64^3 x10:", {k: f"{v:.2e}" for k, v in errs.items()})
    _check(errs)


def test_moist_bubble_128x128x80_10_steps():
    from erf_b200 import Dycore
    case = cases.moist_bubble()
    c = case.cfg
    assert (c.nx, c.ny, c.nz) == (128, 128, 80)
    dy = Dycore(c)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, 10)
    st = dy.status()
    dy.close()
    ref = oracle.advance(c, base, *init, 10)
    assert st == 0
    errs = compare_states(got, ref)
    print("moist_bubble 128x128x80 x10:", {k: f"{v:.2e}" for k, v in errs.items()})
    _check(errs)


def test_terrain_abl_256x256x96_2_steps():
    from erf_b200 import Dycore
    case = T.abl_terrain()
    c = case.cfg
    assert (c.nx, c.ny, c.nz) == (256, 256, 96)
    dy = Dycore(c)
    dy.set_terrain(case.z_nd)
    base = dy.make_base_state_terrain(case)
    dy.set_base_state(base)
    init = case.build_state(base[0])
    got = dy.advance_host(*init, 2)
    st = dy.status()
    dy.close()
    ref = oracle.advance_terrain(c, case.z_nd, base, *init, 2)
    assert st == 0
    errs = compare_states(got, ref)
    print("terrain_abl 256x256x96 x2:", {k: f"{v:.2e}" for k, v in errs.items()})
    _check(errs)
