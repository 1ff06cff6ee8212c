"""erf_b200_kessler_advance (the standalone microphysics entry point, the
column kernel behind Kessler::AdvanceKessler, Microphysics/Kessler/
ERF_Kessler.cpp:11-185) against the CPU oracle's Kessler, on supersaturated,
cloudy and rainy states so every branch runs: a small grid and the moist
bubble's full 128x128x80 grid, with and without rain.  Bar: relative L2
<= 1e-10 per component."""
import ctypes

import numpy as np
import pytest

import oracle
from erf_b200 import config as C

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_l2(a, b):
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


@pytest.mark.parametrize("size,rain", [((24, 20, 40), True), ((128, 128, 80), True), ((24, 20, 40), False)])
def test_context_kessler_matches_oracle(size, rain):
    import torch
    from erf_b200 import Dycore, cases, dycore
    nx, ny, nz = size
    case = cases.moist_bubble(nx=nx, ny=ny, nz=nz)
    cfg = case.cfg
    if not rain:
        cfg.moisture = C.MOIST_KESSLER_NORAIN
        cfg.ncomp = 7
        cfg.buoyancy_type = 1
    dy = Dycore(cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, _, _, _ = case.build_state(base[0])
    cons = np.ascontiguousarray(cons[:cfg.ncomp])
    rng = np.random.default_rng(11)
    cons[5] *= 1.0 + 0.3 * rng.random(cons[5].shape)
    cons[6] = cons[0] * 2.0e-3 * rng.random(cons[0].shape)
    if rain:
        cons[7] = cons[0] * 1.0e-3 * rng.random(cons[0].shape)
    lib = dycore.load_library()
    t = torch.from_numpy(cons.copy()).cuda()
    torch.cuda.synchronize()
    f = dycore.dense_fab(t, 0, nx, ny, nz, cfg.ncomp)
    for _ in range(2):       # two calls in a row, the second from the first's output
        assert lib.erf_b200_kessler_advance(dy.ctx, ctypes.byref(f), cfg.dt) == 0
    assert dy.status() == 0
    got = t.cpu().numpy()
    dy.close()
    ref = oracle.kessler(cfg, oracle.kessler(cfg, cons, cfg.dt), cfg.dt)
    assert not np.array_equal(ref, cons)
    for n in range(cfg.ncomp):
        assert rel_l2(got[n], ref[n]) <= TOL, (n, rel_l2(got[n], ref[n]))
