"""The allocation-free Kessler entry point against the context entry point.

erf_b200_kessler_advance_noalloc serves callers that cannot allocate device
memory (a host code whose memory is all reserved by its own pool, or code
running during CUDA-graph capture).  It must produce what
erf_b200_kessler_advance produces, on consecutive calls that reuse its one
shared scratch array.  This file is collected last so that a failure here
never hides the other tests' results.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_l2(a, b):
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def test_noalloc_kessler_matches_context_entry_point_twice():
    torch = pytest.importorskip("torch")
    from erf_b200 import Dycore, cases, dycore

    case = cases.moist_bubble(nx=24, ny=20, nz=40)
    cfg = case.cfg
    dy = Dycore(cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, _, _, _ = case.build_state(base[0])
    # a supersaturated, cloudy and rainy state so every Kessler branch runs
    rng = np.random.default_rng(7)
    cons[5] *= 1.0 + 0.3 * rng.random(cons[5].shape)
    cons[6] = cons[0] * 2.0e-3 * rng.random(cons[0].shape)
    cons[7] = cons[0] * 1.0e-3 * rng.random(cons[0].shape)
    lib = dycore.load_library()
    nc, nz, ny, nx = cons.shape

    def run_context(x):
        t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        torch.cuda.synchronize()
        f = dycore.dense_fab(t, 0, nx, ny, nz, nc)
        assert lib.erf_b200_kessler_advance(dy.ctx, ctypes.byref(f), cfg.dt) == 0
        assert dy.status() == 0
        return t.cpu().numpy()

    def run_noalloc(x):
        t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        torch.cuda.synchronize()
        f = dycore.dense_fab(t, 0, nx, ny, nz, nc)
        assert lib.erf_b200_kessler_advance_noalloc(ctypes.byref(cfg), ctypes.byref(f), cfg.dt, None) == 0
        torch.cuda.synchronize()
        return t.cpu().numpy()

    x1 = cons
    ref1, got1 = run_context(x1), run_noalloc(x1)
    assert not np.array_equal(ref1, x1)          # the step did something
    for n in range(nc):
        assert rel_l2(got1[n], ref1[n]) <= TOL, n
    # second call in a row: the shared scratch still holds call 1's data
    x2 = got1
    ref2, got2 = run_context(x2), run_noalloc(x2)
    for n in range(nc):
        assert rel_l2(got2[n], ref2[n]) <= TOL, n
    dy.close()


def test_noalloc_rejects_oversize_requests():
    pytest.importorskip("torch")
    from erf_b200 import cases, dycore
    lib = dycore.load_library()
    cfg = cases.moist_bubble(nx=128, ny=128, nz=80).cfg      # 8 * 1.3M doubles > 2^21
    f = dycore.ErfFab()
    f.p = 1  # never dereferenced: the size check comes first
    f.hi[0], f.hi[1], f.hi[2] = cfg.nx - 1, cfg.ny - 1, cfg.nz - 1
    f.ncomp = cfg.ncomp
    assert lib.erf_b200_kessler_advance_noalloc(ctypes.byref(cfg), ctypes.byref(f), cfg.dt, None) == 1
