"""The allocation-free Kessler entry point.

erf_b200_kessler_advance_noalloc serves callers that cannot allocate device
memory: a host code whose device memory is all reserved up front by its own
pool (an AMReX arena, say) and which must not see a second allocator.  It must
produce what erf_b200_kessler_advance produces, on consecutive calls that
reuse its one shared scratch array, for dense views and for views with ghost
cells (whose ghost values it fills like the context entry point), and its
valid region must match the CPU oracle's Kessler.  This file is collected last
so that a failure here never hides the other tests' results.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_l2(a, b):
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def rainy_state(nx=24, ny=20, nz=40):
    """A supersaturated, cloudy and rainy moist-bubble state, so that every
    Kessler branch (condensation, evaporation, autoconversion, accretion,
    rain evaporation, sedimentation) runs."""
    from erf_b200 import Dycore, cases
    case = cases.moist_bubble(nx=nx, ny=ny, nz=nz)
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, _, _, _ = case.build_state(base[0])
    rng = np.random.default_rng(7)
    cons[5] *= 1.0 + 0.3 * rng.random(cons[5].shape)
    cons[6] = cons[0] * 2.0e-3 * rng.random(cons[0].shape)
    cons[7] = cons[0] * 1.0e-3 * rng.random(cons[0].shape)
    return case.cfg, dy, cons


def ghost_fab(t, g, nx, ny, nz, nc):
    """Array4 view with g ghost cells on every side of a (nc, nz+2g, ny+2g,
    nx+2g) device tensor."""
    from erf_b200 import dycore
    f = dycore.ErfFab()
    f.p = t.data_ptr()
    f.lo[0] = f.lo[1] = f.lo[2] = -g
    f.hi[0], f.hi[1], f.hi[2] = nx - 1 + g, ny - 1 + g, nz - 1 + g
    f.jstride = nx + 2 * g
    f.kstride = (nx + 2 * g) * (ny + 2 * g)
    f.nstride = f.kstride * (nz + 2 * g)
    f.ncomp = nc
    return f


def run(entry, cfg, dy, x, g):
    """One Kessler call through the context entry point ('ctx') or the
    allocation-free one ('noalloc') on a view with g ghost cells; returns
    the whole array, ghosts included."""
    import torch
    from erf_b200 import dycore
    lib = dycore.load_library()
    nc, nz, ny, nx = cfg.ncomp, cfg.nz, cfg.ny, cfg.nx
    if g == 0:
        t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        f = dycore.dense_fab(t, 0, nx, ny, nz, nc)
    else:
        t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        f = ghost_fab(t, g, nx, ny, nz, nc)
    torch.cuda.synchronize()
    if entry == "ctx":
        assert lib.erf_b200_kessler_advance(dy.ctx, ctypes.byref(f), cfg.dt) == 0
        assert dy.status() == 0
    else:
        assert lib.erf_b200_kessler_advance_noalloc(ctypes.byref(cfg), ctypes.byref(f), cfg.dt, None) == 0
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_noalloc_kessler_matches_context_entry_point_twice():
    pytest.importorskip("torch")
    cfg, dy, cons = rainy_state()
    nc = cfg.ncomp
    x1 = cons
    ref1, got1 = run("ctx", cfg, dy, x1, 0), run("noalloc", cfg, dy, x1, 0)
    assert not np.array_equal(ref1, x1)          # the step did something
    for n in range(nc):
        assert rel_l2(got1[n], ref1[n]) <= TOL, n
    # second call in a row: the shared scratch still holds call 1's data
    x2 = got1
    ref2, got2 = run("ctx", cfg, dy, x2, 0), run("noalloc", cfg, dy, x2, 0)
    for n in range(nc):
        assert rel_l2(got2[n], ref2[n]) <= TOL, n
    # both entry points against the CPU oracle's Kessler
    orc = oracle.kessler(cfg, x1, cfg.dt)
    for n in range(nc):
        assert rel_l2(got1[n], orc[n]) <= TOL, n
    dy.close()


def test_noalloc_kessler_ghosted_views_match_context_entry_point():
    """Views with two ghost cells on every side (strided, lo < 0): every
    element, ghosts included, equals the context entry point's, on two calls
    in a row; the ghost values start as junk and are overwritten."""
    pytest.importorskip("torch")
    cfg, dy, cons = rainy_state(nx=20, ny=16, nz=24)
    g = 2
    nc, nz, ny, nx = cons.shape
    x = np.full((nc, nz + 2 * g, ny + 2 * g, nx + 2 * g), -7.0)
    x[:, g:g + nz, g:g + ny, g:g + nx] = cons
    for _ in range(2):
        ref, got = run("ctx", cfg, dy, x, g), run("noalloc", cfg, dy, x, g)
        assert np.all(ref != -7.0)
        for n in range(nc):
            assert rel_l2(got[n], ref[n]) <= TOL, n
        x = got
    dy.close()


def test_noalloc_rejects_oversize_and_unsupported_requests():
    pytest.importorskip("torch")
    from erf_b200 import cases, dycore
    lib = dycore.load_library()
    cfg = cases.moist_bubble(nx=128, ny=128, nz=80).cfg      # 8 * 1.3M doubles > 2^21
    f = dycore.ErfFab()
    f.p = 1  # never dereferenced: the checks come first
    f.hi[0], f.hi[1], f.hi[2] = cfg.nx - 1, cfg.ny - 1, cfg.nz - 1
    f.ncomp = cfg.ncomp
    assert lib.erf_b200_kessler_advance_noalloc(ctypes.byref(cfg), ctypes.byref(f), cfg.dt, None) == 1
    # Kessler over terrain is rejected as erf_b200_create rejects it (the
    # sedimentation over terrain divides by detJ, which this call has not)
    small = cases.moist_bubble(nx=8, ny=8, nz=8).cfg
    small.use_terrain = 1
    f.hi[0], f.hi[1], f.hi[2] = 7, 7, 7
    assert lib.erf_b200_kessler_advance_noalloc(ctypes.byref(small), ctypes.byref(f), small.dt, None) == 8
