"""GPU: the per-pass entry points (turbulent_viscosity, slow_rhs_pre,
fast_rhs_N with make_fast_coeffs at substep 0, slow_rhs_post) composed by a
host-side MRISplitIntegrator schedule (ERF_MRI.H:187-369) reproduce the fused
step.  The composed step omits the momentum round trip between substeps that
the fused step applies (a boundary fill of the caller's), so the bar is
relative L2 <= 1e-10 per field after one step.

The library runs on its own stream here (torch is on the legacy default
stream, which a context cannot share), so the host synchronises the device
around every library call that reads or writes tensors made by torch."""
import numpy as np
import pytest

from erf_b200 import cases, config as C
from helpers import compare_states

pytestmark = pytest.mark.gpu


def schedule(cfg, nrk):
    sub = cfg.dt / cfg.mri_ratio
    if nrk == 0:
        return (1, cfg.dt / 3.0, cfg.dt / 3.0) if cfg.force_stage1_single_substep else (cfg.mri_ratio // 3, sub, cfg.dt / 3.0)
    if nrk == 1:
        return cfg.mri_ratio // 2, sub, cfg.dt / 2.0
    return cfg.mri_ratio, sub, cfg.dt


@pytest.mark.parametrize("nosub,most", [(False, False), (True, False), (False, True)])
def test_per_pass_composition_matches_fused_step(nosub, most):
    """With nosub the stages call the no_substep hook entry
    (erf_b200_no_substep) in place of the acoustic substeps, at a time step
    inside the explicit acoustic limit.  With most the ground is a MOST
    surface and the schedule first calls erf_b200_most_update_fluxes on the
    old velocities, as ERF_Advance.cpp:62-86 calls ABLMost::update_fluxes."""
    import ctypes
    import torch
    from erf_b200 import Dycore
    from erf_b200.dycore import dense_fab, ErfFab
    case = cases.abl_most(nx=32, ny=24, nz=16) if most else cases.abl_dry(nx=32, ny=24, nz=16)
    cfg = case.cfg
    if nosub:
        cfg.substepping_type = C.SUBSTEP_NONE
        cfg.dt = 0.05
    nx, ny, nz, nc = cfg.nx, cfg.ny, cfg.nz, cfg.ncomp
    dy = Dycore(cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons0, u0, v0, w0 = case.build_state(base[0])
    fused = dy.advance_host(cons0, u0, v0, w0, 1)
    assert dy.status() == 0

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    zeros = lambda *s: torch.zeros(s, dtype=torch.float64, device="cuda")
    cons, u, v, w = t(cons0), t(u0), t(v0), t(w0)
    rho = cons[0]

    def sums():
        rx = rho + torch.roll(rho, 1, dims=2)
        ry = rho + torch.roll(rho, 1, dims=1)
        rz = rho[1:] + rho[:-1]
        return rx, ry, rz

    def v2m_rt(uu, vv, ww, rx, ry, rz):
        """velocity -> momentum with the fused prologue's round trip; returns momenta and velocities"""
        out_m, out_v = [], []
        for f, rs, kind in ((uu[:, :, :nx], rx, 0), (vv[:, :ny, :], ry, 1), (ww[1:nz], rz, 2)):
            m0 = (f * 0.5) * rs
            v1 = (m0 * 2.0) / rs
            out_m.append((v1 * 0.5) * rs)
            out_v.append(v1)
        return out_m, out_v

    def to_face(a, kind):
        if kind == 0:
            return torch.cat([a, a[:, :, :1]], dim=2).contiguous()
        if kind == 1:
            return torch.cat([a, a[:, :1, :]], dim=1).contiguous()
        z = torch.zeros((1, ny, nx), dtype=a.dtype, device=a.device)
        return torch.cat([z, a, z], dim=0).contiguous()

    rx, ry, rz = sums()
    (mx, my, mz), (u1, v1, w1) = v2m_rt(u, v, w, rx, ry, rz)
    S_old = [cons.clone(), to_face(mx, 0), to_face(my, 1), to_face(mz, 2)]
    vel = [to_face(u1, 0), to_face(v1, 1), to_face(w1, 2)]

    def fabs(S, ncons):
        arr = (ErfFab * 4)()
        arr[0] = dense_fab(S[0], 0, nx, ny, nz, ncons)
        for q, kind in ((1, 1), (2, 2), (3, 3)):
            arr[q] = dense_fab(S[q], kind, nx, ny, nz)
        return arr

    def state(ncons):
        return [zeros(ncons, nz, ny, nx), zeros(nz, ny, nx + 1), zeros(nz, ny + 1, nx), zeros(nz + 1, ny, nx)]

    L = dy.lib
    vf = lambda V: [ctypes.byref(dense_fab(V[q], q + 1, nx, ny, nz)) for q in range(3)]
    L.erf_b200_turbulent_viscosity.argtypes = [ctypes.c_void_p] * 5
    L.erf_b200_slow_rhs_pre.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 6
    L.erf_b200_fast_rhs_N.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5 + [ctypes.c_double] * 2
    L.erf_b200_slow_rhs_post.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 5
    L.erf_b200_no_substep.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_double, ctypes.c_int]
    fc = dense_fab(cons, 0, nx, ny, nz, nc)
    torch.cuda.synchronize()
    assert L.erf_b200_turbulent_viscosity(dy.ctx, *vf([u, v, w]), ctypes.byref(fc)) == 0
    if most:
        L.erf_b200_most_update_fluxes.argtypes = [ctypes.c_void_p] * 3
        assert L.erf_b200_most_update_fluxes(dy.ctx, *vf([u, v, w])[:2]) == 0
    stage = [a.clone() for a in S_old]
    S_rhs, S_scr = state(2), state(2)
    for nrk in range(3):
        nsub, dtau, slow_dt = schedule(cfg, nrk)
        torch.cuda.synchronize()
        assert L.erf_b200_slow_rhs_pre(dy.ctx, nrk, slow_dt, fabs(S_rhs, 2), fabs(stage, nc), fabs(S_scr, 2),
                                       *vf(vel)) == 0
        S_data = [a.clone() for a in S_old]
        if nosub:
            torch.cuda.synchronize()
            assert L.erf_b200_no_substep(dy.ctx, fabs(S_data, nc), fabs(S_old, nc), fabs(S_rhs, 2), slow_dt, nrk) == 0
            torch.cuda.synchronize()
        for ks in range(0 if nosub else nsub):
            prev = S_old if ks == 0 else [a.clone() for a in S_data]
            torch.cuda.synchronize()
            assert L.erf_b200_fast_rhs_N(dy.ctx, ks, nrk, fabs(S_rhs, 2), fabs(prev, nc), fabs(stage, nc),
                                         fabs(S_data, nc), fabs(S_scr, 2), dtau, 1.0 / nsub) == 0
            torch.cuda.synchronize()
        S_new = state(nc)
        torch.cuda.synchronize()
        assert L.erf_b200_slow_rhs_post(dy.ctx, nrk, slow_dt, fabs(S_rhs, 2), fabs(S_old, nc), fabs(S_new, nc),
                                        fabs(S_data, nc), fabs(S_scr, 2)) == 0
        torch.cuda.synchronize()
        # stage velocities: the post's two momentum/velocity round trips of S_data
        rho = S_data[0][0]
        rx, ry, rz = sums()
        vel = []
        for q, rs in ((1, rx), (2, ry), (3, rz)):
            m = S_data[q]
            if q == 1:
                m = m[:, :, :nx]
            elif q == 2:
                m = m[:, :ny, :]
            else:
                m = m[1:nz]
            a1 = (m * 2.0) / rs
            m1 = (a1 * 0.5) * rs
            vel.append(to_face((m1 * 2.0) / rs, q - 1))
        stage = S_new
    assert dy.status() == 0
    got = (stage[0].cpu().numpy(), vel[0].cpu().numpy(), vel[1].cpu().numpy(), vel[2].cpu().numpy())
    dy.close()
    errs = compare_states(got, fused)
    bad = {k: e for k, e in errs.items() if not e <= 1e-10}
    assert not bad, errs


def test_make_fast_coeffs_export():
    """The exported A, 1/B', C, P, Q satisfy the elimination they describe:
    B'_k = B_k - A_k C_{k-1} / B'_{k-1} holds with the stored 1/B'."""
    import ctypes
    import torch
    from erf_b200 import Dycore
    from erf_b200.dycore import dense_fab, ErfFab
    case = cases.abl_dry(nx=16, ny=16, nz=12)
    cfg = case.cfg
    dy = Dycore(cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    cons, u, v, w = case.build_state(base[0])
    S = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (cons, np.zeros((16, 16, 17)),
                                                                     np.zeros((16, 17, 16)), np.zeros((13, 16, 16)))]
    coef = torch.zeros((5, 13, 16, 16), dtype=torch.float64, device="cuda")
    arr = (ErfFab * 4)()
    arr[0] = dense_fab(S[0], 0, 16, 16, 12, cfg.ncomp)
    for q in (1, 2, 3):
        arr[q] = dense_fab(S[q], q, 16, 16, 12)
    fc = dense_fab(coef, 3, 16, 16, 12, 5)
    dy.lib.erf_b200_make_fast_coeffs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
    torch.cuda.synchronize()
    assert dy.lib.erf_b200_make_fast_coeffs(dy.ctx, ctypes.byref(fc), arr, cfg.dt / cfg.mri_ratio) == 0
    torch.cuda.synchronize()
    A, invB, Cc, Pc, Qc = coef.cpu().numpy()
    dy.close()
    assert np.allclose(A[0], 0) and np.allclose(invB[0], 1) and np.allclose(A[12], 0)
    # interior rows: the diagonal of the original system is positive and dominant
    Bp = 1.0 / invB[1:12]
    assert np.all(Bp > 0)
    assert np.all(np.abs(Pc[1:12]) > 0) and np.all(np.abs(Qc[1:12]) > 0)


def _w_walls(z_nd, u, v, dx, dy, zhi_noslip):
    """w on the ground and the lid from Omega = 0 (WFromOmega) for face
    velocities u [nz][ny][nx+1], v [nz+1... ] given as numpy arrays."""
    nz = u.shape[0]
    out = []
    for k in (0, nz):
        z = z_nd[k]
        mx = 0.5 / dx * (z[1:, 1:] + z[:-1, 1:] - z[1:, :-1] - z[:-1, :-1])
        my = 0.5 / dy * (z[1:, 1:] + z[1:, :-1] - z[:-1, 1:] - z[:-1, :-1])
        if k == 0:
            uf = 1.5 * (0.5 * (u[0, :, :-1] + u[0, :, 1:])) - 0.5 * (0.5 * (u[1, :, :-1] + u[1, :, 1:]))
            vf = 1.5 * (0.5 * (v[0, :-1, :] + v[0, 1:, :])) - 0.5 * (0.5 * (v[1, :-1, :] + v[1, 1:, :]))
        else:
            ug = 0.0 * u[nz - 1] if zhi_noslip else u[nz - 1]
            vg = 0.0 * v[nz - 1] if zhi_noslip else v[nz - 1]
            uf = 0.25 * (u[nz - 1, :, :-1] + u[nz - 1, :, 1:] + ug[:, :-1] + ug[:, 1:])
            vf = 0.25 * (v[nz - 1, :-1, :] + v[nz - 1, 1:, :] + vg[:-1, :] + vg[1:, :])
        out.append(0.0 + mx * uf + my * vf)
    return out


def test_per_pass_terrain_composition_matches_fused_step():
    """The per-pass entries over terrain (turbulent_viscosity, slow_rhs_pre,
    fast_rhs_T, slow_rhs_post) composed by the host schedule reproduce the
    fused terrain step; the host supplies w on the ground and the lid."""
    import ctypes
    import torch
    from erf_b200 import Dycore
    from erf_b200 import terrain as T
    from erf_b200.dycore import dense_fab, ErfFab
    case = T.abl_terrain(nx=16, ny=12, nz=16, dx=25.0, dz0=20.0, h0=100.0, r0=100.0, amp=5.0)
    cfg = case.cfg
    nx, ny, nz, nc = cfg.nx, cfg.ny, cfg.nz, cfg.ncomp
    dy = Dycore(cfg)
    dy.set_terrain(case.z_nd)
    base = dy.make_base_state_terrain(case)
    dy.set_base_state(base)
    cons0, u0, v0, w0 = case.build_state(base[0])
    fused = dy.advance_host(cons0, u0, v0, w0, 1)
    assert dy.status() == 0

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    zeros = lambda *s: torch.zeros(s, dtype=torch.float64, device="cuda")
    cons = t(cons0)
    rho = cons[0]
    rx = rho + torch.roll(rho, 1, dims=2)
    ry = rho + torch.roll(rho, 1, dims=1)
    rz = rho[1:] + rho[:-1]

    def faces(a, kind):
        if kind == 0:
            return torch.cat([a, a[:, :, :1]], dim=2).contiguous()
        return torch.cat([a, a[:, :1, :]], dim=1).contiguous()

    def with_walls(wint, uu, vv):
        lo, hi = _w_walls(case.z_nd, uu.cpu().numpy(), vv.cpu().numpy(), cfg.dx, cfg.dy, cfg.zhi_bc == C.BC_NO_SLIP_WALL)
        return torch.cat([t(lo)[None], wint, t(hi)[None]], dim=0).contiguous()

    def mz_of(wf):
        m = torch.empty_like(wf)
        m[1:nz] = (wf[1:nz] * 0.5) * rz
        m[0] = (wf[0] * 0.5) * (rho[0] + rho[0])
        m[nz] = (wf[nz] * 0.5) * (rho[nz - 1] + rho[nz - 1])
        return m

    # the fused prologue: V -> M -> V -> M round trip, w from Omega = 0 on the walls
    u, v, w = t(u0), t(v0), t(w0)
    out = []
    for f, rs in ((u[:, :, :nx], rx), (v[:, :ny, :], ry), (w[1:nz], rz)):
        m0 = (f * 0.5) * rs
        out.append((m0 * 2.0) / rs)
    u1, v1 = faces(out[0], 0), faces(out[1], 1)
    w1 = with_walls(out[2], u1, v1)
    S_old = [cons.clone(), faces((out[0] * 0.5) * rx, 0), faces((out[1] * 0.5) * ry, 1), mz_of(w1)]
    vel = [u1, v1, w1]

    def fabs(S, ncons):
        arr = (ErfFab * 4)()
        arr[0] = dense_fab(S[0], 0, nx, ny, nz, ncons)
        for q, kind in ((1, 1), (2, 2), (3, 3)):
            arr[q] = dense_fab(S[q], kind, nx, ny, nz)
        return arr

    def state(ncons):
        return [zeros(ncons, nz, ny, nx), zeros(nz, ny, nx + 1), zeros(nz, ny + 1, nx), zeros(nz + 1, ny, nx)]

    L = dy.lib
    vf = lambda V: [ctypes.byref(dense_fab(V[q], q + 1, nx, ny, nz)) for q in range(3)]
    L.erf_b200_turbulent_viscosity.argtypes = [ctypes.c_void_p] * 5
    L.erf_b200_slow_rhs_pre.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 6
    L.erf_b200_fast_rhs_T.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5 + [ctypes.c_double] * 2
    L.erf_b200_fast_rhs_N.argtypes = L.erf_b200_fast_rhs_T.argtypes
    L.erf_b200_slow_rhs_post.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 5
    fc = dense_fab(cons, 0, nx, ny, nz, nc)
    wv = dense_fab(w, 3, nx, ny, nz)
    torch.cuda.synchronize()
    assert L.erf_b200_turbulent_viscosity(dy.ctx, ctypes.byref(dense_fab(u, 1, nx, ny, nz)),
                                          ctypes.byref(dense_fab(v, 2, nx, ny, nz)), ctypes.byref(wv),
                                          ctypes.byref(fc)) == 0
    stage = [a.clone() for a in S_old]
    S_rhs, S_scr = state(2), state(2)
    for nrk in range(3):
        nsub, dtau, slow_dt = schedule(cfg, nrk)
        torch.cuda.synchronize()
        assert L.erf_b200_slow_rhs_pre(dy.ctx, nrk, slow_dt, fabs(S_rhs, 2), fabs(stage, nc), fabs(S_scr, 2),
                                       *vf(vel)) == 0
        S_data = [a.clone() for a in S_old]
        for ks in range(nsub):
            prev = S_old if ks == 0 else [a.clone() for a in S_data]
            torch.cuda.synchronize()
            assert L.erf_b200_fast_rhs_T(dy.ctx, ks, nrk, fabs(S_rhs, 2), fabs(prev, nc), fabs(stage, nc),
                                         fabs(S_data, nc), fabs(S_scr, 2), dtau, 1.0 / nsub) == 0
            torch.cuda.synchronize()
        if nrk == 0:   # the flat-grid substep is refused in a terrain context
            assert L.erf_b200_fast_rhs_N(dy.ctx, 0, 0, fabs(S_rhs, 2), fabs(prev, nc), fabs(stage, nc),
                                         fabs(S_data, nc), fabs(S_scr, 2), dtau, 1.0) != 0
        S_new = state(nc)
        torch.cuda.synchronize()
        assert L.erf_b200_slow_rhs_post(dy.ctx, nrk, slow_dt, fabs(S_rhs, 2), fabs(S_old, nc), fabs(S_new, nc),
                                        fabs(S_data, nc), fabs(S_scr, 2)) == 0
        torch.cuda.synchronize()
        rho = S_data[0][0]
        rx = rho + torch.roll(rho, 1, dims=2)
        ry = rho + torch.roll(rho, 1, dims=1)
        rz = rho[1:] + rho[:-1]
        vv = []
        for q, rs in ((1, rx), (2, ry), (3, rz)):
            m = S_data[q]
            m = m[:, :, :nx] if q == 1 else (m[:, :ny, :] if q == 2 else m[1:nz])
            a1 = (m * 2.0) / rs
            m1 = (a1 * 0.5) * rs
            vv.append((m1 * 2.0) / rs)
        u2, v2 = faces(vv[0], 0), faces(vv[1], 1)
        vel = [u2, v2, with_walls(vv[2], u2, v2)]
        stage = S_new
    assert dy.status() == 0
    got = (stage[0].cpu().numpy(), vel[0].cpu().numpy(), vel[1].cpu().numpy(), vel[2].cpu().numpy())
    dy.close()
    errs = compare_states(got, fused)
    bad = {k: e for k, e in errs.items() if not e <= 1e-10}
    assert not bad, errs
