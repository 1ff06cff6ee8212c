"""Learned subgrid closure: ctypes binding of the erf_b200_mlp C-ABI.

The network (13 -> 64 -> 64 -> 64 -> 9, GELU, BF16 weights, FP32 accumulation
on the tcgen05 tensor cores) is trained and evaluated by the CUDA kernels of
erf_b200/csrc/mlp.cu; this module only moves arrays and calls them.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .dycore import load_library

NIN, NOUT = 13, 9


def _lib():
    L = load_library()
    if not getattr(L, "_mlp_bound", False):
        vp, fp, i = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int
        L.erf_b200_mlp_num_params.argtypes = []
        L.erf_b200_mlp_create.argtypes = [ctypes.POINTER(vp), vp]
        L.erf_b200_mlp_destroy.argtypes = [vp]
        L.erf_b200_mlp_set_params.argtypes = [vp, fp]
        L.erf_b200_mlp_get_params.argtypes = [vp, fp]
        L.erf_b200_mlp_set_normalization.argtypes = [vp, fp, fp, fp, fp, fp, fp]
        L.erf_b200_mlp_gradient.argtypes = [vp, fp, fp, i, fp, fp]
        L.erf_b200_mlp_train.argtypes = [vp, fp, fp, i, i, i, ctypes.c_float, fp]
        L.erf_b200_mlp_infer.argtypes = [vp, fp, i, fp]
        L._mlp_bound = True
    return L


def _fptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class MLP:
    """One network on the current CUDA device (stream: a raw cudaStream_t or None)."""

    def __init__(self, stream=None):
        self.lib = _lib()
        self.npar = self.lib.erf_b200_mlp_num_params()
        self.h = ctypes.c_void_p()
        rc = self.lib.erf_b200_mlp_create(ctypes.byref(self.h), stream)
        if rc:
            raise RuntimeError(f"erf_b200_mlp_create failed: {rc}")

    def close(self):
        if self.h:
            self.lib.erf_b200_mlp_destroy(self.h)
            self.h = ctypes.c_void_p()

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.npar
        self._check(self.lib.erf_b200_mlp_set_params(self.h, _fptr(p)))

    def get_params(self):
        p = np.zeros(self.npar, dtype=np.float32)
        self._check(self.lib.erf_b200_mlp_get_params(self.h, _fptr(p)))
        return p

    def set_normalization(self, in_mean, in_std, out_mean, out_std, in_lo=None, in_hi=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (in_mean, in_std, out_mean, out_std)]
        lo = np.ascontiguousarray(in_lo, dtype=np.float32) if in_lo is not None else None
        hi = np.ascontiguousarray(in_hi, dtype=np.float32) if in_hi is not None else None
        self._check(self.lib.erf_b200_mlp_set_normalization(
            self.h, *[_fptr(a) for a in arrs], _fptr(lo) if lo is not None else None,
            _fptr(hi) if hi is not None else None))
        self.norm = (tuple(arrs), lo, hi)

    def gradient(self, xn_dev, tn_dev, n):
        """(loss, gradient) for device tensors of normalised inputs/targets."""
        g = np.zeros(self.npar, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        self._check(self.lib.erf_b200_mlp_gradient(self.h, xn_dev.data_ptr(), tn_dev.data_ptr(), n, _fptr(g),
                                                   _fptr(loss)))
        return float(loss[0]), g

    def train(self, xn_dev, tn_dev, n, batch, iters, lr):
        loss = np.zeros(1, dtype=np.float32)
        self._check(self.lib.erf_b200_mlp_train(self.h, xn_dev.data_ptr(), tn_dev.data_ptr(), n, batch, iters,
                                                ctypes.c_float(lr), _fptr(loss)))
        return float(loss[0])

    def infer(self, x_dev, y_dev, n):
        self._check(self.lib.erf_b200_mlp_infer(self.h, x_dev.data_ptr(), n, y_dev.data_ptr()))

    @staticmethod
    def _check(rc):
        if rc:
            raise RuntimeError(f"erf_b200_mlp call failed: {rc}")


# ---------------------------------------------------------------------------
# Training data, training and evaluation of the closure
# ---------------------------------------------------------------------------
FEATURES = ("du/dx", "du/dy", "du/dz", "dv/dx", "dv/dy", "dv/dz", "dw/dx", "dw/dy", "dw/dz",
            "dT/dx", "dT/dy", "dT/dz", "Delta")
OUTPUTS = ("tau11", "tau22", "tau33", "tau12", "tau13", "tau23", "q1", "q2", "q3")


def _block_mean(a, fz, fy, fx):
    nz, ny, nx = a.shape
    return a.reshape(nz // fz, fz, ny // fy, fy, nx // fx, fx).mean(axis=(1, 3, 5))


def coarse_grain(cons, u, v, w, r):
    """Box filter of width r and coarse-graining by r of a dense fine state.

    Returns the coarse state (cons, u, v, w in the dense layout of the coarse
    grid: cells by block means, face velocities by means over the coincident
    fine faces) and the subgrid targets [Nc][9] (kinematic deviatoric stresses
    <u_i u_j> - <u_i><u_j> and heat fluxes <u_j T> - <u_j><T> of the fine
    cell-centred fields)."""
    nc, nz, ny, nx = cons.shape
    cc = np.stack([_block_mean(cons[n], r, r, r) for n in range(nc)])
    uc = _block_mean(u[:, :, ::r][:, :, :nx // r + 1], r, r, 1)
    vc = _block_mean(v[:, ::r, :][:, :ny // r + 1, :], r, 1, r)
    wc = _block_mean(w[::r, :, :][:nz // r + 1], 1, r, r)
    U = 0.5 * (u[:, :, :-1] + u[:, :, 1:])
    V = 0.5 * (v[:, :-1, :] + v[:, 1:, :])
    W = 0.5 * (w[:-1] + w[1:])
    T = cons[1] / cons[0]
    m = {nm: _block_mean(f, r, r, r) for nm, f in (("u", U), ("v", V), ("w", W), ("T", T))}

    def cov(a, b, na, nb):
        return _block_mean(a * b, r, r, r) - m[na] * m[nb]
    t11, t22, t33 = cov(U, U, "u", "u"), cov(V, V, "v", "v"), cov(W, W, "w", "w")
    tr = (t11 + t22 + t33) / 3.0
    tgt = np.stack([t11 - tr, t22 - tr, t33 - tr, cov(U, V, "u", "v"), cov(U, W, "u", "w"), cov(V, W, "v", "w"),
                    cov(U, T, "u", "T"), cov(V, T, "v", "T"), cov(W, T, "w", "T")], axis=-1)
    return (cc, uc, vc, wc), tgt.reshape(-1, 9)


def smagorinsky_prediction(feat, Cs, Pr_t):
    """The Smagorinsky stress and heat flux (kinematic) from the features, the
    same formula as the closure kernel's fallback."""
    f = feat.astype(np.float64)
    s11, s22, s33 = f[:, 0], f[:, 4], f[:, 8]
    s12, s13, s23 = 0.5 * (f[:, 1] + f[:, 3]), 0.5 * (f[:, 2] + f[:, 6]), 0.5 * (f[:, 5] + f[:, 7])
    ss = s11 ** 2 + s22 ** 2 + s33 ** 2 + 2 * (s12 ** 2 + s13 ** 2 + s23 ** 2)
    nut = (Cs * f[:, 12]) ** 2 * np.sqrt(2.0 * ss)
    tr = (s11 + s22 + s33) / 3.0
    out = np.stack([-2 * nut * (s11 - tr), -2 * nut * (s22 - tr), -2 * nut * (s33 - tr), -2 * nut * s12,
                    -2 * nut * s13, -2 * nut * s23, -nut / Pr_t * f[:, 9], -nut / Pr_t * f[:, 10],
                    -nut / Pr_t * f[:, 11]], axis=-1)
    return out


def fine_snapshots(case, spinup, nsnap, every):
    """Run the fine case in FP64 on the GPU; return nsnap dense host states."""
    from .dycore import Dycore
    dy = Dycore(case.cfg)
    base = dy.make_base_state(case)
    dy.set_base_state(base)
    st = case.build_state(base[0])
    st = dy.advance_host(*st, spinup)
    snaps = []
    for _ in range(nsnap):
        st = dy.advance_host(*st, every)
        snaps.append(st)
    if dy.status() != 0:
        raise RuntimeError("fine run reported a bad state")
    dy.close()
    return snaps, base


def coarse_case(fine_case, r):
    """The coarse-grid configuration matching a fine case.  Its seeded noise
    amplitudes are those of the fine case's noise block-averaged over r^3
    cells (the standard deviation of a mean of r^3 independent samples is
    r^-3/2 of theirs), so that a coarse run starts with the coarse-grained
    statistics the closure is trained on, not with grid-scale noise r^3/2
    times stronger."""
    import copy
    c = copy.deepcopy(fine_case)
    for key in ("noise_amp", "vel_noise_amp"):
        if key in c.pert:
            c.pert[key] = c.pert[key] * float(r) ** -1.5
    cfg = c.cfg.copy()
    cfg.nx, cfg.ny, cfg.nz = fine_case.cfg.nx // r, fine_case.cfg.ny // r, fine_case.cfg.nz // r
    cfg.dx, cfg.dy, cfg.dz = fine_case.cfg.dx * r, fine_case.cfg.dy * r, fine_case.cfg.dz * r
    cfg.dt = fine_case.cfg.dt * r
    c.cfg = cfg
    z = (np.arange(cfg.nz) + 0.5) * cfg.dz
    c.theta_cc = np.interp(z, (np.arange(fine_case.cfg.nz) + 0.5) * fine_case.cfg.dz, fine_case.theta_cc)
    c.qv_cc = np.zeros(cfg.nz)
    c.u_cc = np.interp(z, (np.arange(fine_case.cfg.nz) + 0.5) * fine_case.cfg.dz, fine_case.u_cc)
    c.v_cc = np.zeros(cfg.nz)
    return c


def build_dataset(fine_cases, r, spinup, nsnap, every):
    """Features and targets of coarse-grained snapshots of the fine cases."""
    from .dycore import Dycore
    X, Y = [], []
    for fc in fine_cases:
        snaps, _ = fine_snapshots(fc, spinup, nsnap, every)
        cc = coarse_case(fc, r)
        dyc = Dycore(cc.cfg)
        for s in snaps:
            coarse, tgt = coarse_grain(*s, r)
            X.append(dyc.closure_features(*coarse))
            Y.append(tgt.astype(np.float32))
        dyc.close()
    return X, Y


def normalization(X):
    x = np.concatenate(X)
    mean = x.mean(axis=0)
    std = x.std(axis=0)
    std = np.where(std > 1e-12 * np.maximum(np.abs(mean), 1e-30), std, 1.0)
    return mean.astype(np.float32), std.astype(np.float32), x.min(axis=0), x.max(axis=0)


def _init_params(seed):
    """He-style initial weights in the padded parameter layout, zero biases."""
    rng = np.random.default_rng(seed)
    HID, KIN, NOUTP = 64, 16, 16
    p = np.zeros(HID * KIN + 2 * HID * HID + NOUTP * HID + 3 * HID + NOUTP, dtype=np.float32)
    o = 0
    p[o:o + HID * KIN] = (rng.standard_normal((HID, KIN)) * np.sqrt(2.0 / NIN) * (np.arange(KIN) < NIN)).ravel()
    o += HID * KIN
    for _ in range(2):
        p[o:o + HID * HID] = (rng.standard_normal((HID, HID)) * np.sqrt(2.0 / HID)).ravel()
        o += HID * HID
    p[o:o + NOUTP * HID] = (rng.standard_normal((NOUTP, HID)) * np.sqrt(1.0 / HID)
                            * (np.arange(NOUTP) < NOUT)[:, None]).ravel()
    return p


def train_closure(X, Y, iters=3000, batch=8192, lr=2e-3, seed=0, stream=None):
    """Train a network on lists of feature / target arrays; returns (net, info)."""
    import torch
    xm, xs, lo, hi = normalization(X)
    y = np.concatenate(Y)
    ym, ys = y.mean(axis=0).astype(np.float32), np.maximum(y.std(axis=0), 1e-30).astype(np.float32)
    x = np.concatenate(X)
    perm = np.random.default_rng(seed).permutation(len(x))
    xn = ((x[perm] - xm) / xs).astype(np.float32)
    yn = ((y[perm] - ym) / ys).astype(np.float32)
    net = MLP(stream)
    net.set_params(_init_params(seed))
    net.set_normalization(xm, xs, ym, ys, lo, hi)
    xd, yd = torch.from_numpy(xn).cuda(), torch.from_numpy(yn).cuda()
    n = len(xn)
    l0, _ = net.gradient(xd, yd, min(n, 65536))
    torch.cuda.synchronize()
    import time
    t0 = time.perf_counter()
    last = net.train(xd, yd, n, min(batch, n), iters, lr)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    l1, _ = net.gradient(xd, yd, min(n, 65536))
    return net, {"samples": n, "iters": iters, "batch": batch, "lr": lr, "loss_initial": l0, "loss_final": l1,
                 "loss_last_batch": last, "train_seconds": t_train}


def apriori(net, X, Y, Cs, Pr_t):
    """Relative L2 error of the network and of Smagorinsky against the
    coarse-grained truth, per output and over all outputs (each output
    scaled by its standard deviation)."""
    import torch
    x = np.concatenate(X).astype(np.float32)
    y = np.concatenate(Y).astype(np.float64)
    yd = torch.zeros((len(x), 9), dtype=torch.float32, device="cuda")
    net.infer(torch.from_numpy(x).cuda(), yd, len(x))
    ym = yd.cpu().numpy().astype(np.float64)
    ys = smagorinsky_prediction(x, Cs, Pr_t)
    sd = np.maximum(y.std(axis=0), 1e-30)

    def err(p):
        per = {OUTPUTS[q]: float(np.linalg.norm(p[:, q] - y[:, q]) / max(np.linalg.norm(y[:, q]), 1e-30))
               for q in range(9)}
        tot = float(np.linalg.norm((p - y) / sd) / np.linalg.norm(y / sd))
        return tot, per
    tm, pm = err(ym)
    tsm, psm = err(ys)
    return {"mlp": tm, "smagorinsky": tsm, "mlp_per_output": pm, "smagorinsky_per_output": psm}


def aposteriori(net, fine_case, r, spinup, nsteps_coarse, precision=None):
    """Coarse runs with the learned closure and with Smagorinsky from the
    coarse-grained fine state, against the coarse-grained fine run after
    nsteps_coarse coarse steps (r fine steps each).  Returns the relative L2
    of u, v, w, theta for both closures."""
    from . import config as C
    from .dycore import Dycore
    dy = Dycore(fine_case.cfg)
    base = dy.make_base_state(fine_case)
    dy.set_base_state(base)
    st = dy.advance_host(*fine_case.build_state(base[0]), spinup)
    start, _ = coarse_grain(*st, r)
    st = dy.advance_host(*st, nsteps_coarse * r)
    truth, _ = coarse_grain(*st, r)
    dy.close()
    out = {}
    for name, les in (("mlp", C.LES_MLP), ("smagorinsky", C.LES_SMAGORINSKY)):
        cc = coarse_case(fine_case, r)
        cc.cfg.les_type = les
        if precision is not None:
            cc.cfg.precision = precision
        d = Dycore(cc.cfg)
        d.set_base_state(d.make_base_state(cc))
        if les == C.LES_MLP:
            d.set_closure(net)
        got = d.advance_host(*start, nsteps_coarse)
        res = {"status": d.status()}
        if les == C.LES_MLP:
            res["fallback_cells"] = d.closure_fallbacks()
        d.close()
        for nm, a, b in (("u", got[1], truth[1]), ("v", got[2], truth[2]), ("w", got[3], truth[3]),
                         ("theta", got[0][1] / got[0][0], truth[0][1] / truth[0][0])):
            ref = b - (b.mean() if nm == "theta" else 0.0)
            res[nm] = float(np.linalg.norm(a - b) / max(np.linalg.norm(ref), 1e-30))
        out[name] = res
    return out


def save_closure(path, net, info=None):
    """Parameters, normalisation and envelope of a trained network (npz)."""
    (xm, xs, ym, ys), lo, hi = net.norm
    np.savez(path, params=net.get_params(), in_mean=xm, in_std=xs, out_mean=ym, out_std=ys, in_lo=lo, in_hi=hi,
             info=np.array(json_dumps(info or {})))


def load_closure(path, stream=None):
    """A network on the current device from a save_closure file."""
    d = np.load(path)
    net = MLP(stream)
    net.set_params(d["params"])
    net.set_normalization(d["in_mean"], d["in_std"], d["out_mean"], d["out_std"], d["in_lo"], d["in_hi"])
    return net


def json_dumps(obj):
    import json
    return json.dumps(obj, default=float)


def main(argv=None):
    """Train the closure on coarse-grained fine-grid ABL runs and evaluate it.

        python -m erf_b200.closure [--fine NX NY NZ] [--factor R] [--out model.npz] [--report report.json]

    Fine runs: the abl_fine case (abl_dry physics, dx = dz = 10 m) at five
    seeds and geostrophic winds 5, 7.5, 10, 12.5, 15 m/s; the last one is held
    out for the a-priori and a-posteriori evaluation."""
    import argparse
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--fine", type=int, nargs=3, default=[512, 512, 128])
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--spinup", type=int, default=400)
    ap.add_argument("--snapshots", type=int, default=4)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--iters", type=int, default=4000)
    ap.add_argument("--post-steps", type=int, default=25)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    from . import cases
    nx, ny, nz = a.fine
    winds = (5.0, 7.5, 10.0, 12.5, 15.0)
    fine = [cases.abl_fine(nx=nx, ny=ny, nz=nz, u_g=ug, seed=s) for s, ug in enumerate(winds)]
    t0 = time.perf_counter()
    X, Y = build_dataset(fine[:4], a.factor, a.spinup, a.snapshots, a.every)
    Xh, Yh = build_dataset(fine[4:], a.factor, a.spinup, a.snapshots, a.every)
    t_data = time.perf_counter() - t0
    net, info = train_closure(X, Y, iters=a.iters)
    pri = apriori(net, Xh, Yh, fine[0].cfg.Cs, fine[0].cfg.Pr_t)
    from . import config as C
    post = aposteriori(net, fine[4], a.factor, a.spinup, a.post_steps)
    post_mixed = aposteriori(net, fine[4], a.factor, a.spinup, a.post_steps, precision=C.PREC_MIXED)
    report = {"fine_grid": [nx, ny, nz], "dx_fine": fine[0].cfg.dx, "factor": a.factor,
              "coarse_grid": [nx // a.factor, ny // a.factor, nz // a.factor], "winds": winds, "held_out": winds[4],
              "spinup_steps": a.spinup, "snapshots": a.snapshots, "every": a.every, "data_seconds": t_data,
              "training": info, "apriori": pri, "aposteriori_fp64": post, "aposteriori_mixed": post_mixed}
    print(json_dumps(report))
    if a.out:
        save_closure(a.out, net, info)
    if a.report:
        with open(a.report, "w") as fh:
            fh.write(json_dumps(report))
    net.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
