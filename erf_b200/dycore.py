"""Python host binding of the C-ABI (include/erf_b200.h) through ctypes.

The product path is liberf_b200.so; there is no CPU fallback: constructing a
Dycore without the built library or without a CUDA device raises.  Device
memory for the Python-level entry points comes from torch tensors (plumbing
only); all arithmetic runs in the library's kernels.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import config as C

_HERE = os.path.dirname(os.path.abspath(__file__))
# ERF_B200_LIB selects another build of the library for this process (the
# bounds-checked liberf_b200_bounds.so); the default is the in-tree build
LIB_PATH = os.environ.get("ERF_B200_LIB", os.path.join(_HERE, "liberf_b200.so"))
_lib = None

ERRORS = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "EBADSTATE", 5: "ENAN", 6: "EPIVOT",
          7: "ETIMEOUT", 8: "ECONFIG", 9: "EABORTED", 10: "EBOUNDS"}
EABORTED = 9

EXPORTS = [
    "erf_b200_config_defaults", "erf_b200_create", "erf_b200_destroy", "erf_b200_set_stream",
    "erf_b200_get_status", "erf_b200_scratch_bytes", "erf_b200_make_base_state", "erf_b200_set_base_state",
    "erf_b200_advance", "erf_b200_advance_host", "erf_b200_turbulent_viscosity", "erf_b200_slow_rhs_pre",
    "erf_b200_make_fast_coeffs", "erf_b200_fast_rhs_N", "erf_b200_slow_rhs_post", "erf_b200_kessler_advance",
    "erf_b200_advance_profiled", "erf_b200_kernels_per_step", "erf_b200_kessler_advance_noalloc",
    "erf_b200_mlp_num_params", "erf_b200_mlp_create", "erf_b200_mlp_destroy", "erf_b200_mlp_set_params",
    "erf_b200_mlp_get_params", "erf_b200_mlp_set_normalization", "erf_b200_mlp_gradient", "erf_b200_mlp_train",
    "erf_b200_mlp_infer", "erf_b200_set_closure", "erf_b200_closure_fallbacks", "erf_b200_closure_features_host",
    "erf_b200_load_state", "erf_b200_store_state", "erf_b200_advance_resident", "erf_b200_autotune",
    "erf_b200_ensemble_create", "erf_b200_ensemble_advance", "erf_b200_ensemble_sync", "erf_b200_ensemble_destroy",
    "erf_b200_last_cuda_error", "erf_b200_set_terrain", "erf_b200_make_base_state_terrain",
    "erf_b200_fast_rhs_T", "erf_b200_write_plotfile", "erf_b200_write_checkpoint", "erf_b200_read_checkpoint",
    "erf_b200_selftest_bounded_wait", "erf_b200_no_substep", "erf_b200_most_update_fluxes",
    "erf_b200_ensemble_abort", "erf_b200_ensemble_steps", "erf_b200_set_time", "erf_b200_moving_terrain_state",
    "erf_b200_diagnostics",
]
KERNEL_SLOTS = ["step_begin", "stress", "slow_cell", "plane_avg", "slow_mom", "fast_horizontal", "fast_column",
                "slow_post", "kessler", "fast_coeffs", "no_substep"]


class ErfFab(ctypes.Structure):
    _fields_ = [("p", ctypes.c_void_p), ("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3),
                ("jstride", ctypes.c_int64), ("kstride", ctypes.c_int64), ("nstride", ctypes.c_int64),
                ("ncomp", ctypes.c_int)]


class ErfError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed: {ERRORS.get(code, code)}")
        self.code = code


def load_library():
    """Load liberf_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m erf_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, i = ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int
    L.erf_b200_config_defaults.argtypes = [vp]
    L.erf_b200_create.argtypes = [ctypes.POINTER(vp), vp, vp]
    L.erf_b200_destroy.argtypes = [vp]
    L.erf_b200_set_stream.argtypes = [vp, vp]
    L.erf_b200_get_status.argtypes = [vp]
    L.erf_b200_scratch_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    L.erf_b200_make_base_state.argtypes = [vp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           dp, dp, dp, dp]
    L.erf_b200_set_base_state.argtypes = [vp, dp, dp, dp, dp]
    L.erf_b200_set_terrain.argtypes = [vp, dp]
    L.erf_b200_set_time.argtypes = [vp, ctypes.c_double]
    L.erf_b200_moving_terrain_state.argtypes = [vp, dp, dp, dp, dp]
    L.erf_b200_diagnostics.argtypes = [vp, dp]
    L.erf_b200_make_base_state_terrain.argtypes = [vp, dp, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                   dp, dp, dp, dp]
    fabp = ctypes.POINTER(ErfFab)
    L.erf_b200_advance.argtypes = [vp, fabp, fabp, fabp, fabp, i]
    L.erf_b200_advance_host.argtypes = [vp, dp, dp, dp, dp, i]
    L.erf_b200_kessler_advance.argtypes = [vp, fabp, ctypes.c_double]
    L.erf_b200_advance_profiled.argtypes = [vp, fabp, fabp, fabp, fabp, i, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_int), i]
    L.erf_b200_kernels_per_step.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.erf_b200_kessler_advance_noalloc.argtypes = [vp, fabp, ctypes.c_double, vp]
    L.erf_b200_set_closure.argtypes = [vp, vp]
    L.erf_b200_closure_fallbacks.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    L.erf_b200_closure_features_host.argtypes = [vp, dp, dp, dp, dp, dp]
    L.erf_b200_load_state.argtypes = [vp, fabp, fabp, fabp, fabp]
    L.erf_b200_store_state.argtypes = [vp, fabp, fabp, fabp, fabp]
    L.erf_b200_advance_resident.argtypes = [vp, i]
    L.erf_b200_autotune.argtypes = [vp, i, ctypes.POINTER(ctypes.c_double)]
    L.erf_b200_ensemble_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), i, vp]
    L.erf_b200_ensemble_advance.argtypes = [vp, i]
    L.erf_b200_ensemble_sync.argtypes = [vp]
    L.erf_b200_ensemble_abort.argtypes = [vp, i]
    L.erf_b200_ensemble_steps.argtypes = [vp, ctypes.POINTER(i)]
    L.erf_b200_ensemble_destroy.argtypes = [vp]
    L.erf_b200_selftest_bounded_wait.argtypes = [i, ctypes.POINTER(i)]
    L.erf_b200_write_plotfile.argtypes = [vp, ctypes.c_char_p, dp, dp, dp, dp, dp, dp, dp, ctypes.c_double, i]
    L.erf_b200_write_checkpoint.argtypes = [vp, ctypes.c_char_p] + [dp] * 9 + [i, ctypes.c_double, ctypes.c_double]
    L.erf_b200_read_checkpoint.argtypes = [vp, ctypes.c_char_p] + [dp] * 9 + [ctypes.POINTER(i),
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    for name in EXPORTS:
        getattr(L, name).restype = ctypes.c_int
    L.erf_b200_last_cuda_error.argtypes = []
    L.erf_b200_last_cuda_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(rc: int, what: str):
    if rc != 0:
        if rc in (2, 3) and _lib is not None:   # ECUDA / ENOMEM: name the CUDA error
            what = f"{what} ({_lib.erf_b200_last_cuda_error().decode()})"
        raise ErfError(rc, what)


def dense_fab(t, kind: int, nx: int, ny: int, nz: int, ncomp: int = 1) -> ErfFab:
    """Array4 view of a dense contiguous device tensor (valid region only)."""
    hx = nx - 1 + (kind == 1)
    hy = ny - 1 + (kind == 2)
    hz = nz - 1 + (kind == 3)
    f = ErfFab()
    f.p = t.data_ptr()
    f.lo[0] = f.lo[1] = f.lo[2] = 0
    f.hi[0], f.hi[1], f.hi[2] = hx, hy, hz
    f.jstride = hx + 1
    f.kstride = (hx + 1) * (hy + 1)
    f.nstride = f.kstride * (hz + 1)
    f.ncomp = ncomp
    return f


class Ensemble:
    """Contexts with resident states advanced together: a device-side loop
    over steps inside one graph launch, stoppable through an abort word."""

    def __init__(self, members, stream=None):
        self.lib = load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.ctx.value for m in self.members])
        self.h = ctypes.c_void_p()
        _check(self.lib.erf_b200_ensemble_create(ctypes.byref(self.h), arr, len(self.members), stream),
               "ensemble_create")

    def advance(self, nsteps: int):
        _check(self.lib.erf_b200_ensemble_advance(self.h, int(nsteps)), "ensemble_advance")

    def sync(self) -> bool:
        """Wait for the ensemble's work; False when an abort stopped it."""
        rc = self.lib.erf_b200_ensemble_sync(self.h)
        if rc == EABORTED:
            return False
        _check(rc, "ensemble_sync")
        return True

    def abort(self, flag: bool = True):
        _check(self.lib.erf_b200_ensemble_abort(self.h, 1 if flag else 0), "ensemble_abort")

    def steps(self) -> int:
        n = ctypes.c_int()
        _check(self.lib.erf_b200_ensemble_steps(self.h, ctypes.byref(n)), "ensemble_steps")
        return n.value

    def close(self):
        if self.h:
            self.lib.erf_b200_ensemble_destroy(self.h)
            self.h = ctypes.c_void_p()


class Dycore:
    """One dycore context on the current CUDA device.

    The context runs on `stream` (a cudaStream_t handle), by default torch's
    current stream.  When that is the legacy default stream (handle 0) the
    library creates a non-blocking stream of its own, which does not order
    after torch's work: synchronise (torch.cuda.synchronize) between torch
    operations on tensors and library calls that read or write them.
    advance_host and the make_base_state* methods return synchronised host
    results."""

    def __init__(self, cfg: C.ErfConfig, stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("erf_b200 needs a CUDA device")
        self.lib = load_library()
        self.cfg = cfg.copy()
        self._ctx = ctypes.c_void_p()
        s = ctypes.c_void_p(stream) if stream is not None else ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _check(self.lib.erf_b200_create(ctypes.byref(self._ctx), ctypes.byref(self.cfg), s), "erf_b200_create")
        self.base = None

    def close(self):
        if self._ctx:
            self.lib.erf_b200_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ctx(self):
        return self._ctx

    def status(self) -> int:
        return self.lib.erf_b200_get_status(self._ctx)

    def scratch_bytes(self) -> int:
        n = ctypes.c_size_t()
        _check(self.lib.erf_b200_scratch_bytes(self._ctx, ctypes.byref(n)), "scratch_bytes")
        return n.value

    def make_base_state(self, case):
        """FP64 hydrostatic base state computed on the GPU; returns 4 numpy arrays (nz+2)."""
        import torch
        nz = self.cfg.nz
        th = torch.tensor(np.asarray(case.theta_cc, dtype=np.float64), device="cuda")
        qv = torch.tensor(np.asarray(case.qv_cc, dtype=np.float64), device="cuda")
        out = [torch.zeros(nz + 2, dtype=torch.float64, device="cuda") for _ in range(4)]
        torch.cuda.synchronize()
        _check(self.lib.erf_b200_make_base_state(self._ctx, th.data_ptr(), qv.data_ptr(), case.theta_sfc,
                                                 case.qv_sfc, case.p_sfc, *[o.data_ptr() for o in out]),
               "make_base_state")
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in out]

    def set_terrain(self, z_nd):
        """Install z_phys_nd ([nz+1][ny+1][nx+1] node heights, periodic)."""
        z = np.ascontiguousarray(z_nd, dtype=np.float64)
        cfg = self.cfg
        assert z.shape == (cfg.nz + 1, cfg.ny + 1, cfg.nx + 1)
        _check(self.lib.erf_b200_set_terrain(self._ctx, z.ctypes.data), "set_terrain")

    def diagnostics(self) -> dict:
        """Mass and rho-theta integrals (dx dy dz detJ per cell) and max |w|
        of the latest state (a device reduction; synchronises)."""
        out = np.zeros(3)
        _check(self.lib.erf_b200_diagnostics(self._ctx, out.ctypes.data), "diagnostics")
        return {"mass": float(out[0]), "rhotheta": float(out[1]), "max_w": float(out[2])}

    def set_time(self, t: float):
        """Moving terrain: the device clock (the old time of the next step)."""
        _check(self.lib.erf_b200_set_time(self._ctx, float(t)), "set_time")

    def moving_terrain_state(self):
        """Moving terrain: (time, z_nd [nz+1][ny+1][nx+1], rho0, p0 ((nz+2)*ny*nx))."""
        cfg = self.cfg
        t = np.zeros(1)
        z = np.zeros((cfg.nz + 1, cfg.ny + 1, cfg.nx + 1))
        r0 = np.zeros((cfg.nz + 2) * cfg.ny * cfg.nx)
        p0 = np.zeros((cfg.nz + 2) * cfg.ny * cfg.nx)
        _check(self.lib.erf_b200_moving_terrain_state(self._ctx, t.ctypes.data, z.ctypes.data, r0.ctypes.data,
                                                      p0.ctypes.data), "moving_terrain_state")
        return float(t[0]), z, r0, p0

    def make_base_state_terrain(self, case):
        """Base state over the terrain on the GPU: 4 arrays of (nz+2)*ny*nx."""
        import torch
        cfg = self.cfg
        th = torch.tensor(np.ascontiguousarray(case.theta3, dtype=np.float64), device="cuda")
        qv = torch.tensor(np.ascontiguousarray(case.qv3, dtype=np.float64), device="cuda")
        n = (cfg.nz + 2) * cfg.ny * cfg.nx
        out = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
        torch.cuda.synchronize()
        _check(self.lib.erf_b200_make_base_state_terrain(self._ctx, th.data_ptr(), qv.data_ptr(), case.theta_sfc,
                                                         case.qv_sfc, case.p_sfc, *[o.data_ptr() for o in out]),
               "make_base_state_terrain")
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in out]

    def set_base_state(self, base):
        import torch
        self._base_dev = [torch.tensor(np.asarray(b, dtype=np.float64), device="cuda") for b in base]
        torch.cuda.synchronize()
        _check(self.lib.erf_b200_set_base_state(self._ctx, *[b.data_ptr() for b in self._base_dev]),
               "set_base_state")
        _check(self.lib.erf_b200_get_status(self._ctx), "set_base_state sync")
        self.base = base

    def advance_host(self, cons, u, v, w, nsteps: int):
        """Advance dense host arrays; returns new arrays (host buffers in, host buffers out)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in (cons, u, v, w)]
        _check(self.lib.erf_b200_advance_host(self._ctx, *[a.ctypes.data for a in arrs], int(nsteps)),
               "advance_host")
        return tuple(arrs)

    def write_plotfile(self, path: str, cons, u, v, w, z_nd=None, time: float = 0.0, step: int = 0):
        """AMReX plotfile of a host state of this context's grid (base state
        from set_base_state for pres_hse / dens_hse)."""
        from .plotfile import write_plotfile
        write_plotfile(self.cfg, path, cons, u, v, w, base=self.base, z_nd=z_nd, time=time, step=step)

    def write_checkpoint(self, path: str, cons, u, v, w, z_nd=None, step: int = 0, time: float = 0.0):
        """ERF-layout checkpoint of a host state with this context's base state."""
        from .checkpoint import write_checkpoint
        if self.base is None:
            raise RuntimeError("write_checkpoint needs the base state (set_base_state)")
        write_checkpoint(self.cfg, path, cons, u, v, w, self.base, z_nd=z_nd, step=step, dt=self.cfg.dt, time=time)

    def advance(self, cons_t, u_t, v_t, w_t, nsteps: int):
        """Advance dense device tensors in place (asynchronous on the context stream)."""
        c = self.cfg
        fc = dense_fab(cons_t, 0, c.nx, c.ny, c.nz, c.ncomp)
        fu = dense_fab(u_t, 1, c.nx, c.ny, c.nz)
        fv = dense_fab(v_t, 2, c.nx, c.ny, c.nz)
        fw = dense_fab(w_t, 3, c.nx, c.ny, c.nz)
        _check(self.lib.erf_b200_advance(self._ctx, ctypes.byref(fc), ctypes.byref(fu), ctypes.byref(fv),
                                         ctypes.byref(fw), int(nsteps)), "advance")

    def set_closure(self, net):
        """Attach a trained erf_b200.closure.MLP (les_type MLP contexts)."""
        _check(self.lib.erf_b200_set_closure(self._ctx, net.h), "set_closure")
        self._net = net

    def closure_fallbacks(self) -> int:
        n = ctypes.c_ulonglong()
        _check(self.lib.erf_b200_closure_fallbacks(self._ctx, ctypes.byref(n)), "closure_fallbacks")
        return n.value

    def closure_features(self, cons, u, v, w):
        """The 13 closure features of every cell of a dense host state: [nz*ny*nx][13] float32."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (cons, u, v, w)]
        c = self.cfg
        out = np.zeros((c.nx * c.ny * c.nz, 13), dtype=np.float32)
        _check(self.lib.erf_b200_closure_features_host(self._ctx, *[a.ctypes.data for a in arrs], out.ctypes.data),
               "closure_features")
        return out

    def load_state(self, cons, u, v, w):
        """Make a dense host state resident on the device (graph steps then
        advance it in place: advance_resident, Ensemble)."""
        import torch
        self._res = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda() for a in (cons, u, v, w)]
        torch.cuda.synchronize()
        c = self.cfg
        f = [dense_fab(self._res[0], 0, c.nx, c.ny, c.nz, c.ncomp)] + \
            [dense_fab(self._res[q], q, c.nx, c.ny, c.nz) for q in (1, 2, 3)]
        _check(self.lib.erf_b200_load_state(self._ctx, *[ctypes.byref(x) for x in f]), "load_state")
        _check(self.lib.erf_b200_get_status(self._ctx), "load_state sync")

    def store_state(self, cons, u, v, w):
        """Copy the resident state into new dense host arrays shaped like the given ones."""
        import torch
        out = [torch.zeros(np.shape(a), dtype=torch.float64, device="cuda") for a in (cons, u, v, w)]
        torch.cuda.synchronize()
        c = self.cfg
        f = [dense_fab(out[0], 0, c.nx, c.ny, c.nz, c.ncomp)] + [dense_fab(out[q], q, c.nx, c.ny, c.nz) for q in (1, 2, 3)]
        _check(self.lib.erf_b200_store_state(self._ctx, *[ctypes.byref(x) for x in f]), "store_state")
        _check(self.lib.erf_b200_get_status(self._ctx), "store_state sync")
        return tuple(t.cpu().numpy() for t in out)

    def advance_resident(self, nsteps: int):
        _check(self.lib.erf_b200_advance_resident(self._ctx, int(nsteps)), "advance_resident")

    def autotune(self, reps: int = 3) -> float:
        """Tune the launch shapes on the resident state; returns the tuned step time (ms)."""
        ms = ctypes.c_double()
        _check(self.lib.erf_b200_autotune(self._ctx, int(reps), ctypes.byref(ms)), "autotune")
        return ms.value

    def kernels_per_step(self) -> int:
        n = ctypes.c_int()
        _check(self.lib.erf_b200_kernels_per_step(self._ctx, ctypes.byref(n)), "kernels_per_step")
        return n.value

    def advance_profiled(self, cons_t, u_t, v_t, w_t, nsteps: int):
        """Eager (graph-less) advance with CUDA events around every kernel.

        Returns {slot name: (total_ms, launches)}."""
        c = self.cfg
        fc = dense_fab(cons_t, 0, c.nx, c.ny, c.nz, c.ncomp)
        fu = dense_fab(u_t, 1, c.nx, c.ny, c.nz)
        fv = dense_fab(v_t, 2, c.nx, c.ny, c.nz)
        fw = dense_fab(w_t, 3, c.nx, c.ny, c.nz)
        n = len(KERNEL_SLOTS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int * n)()
        _check(self.lib.erf_b200_advance_profiled(self._ctx, ctypes.byref(fc), ctypes.byref(fu), ctypes.byref(fv),
                                                  ctypes.byref(fw), int(nsteps), ms, cnt, n), "advance_profiled")
        return {KERNEL_SLOTS[q]: (ms[q], cnt[q]) for q in range(n)}
