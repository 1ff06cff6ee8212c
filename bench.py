#!/usr/bin/env python
"""Benchmark of the multirate RK3 dycore step: cell-RK3-steps/s on B200.

Workload (default): the moist warm-bubble case, 128 x 128 x 80 cells,
Kessler microphysics, Upwind_5th dycore, WENO5 scalars, buoyancy type 2,
dt = 2 s with 6 acoustic substeps per RK3 stage 3 (10 substeps per step),
plain FP64 arithmetic.  A "step" is one full RK3 step of the whole domain
including all acoustic substeps and the Kessler pass.  Inputs are synthetic
and seeded (erf_b200/cases.py); the device working set (~0.9 GB) is larger
than the 126 MB L2, so no L2 flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

One JSON line is printed by rank 0.  Under torchrun each rank advances its
own replica of the workload (the path does not shard: replicas only) and the
time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from erf_b200 import cases  # noqa: E402

METRIC = "cell-RK3-steps/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


# ---------------------------------------------------------------------------
# Algorithmic traffic per cell for each kernel slot: every array the pass must
# read or write, counted once, as (FP64 values, bulk values).  Bulk values are
# 8 bytes in the plain form and 4 bytes in the mixed form; the prognostic
# state, velocities and base state are FP64 in both.
# ---------------------------------------------------------------------------
def algorithmic_values_per_cell(cfg):
    moist = cfg.moisture != 0
    m2 = 2 if moist else 0
    nq = cfg.ncomp - 5
    diff = cfg.les_type != 0 or cfg.molec_diff_type != 0
    les = 1 if cfg.les_type == 1 else 0
    d = 1 if diff else 0
    return {
        # reads cons(ncomp) + u,v,w; writes 3 momenta, 3 velocities | prim (ncomp-1), pi, p', (mu_t)
        "step_begin": (cfg.ncomp + 3 + 3 + 3, (cfg.ncomp - 1) + 2 + les),
        # reads u,v,w, rho | mu_t; writes 6 stresses
        "stress": (4, d + 6),
        # reads 3 momenta, (rho) | theta, (mu_t); writes rhs rho, rho-theta, 3 avg momenta
        "slow_cell": (3 + d, 1 + d + 2 + 3),
        # reads rho | theta, (qv, qc, qp)
        "plane_avg": (1, 4 if moist else 1),
        # reads 3 momenta, 3 velocities, rho | p', (qv, qc), (6 stresses); writes 3 rhs
        "slow_mom": (7, 1 + m2 + 6 * d + 3),
        # reads prev 2 mom, rho-theta, rho; stage 2 mom, rho-theta; writes new 2 mom |
        # reads 2 rhs, lag, pi, (qv, qc), avg 2; writes avg 2, lag
        "fast_horizontal": (9, 9 + m2),
        # reads prev rho, rho-theta, w-mom; stage rho, rho-theta, 3 mom; new 2 mom; writes rho,
        # rho-theta, w-mom | theta, 5 coefficients, rhs rho, rho-theta, w; avg w read+write
        "fast_column": (13, 11),
        # reads old scalars (1+nq), sum rho, rho-theta, 3 mom; writes ncomp, 3 mom, 3 vel |
        # reads scalar prims (1+nq), 3 avg mom; writes next prim (ncomp-1), pi, p'
        "slow_post": ((1 + nq) + 5 + cfg.ncomp + 6, (1 + nq) + 3 + (cfg.ncomp - 1) + 2),
        # reads rho, rho-theta, 3 moisture; writes all ncomp (into the other buffer)
        "kessler": ((5 + cfg.ncomp) if moist else 0, 0),
        # reads stage rho-theta | theta, pi, (qv, qc); writes A, 1/B', C/B', P, Q
        "fast_coeffs": (1, 1 + 1 + m2 + 5),
    }


def survey_bytes_per_cell_step(cfg, substeps):
    """The pass model of the benchmark's byte budget: each value counted once
    per forced pass at 8 bytes.  Per cell per step: slow-pre 3 x (5 read +
    5 write); each acoustic substep prev 5 + stage 5 + rhs 5 + new 5 + average
    momenta 3 read + 3 write; slow-post 3 x (3 + 3 S) with S slow scalars
    (the passive scalar, rho*KE with Deardorff, the moisture species);
    closure 7 values (Smagorinsky) or 9 (Deardorff); Kessler 9; terrain adds
    4 values to each slow-pre and substep pass.  Dry ABL 64^3: 315 values
    (2520 B); moist bubble: 344 (2752 B); terrain ABL: 378 (3024 B)."""
    nq = cfg.ncomp - 5
    S = 1 + (1 if cfg.les_type == 2 else 0) + nq
    vals = 3 * 10 + substeps * 26 + 3 * (3 + 3 * S)
    vals += {0: 0, 1: 7, 2: 9}.get(cfg.les_type, 7)
    vals += 9 if cfg.moisture != 0 else 0
    vals += 4 * (3 + substeps) if cfg.use_terrain else 0
    return 8 * vals


def substeps_per_step(cfg):
    """Acoustic substeps per RK3 step (ERF_MRI.H:255-282): R/3 (or 1 with
    force_stage1_single_substep), R/2 and R; none without substepping."""
    if getattr(cfg, "substepping_type", 0) == 1:
        return 0
    r = cfg.mri_ratio
    return (1 if cfg.force_stage1_single_substep else r // 3) + r // 2 + r


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def bytes_per_cell(vals, bulk_bytes):
    return {k: 8 * a + bulk_bytes * b for k, (a, b) in vals.items()}


def sample_clocks(stop, out):
    cmd = ["nvidia-smi", "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        p = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except Exception:
        return
    dev = os.environ.get("LOCAL_RANK", "0")
    try:
        while not stop.is_set():
            line = p.stdout.readline()
            if not line:
                break
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9 and f[0] == dev:
                out.append(f)
    finally:
        p.terminate()
        try:
            p.wait(timeout=2)
        except Exception:
            p.kill()


def summarize_clocks(samples):
    if not samples:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
    mx = [float(s[2]) for s in samples if s[2].replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = []
    for q, nm in enumerate(names):
        if any(s[5 + q].lower().startswith("active") for s in samples):
            reasons.append(nm)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": reasons, "samples": len(samples)}


def max_over_ranks(x, world, device):
    """Max of a per-rank scalar over all ranks (the timing rule for replicas)."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return x


def replica_throughput(world, n_cells, steps, seconds):
    """Whole-job cell-steps/s: every rank advances its own full replica."""
    return world * n_cells * steps / seconds


CLOSURE_MODEL = os.path.join(ROOT, "erf_b200", "data", "closure_abl.npz")


def learned_arm(measure, form_error, C):
    """The learned closure on the coarse ABL grid it was trained for
    (128 x 128 x 32, dx = dz = 40 m): plain FP64 with Smagorinsky, FP64 with
    the network, and the mixed form with the network; the mixed form's error
    is taken against FP64 with the same network after 100 steps."""
    if not os.path.exists(CLOSURE_MODEL):
        return {"unavailable": "no trained closure model (python -m erf_b200.closure --out ...)"}
    from erf_b200.closure import coarse_case, load_closure
    net = load_closure(CLOSURE_MODEL)
    mk = lambda: coarse_case(cases.abl_fine(nx=512, ny=512, nz=128), 4)
    smag, _, _ = measure(C.PREC_FP64, None, case=mk(), les=C.LES_SMAGORINSKY, light=True)
    l64, base, init = measure(C.PREC_FP64, None, case=mk(), net=net, les=C.LES_MLP, light=True)
    l32, _, _ = measure(C.PREC_MIXED, None, case=mk(), net=net, les=C.LES_MLP, light=True)
    ce = mk()
    ce.cfg.les_type = C.LES_MLP
    err = form_error(base, init, 100, case=ce, net=net)
    # the same mixed-vs-FP64 comparison with Smagorinsky: the share of the
    # error that the flow's sensitivity to FP32 rounding gives by itself
    cs = mk()
    cs.cfg.les_type = C.LES_SMAGORINSKY
    err_smag = form_error(base, init, 100, case=cs)
    net.close()
    return {"workload": "abl coarse 128x128x32, dx=dz=40 m, dt=0.32 s, learned closure (tcgen05 BF16 MLP)",
            "fp64_smagorinsky": smag, "fp64_learned": l64, "mixed_learned": l32,
            "speedup_mixed_learned_vs_fp64_smagorinsky": l32["value"] / smag["value"],
            "rel_l2_mixed_vs_fp64_learned_after_100_steps": err,
            "rel_l2_mixed_vs_fp64_smagorinsky_after_100_steps": err_smag}


def ensemble_members(n=32, seed=100):
    """Member sizes (64^3 up to 192 x 192 x 96, multiples of 32 / 16) and
    geostrophic winds (4-16 m/s), seeded."""
    import numpy as _np
    rng = _np.random.default_rng(seed)
    out = []
    for q in range(n):
        nx = int(rng.integers(2, 7)) * 32
        ny = int(rng.integers(2, 7)) * 32
        nz = int(rng.integers(4, 7)) * 16
        out.append((nx, ny, nz, float(rng.uniform(4.0, 16.0)), seed + q))
    return out


def ensemble_arm(args, C, Dycore, Ensemble, stream, n_err=32):
    """32 ABL members of uneven sizes at dx = dz = 40 m (the learned closure's
    grid spacing), mixed form with the learned closure, each member
    autotuned, advanced together for args.ens_steps steps in one graph
    launch (a device-side loop over pairs of steps); each member's error
    against the plain FP64 form (same closure) after the run."""
    import torch
    if not os.path.exists(CLOSURE_MODEL):
        return {"unavailable": "no trained closure model"}
    from erf_b200.closure import coarse_case, load_closure
    net = load_closure(CLOSURE_MODEL)
    specs = ensemble_members()

    def member_case(nx, ny, nz, ug, seed, precision):
        # the coarse (dx = dz = 40 m) counterpart of a fine training run, with
        # the fine case's noise at coarse-grained amplitude
        case = coarse_case(cases.abl_fine(nx=4 * nx, ny=4 * ny, nz=4 * nz, u_g=ug, seed=seed), 4)
        case.cfg.precision = precision
        case.cfg.les_type = C.LES_MLP
        return case

    def make(spec, precision):
        case = member_case(*spec, precision)
        dy = Dycore(case.cfg, stream=stream.cuda_stream)
        base = dy.make_base_state(case)
        dy.set_base_state(base)
        dy.set_closure(net)
        st = case.build_state(base[0])
        dy.load_state(*st)
        return dy, st

    members = [make(sp, C.PREC_MIXED) for sp in specs]
    tuned = [dy.autotune(2) for dy, _ in members]
    for dy, _ in members:
        dy.closure_fallbacks()   # reset: count only the warm-up and timed steps
    cells = sum(sp[0] * sp[1] * sp[2] for sp in specs)
    ens = Ensemble([dy for dy, _ in members], stream=stream.cuda_stream)
    nsteps_t = args.ens_steps
    ens.advance(args.warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.advance(nsteps_t)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    finished = ens.sync()
    steps_run = ens.steps()
    status = [dy.status() for dy, _ in members]
    # fraction of closure evaluations (one per cell per RK stage) that took the
    # Smagorinsky fallback
    fb_frac = sum(dy.closure_fallbacks() for dy, _ in members) / (3.0 * cells * (args.warmup + nsteps_t))
    # per-member error of the mixed form against FP64 (same closure) after
    # warmup + ens_steps steps
    errs = []
    nsteps = args.warmup + nsteps_t

    def rl2(a, b):
        return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
    for q in range(n_err):
        dy, st = members[q]
        got = dy.store_state(*st)
        ref_dy, _ = make(specs[q], C.PREC_FP64)
        ref_dy.advance_resident(nsteps)
        ref = ref_dy.store_state(*st)
        ref_dy.close()
        errs.append({"size": specs[q][:3], "u": rl2(got[1], ref[1]), "v": rl2(got[2], ref[2]), "w": rl2(got[3], ref[3]),
                     "theta": rl2(got[0][1] / got[0][0], ref[0][1] / ref[0][0])})
    ens.close()
    for dy, _ in members:
        dy.close()
    net.close()
    worst = {f: max(e[f] for e in errs) for f in ("u", "v", "w", "theta")} if errs else {}
    # the same comparison with the Smagorinsky closure for the first members:
    # if these also decorrelate, the learned run's v / w error is the flow's
    # sensitivity to FP32 rounding, not the network's
    smag_errs = []
    for q in range(2):
        outs = {}
        for prec in (C.PREC_FP64, C.PREC_MIXED):
            case = member_case(*specs[q], prec)
            case.cfg.les_type = C.LES_SMAGORINSKY
            dy = Dycore(case.cfg, stream=stream.cuda_stream)
            base = dy.make_base_state(case)
            dy.set_base_state(base)
            st = case.build_state(base[0])
            dy.load_state(*st)
            dy.advance_resident(nsteps)
            outs[prec] = dy.store_state(*st)
            dy.close()
        got, ref = outs[C.PREC_MIXED], outs[C.PREC_FP64]
        smag_errs.append({"size": specs[q][:3], "u": rl2(got[1], ref[1]), "v": rl2(got[2], ref[2]),
                          "w": rl2(got[3], ref[3]), "theta": rl2(got[0][1] / got[0][0], ref[0][1] / ref[0][0])})
    return {"workload": f"{len(specs)} ABL members 64^3..192x192x96 (seeded), dx=dz=40 m, u_g 4-16 m/s, "
                        "mixed form + learned closure, all steps in one graph launch (device-side loop over "
                        "pairs of steps, host-polled abort word), autotuned",
            "members": len(specs), "cells": cells, "steps": nsteps_t, "steps_run": steps_run,
            "finished": finished, "ms_per_step": ms / nsteps_t,
            "value": cells * nsteps_t / (ms * 1e-3), "unit": "cell-steps/s",
            "autotuned_ms_per_member_step": tuned, "status": max(status), "fallback_fraction": fb_frac,
            "rel_l2_mixed_vs_fp64_per_member": errs, "rel_l2_mixed_vs_fp64_worst_member": worst,
            "rel_l2_mixed_vs_fp64_smagorinsky_first_members": smag_errs}


def terrain_arm(args, C, Dycore, stream, n_err=100):
    """Terrain-following ABL (static terrain, Deardorff): throughput of the
    plain and mixed forms (graph replay, device-resident state) and the
    mixed form's error against the plain form after n_err steps."""
    import torch
    from erf_b200 import terrain as T
    tn = [int(x) for x in args.terrain_size.split("x")]
    case = T.abl_terrain(nx=tn[0], ny=tn[1], nz=tn[2], dt=0.25)
    cfg = case.cfg
    n_cells = cfg.nx * cfg.ny * cfg.nz
    out = {"workload": f"terrain ABL {cfg.nx}x{cfg.ny}x{cfg.nz}, dx={cfg.dx:g} m, levels stretched from 5 m "
                       f"(ratio 1.04, top {case.z_nd[-1, 0, 0]:.0f} m), 300 m hill + 20 m sinusoids, Deardorff, "
                       f"dt={cfg.dt} s, {cfg.mri_ratio} substeps/RK stage 3",
           "cells": n_cells}
    base = init = None
    res = {}
    for prec, name in ((C.PREC_FP64, "fp64"), (C.PREC_MIXED, "mixed")):
        c = cfg.copy()
        c.precision = prec
        dy = Dycore(c, stream=stream.cuda_stream)
        dy.set_terrain(case.z_nd)
        if base is None:
            base = dy.make_base_state_terrain(case)
            init = case.build_state(base[0])
        dy.set_base_state(base)
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in init]
        torch.cuda.synchronize()
        dy.advance(*dev, args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dy.advance(*dev, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        prof = dy.advance_profiled(*dev, 2)
        kern = {k: {"launches": n, "ms_per_launch": t / n} for k, (t, n) in prof.items() if n}
        out[name] = {"value": n_cells * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
                     "status": dy.status(), "kernels": kern}
        # error run from the initial state
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in init]
        torch.cuda.synchronize()   # the copies run on torch's default stream
        dy.advance(*dev, n_err)
        torch.cuda.synchronize()
        res[name] = [t.cpu().numpy() for t in dev]
        out[name]["status_after_error_run"] = dy.status()
        dy.close()

    def rl2(a, b):
        return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
    (c64, u64, v64, w64), (c32, u32, v32, w32) = res["fp64"], res["mixed"]
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["mixed"][f"rel_l2_vs_fp64_after_{n_err}_steps"] = {
        "u": rl2(u32, u64), "v": rl2(v32, v64), "w": rl2(w32, w64),
        "theta": rl2(c32[1] / c32[0], c64[1] / c64[0]), "tke": rl2(c32[2] / c32[0], c64[2] / c64[0])}
    return out


def moving_terrain_arm(args, C, Dycore, stream):
    """Moving terrain: the reference's MovingTerrain physics (Sullivan grid
    under a travelling surface wave, Centered_2nd, buoyancy type 1) at the
    gold size (40 x 8 x 79, with 20 acoustic substeps per step) and on a
    larger periodic grid with and without substeps; graph replay on a
    device-resident state, plain FP64.  Each step regenerates the grid on
    the device at every geometry time."""
    import torch
    from erf_b200 import terrain as T
    runs = {
        "gold_size_substeps": T.moving_terrain(substeps=True),
        "large_substeps": T.moving_terrain(nx=512, ny=128, nz=79, Lx=2560.0, Ly=640.0, substeps=True),
        "large_no_substep": T.moving_terrain(nx=512, ny=128, nz=79, Lx=2560.0, Ly=640.0),
    }
    out = {"workload": "moving terrain (MovingTerrain physics): 40x8x79 and 512x128x79 cells, dx=dy=5 m, "
                       "400 m deep, 0.16 m wave of 100 m; dt 0.1 s with 20 substeps / dt 0.005 s without"}
    for name, case in runs.items():
        cfg = case.cfg
        n_cells = cfg.nx * cfg.ny * cfg.nz
        dy = Dycore(cfg, stream=stream.cuda_stream)
        dy.set_base_state(case.base)
        dy.load_state(*case.build_state())
        dy.advance_resident(args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dy.advance_resident(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        d = dy.diagnostics()
        out[name] = {"cells": n_cells, "value": n_cells * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
                     "substeps_per_step": (cfg.mri_ratio if cfg.substepping_type == C.SUBSTEP_IMPLICIT else 0),
                     "status": dy.status(), "mass": d["mass"]}
        dy.close()
    return out


def cpu_baseline_run(case_fn, nx, ny, nz, nsteps):
    """Time the FP64 CPU oracle on a bounded sample of the workload; returns
    cell-steps/s, seconds, cores and the seconds of each pass."""
    import oracle
    case = case_fn(nx=nx, ny=ny, nz=nz)
    base = oracle.make_base_state(case.cfg, case)
    cons, u, v, w = case.build_state(base[0])
    oracle.advance(case.cfg, base, cons, u, v, w, 1)  # warm the library / page in
    t0 = time.perf_counter()
    _, passes = oracle.advance_timed(case.cfg, base, cons, u, v, w, nsteps)
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return nx * ny * nz * nsteps / dt, dt, cores, passes


def run_reference(args, rank, world):
    """Reference arm: the CPU FP64 oracle (a restatement of the reference's own
    CPU path; the reference itself cannot be built here) on the host cores."""
    if rank != 0:
        return 0
    case_fn = cases.CASES[args.case]
    full = case_fn()
    import oracle
    # the whole grid of the workload when its steps fit in about three
    # minutes of host time, else a 64 x 64 column block of the same case
    # (timed from one untimed warm-up step of the whole grid)
    case = full
    base = oracle.make_base_state(case.cfg, case)
    st = case.build_state(base[0])
    t0 = time.perf_counter()
    st = oracle.advance(case.cfg, base, *st, 1)
    per_step = time.perf_counter() - t0
    if per_step * (args.steps + max(args.warmup - 1, 0)) > 180.0:
        case = case_fn(nx=min(64, full.cfg.nx), ny=min(64, full.cfg.ny), nz=full.cfg.nz)
        base = oracle.make_base_state(case.cfg, case)
        st = case.build_state(base[0])
        st = oracle.advance(case.cfg, base, *st, 1)
    nx, ny, nz = case.cfg.nx, case.cfg.ny, case.cfg.nz
    for _ in range(args.warmup - 1):
        st = oracle.advance(case.cfg, base, *st, 1)
    passes = {}
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st, p = oracle.advance_timed(case.cfg, base, *st, 1)
        for kq, vq in p.items():
            passes[kq] = passes.get(kq, 0.0) + vq
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    value = nx * ny * nz * args.steps / dt
    whole = (nx, ny, nz) == (full.cfg.nx, full.cfg.ny, full.cfg.nz)
    sample = (f"{args.steps} steps of the whole {nx}x{ny}x{nz} grid" if whole else
              f"{args.steps} steps of a {nx}x{ny}x{nz} block") + f" of the {args.case} case, FP64, OpenMP"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.case} {full.cfg.nx}x{full.cfg.ny}x{full.cfg.nz}" +
                               ("" if whole else f" (sampled {nx}x{ny}x{nz})"),
                   "parallelism": "cpu-openmp"},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": "port", "sample": sample,
                         "cpu_model": cpu_model(), "build": "g++ -O3 -fopenmp -ffp-contract=off",
                         "seconds_per_pass": passes},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--case", default="moist_bubble", choices=sorted(cases.CASES))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="both", choices=["both", "fp64", "mixed", "learned", "ensemble", "terrain",
                                                       "moving_terrain"],
                    help="precision forms to time (the JSON line needs both; single forms are for profiling)")
    ap.add_argument("--terrain-size", default="256x256x96",
                    help="cells of the terrain ABL (nx x ny x nz); smaller only for profiling")
    ap.add_argument("--ens-steps", type=int, default=200,
                    help="steps of the ensemble arm (one graph launch)")
    ap.add_argument("--err-steps", type=int, default=100,
                    help="steps of the mixed-vs-plain error runs (100; fewer only to shorten profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from erf_b200 import Dycore, config as C
    case = cases.CASES[args.case]()
    cfg = case.cfg
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    n_cells = cfg.nx * cfg.ny * cfg.nz
    peaks, peak_kind = load_peaks()
    hbm = float(peaks["hbm_gbs"])
    vals = algorithmic_values_per_cell(cfg)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def measure(precision, clocks, case=case, net=None, les=None, light=False):
        """Time one precision form: graph replay (device-resident state),
        eager per-kernel events, and end to end through the host entry point
        (graph replay only when light)."""
        cfg = case.cfg
        n_cells = cfg.nx * cfg.ny * cfg.nz
        vals = algorithmic_values_per_cell(cfg)
        cfg.precision = precision
        if les is not None:
            cfg.les_type = les
        dy = Dycore(cfg, stream=stream.cuda_stream)
        base = dy.make_base_state(case)
        dy.set_base_state(base)
        if net is not None:
            dy.set_closure(net)
        cons, u, v, w = case.build_state(base[0])
        # launch shapes picked by the library's autotuner on this state
        dy.load_state(cons, u, v, w)
        tuned_ms = dy.autotune(3)
        if net is not None:
            dy.closure_fallbacks()   # reset: count only the warm-up and timed steps below
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (cons, u, v, w)]
        torch.cuda.synchronize()
        dy.advance(*dev, args.warmup)
        barrier()
        # ---- timed region 1: device-resident state, CUDA graph replay
        stop = threading.Event()
        th = None
        if clocks is not None:
            th = threading.Thread(target=sample_clocks, args=(stop, clocks), daemon=True)
            th.start()
            time.sleep(0.3)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dy.advance(*dev, args.steps)
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        stop.set()
        if th is not None:
            th.join(timeout=5)
        ms = max_over_ranks(ms, world, "cuda")
        st = dy.status()
        value = replica_throughput(world, n_cells, args.steps, ms * 1e-3)
        if light:
            out = {"value": value, "ms_per_step": ms / args.steps, "status": st, "autotuned_ms": tuned_ms}
            if net is not None:
                per_step = dy.closure_fallbacks() / max(args.warmup + args.steps, 1)
                out["fallback_cells_per_step"] = per_step
                # the closure runs once per RK stage
                out["fallback_fraction"] = per_step / (3.0 * n_cells)
            dy.close()
            return out, base, (cons, u, v, w)
        # ---- timed region 2: same K steps, eager launches with per-kernel events
        barrier()
        prof = dy.advance_profiled(*dev, args.steps)
        barrier()
        # ---- timed region 3: end to end through the host-buffer entry point,
        #      pinned host memory in and out every step
        host = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (cons, u, v, w)]
        # bytes the host entry moves each way: every velocity and the live cons
        # components (rho*QKE, and rho*KE without Deardorff, are not copied)
        dead = 1 + (1 if cfg.les_type != C.LES_DEARDORFF else 0)
        h2d = sum(t.numel() * 8 for t in host) - dead * n_cells * 8
        dy.lib.erf_b200_advance_host(dy.ctx, *[t.data_ptr() for t in host], 1)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            rc = dy.lib.erf_b200_advance_host(dy.ctx, *[t.data_ptr() for t in host], 1)
            if rc:
                raise RuntimeError(f"advance_host rc={rc}")
        barrier()
        e2e_s = max_over_ranks(time.perf_counter() - t0, world, "cuda")
        e2e = replica_throughput(world, n_cells, args.steps, e2e_s)
        bpc = bytes_per_cell(vals, 4 if precision == C.PREC_MIXED else 8)
        kern = {}
        for name, (kms, cnt) in prof.items():
            if cnt == 0:
                continue
            per_launch_ms = kms / cnt
            nb = bpc.get(name, 0) * n_cells
            kern[name] = {"launches": cnt, "total_ms": kms, "ms_per_launch": per_launch_ms, "algo_bytes": nb,
                          "gbs": nb / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else None}
        dominant = max(kern, key=lambda k: kern[k]["total_ms"])
        dk = kern[dominant]
        form = "mixed" if precision == C.PREC_MIXED else "fp64"
        # DRAM bytes per launch of the dominant kernel from the committed ncu
        # capture (dram__bytes_read.sum + dram__bytes_write.sum); the capture
        # names the library build it measured, reported beside the figure
        traffic, traffic_src = None, None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as fh:
                tj = json.load(fh)
            traffic = tj.get(f"{args.case}/{form}", {}).get(dominant)
            if traffic is not None:
                traffic_src = {k: tj.get(k) for k in ("captured", "library_sha16", "command")}
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": dk["gbs"], "peak": hbm, "unit": "GB/s",
                    "frac": dk["gbs"] / hbm, "traffic": traffic, "traffic_source": traffic_src,
                    "peak_kind": peak_kind,
                    "algo_bytes_per_launch": dk["algo_bytes"], "ms_per_launch": dk["ms_per_launch"]}
        step_bytes = sum(bpc[k] * n_cells * (kern[k]["launches"] / args.steps) for k in kern)
        roof_cells = hbm * 1e9 / (step_bytes / n_cells)
        sb = survey_bytes_per_cell_step(cfg, substeps_per_step(cfg))
        survey_roof = {"bytes_per_cell_step": sb, "hbm_roof_cell_steps_per_s": hbm * 1e9 / sb,
                       "frac": value / world / (hbm * 1e9 / sb), "peak_gbs": hbm, "peak_kind": peak_kind}
        out = {"value": value, "ms_per_step": ms / args.steps, "status": st, "autotuned_ms": tuned_ms,
               "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d},
               "roofline": roofline,
               "step_roofline": {"algo_bytes_per_cell_step": step_bytes / n_cells,
                                 "hbm_roof_cell_steps_per_s": roof_cells, "frac": value / world / roof_cells},
               "survey_roofline": survey_roof,
               "kernels": kern, "launches": dy.kernels_per_step() * args.steps}
        dy.close()
        return out, base, (cons, u, v, w)

    def form_error(base, init, nsteps, case=case, net=None):
        """Per-field relative L2 of the mixed form against the plain FP64 form
        (parity-pinned to the oracle) after nsteps from the same state."""
        cfg = case.cfg
        res = {}
        for prec in (C.PREC_FP64, C.PREC_MIXED):
            cfg.precision = prec
            dy = Dycore(cfg, stream=stream.cuda_stream)
            dy.set_base_state(base)
            if net is not None:
                dy.set_closure(net)
            dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in init]
            torch.cuda.synchronize()   # the copies run on torch's default stream
            dy.advance(*dev, nsteps)
            torch.cuda.synchronize()
            res[prec] = [t.cpu().numpy() for t in dev]
            dy.close()
        cfg.precision = C.PREC_FP64
        (c64, u64, v64, w64), (c32, u32, v32, w32) = res[C.PREC_FP64], res[C.PREC_MIXED]

        def rl2(a, b):
            return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
        err = {"u": rl2(u32, u64), "v": rl2(v32, v64), "w": rl2(w32, w64), "theta": rl2(c32[1] / c32[0], c64[1] / c64[0])}
        if cfg.moisture != 0:
            for n, nm in ((5, "qv"), (6, "qc"), (7, "qr")):
                if n < c64.shape[0]:
                    err[nm] = rl2(c32[n] / c32[0], c64[n] / c64[0])
        qv32 = c32[5, 0] / c32[0, 0] if cfg.moisture != 0 else 0.0
        qv64 = c64[5, 0] / c64[0, 0] if cfg.moisture != 0 else 0.0
        ps = lambda c, qv: 1.0e5 * (287.0 * c[1, 0] * (1.0 + 461.505 / 287.0 * qv) / 1.0e5) ** 1.4
        err["p_sfc"] = rl2(ps(c32, qv32), ps(c64, qv64))
        if cfg.moisture != 0 and c64.shape[0] > 7:
            # the condensate present, so that a zero qc / qr error means agreement
            err["max_qc"] = float(np.max(c64[6] / c64[0]))
            err["max_qr"] = float(np.max(c64[7] / c64[0]))
        return err

    clock_samples = []
    if args.form == "ensemble":
        from erf_b200.dycore import Ensemble
        if rank == 0:
            print(json.dumps({"form": "ensemble", "ensemble": ensemble_arm(args, C, Dycore, Ensemble, stream)}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return 0
    if args.form == "terrain":
        if rank == 0:
            print(json.dumps({"form": "terrain", "terrain": terrain_arm(args, C, Dycore, stream, n_err=args.err_steps)}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return 0
    if args.form == "moving_terrain":
        if rank == 0:
            print(json.dumps({"form": "moving_terrain", "moving_terrain": moving_terrain_arm(args, C, Dycore, stream)}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return 0
    if args.form == "learned":
        if rank == 0:
            print(json.dumps({"form": "learned", "learned": learned_arm(measure, form_error, C)}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return 0
    if args.form != "both":
        res, _, _ = measure(C.PREC_MIXED if args.form == "mixed" else C.PREC_FP64, clock_samples)
        if rank == 0:
            print(json.dumps({"form": args.form, "value": res["value"], "ms_per_step": res["ms_per_step"],
                              "kernels": res["kernels"], "status": res["status"]}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return 0
    plain, base, init = measure(C.PREC_FP64, clock_samples)
    mixed, _, _ = measure(C.PREC_MIXED, None)
    # the dry neutral ABL 64^3 (Smagorinsky, dt 0.5 s, 6 substeps), plain form
    c0 = None
    if args.case != "abl_dry":
        c0_res, _, _ = measure(C.PREC_FP64, None, case=cases.abl_dry())
        c0 = {"workload": "abl_dry 64x64x64, Smagorinsky, no-slip ground, Coriolis + geostrophic, dt=0.5 s, "
                          "6 substeps/RK stage 3, FP64 plain form",
              "value": c0_res["value"], "ms_per_step": c0_res["ms_per_step"], "e2e": c0_res["e2e"],
              "survey_roofline": c0_res["survey_roofline"], "step_roofline": c0_res["step_roofline"],
              "roofline": c0_res["roofline"], "status": c0_res["status"]}
    cfg.precision = C.PREC_FP64
    mixed_err = form_error(base, init, 100) if rank == 0 else None
    # a longer run in which the bubble condenses and rains, so that the qc /
    # qr errors are taken where both fields are non-zero
    mixed_err_cloud = form_error(base, init, 600) if (rank == 0 and cfg.moisture) else None
    cfg.precision = C.PREC_FP64
    learned = learned_arm(measure, form_error, C) if rank == 0 else None
    from erf_b200.dycore import Ensemble
    ensemble = ensemble_arm(args, C, Dycore, Ensemble, stream) if rank == 0 else None
    terrain_res = terrain_arm(args, C, Dycore, stream) if rank == 0 else None
    mt_res = moving_terrain_arm(args, C, Dycore, stream) if rank == 0 else None

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        bx, by = min(64, cfg.nx), min(64, cfg.ny)
        v_cpu, t_cpu, cores, passes = cpu_baseline_run(cases.CASES[args.case], bx, by, cfg.nz, 2)
        cpu = {"value": v_cpu, "unit": "cell-steps/s", "cores": cores, "kind": "port",
               "sample": f"2 steps of a {bx}x{by}x{cfg.nz} block of the {args.case} case "
                         f"({t_cpu:.1f} s, FP64 oracle, OpenMP)",
               "cpu_model": cpu_model(), "build": "g++ -O3 -fopenmp -ffp-contract=off",
               "seconds_per_pass": passes}

    if rank == 0:
        line = {
            "metric": METRIC, "value": plain["value"], "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": plain["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.case} {cfg.nx}x{cfg.ny}x{cfg.nz}, "
                                   f"{'Kessler, ' if cfg.moisture else ''}dt={cfg.dt} s, "
                                   f"{cfg.mri_ratio} substeps/RK stage 3, FP64 plain form",
                       "cells": n_cells, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "working set > 126 MB L2 (no flush needed)"},
            "e2e": plain["e2e"],
            "roofline": plain["roofline"],
            "step_roofline": plain["step_roofline"],
            "survey_roofline": plain["survey_roofline"],
            "kernels": plain["kernels"],
            "abl_dry_64": c0,
            "mixed": {"value": mixed["value"], "ms_per_step": mixed["ms_per_step"],
                      "speedup_vs_fp64": mixed["value"] / plain["value"], "dtype": "f32 bulk / f64 state",
                      "e2e": mixed["e2e"], "roofline": mixed["roofline"], "step_roofline": mixed["step_roofline"],
                      "kernels": {k: {"ms_per_launch": v["ms_per_launch"], "gbs": v["gbs"]}
                                  for k, v in mixed["kernels"].items()},
                      "rel_l2_vs_fp64_after_100_steps": mixed_err,
                      "rel_l2_vs_fp64_after_600_steps_cloudy": mixed_err_cloud, "status": mixed["status"]},
            "learned": learned,
            "ensemble": ensemble,
            "terrain": terrain_res,
            "moving_terrain": mt_res,
            "cpu_baseline": cpu,
            "clocks": summarize_clocks(clock_samples),
            "gpu_launches": plain["launches"],
            "status": plain["status"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
