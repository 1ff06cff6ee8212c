// kernels.cu -- FP64 dycore kernels for sm_100a.
//
// Each kernel fuses one or more of the reference's AMReX ParallelFor passes
// (file:line cited per kernel).  Lateral neighbours are addressed through
// periodic index wrapping and vertical ghost values through the wall
// conditions, so no separate ghost-fill pass is launched between stages and
// substeps; the reference's momentum<->velocity round trips at every boundary
// fill (BoundaryConditions/ERF_FillIntermediatePatch.cpp:63-67, 224-236) are
// applied inline where the filled values are next read.
#include "kernels.cuh"

namespace erfb {

// ---------------------------------------------------------------------------
// Accessors with boundary conditions
// ---------------------------------------------------------------------------
// Tangential velocity at (i,j,k), i,j already wrapped; below/above the walls
// the ghost value is 0 (no-slip, ext_dir) or the nearest interior value
// (slip, foextrap): ERF_BoundaryConditions_xvel.cpp:190-230.
__device__ __forceinline__ double tang(const double* __restrict__ f, const Geo& g, int i, int j, int k) {
    if (k < 0) return g.zlo_noslip ? 0.0 : __ldg(f + cidx(g, i, j, 0));
    if (k >= g.nz) return g.zhi_noslip ? 0.0 : __ldg(f + cidx(g, i, j, g.nz - 1));
    return __ldg(f + cidx(g, i, j, k));
}
// Cell-centred scalar with foextrap in z.
__device__ __forceinline__ double ccz(const double* __restrict__ f, const Geo& g, int i, int j, int k) {
    return __ldg(f + cidx(g, i, j, clampk(k, g.nz)));
}

// ---------------------------------------------------------------------------
// Strain-rate components (Diffusion/ERF_ComputeStrain_N.cpp:28-229) with the
// one-sided wall stencils at no-slip walls.  Edge (i,j,k) of an xy/xz/yz edge
// array sits at the low corner of cell (i,j,k).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double strain12(const double* u, const double* v, const Geo& g, int i, int j, int k) {
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    return 0.5 * ((__ldg(u + cidx(g, i, j, k)) - __ldg(u + cidx(g, i, jm, k))) * g.dyi +
                  (__ldg(v + cidx(g, i, j, k)) - __ldg(v + cidx(g, im, j, k))) * g.dxi);
}
__device__ __forceinline__ double strain13(const double* u, const double* w, const Geo& g, int i, int j, int k) {
    int im = wrap(i - 1, g.nx);
    double wx = (__ldg(w + cidx(g, i, j, k)) - __ldg(w + cidx(g, im, j, k))) * g.dxi;
    if (k == 0 && g.zlo_noslip)
        return 0.5 * ((-(8. / 3.) * tang(u, g, i, j, k - 1) + 3. * tang(u, g, i, j, k) - (1. / 3.) * tang(u, g, i, j, k + 1)) * g.dzi + wx);
    if (k == g.nz && g.zhi_noslip)
        return 0.5 * (-(-(8. / 3.) * tang(u, g, i, j, k) + 3. * tang(u, g, i, j, k - 1) - (1. / 3.) * tang(u, g, i, j, k - 2)) * g.dzi + wx);
    return 0.5 * ((tang(u, g, i, j, k) - tang(u, g, i, j, k - 1)) * g.dzi + wx);
}
__device__ __forceinline__ double strain23(const double* v, const double* w, const Geo& g, int i, int j, int k) {
    int jm = wrap(j - 1, g.ny);
    double wy = (__ldg(w + cidx(g, i, j, k)) - __ldg(w + cidx(g, i, jm, k))) * g.dyi;
    if (k == 0 && g.zlo_noslip)
        return 0.5 * ((-(8. / 3.) * tang(v, g, i, j, k - 1) + 3. * tang(v, g, i, j, k) - (1. / 3.) * tang(v, g, i, j, k + 1)) * g.dzi + wy);
    if (k == g.nz && g.zhi_noslip)
        return 0.5 * (-(-(8. / 3.) * tang(v, g, i, j, k) + 3. * tang(v, g, i, j, k - 1) - (1. / 3.) * tang(v, g, i, j, k - 2)) * g.dzi + wy);
    return 0.5 * ((tang(v, g, i, j, k) - tang(v, g, i, j, k - 1)) * g.dzi + wy);
}

__device__ __forceinline__ bool cell_coords(const Geo& g, int& i, int& j, int& k) {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y * blockDim.y + threadIdx.y;
    k = blockIdx.z;
    return i < g.nx && j < g.ny && k < g.nz;
}

// Derived stage quantities of one cell: cons_to_prim + pi_stage
// (TimeIntegration/ERF_TI_utils.H:4-45) and p' (ERF_slow_rhs_pre.cpp:337-358).
__device__ __forceinline__ void stage_aux_cell(const Params& P, const double* __restrict__ cons, StageAux A,
                                               int64_t c, int k) {
    const int64_t N = P.g.ncell;
    double rho = cons[c];
    double rt = cons[N + c];
    A.prim[c] = rt / rho;
    for (int n = 1; n < P.nprim; ++n) A.prim[n * N + c] = cons[(n + 1) * N + c] / rho;
    A.pi[c] = eos_exner(rt, P.rdOcp);
    double qv = P.moist ? cons[5 * N + c] / rho : 0.0;
    A.pp[c] = eos_p(rt, qv) - P.p0[k + 1];
    if (!(rt > 0.0) || !(rho > 0.0)) atomicOr(P.status, ST_BADSTATE);
}

// ---------------------------------------------------------------------------
// Step prologue.  Fuses, for the step's old state:
//   * ComputeStrain_N + ComputeTurbulentViscosityLES (Smagorinsky) from the
//     old velocities (ERF_advance_dycore.cpp:114-223,
//     ERF_ComputeTurbulentViscosity.cpp:85-126; EddyViscosity.H:31-83);
//   * VelocityToMomentum of the old velocities, the MomentumToVelocity /
//     VelocityToMomentum round trip of apply_bcs(state_old)
//     (ERF_advance_dycore.cpp:260-276);
//   * cons_to_prim / pi_stage / p' of the old state.
// ---------------------------------------------------------------------------
__global__ void k_step_begin(Params P, const double* __restrict__ cons, const double* __restrict__ uo,
                             const double* __restrict__ vo, const double* __restrict__ wo, StateBuf S,
                             double* __restrict__ un, double* __restrict__ vn, double* __restrict__ wn,
                             StageAux A, double* __restrict__ mut) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    int64_t c = cidx(g, i, j, k);
    double rho = cons[c];
    {
        double rs = rho + cons[cidx(g, im, j, k)];
        double m0 = (uo[c] * 0.5) * rs, u1 = (m0 * 2.0) / rs;
        S.mx[c] = (u1 * 0.5) * rs; un[c] = u1;
    }
    {
        double rs = rho + cons[cidx(g, i, jm, k)];
        double m0 = (vo[c] * 0.5) * rs, v1 = (m0 * 2.0) / rs;
        S.my[c] = (v1 * 0.5) * rs; vn[c] = v1;
    }
    if (k == 0) {
        S.mz[c] = 0.0; wn[c] = 0.0;
    } else {
        double rs = rho + cons[cidx(g, i, j, k - 1)];
        double m0 = (wo[c] * 0.5) * rs, w1 = (m0 * 2.0) / rs;
        S.mz[c] = (w1 * 0.5) * rs; wn[c] = w1;
    }
    if (k == g.nz - 1) { S.mz[c + g.sk] = 0.0; wn[c + g.sk] = 0.0; }
    stage_aux_cell(P, cons, A, c, k);

    if (P.les == ERF_LES_SMAGORINSKY) {
        int ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
        double s11 = (uo[cidx(g, ip, j, k)] - uo[c]) * g.dxi;
        double s22 = (vo[cidx(g, i, jp, k)] - vo[c]) * g.dyi;
        double s33 = (wo[c + g.sk] - wo[c]) * g.dzi;
        double s12 = 0.25 * (strain12(uo, vo, g, i, j, k) + strain12(uo, vo, g, i, jp, k) +
                             strain12(uo, vo, g, ip, j, k) + strain12(uo, vo, g, ip, jp, k));
        double s13 = 0.25 * (strain13(uo, wo, g, i, j, k) + strain13(uo, wo, g, i, j, k + 1) +
                             strain13(uo, wo, g, ip, j, k) + strain13(uo, wo, g, ip, j, k + 1));
        double s23 = 0.25 * (strain23(vo, wo, g, i, j, k) + strain23(vo, wo, g, i, j, k + 1) +
                             strain23(vo, wo, g, i, jp, k) + strain23(vo, wo, g, i, jp, k + 1));
        double S2 = s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * s12 * s12 + 2.0 * s13 * s13 + 2.0 * s23 * s23;
        mut[c] = P.CsDeltaSqr * rho * sqrt(2.0 * S2);
    }
}

// ---------------------------------------------------------------------------
// Stress tensor (erf_make_tau_terms, TimeIntegration/ERF_make_tau_terms.cpp:
// 320-424 with ComputeStress{Cons,Var}Visc_N, Diffusion/ERF_ComputeStress_N.cpp):
// tau_ii at cell centres, tau_12/13/23 on edges.
// ---------------------------------------------------------------------------
__global__ void k_tau(Params P, const double* __restrict__ cons, const double* __restrict__ u,
                      const double* __restrict__ v, const double* __restrict__ w, const double* __restrict__ mut,
                      double* __restrict__ t11, double* __restrict__ t22, double* __restrict__ t33,
                      double* __restrict__ t12, double* __restrict__ t13, double* __restrict__ t23) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny), ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
    int64_t c = cidx(g, i, j, k);
    const double OneThird = 1. / 3.;
    double s11 = (u[cidx(g, ip, j, k)] - u[c]) * g.dxi;
    double s22 = (v[cidx(g, i, jp, k)] - v[c]) * g.dyi;
    double s33 = (w[c + g.sk] - w[c]) * g.dzi;
    double er = s11 + s22 + s33;
    double base = P.use_consA ? cons[c] * P.mu_eff : P.mu_eff;
    double m11 = P.use_turb ? base + 2.0 * mut[c] : base;
    t11[c] = -m11 * (s11 - OneThird * er);
    t22[c] = -m11 * (s22 - OneThird * er);
    t33[c] = -m11 * (s33 - OneThird * er);
    auto mu = [&](int ii, int jj, int kk) { return __ldg(mut + cidx(g, ii, jj, clampk(kk, g.nz))); };
    auto rho = [&](int ii, int jj, int kk) { return __ldg(cons + cidx(g, ii, jj, clampk(kk, g.nz))); };
    {
        double m = P.use_consA ? 0.25 * (rho(im, j, k) + rho(i, j, k) + rho(im, jm, k) + rho(i, jm, k)) * P.mu_eff : P.mu_eff;
        if (P.use_turb) m = m + 2.0 * (0.25 * (mu(im, j, k) + mu(i, j, k) + mu(im, jm, k) + mu(i, jm, k)));
        t12[c] = strain12(u, v, g, i, j, k) * -m;
    }
    for (int kk = k; kk <= (k == g.nz - 1 ? g.nz : k); ++kk) {
        int64_t e = cidx(g, i, j, kk);
        double m = P.use_consA ? 0.25 * (rho(im, j, kk) + rho(i, j, kk) + rho(im, j, kk - 1) + rho(i, j, kk - 1)) * P.mu_eff : P.mu_eff;
        if (P.use_turb) m = m + 2.0 * (0.25 * (mu(im, j, kk) + mu(i, j, kk) + mu(im, j, kk - 1) + mu(i, j, kk - 1)));
        t13[e] = strain13(u, w, g, i, j, kk) * -m;
        double m2 = P.use_consA ? 0.25 * (rho(i, jm, kk) + rho(i, j, kk) + rho(i, jm, kk - 1) + rho(i, j, kk - 1)) * P.mu_eff : P.mu_eff;
        if (P.use_turb) m2 = m2 + 2.0 * (0.25 * (mu(i, jm, kk) + mu(i, j, kk) + mu(i, jm, kk - 1) + mu(i, j, kk - 1)));
        t23[e] = strain23(v, w, g, i, j, kk) * -m2;
    }
}

// ---------------------------------------------------------------------------
// Scalar flux helpers
// ---------------------------------------------------------------------------
// Advective flux of primitive component `pc` through the low x/y/z face of
// cell (i,j,k): mom * interp(phi) (Advection/ERF_AdvectionSrcForScalars.H:7-58).
template <int T = -1>
__device__ __forceinline__ double adv_flux_x(const Geo& g, const double* __restrict__ phi, const double* __restrict__ mom,
                                             int type, double frac, int i, int j, int k) {
    double s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? __ldg(phi + cidx(g, wrap(i + off, g.nx), j, k)) : 0.0;
    }
    double a = __ldg(mom + cidx(g, i, j, k));
    return a * interp_of<T>(type, s, a, frac);
}
template <int T = -1>
__device__ __forceinline__ double adv_flux_y(const Geo& g, const double* __restrict__ phi, const double* __restrict__ mom,
                                             int type, double frac, int i, int j, int k) {
    double s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? __ldg(phi + cidx(g, i, wrap(j + off, g.ny), k)) : 0.0;
    }
    double a = __ldg(mom + cidx(g, i, j, k));
    return a * interp_of<T>(type, s, a, frac);
}
template <int T = -1>
__device__ __forceinline__ double adv_flux_z(const Geo& g, const double* __restrict__ phi, const double* __restrict__ mom,
                                             int type, double frac, int i, int j, int k) {
    double s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? ccz(phi, g, i, j, k + off) : 0.0;
    }
    double a = __ldg(mom + cidx(g, i, j, k));
    return a * interp_of<T>(type, s, a, frac);
}

// Advective tendency of one scalar (assigns, like AdvectionSrcForScalars,
// Advection/ERF_AdvectionSrcForState.cpp:359-370)
__device__ __forceinline__ double scalar_adv_tend(const Params& P, const double* phi, const double* ax,
                                                  const double* ay, const double* az, int th, int tv, double fh,
                                                  double fv, int i, int j, int k) {
    const Geo& g = P.g;
    int ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
    double fxl = adv_flux_x(g, phi, ax, th, fh, i, j, k), fxh = adv_flux_x(g, phi, ax, th, fh, ip, j, k);
    double fyl = adv_flux_y(g, phi, ay, th, fh, i, j, k), fyh = adv_flux_y(g, phi, ay, th, fh, i, jp, k);
    double fzl = adv_flux_z(g, phi, az, tv, fv, i, j, k), fzh = adv_flux_z(g, phi, az, tv, fv, i, j, k + 1);
    return -1.0 * 1.0 * ((fxh - fxl) * g.dxi + (fyh - fyl) * g.dyi + (fzh - fzl) * g.dzi);
}

// Diffusive tendency -div(-rhoAlpha grad phi) (Diffusion/ERF_DiffusionSrcForState_N.cpp:
// 196-667), scalars foextrap at the walls; returns the amount subtracted.
__device__ __forceinline__ double scalar_diff(const Params& P, const double* __restrict__ rhoarr,
                                              const double* __restrict__ phi, const double* __restrict__ mut,
                                              double ae, double fac, int i, int j, int k) {
    const Geo& g = P.g;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny), ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
    auto ph = [&](int ii, int jj, int kk) { return ccz(phi, g, ii, jj, kk); };
    auto rA = [&](int i0, int j0, int k0, int i1, int j1, int k1) {
        double r = P.use_consA ? 0.5 * (ccz(rhoarr, g, i0, j0, k0) + ccz(rhoarr, g, i1, j1, k1)) * ae : ae;
        if (P.use_turb) r += 0.5 * (ccz(mut, g, i0, j0, k0) * fac + ccz(mut, g, i1, j1, k1) * fac);
        return r;
    };
    double fxl = -rA(i, j, k, im, j, k) * (ph(i, j, k) - ph(im, j, k)) * g.dxi * 1.0;
    double fxh = -rA(ip, j, k, i, j, k) * (ph(ip, j, k) - ph(i, j, k)) * g.dxi * 1.0;
    double fyl = -rA(i, j, k, i, jm, k) * (ph(i, j, k) - ph(i, jm, k)) * g.dyi * 1.0;
    double fyh = -rA(i, jp, k, i, j, k) * (ph(i, jp, k) - ph(i, j, k)) * g.dyi * 1.0;
    double fzl = -rA(i, j, k, i, j, k - 1) * (ph(i, j, k) - ph(i, j, k - 1)) * g.dzi;
    double fzh = -rA(i, j, k + 1, i, j, k) * (ph(i, j, k + 1) - ph(i, j, k)) * g.dzi;
    return (fxh - fxl) * g.dxi * 1.0 + (fyh - fyl) * g.dyi * 1.0 + (fzh - fzl) * g.dzi;
}

// Horizontal plane averages of rho, theta, qv, qc, qp for buoyancy type 2
// (SourceTerms/ERF_make_buoyancy.cpp:212-249): one block per level.
__global__ void k_plane_avg(Params P, const double* __restrict__ cons, const double* __restrict__ prim,
                            double* __restrict__ avg) {
    const Geo& g = P.g;
    int k = blockIdx.x;
    const int64_t N = g.ncell;
    double denom = 1.0 / (double)(g.nx * g.ny);
    int nq = P.ncomp - ERF_RHOQ1_COMP;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int64_t t = threadIdx.x; t < g.sk; t += blockDim.x) {
        int64_t c = g.sk * k + t;
        acc[0] += cons[c] * denom;
        acc[1] += prim[c] * denom;
        if (nq >= 1) acc[2] += prim[4 * N + c] * denom;
        if (nq >= 2) acc[3] += prim[5 * N + c] * denom;
        if (nq >= 3) acc[4] += prim[6 * N + c] * denom;
    }
    __shared__ double sh[5][256];
    for (int q = 0; q < 5; ++q) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 5; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 5; ++q) avg[q * g.nz + k] = sh[q][0];
}

// Momentum flux of component `phi` (a face velocity) through a face, with the
// interpolant selected at run time (ERF_AdvectionSrcForMom_N.H:17-274).
template <int T = -1>
__device__ __forceinline__ double gatherx_interp(const Geo& g, const double* f, int type, double upw, double frac,
                                                 int i, int j, int k) {
    double s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? __ldg(f + cidx(g, wrap(i + off, g.nx), j, k)) : 0.0;
    }
    return interp_of<T>(type, s, upw, frac);
}
template <int T = -1>
__device__ __forceinline__ double gathery_interp(const Geo& g, const double* f, int type, double upw, double frac,
                                                 int i, int j, int k) {
    double s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? __ldg(f + cidx(g, i, wrap(j + off, g.ny), k)) : 0.0;
    }
    return interp_of<T>(type, s, upw, frac);
}
template <int T = -1>
__device__ __forceinline__ double gatherz_tang(const Geo& g, const double* f, int type, double upw, double frac,
                                               int i, int j, int k) {
    double s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? tang(f, g, i, j, k + off) : 0.0;
    }
    return interp_of<T>(type, s, upw, frac);
}

// ---------------------------------------------------------------------------
// Acoustic substep, horizontal part (ERF_fast_rhs_N.cpp:115-256): lagged
// d(rho theta) and its forward extrapolation, explicit U'' / V'' update and
// the average-momentum accumulation.  For substeps after the first, the
// previous momenta are first passed through the momentum->velocity->momentum
// round trip of apply_bcs (ERF_TI_fast_rhs_fun.H:183-189).
// ---------------------------------------------------------------------------
__global__ void k_fast_h(Params P, int step, int nrk, double dtau, double facinv, StateBuf Sprev, int prev_rt,
                         StateBuf Sst, StageAux A, const double* __restrict__ Fmx, const double* __restrict__ Fmy,
                         const double* __restrict__ lag_in, double* __restrict__ lag_out, double* __restrict__ avx,
                         double* __restrict__ avy, double* __restrict__ outx, double* __restrict__ outy) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    const int64_t N = g.ncell;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    int64_t c = cidx(g, i, j, k), cxm = cidx(g, im, j, k), cym = cidx(g, i, jm, k);
    const double beta_d = 0.1;
    auto extrap = [&](int64_t cc) {
        double drt = Sprev.cons[N + cc] - Sst.cons[N + cc];
        if (step == 0) return drt;
        return drt + beta_d * (drt - lag_in[cc]);
    };
    double drt_c = Sprev.cons[N + c] - Sst.cons[N + c];
    lag_out[c] = drt_c;
    double px = Sprev.mx[c], py = Sprev.my[c];
    if (prev_rt) {
        double rs = Sprev.cons[c] + Sprev.cons[cxm];
        double ut = (px * 2.0) / rs;
        px = (ut * 0.5) * rs;
        rs = Sprev.cons[c] + Sprev.cons[cym];
        double vt = (py * 2.0) / rs;
        py = (vt * 0.5) * rs;
    }
    double ndx, ndy;
    if (nrk == 0 && step == 0) {
        ndx = px - Sst.mx[c] + dtau * Fmx[c];
        ndy = py - Sst.my[c] + dtau * Fmy[c];
    } else {
        double ec = extrap(c);
        double gpx = (ec - extrap(cxm)) * g.dxi;
        gpx *= 1.0;
        double gpy = (ec - extrap(cym)) * g.dyi;
        gpy *= 1.0;
        if (P.moist) {
            const double* pr = A.prim;
            double qx = 0.5 * (pr[4 * N + c] + pr[4 * N + cxm] + pr[5 * N + c] + pr[5 * N + cxm]);
            double qy = 0.5 * (pr[4 * N + c] + pr[4 * N + cym] + pr[5 * N + c] + pr[5 * N + cym]);
            gpx /= (1.0 + qx);
            gpy /= (1.0 + qy);
        }
        double pix = 0.5 * (A.pi[cxm] + A.pi[c]);
        double piy = 0.5 * (A.pi[cym] + A.pi[c]);
        double fx = -Gamma_ * R_d * pix * gpx;
        double fy = -Gamma_ * R_d * piy * gpy;
        ndx = px - Sst.mx[c] + dtau * fx + dtau * Fmx[c];
        ndy = py - Sst.my[c] + dtau * fy + dtau * Fmy[c];
    }
    avx[c] += facinv * ndx;
    avy[c] += facinv * ndy;
    outx[c] = Sst.mx[c] + ndx;
    outy[c] = Sst.my[c] + ndy;
}

// ---------------------------------------------------------------------------
// Acoustic substep, vertical part: one thread per column.  Fuses
//   * make_fast_coeffs (ERF_make_fast_coeffs.cpp:160-290): P, Q, A, B, C and
//     the Thomas forward elimination of B, evaluated from the stage state
//     (they are constant over a stage, so recomputing them per substep
//     reproduces the stored values);
//   * the horizontal rho / rho*theta fluxes from the new U'', V''
//     (ERF_fast_rhs_N.cpp:328-357);
//   * the right-hand side of the implicit w system (:374-432);
//   * the tridiagonal solve (:437-453);
//   * vertical fluxes, average z-momentum and the rho, rho*theta update
//     (:518-592).
// Scratch (per column, face/cell layout): soln, C/B', and the horizontal
// parts of temp_rhs.
// ---------------------------------------------------------------------------
__global__ void k_fast_col(Params P, int step, double dtau, double facinv, double D, double beta_1, double beta_2,
                           StateBuf Sprev, int prev_rt, StateBuf Sst, StageAux A, const double* __restrict__ Fcons,
                           const double* __restrict__ Fmz, const double* __restrict__ newx,
                           const double* __restrict__ newy, double* __restrict__ avz, double* __restrict__ out_cons,
                           double* __restrict__ out_mz, double* __restrict__ sc_soln, double* __restrict__ sc_cb,
                           double* __restrict__ sc_tr0, double* __restrict__ sc_tr1) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    (void)step;
    const int64_t N = g.ncell;
    const int nz = g.nz;
    int ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny), im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    const double* th = A.prim;
    const double halfg = P.halfg;
    const double dzi = g.dzi;
    auto thz = [&](int k) { return th[cidx(g, i, j, clampk(k, nz))]; };
    // horizontal part of temp_rhs for cell k
    auto trh = [&](int k, double& t0, double& t1) {
        int64_t c = cidx(g, i, j, k);
        double xl = (newx[c] - Sst.mx[c]) / 1.0;
        double xh = (newx[cidx(g, ip, j, k)] - Sst.mx[cidx(g, ip, j, k)]) / 1.0;
        double yl = (newy[c] - Sst.my[c]) / 1.0;
        double yh = (newy[cidx(g, i, jp, k)] - Sst.my[cidx(g, i, jp, k)]) / 1.0;
        double mfsq = 1.0;
        double tc = th[c];
        t0 = (xh - xl) * g.dxi * mfsq + (yh - yl) * g.dyi * mfsq;
        t1 = ((xh * (tc + th[cidx(g, ip, j, k)]) - xl * (tc + th[cidx(g, im, j, k)])) * g.dxi * mfsq +
              (yh * (tc + th[cidx(g, i, jp, k)]) - yl * (tc + th[cidx(g, i, jm, k)])) * g.dyi * mfsq) * 0.5;
    };
    // previous z-momentum at face k (with the apply_bcs round trip)
    auto prev_mz = [&](int k) {
        int64_t f = cidx(g, i, j, k);
        double m = Sprev.mz[f];
        if (prev_rt) {
            if (k == 0 || k == nz) return 0.0;
            double rs = Sprev.cons[f] + Sprev.cons[f - g.sk];
            double wt = (m * 2.0) / rs;
            m = (wt * 0.5) * rs;
        }
        return m;
    };
    auto qcell = [&](int k) {
        int64_t c = cidx(g, i, j, k);
        return P.moist ? (th[4 * N + c] + th[5 * N + c]) : 0.0;
    };
    (void)qcell;

    // ---- forward sweep over faces
    double Om = prev_mz(0) - Sst.mz[cidx(g, i, j, 0)];  // Omega at face k-1 (starts as face 0)
    double Ok = 0.0;
    double soln_prev, bet, Cprev;
    {
        int64_t f0 = cidx(g, i, j, 0);
        double rhs0 = prev_mz(0) - Sst.mz[f0] + dtau * Fmz[f0];
        soln_prev = rhs0 * 1.0;
        sc_soln[f0] = soln_prev;
        sc_cb[f0] = 0.0 * 1.0;
        bet = 1.0;
        Cprev = 0.0;
    }
    // rolling cell data for cells k-1 and k
    double tr0_lo, tr1_lo;
    trh(0, tr0_lo, tr1_lo);
    sc_tr0[cidx(g, i, j, 0)] = tr0_lo;
    sc_tr1[cidx(g, i, j, 0)] = tr1_lo;
    Ok = prev_mz(1) - Sst.mz[cidx(g, i, j, 1)];
    for (int k = 1; k <= nz - 1; ++k) {
        int64_t c = cidx(g, i, j, k), cm = c - g.sk;
        double tr0_hi, tr1_hi;
        trh(k, tr0_hi, tr1_hi);
        sc_tr0[c] = tr0_hi;
        sc_tr1[c] = tr1_hi;
        double Okp1 = prev_mz(k + 1) - Sst.mz[c + g.sk];
        // coefficients (make_fast_coeffs, no terrain)
        double pi_c = 0.5 * (A.pi[cm] + A.pi[c]);
        double cP = -Gamma_ * R_d * dzi + halfg * R_d * P.r0[k + 1] / (P.c_v * P.pi0[k + 1] * Sst.cons[N + c]);
        cP *= pi_c;
        double cQ = Gamma_ * R_d * dzi + halfg * R_d * P.r0[k] / (P.c_v * P.pi0[k] * Sst.cons[N + cm]);
        cQ *= pi_c;
        if (P.moist) {
            double q = 0.5 * (th[4 * N + c] + th[4 * N + cm] + th[5 * N + c] + th[5 * N + cm]);
            cP /= (1.0 + q);
            cQ /= (1.0 + q);
        }
        double tlo = 0.5 * (thz(k - 2) + thz(k - 1));
        double tmid = 0.5 * (thz(k - 1) + thz(k));
        double thi = 0.5 * (thz(k) + thz(k + 1));
        double Acoef = D * (halfg - cQ * tlo);
        double Ccoef = D * (-halfg + cP * thi);
        double Bcoef = 1.0 + D * (cQ - cP) * tmid;
        // right-hand side
        double drt_k = Sprev.cons[N + c] - Sst.cons[N + c];
        double drt_km = Sprev.cons[N + cm] - Sst.cons[N + cm];
        double odk = Sprev.cons[c] - Sst.cons[c];
        double odkm = Sprev.cons[cm] - Sst.cons[cm];
        double R0 = cP * drt_k + cQ * drt_km - halfg * (odk + odkm);
        double R1 = halfg * (-Fcons[c] - Fcons[cm] + tr0_hi + tr0_lo) +
                    (cP * (Fcons[N + c] - tr1_hi) + cQ * (Fcons[N + cm] - tr1_lo));
        R1 += beta_1 * dzi * ((Okp1 - Om) * halfg - (Okp1 * thi - Ok * tmid) * cP - (Ok * tmid - Om * tlo) * cQ);
        double rhs = Ok + dtau * (Fmz[c] + R0 + dtau * beta_2 * R1);
        // Thomas forward elimination
        double gam = Cprev / bet;
        bet = Bcoef - Acoef * gam;
        double invB = 1.0 / bet;
        double sol = (rhs - Acoef * soln_prev) * invB;
        sc_soln[c] = sol;
        sc_cb[c] = Ccoef * invB;
        if (!(fabs(bet) > 1e-300)) atomicOr(P.status, ST_BADSTATE);
        soln_prev = sol;
        Cprev = Ccoef;
        Om = Ok;
        Ok = Okp1;
        tr0_lo = tr0_hi;
        tr1_lo = tr1_hi;
    }
    // top face (A = 0, B = 1, C = 0; B' = 1 is not inverted by the reference)
    int64_t ftop = cidx(g, i, j, nz);
    double rhs_top = prev_mz(nz) - Sst.mz[ftop] + dtau * Fmz[ftop];
    double gam = Cprev / bet;
    double bet_top = 1.0 - 0.0 * gam;
    double sol_top = (rhs_top - 0.0 * soln_prev) * bet_top;
    // ---- back substitution and cell updates, top to bottom
    double drw_hi = prev_mz(nz) - Sst.mz[ftop];
    out_mz[ftop] = Sst.mz[ftop] + sol_top;
    double sol_hi = sol_top;
    for (int k = nz - 1; k >= 0; --k) {
        int64_t c = cidx(g, i, j, k);
        double sol = sc_soln[c];
        sol -= sc_cb[c] * sol_hi;
        double pmz = prev_mz(k);
        double drw_lo = pmz - Sst.mz[c];
        out_mz[c] = Sst.mz[c] + sol;
        double zl = beta_2 * sol + beta_1 * drw_lo;
        double zh = beta_2 * sol_hi + beta_1 * drw_hi;
        avz[c] += facinv * zl / (1.0 * 1.0);
        if (k == nz - 1) avz[c + g.sk] += facinv * zh / (1.0 * 1.0);
        double tc = th[c];
        double t0 = sc_tr0[c] + dzi * (zh - zl);
        double t1 = sc_tr1[c] + 0.5 * dzi * (zh * (tc + thz(k + 1)) - zl * (tc + thz(k - 1)));
        double pr = Sprev.cons[c], prt = Sprev.cons[N + c];
        out_cons[c] = pr + dtau * (Fcons[c] - t0);
        out_cons[N + c] = prt + dtau * (Fcons[N + c] - t1);
        sol_hi = sol;
        drw_hi = drw_lo;
    }
}

// ---------------------------------------------------------------------------
// Kessler warm-rain microphysics, one thread per column, in place
// (Microphysics/Kessler/ERF_Kessler.cpp:11-185, ERF_Init_Kessler.cpp:64-99,
// ERF_Update_Kessler.cpp:14-40).  The rain flux through face k+1 is computed
// from the pre-update cells k and k+1 before cell k is updated.
// ---------------------------------------------------------------------------
__global__ void k_kessler(Params P, double* __restrict__ cons, double dtn, double dz) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int64_t N = g.ncell;
    const int nz = g.nz;
    const bool rain = P.kessler_rain;
    const bool has_qp = P.ncomp > 7;
    const double fac_cond = lcond / P.c_p;
    auto qp_of = [&](int64_t c) { return has_qp ? cons[7 * N + c] / cons[c] : 0.0; };
    auto flux = [&](double ra, double qa) {
        qa = fmax(0.0, qa);
        double Vt = 36.34 * pow(ra * 0.001 * qa, 0.1346) * pow(ra / 1.16, -0.5);
        double f = ra * Vt * qa;
        return (fabs(f) < 1e-14) ? 0.0 : f;
    };
    double fz_lo = 0.0;
    if (rain) {
        int64_t c0 = cidx(g, i, j, 0);
        fz_lo = flux(cons[c0], qp_of(c0));
    }
    for (int k = 0; k < nz; ++k) {
        int64_t c = cidx(g, i, j, k);
        double rho = cons[c];
        double rt = cons[N + c];
        double theta = rt / rho;
        double qv = cons[5 * N + c] / rho;
        double qc = cons[6 * N + c] / rho;
        double qp = qp_of(c);
        double tabs = eos_T(rho, rt, qv);
        double pres = eos_p(rt, qv) / 100.;
        if (rain) {
            double fz_hi;
            if (k == nz - 1) fz_hi = flux(rho, qp);
            else {
                int64_t cu = c + g.sk;
                fz_hi = flux(0.5 * (rho + cons[cu]), 0.5 * (qp + qp_of(cu)));
            }
            qv = fmax(0.0, qv); qc = fmax(0.0, qc); qp = fmax(0.0, qp);
            double es = esatw(tabs);
            double qs = Rd_on_Rv * es / fmax(es, pres - es);
            double dqs = Rd_on_Rv * dtesatw(tabs) / pres;
            if (qs <= 0.0) qs = 0.0;
            double d_c2r = 0.0, d_r2v = 0.0, d_v2c = 0.0, d_c2v = 0.0;
            double fac = 1.0 + (L_v / Cp_d) * dqs;
            if (qv > qs) d_v2c = fmin(qv, (qv - qs) / (1.0 + fac));
            if (qv < qs && qc > 0.0) d_c2v = fmin(qc, (qs - qv) / (1.0 + fac));
            if (qp > 0.0 && qv < qs) {
                double C = 1.6 + 124.9 * pow(0.001 * rho * qp, 0.2046);
                d_r2v = 1.0 / (0.001 * rho) * (1.0 - qv / qs) * C * pow(0.001 * rho * qp, 0.525) / (5.4e5 + 2.55e6 / (pres * qs)) * dtn;
                d_r2v = fmin(qp, d_r2v);
            }
            if (qc > 0.0) {
                double auto_r = (qc > 1.e-3) ? 1.e-3 : 0.0;
                double accrr = 2.2 * pow(qp, 0.875);
                d_c2r = dtn * (accrr * qc + auto_r * (qc - 1.e-3));
                d_c2r = fmin(d_c2r, qc);
            }
            double dq_sed = dtn * 1.0 * (1.0 / rho) * (fz_hi - fz_lo) / dz;
            if (fabs(dq_sed) < 1e-14) dq_sed = 0.0;
            qv += -d_v2c + d_c2v + d_r2v;
            qc += d_v2c - d_c2v - d_c2r;
            qp += dq_sed + d_c2r - d_r2v;
            theta += theta / tabs * fac_cond * (d_v2c - d_c2v - d_r2v);
            qv = fmax(0.0, qv); qc = fmax(0.0, qc); qp = fmax(0.0, qp);
            fz_lo = fz_hi;
        } else {
            qc = fmax(0.0, qc);
            double es = esatw(tabs);
            double qs = Rd_on_Rv * es / fmax(es, pres - es);
            double dqs = Rd_on_Rv * dtesatw(tabs) / pres;
            double d_v2c = 0.0, d_c2v = 0.0;
            double fac = 1.0 + (L_v / Cp_d) * dqs;
            if (qv > qs) d_v2c = fmin(qv, (qv - qs) / (1.0 + fac));
            if (qv < qs && qc > 0.0) d_c2v = fmin(qc, (qs - qv) / (1.0 + fac));
            qv += -d_v2c + d_c2v;
            qc += d_v2c - d_c2v;
            theta += theta / tabs * fac_cond * (d_v2c - d_c2v);
            qv = fmax(0.0, qv); qc = fmax(0.0, qc);
        }
        cons[N + c] = rho * theta;
        cons[5 * N + c] = rho * qv;
        cons[6 * N + c] = rho * qc;
        if (has_qp) cons[7 * N + c] = rho * qp;
    }
}

// ---------------------------------------------------------------------------
// Hydrostatic base state, one thread: calc_rho_p Newton integration at cell
// centres (ERF_InputSoundingData.H:176-256, ERF_HSE_utils.H:34-72) and
// erf_enforce_hse (ERF_init1d.cpp:152-260).  FP64, run once at set-up.
// ---------------------------------------------------------------------------
__global__ void k_base_state(int nz, double dz, double g, double rdOcp, const double* __restrict__ th_cc,
                             const double* __restrict__ qv_cc, double th_s, double qv_s, double p_s,
                             double* __restrict__ rho0, double* __restrict__ p0o, double* __restrict__ pi0o,
                             double* __restrict__ th0o) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double tol = 1.0e-12;
    const double RdOCp = R_d / Cp_d;
    double pm = p_s;
    double rd = eos_rho_given_theta_p(th_s, p_s, RdOCp, qv_s);
    double zprev = 0.0, qprev = qv_s;
    for (int k = 1; k <= nz; ++k) {
        double z = (k - 1 + 0.5) * dz;
        double th = th_cc[k - 1], qv = qv_cc[k - 1];
        double dzl = z - zprev;
        double rlo = rd * (1. + qprev);
        double C = -pm + 0.5 * rlo * g * dzl;
        double pk = pm;
        double rk = eos_rho_given_theta_p(th, pk, RdOCp, qv);
        double rhi = rk * (1. + qv);
        double F = pk + 0.5 * rhi * g * dzl + C;
        if (fabs(F) > tol) {
            int iter = 0;
            double eps = 1.0e-6, ieps = 1.0e6;
            do {
                double hi = eos_rho_given_theta_p(th, pk + eps, RdOCp, qv);
                double lo = eos_rho_given_theta_p(th, pk - eps, RdOCp, qv);
                double dFdp = 1.0 + 0.25 * ieps * (hi - lo) * g * dzl;
                pk -= F / dFdp;
                rk = eos_rho_given_theta_p(th, pk, RdOCp, qv);
                double rt = rk * (1. + qv);
                F = pk + 0.5 * rt * g * dzl + C;
                ++iter;
            } while (fabs(F) > tol && iter < 30);
        }
        rho0[k] = rk;
        pm = pk; rd = rk; zprev = z; qprev = qv;
    }
    rho0[0] = rho0[1];
    rho0[nz + 1] = rho0[nz];
    double hz = 0.5 * dz;
    p0o[1] = p_0 - hz * rho0[1] * g;
    pi0o[1] = eos_exner_p(p0o[1], rdOcp);
    th0o[1] = eos_rt_given_p(p0o[1]) / rho0[1];
    p0o[0] = p_0 + hz * rho0[1] * g;
    pi0o[0] = eos_exner_p(p0o[0], rdOcp);
    th0o[0] = eos_rt_given_p(p0o[0]) / rho0[0];
    for (int k = 1; k <= nz; ++k) {
        int kk = k + 1;
        double di = 0.5 * (rho0[kk] + rho0[kk - 1]);
        p0o[kk] = p0o[kk - 1] - dz * di * g;
        pi0o[kk] = eos_exner_p(p0o[kk], rdOcp);
        th0o[kk] = eos_rt_given_p(p0o[kk]) / rho0[kk];
    }
}

// ---------------------------------------------------------------------------
// Layout conversion between a caller's Array4 view and the internal arrays.
// kind: 0 cell, 1 x-face, 2 y-face, 3 z-face.  Unpack writes the caller's
// valid region and every ghost cell the view covers (periodic laterally,
// wall conditions vertically).
// ---------------------------------------------------------------------------
__global__ void k_pack(Geo g, erf_b200_fab f, int kind, int ncomp, double* __restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z;
    int nzk = (kind == 3) ? g.nz + 1 : g.nz;
    if (i >= g.nx || j >= g.ny || k >= nzk) return;
    int64_t src0 = (int64_t)(i - f.lo[0]) + (int64_t)(j - f.lo[1]) * f.jstride + (int64_t)(k - f.lo[2]) * f.kstride;
    int64_t per = (kind == 3) ? g.nzf : g.ncell;
    for (int n = 0; n < ncomp; ++n) dst[n * per + cidx(g, i, j, k)] = f.p[src0 + n * f.nstride];
}

__global__ void k_unpack(Geo g, erf_b200_fab f, int kind, int ncomp, const double* __restrict__ src,
                         int tang_lo_zero, int tang_hi_zero) {
    // thread over the caller's whole box
    int64_t nxb = f.hi[0] - f.lo[0] + 1, nyb = f.hi[1] - f.lo[1] + 1;
    int ib = blockIdx.x * blockDim.x + threadIdx.x;
    int jb = blockIdx.y * blockDim.y + threadIdx.y;
    int kb = blockIdx.z;
    if (ib >= nxb || jb >= nyb || kb > f.hi[2] - f.lo[2]) return;
    int i = f.lo[0] + ib, j = f.lo[1] + jb, k = f.lo[2] + kb;
    int64_t dst0 = (int64_t)ib + (int64_t)jb * f.jstride + (int64_t)kb * f.kstride;
    int64_t per = (kind == 3) ? g.nzf : g.ncell;
    int ii = ((i % g.nx) + g.nx) % g.nx, jj = ((j % g.ny) + g.ny) % g.ny;
    for (int n = 0; n < ncomp; ++n) {
        double val;
        if (kind == 3) {
            if (k <= 0 || k >= g.nz) val = 0.0;  // walls (and beyond): w = 0
            else val = src[n * per + cidx(g, ii, jj, k)];
        } else if (k < 0 || k >= g.nz) {
            bool lo = k < 0;
            int ks = lo ? 0 : g.nz - 1;
            bool zero = (kind == 1 || kind == 2) && (lo ? tang_lo_zero : tang_hi_zero);
            val = zero ? 0.0 : src[n * per + cidx(g, ii, jj, ks)];
        } else {
            val = src[n * per + cidx(g, ii, jj, k)];
        }
        f.p[dst0 + n * f.nstride] = val;
    }
}

}  // namespace erfb

namespace erfb {

// ---------------------------------------------------------------------------
// Tile layout shared by the two vertical kernels below: a block owns TX
// adjacent columns (i = blockIdx.x*TX + threadIdx.x, j = blockIdx.y) and
// blockDim.y warps split the levels; per-column data live in shared memory as
// [level][column] so a warp touches consecutive banks.
// ---------------------------------------------------------------------------
struct Tile {
    int i, j, lane, w, nw, tx;
    bool ok;
    __device__ Tile(const Geo& g) {
        tx = blockDim.x; lane = threadIdx.x; w = threadIdx.y; nw = blockDim.y;
        i = blockIdx.x * tx + lane; j = blockIdx.y;
        ok = i < g.nx;
    }
};

// ---------------------------------------------------------------------------
// Fast coefficients of one RK stage (make_fast_coeffs,
// TimeIntegration/ERF_make_fast_coeffs.cpp:160-290, no terrain): P and Q
// (divided by 1+q when moist), A, B, C on interior z-faces, Dirichlet rows at
// the walls, then the Thomas forward elimination of B.  Stored per face:
// A, 1/B' (B' at the wall rows, which the reference leaves uninverted),
// C/B', P, Q.  Levels are computed in parallel; the B' recurrence runs in one
// warp from shared memory.
// ---------------------------------------------------------------------------
__global__ void k_fast_coef(Params P, double D, StateBuf Sst, StageAux A, double* __restrict__ cA,
                            double* __restrict__ cInvB, double* __restrict__ cCB, double* __restrict__ cP,
                            double* __restrict__ cQ) {
    extern __shared__ double sm[];
    const Geo& g = P.g;
    Tile t(g);
    const int nz = g.nz, TX = t.tx;
    double* sA = sm;
    double* sB = sA + (nz + 1) * TX;
    double* sC = sB + (nz + 1) * TX;
    const int64_t N = g.ncell;
    const double dzi = g.dzi, halfg = P.halfg;
    const double* th = A.prim;
    if (t.ok) {
        for (int k = 1 + t.w; k <= nz - 1; k += t.nw) {
            int64_t c = cidx(g, t.i, t.j, k), cm = c - g.sk;
            double pi_c = 0.5 * (A.pi[cm] + A.pi[c]);
            double P_ = -Gamma_ * R_d * dzi + halfg * R_d * P.r0[k + 1] / (P.c_v * P.pi0[k + 1] * Sst.cons[N + c]);
            P_ *= pi_c;
            double Q_ = Gamma_ * R_d * dzi + halfg * R_d * P.r0[k] / (P.c_v * P.pi0[k] * Sst.cons[N + cm]);
            Q_ *= pi_c;
            if (P.moist) {
                double q = 0.5 * (th[4 * N + c] + th[4 * N + cm] + th[5 * N + c] + th[5 * N + cm]);
                P_ /= (1.0 + q);
                Q_ /= (1.0 + q);
            }
            double tlo = 0.5 * (th[cidx(g, t.i, t.j, clampk(k - 2, nz))] + th[cm]);
            double tmid = 0.5 * (th[cm] + th[c]);
            double thi = 0.5 * (th[c] + th[cidx(g, t.i, t.j, clampk(k + 1, nz))]);
            double a = D * (halfg - Q_ * tlo);
            double cc = D * (-halfg + P_ * thi);
            double b = 1.0 + D * (Q_ - P_) * tmid;
            sA[k * TX + t.lane] = a; sB[k * TX + t.lane] = b; sC[k * TX + t.lane] = cc;
            cA[c] = a; cP[c] = P_; cQ[c] = Q_;
        }
        if (t.w == 0) {
            for (int k : {0, nz}) {
                sA[k * TX + t.lane] = 0.0; sB[k * TX + t.lane] = 1.0; sC[k * TX + t.lane] = 0.0;
                int64_t f = cidx(g, t.i, t.j, k);
                cA[f] = 0.0; cP[f] = 0.0; cQ[f] = 0.0;
            }
        }
    }
    __syncthreads();
    if (t.w == 0 && t.ok) {
        double bet = sB[t.lane];
        int64_t f0 = cidx(g, t.i, t.j, 0);
        cInvB[f0] = bet;               // B at the bottom row stays uninverted (== 1)
        cCB[f0] = sC[t.lane] * bet;
        for (int k = 1; k <= nz; ++k) {
            double gam = sC[(k - 1) * TX + t.lane] / bet;
            bet = sB[k * TX + t.lane] - sA[k * TX + t.lane] * gam;
            if (!(fabs(bet) > 1e-300)) atomicOr(P.status, ST_BADSTATE);
            double inv = (k < nz) ? 1.0 / bet : bet;
            int64_t f = cidx(g, t.i, t.j, k);
            cInvB[f] = inv;
            cCB[f] = sC[k * TX + t.lane] * inv;
        }
    }
}

// ---------------------------------------------------------------------------
// Acoustic substep, vertical part (erf_fast_rhs_N, ERF_fast_rhs_N.cpp:259-592):
//   phase 1  horizontal rho / rho*theta fluxes from the new U'', V'' per cell;
//   phase 2  right-hand side of the implicit w system per face, and
//            d(rho w) of the previous solution;
//   phase 3  Thomas forward / back substitution (one warp; FMA only, the
//            stage's 1/B' and C/B' come from k_fast_coef);
//   phase 4  vertical fluxes, average z-momentum, rho and rho*theta update.
// All reads of the previous state happen in phases 1-2, before any write,
// because the previous and new states may be the same buffers.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_fast_vert(Params P, double dtau, double facinv, double beta_1, double beta_2, StateBuf Sprev,
                            int prev_rt, StateBuf Sst, StageAux A, const double* __restrict__ Fcons,
                            const double* __restrict__ Fmz, const double* __restrict__ newx,
                            const double* __restrict__ newy, const double* __restrict__ cA,
                            const double* __restrict__ cInvB, const double* __restrict__ cCB,
                            const double* __restrict__ cP, const double* __restrict__ cQ, double* __restrict__ avz,
                            double* out_cons, double* out_mz) {
    extern __shared__ double sm[];
    const Geo& g = P.g;
    Tile t(g);
    const int nz = g.nz, TX = t.tx, L = t.lane;
    double* sT0 = sm;
    double* sT1 = sT0 + nz * TX;
    double* sR = sT1 + nz * TX;
    double* sD = sR + (nz + 1) * TX;
    double* sA = sD + (nz + 1) * TX;
    double* sI = sA + (nz + 1) * TX;
    double* sCB = sI + (nz + 1) * TX;
    const int64_t N = g.ncell;
    const double dzi = g.dzi, halfg = P.halfg;
    const double* th = A.prim;
    const int i = t.i, j = t.j;
    int ip = 0, im = 0, jp = 0, jm = 0;
    if (t.ok) { ip = wrap(i + 1, g.nx); im = wrap(i - 1, g.nx); jp = wrap(j + 1, g.ny); jm = wrap(j - 1, g.ny); }
    auto prev_mz = [&](int k) {
        int64_t f = cidx(g, i, j, k);
        double m = Sprev.mz[f];
        if (prev_rt) {
            if (k == 0 || k == nz) return 0.0;
            double rs = Sprev.cons[f] + Sprev.cons[f - g.sk];
            double wt = (m * 2.0) / rs;
            m = (wt * 0.5) * rs;
        }
        return m;
    };
    auto thz = [&](int k) { return th[cidx(g, i, j, clampk(k, nz))]; };
    // ---- phase 1
    if (t.ok) {
        for (int k = t.w; k < nz; k += t.nw) {
            int64_t c = cidx(g, i, j, k);
            double xl = (newx[c] - Sst.mx[c]) / 1.0;
            double xh = (newx[cidx(g, ip, j, k)] - Sst.mx[cidx(g, ip, j, k)]) / 1.0;
            double yl = (newy[c] - Sst.my[c]) / 1.0;
            double yh = (newy[cidx(g, i, jp, k)] - Sst.my[cidx(g, i, jp, k)]) / 1.0;
            double mfsq = 1.0;
            double tc = th[c];
            sT0[k * TX + L] = (xh - xl) * g.dxi * mfsq + (yh - yl) * g.dyi * mfsq;
            sT1[k * TX + L] = ((xh * (tc + th[cidx(g, ip, j, k)]) - xl * (tc + th[cidx(g, im, j, k)])) * g.dxi * mfsq +
                               (yh * (tc + th[cidx(g, i, jp, k)]) - yl * (tc + th[cidx(g, i, jm, k)])) * g.dyi * mfsq) * 0.5;
        }
    }
    __syncthreads();
    // ---- phase 2
    if (t.ok) {
        for (int k = t.w; k <= nz; k += t.nw) {
            int64_t f = cidx(g, i, j, k);
            double Ok = prev_mz(k) - Sst.mz[f];
            sD[k * TX + L] = Ok;
            sA[k * TX + L] = cA[f];
            sI[k * TX + L] = cInvB[f];
            sCB[k * TX + L] = cCB[f];
            double rhs;
            if (k == 0 || k == nz) {
                rhs = Ok + dtau * Fmz[f];
            } else {
                int64_t cm = f - g.sk;
                double Okp1 = prev_mz(k + 1) - Sst.mz[f + g.sk];
                double Okm1 = prev_mz(k - 1) - Sst.mz[cm];
                double cPk = cP[f], cQk = cQ[f];
                double tlo = 0.5 * (thz(k - 2) + thz(k - 1));
                double tmid = 0.5 * (thz(k - 1) + thz(k));
                double thi = 0.5 * (thz(k) + thz(k + 1));
                double drt_k = Sprev.cons[N + f] - Sst.cons[N + f];
                double drt_km = Sprev.cons[N + cm] - Sst.cons[N + cm];
                double odk = Sprev.cons[f] - Sst.cons[f];
                double odkm = Sprev.cons[cm] - Sst.cons[cm];
                double R0 = cPk * drt_k + cQk * drt_km - halfg * (odk + odkm);
                double R1 = halfg * (-Fcons[f] - Fcons[cm] + sT0[k * TX + L] + sT0[(k - 1) * TX + L]) +
                            (cPk * (Fcons[N + f] - sT1[k * TX + L]) + cQk * (Fcons[N + cm] - sT1[(k - 1) * TX + L]));
                R1 += beta_1 * dzi * ((Okp1 - Okm1) * halfg - (Okp1 * thi - Ok * tmid) * cPk - (Ok * tmid - Okm1 * tlo) * cQk);
                rhs = Ok + dtau * (Fmz[f] + R0 + dtau * beta_2 * R1);
            }
            sR[k * TX + L] = rhs;
        }
    }
    __syncthreads();
    // ---- phase 3: tridiagonal solve, one warp
    if (t.w == 0 && t.ok) {
        double s = sR[L] * sI[L];
        sR[L] = s;
        for (int k = 1; k <= nz; ++k) {
            s = (sR[k * TX + L] - sA[k * TX + L] * s) * sI[k * TX + L];
            sR[k * TX + L] = s;
        }
        for (int k = nz - 1; k >= 0; --k) {
            s = sR[k * TX + L] - sCB[k * TX + L] * s;
            sR[k * TX + L] = s;
        }
    }
    __syncthreads();
    // ---- phase 4
    if (t.ok) {
        for (int k = t.w; k < nz; k += t.nw) {
            int64_t c = cidx(g, i, j, k);
            double sol = sR[k * TX + L], sol_hi = sR[(k + 1) * TX + L];
            double zl = beta_2 * sol + beta_1 * sD[k * TX + L];
            double zh = beta_2 * sol_hi + beta_1 * sD[(k + 1) * TX + L];
            avz[c] += facinv * zl / (1.0 * 1.0);
            if (k == nz - 1) avz[c + g.sk] += facinv * zh / (1.0 * 1.0);
            double tc = th[c];
            double t0 = sT0[k * TX + L] + dzi * (zh - zl);
            double t1 = sT1[k * TX + L] + 0.5 * dzi * (zh * (tc + thz(k + 1)) - zl * (tc + thz(k - 1)));
            double pr = Sprev.cons[c], prt = Sprev.cons[N + c];
            out_cons[c] = pr + dtau * (Fcons[c] - t0);
            out_cons[N + c] = prt + dtau * (Fcons[N + c] - t1);
            double smz = Sst.mz[c];
            out_mz[c] = smz + sol;
            if (k == nz - 1) out_mz[c + g.sk] = Sst.mz[c + g.sk] + sol_hi;
        }
    }
}

// ---------------------------------------------------------------------------
// Kessler, one thread per cell: the fall fluxes through the cell's bottom and
// top faces are evaluated from the pre-update neighbours, so cells are
// independent (same arithmetic as k_kessler).
// ---------------------------------------------------------------------------
__global__ void k_kessler_cells(Params P, const double* __restrict__ cin, double* __restrict__ cout, double dtn,
                                double dz) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    const int64_t N = g.ncell;
    const int nz = g.nz;
    const bool rain = P.kessler_rain;
    const bool has_qp = P.ncomp > 7;
    const double fac_cond = lcond / P.c_p;
    int64_t c = cidx(g, i, j, k);
    auto qp_of = [&](int64_t cc) { return has_qp ? cin[7 * N + cc] / cin[cc] : 0.0; };
    auto flux = [&](double ra, double qa) {
        qa = fmax(0.0, qa);
        double Vt = 36.34 * pow(ra * 0.001 * qa, 0.1346) * pow(ra / 1.16, -0.5);
        double f = ra * Vt * qa;
        return (fabs(f) < 1e-14) ? 0.0 : f;
    };
    double rho = cin[c];
    double rt = cin[N + c];
    double theta = rt / rho;
    double qv = cin[5 * N + c] / rho;
    double qc = cin[6 * N + c] / rho;
    double qp = qp_of(c);
    double tabs = eos_T(rho, rt, qv);
    double pres = eos_p(rt, qv) / 100.;
    if (rain) {
        double fz_lo, fz_hi;
        if (k == 0) fz_lo = flux(rho, qp);
        else fz_lo = flux(0.5 * (cin[c - g.sk] + rho), 0.5 * (qp_of(c - g.sk) + qp));
        if (k == nz - 1) fz_hi = flux(rho, qp);
        else fz_hi = flux(0.5 * (rho + cin[c + g.sk]), 0.5 * (qp + qp_of(c + g.sk)));
        qv = fmax(0.0, qv); qc = fmax(0.0, qc); qp = fmax(0.0, qp);
        double es = esatw(tabs);
        double qs = Rd_on_Rv * es / fmax(es, pres - es);
        double dqs = Rd_on_Rv * dtesatw(tabs) / pres;
        if (qs <= 0.0) qs = 0.0;
        double d_c2r = 0.0, d_r2v = 0.0, d_v2c = 0.0, d_c2v = 0.0;
        double fac = 1.0 + (L_v / Cp_d) * dqs;
        if (qv > qs) d_v2c = fmin(qv, (qv - qs) / (1.0 + fac));
        if (qv < qs && qc > 0.0) d_c2v = fmin(qc, (qs - qv) / (1.0 + fac));
        if (qp > 0.0 && qv < qs) {
            double C = 1.6 + 124.9 * pow(0.001 * rho * qp, 0.2046);
            d_r2v = 1.0 / (0.001 * rho) * (1.0 - qv / qs) * C * pow(0.001 * rho * qp, 0.525) / (5.4e5 + 2.55e6 / (pres * qs)) * dtn;
            d_r2v = fmin(qp, d_r2v);
        }
        if (qc > 0.0) {
            double auto_r = (qc > 1.e-3) ? 1.e-3 : 0.0;
            double accrr = 2.2 * pow(qp, 0.875);
            d_c2r = dtn * (accrr * qc + auto_r * (qc - 1.e-3));
            d_c2r = fmin(d_c2r, qc);
        }
        double dq_sed = dtn * 1.0 * (1.0 / rho) * (fz_hi - fz_lo) / dz;
        if (fabs(dq_sed) < 1e-14) dq_sed = 0.0;
        qv += -d_v2c + d_c2v + d_r2v;
        qc += d_v2c - d_c2v - d_c2r;
        qp += dq_sed + d_c2r - d_r2v;
        theta += theta / tabs * fac_cond * (d_v2c - d_c2v - d_r2v);
        qv = fmax(0.0, qv); qc = fmax(0.0, qc); qp = fmax(0.0, qp);
    } else {
        qc = fmax(0.0, qc);
        double es = esatw(tabs);
        double qs = Rd_on_Rv * es / fmax(es, pres - es);
        double dqs = Rd_on_Rv * dtesatw(tabs) / pres;
        double d_v2c = 0.0, d_c2v = 0.0;
        double fac = 1.0 + (L_v / Cp_d) * dqs;
        if (qv > qs) d_v2c = fmin(qv, (qv - qs) / (1.0 + fac));
        if (qv < qs && qc > 0.0) d_c2v = fmin(qc, (qs - qv) / (1.0 + fac));
        qv += -d_v2c + d_c2v;
        qc += d_v2c - d_c2v;
        theta += theta / tabs * fac_cond * (d_v2c - d_c2v);
        qv = fmax(0.0, qv); qc = fmax(0.0, qc);
    }
    for (int n = 0; n < P.ncomp; ++n) cout[n * N + c] = cin[n * N + c];
    cout[N + c] = rho * theta;
    cout[5 * N + c] = rho * qv;
    cout[6 * N + c] = rho * qc;
    if (has_qp) cout[7 * N + c] = rho * qp;
}

}  // namespace erfb

namespace erfb {

// ---------------------------------------------------------------------------
// Scalar and momentum transport on x-y tiles marching up in k.  A block owns
// TTX x TTY columns and `kz` consecutive levels.  At each level every thread
// evaluates the advective flux through its cell's low x and y faces into
// shared memory (the tile's high edge also evaluates the high faces) and
// carries the flux through its top face to the next level, so each face flux
// is evaluated once per block.  All fluxes of one level are staged before a
// single barrier.  `kz` is chosen on the host so that the whole grid is one
// wave of resident blocks.
// Divergence as in AdvectionSrcForScalars (ERF_AdvectionSrcForState.cpp:359-370).
// ---------------------------------------------------------------------------
// Minimum resident blocks per SM requested from the register allocator for
// each tiled kernel (trades instruction-level for warp-level parallelism).
#ifndef ERFB_MINB_CELL
#define ERFB_MINB_CELL 4
#endif
#ifndef ERFB_MINB_MOM
#define ERFB_MINB_MOM 4
#endif
#ifndef ERFB_MINB_POST
#define ERFB_MINB_POST 4
#endif

struct FluxTile {
    double fx[TTY][TTX + 1];
    double fy[TTY + 1][TTX];
};

// Fluxes of one scalar for cell (i,j,k): x/y into the tile, z through zl/zh
// (zl is computed only on the block's first level; otherwise it is the
// carried top flux of the level below).
template <int TH, int TV>
__device__ __forceinline__ void tile_put(const Geo& g, FluxTile& t, const double* __restrict__ phi,
                                         const double* __restrict__ ax, const double* __restrict__ ay,
                                         const double* __restrict__ az, int th, int tv, double fh, double fv, int i,
                                         int j, int k, bool first, double& zl, double& zh) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    t.fx[ty][tx] = adv_flux_x<TH>(g, phi, ax, th, fh, i, j, k);
    if (tx == TTX - 1 || i == g.nx - 1) t.fx[ty][tx + 1] = adv_flux_x<TH>(g, phi, ax, th, fh, wrap(i + 1, g.nx), j, k);
    t.fy[ty][tx] = adv_flux_y<TH>(g, phi, ay, th, fh, i, j, k);
    if (ty == TTY - 1 || j == g.ny - 1) t.fy[ty + 1][tx] = adv_flux_y<TH>(g, phi, ay, th, fh, i, wrap(j + 1, g.ny), k);
    if (first) zl = adv_flux_z<TV>(g, phi, az, tv, fv, i, j, k);
    zh = adv_flux_z<TV>(g, phi, az, tv, fv, i, j, k + 1);
}
__device__ __forceinline__ double tile_div(const Geo& g, const FluxTile& t, double zl, double zh) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    return -1.0 * 1.0 * ((t.fx[ty][tx + 1] - t.fx[ty][tx]) * g.dxi + (t.fy[ty + 1][tx] - t.fy[ty][tx]) * g.dyi +
                         (zh - zl) * g.dzi);
}

// ---------------------------------------------------------------------------
// Slow RHS for rho and rho*theta (erf_slow_rhs_pre cell part,
// ERF_slow_rhs_pre.cpp:462-526): AdvectionSrcForRho (also initialises the
// average momenta to the stage mass fluxes, ERF_AdvectionSrcForState.cpp:56-71),
// AdvectionSrcForScalars for theta with the dycore scheme
// (ERF_slow_rhs_pre.cpp:139-142, 469-477), DiffusionSrcForState_N for theta.
// ---------------------------------------------------------------------------
template <int TH, int TV>
__global__ void __launch_bounds__(TTX * TTY, ERFB_MINB_CELL) k_slow_cell(Params P, int kz, StateBuf S, StageAux A,
                                                         const double* __restrict__ mut, double* __restrict__ Fcons,
                                                         double* __restrict__ avx, double* __restrict__ avy,
                                                         double* __restrict__ avz) {
    __shared__ FluxTile sh;
    const Geo& g = P.g;
    const int i = blockIdx.x * TTX + threadIdx.x, j = blockIdx.y * TTY + threadIdx.y;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const int ip = ok ? wrap(i + 1, g.nx) : 0, jp = ok ? wrap(j + 1, g.ny) : 0;
    double zl = 0.0, zh = 0.0;
    for (int k = k0; k < k1; ++k) {
        if (ok)
            tile_put<TH, TV>(g, sh, A.prim, S.mx, S.my, S.mz, P.dyc_h, P.dyc_v, P.f_dyc_h, P.f_dyc_v, i, j, k,
                             k == k0, zl, zh);
        __syncthreads();
        if (ok) {
            double frt = tile_div(g, sh, zl, zh);
            zl = zh;
            int64_t c = cidx(g, i, j, k);
            avx[c] = S.mx[c];
            avy[c] = S.my[c];
            avz[c] = S.mz[c];
            if (k == g.nz - 1) avz[c + g.sk] = S.mz[c + g.sk];
            Fcons[c] = -1.0 / 1.0 * ((S.mx[cidx(g, ip, j, k)] - S.mx[c]) * g.dxi +
                                     (S.my[cidx(g, i, jp, k)] - S.my[c]) * g.dyi + (S.mz[c + g.sk] - S.mz[c]) * g.dzi);
            if (P.use_diff) frt -= scalar_diff(P, S.cons, A.prim, mut, P.alphaT_eff, P.invPr, i, j, k);
            Fcons[g.ncell + c] = frt;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Slow RHS post + stage finalisation (erf_slow_rhs_post,
// ERF_slow_rhs_post.cpp:228-531, and post_update = apply_bcs(S_new),
// ERF_TI_slow_rhs_fun.H:284-288):
//   * advection (average momenta) and diffusion of the slow scalars
//     (passive scalar with the dry-scalar scheme; moisture with the moist
//     scheme), S_new = S_old + slow_dt * RHS, moisture clipped at 0;
//   * rho, rho*theta and the momenta copied from the fast solution, with the
//     momentum/velocity round trips of the two boundary fills;
//   * the stage velocities, and (unless last) the next stage's primitive
//     variables, Exner function and p'.
// ---------------------------------------------------------------------------
constexpr int MAX_SLOW = 4;  // passive scalar + up to three moisture species
template <int DH, int DV, int MH, int MV>
__global__ void __launch_bounds__(TTX * TTY, ERFB_MINB_POST) k_post(Params P, int kz, double slow_dt, StateBuf Sold, StateBuf Sst,
                                                    StateBuf Ssum, StateBuf Snew, StageAux Acur, StageAux Anext,
                                                    int make_next, const double* __restrict__ mut,
                                                    const double* __restrict__ avx, const double* __restrict__ avy,
                                                    const double* __restrict__ avz, double* __restrict__ un,
                                                    double* __restrict__ vn, double* __restrict__ wn) {
    __shared__ FluxTile sh[MAX_SLOW];
    const Geo& g = P.g;
    const int64_t N = g.ncell;
    const int i = blockIdx.x * TTX + threadIdx.x, j = blockIdx.y * TTY + threadIdx.y;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const int im = ok ? wrap(i - 1, g.nx) : 0, jm = ok ? wrap(j - 1, g.ny) : 0;
    const int nslow = P.moist ? 1 + (P.ncomp - ERF_RHOQ1_COMP) : 1;
    double zl[MAX_SLOW], zh[MAX_SLOW];
#pragma unroll
    for (int q = 0; q < MAX_SLOW; ++q) zl[q] = zh[q] = 0.0;
    for (int k = k0; k < k1; ++k) {
        if (ok) {
#pragma unroll
            for (int q = 0; q < MAX_SLOW; ++q) {
                if (q >= nslow) break;
                if (q == 0)
                    tile_put<DH, DV>(g, sh[0], Acur.prim + (int64_t)(ERF_RHOSCALAR_COMP - 1) * N, avx, avy, avz,
                                     P.dry_h, P.dry_v, P.f_dry_h, P.f_dry_v, i, j, k, k == k0, zl[0], zh[0]);
                else
                    tile_put<MH, MV>(g, sh[q], Acur.prim + (int64_t)(ERF_RHOQ1_COMP + q - 2) * N, avx, avy, avz,
                                     P.moi_h, P.moi_v, P.f_moi_h, P.f_moi_v, i, j, k, k == k0, zl[q], zh[q]);
            }
        }
        __syncthreads();
        if (ok) {
            int64_t c = cidx(g, i, j, k);
#pragma unroll
            for (int q = 0; q < MAX_SLOW; ++q) {
                if (q >= nslow) break;
                int n = (q == 0) ? ERF_RHOSCALAR_COMP : ERF_RHOQ1_COMP + q - 1;
                double r = tile_div(g, sh[q], zl[q], zh[q]);
                zl[q] = zh[q];
                if (P.use_diff)
                    r -= scalar_diff(P, Sst.cons, Acur.prim + (int64_t)(n - 1) * N, mut, P.alphaC_eff, P.invSc, i, j, k);
                double v_ = Sold.cons[n * N + c] + slow_dt * r;
                Snew.cons[n * N + c] = (q == 0) ? v_ : fmax(v_, 0.0);
            }
            Snew.cons[c] = Ssum.cons[c];
            Snew.cons[N + c] = Ssum.cons[N + c];
            Snew.cons[2 * N + c] = Sst.cons[2 * N + c];
            Snew.cons[3 * N + c] = Sst.cons[3 * N + c];
            double rho = Ssum.cons[c];
            {
                double rs = rho + Ssum.cons[cidx(g, im, j, k)];
                double m = Ssum.mx[c];
                double u1 = (m * 2.0) / rs; m = (u1 * 0.5) * rs;
                double u2 = (m * 2.0) / rs; m = (u2 * 0.5) * rs;
                Snew.mx[c] = m; un[c] = u2;
            }
            {
                double rs = rho + Ssum.cons[cidx(g, i, jm, k)];
                double m = Ssum.my[c];
                double v1 = (m * 2.0) / rs; m = (v1 * 0.5) * rs;
                double v2 = (m * 2.0) / rs; m = (v2 * 0.5) * rs;
                Snew.my[c] = m; vn[c] = v2;
            }
            if (k == 0) {
                Snew.mz[c] = 0.0; wn[c] = 0.0;
            } else {
                double rs = rho + Ssum.cons[c - g.sk];
                double m = Ssum.mz[c];
                double w1 = (m * 2.0) / rs; m = (w1 * 0.5) * rs;
                double w2 = (m * 2.0) / rs; m = (w2 * 0.5) * rs;
                Snew.mz[c] = m; wn[c] = w2;
            }
            if (k == g.nz - 1) { Snew.mz[c + g.sk] = 0.0; wn[c + g.sk] = 0.0; }
            if (make_next) stage_aux_cell(P, Snew.cons, Anext, c, k);
        }
        __syncthreads();
    }
}

// Momentum fluxes of AdvectionSrcFor{X,Y,Z}Mom_N (ERF_AdvectionSrcForMom_N.H:
// 17-274).  Each is the flux through the low side of the face's control
// volume in one direction; the high side is the same function one index up.
template <int HT>
__device__ __forceinline__ double xmom_flux_x(const Params& P, const double* ru, const double* u, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (ru[cidx(g, wrap(i - 1, g.nx), j, k)] + ru[cidx(g, i, j, k)]);
    return a * gatherx_interp<HT>(g, u, P.dyc_h, a, P.f_dyc_h, i, j, k);
}
template <int HT>
__device__ __forceinline__ double xmom_flux_y(const Params& P, const double* rv, const double* u, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (rv[cidx(g, i, j, k)] + rv[cidx(g, wrap(i - 1, g.nx), j, k)]);
    return a * gathery_interp<HT>(g, u, P.dyc_h, a, P.f_dyc_h, i, j, k);
}
template <int VT>
__device__ __forceinline__ double xmom_flux_z(const Params& P, const double* rw, const double* u, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (rw[cidx(g, i, j, k)] + rw[cidx(g, wrap(i - 1, g.nx), j, k)]);
    return a * gatherz_tang<VT>(g, u, P.dyc_v, a, P.f_dyc_v, i, j, k);
}
template <int HT>
__device__ __forceinline__ double ymom_flux_x(const Params& P, const double* ru, const double* v, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (ru[cidx(g, i, j, k)] + ru[cidx(g, i, wrap(j - 1, g.ny), k)]);
    return a * gatherx_interp<HT>(g, v, P.dyc_h, a, P.f_dyc_h, i, j, k);
}
template <int HT>
__device__ __forceinline__ double ymom_flux_y(const Params& P, const double* rv, const double* v, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (rv[cidx(g, i, j, k)] + rv[cidx(g, i, wrap(j - 1, g.ny), k)]);
    return a * gathery_interp<HT>(g, v, P.dyc_h, a, P.f_dyc_h, i, j, k);
}
template <int VT>
__device__ __forceinline__ double ymom_flux_z(const Params& P, const double* rw, const double* v, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (rw[cidx(g, i, j, k)] + rw[cidx(g, i, wrap(j - 1, g.ny), k)]);
    return a * gatherz_tang<VT>(g, v, P.dyc_v, a, P.f_dyc_v, i, j, k);
}
template <int HT>
__device__ __forceinline__ double zmom_flux_x(const Params& P, const double* ru, const double* w, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (ru[cidx(g, i, j, k)] + ru[cidx(g, i, j, k - 1)]) * 1.0;
    return a * gatherx_interp<HT>(g, w, P.dyc_h, a, P.f_dyc_h, i, j, k);
}
template <int HT>
__device__ __forceinline__ double zmom_flux_y(const Params& P, const double* rv, const double* w, int i, int j, int k) {
    const Geo& g = P.g;
    double a = 0.5 * (rv[cidx(g, i, j, k)] + rv[cidx(g, i, j, k - 1)]) * 1.0;
    return a * gathery_interp<HT>(g, w, P.dyc_h, a, P.f_dyc_h, i, j, k);
}
// Vertical flux of w between faces kk-1 and kk (the "lo" flux of face kk),
// with the order reduction next to the walls (ERF_AdvectionSrcForMom_N.H:
// 220-265); for kk == nz it is the "hi" flux of the top interior face,
// which the reference takes centred.
template <int VT>
__device__ __forceinline__ double zmom_flux_z(const Params& P, const double* rw, const double* w, int i, int j, int kk) {
    const Geo& g = P.g;
    const int vt = P.dyc_v, lo_z_face = 0, hi_z_face = g.nz;
    const double vf = P.f_dyc_v;
    auto wz = [&](int q) { return __ldg(w + cidx(g, i, j, q)); };
    auto all = [&](int q, double upw, double frac, int type) {
        double sv[6];
        bool wide = (type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH);
        sv[0] = wide ? wz(q - 3) : 0.0;
        sv[1] = (type == ERF_ADV_CENTERED_2ND) ? 0.0 : wz(q - 2);
        sv[2] = wz(q - 1);
        sv[3] = wz(q);
        sv[4] = (type == ERF_ADV_CENTERED_2ND) ? 0.0 : wz(q + 1);
        sv[5] = wide ? wz(q + 2) : 0.0;
        return interp_all(type, sv, upw, frac);
    };
    auto normal = [&](int q, double upw) {
        double sv[6];
        const int wd = width_of<VT>(vt);
        for (int m = 0; m < 6; ++m) {
            int off = m - 3;
            sv[m] = (off >= -wd && off <= wd - 1) ? wz(q + off) : 0.0;
        }
        return interp_of<VT>(vt, sv, upw, vf);
    };
    double a = 0.5 * (rw[cidx(g, i, j, kk)] + rw[cidx(g, i, j, kk - 1)]);
    double iv;
    if (kk == hi_z_face || kk == lo_z_face + 1) iv = all(kk, a, 0, ERF_ADV_CENTERED_2ND);
    else if (kk == lo_z_face + 2 || kk == hi_z_face - 1) {
        if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) iv = all(kk, a, 0, ERF_ADV_CENTERED_4TH);
        else iv = all(kk, a, vf, vt);
    } else iv = normal(kk, a);
    return a * iv;
}

// ---------------------------------------------------------------------------
// Slow RHS for the three momenta (erf_slow_rhs_pre face part,
// ERF_slow_rhs_pre.cpp:556-744): AdvectionSrcForMom (N), DiffusionSrcForMom_N,
// pressure gradient of p', buoyancy / Coriolis / geostrophic sources
// (make_mom_sources, make_buoyancy).  Same tiles as the scalar transport;
// the three momenta's x/y fluxes of a level are staged before one barrier.
// ---------------------------------------------------------------------------
template <int HT, int VT>
__global__ void __launch_bounds__(TTX * TTY, ERFB_MINB_MOM) k_slow_mom(Params P, int kz, StateBuf S, StageAux A,
                                                        const double* __restrict__ u, const double* __restrict__ v,
                                                        const double* __restrict__ w, const double* __restrict__ t11,
                                                        const double* __restrict__ t22, const double* __restrict__ t33,
                                                        const double* __restrict__ t12, const double* __restrict__ t13,
                                                        const double* __restrict__ t23, const double* __restrict__ pavg,
                                                        double* __restrict__ Fmx, double* __restrict__ Fmy,
                                                        double* __restrict__ Fmz) {
    __shared__ FluxTile sh[3];
    const Geo& g = P.g;
    const int64_t N = g.ncell;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * TTX + tx, j = blockIdx.y * TTY + ty;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const int im = ok ? wrap(i - 1, g.nx) : 0, jm = ok ? wrap(j - 1, g.ny) : 0;
    const int ip = ok ? wrap(i + 1, g.nx) : 0, jp = ok ? wrap(j + 1, g.ny) : 0;
    const bool xedge = ok && (tx == TTX - 1 || i == g.nx - 1);
    const bool yedge = ok && (ty == TTY - 1 || j == g.ny - 1);
    const double* ru = S.mx;
    const double* rv = S.my;
    const double* rw = S.mz;
    const double* cd = S.cons;
    const double* prim = A.prim;
    const double* pp = A.pp;
    double zlu = 0.0, zhu = 0.0, zlv = 0.0, zhv = 0.0, zlw = 0.0, zhw = 0.0;
    for (int k = k0; k < k1; ++k) {
        const int64_t c = ok ? cidx(g, i, j, k) : 0;
        const bool zk = ok && k >= 1;   // z-momentum on interior faces only
        if (ok) {
            sh[0].fx[ty][tx] = xmom_flux_x<HT>(P, ru, u, i, j, k);
            if (xedge) sh[0].fx[ty][tx + 1] = xmom_flux_x<HT>(P, ru, u, ip, j, k);
            sh[0].fy[ty][tx] = xmom_flux_y<HT>(P, rv, u, i, j, k);
            if (yedge) sh[0].fy[ty + 1][tx] = xmom_flux_y<HT>(P, rv, u, i, jp, k);
            if (k == k0) zlu = xmom_flux_z<VT>(P, rw, u, i, j, k);
            zhu = xmom_flux_z<VT>(P, rw, u, i, j, k + 1);
            sh[1].fx[ty][tx] = ymom_flux_x<HT>(P, ru, v, i, j, k);
            if (xedge) sh[1].fx[ty][tx + 1] = ymom_flux_x<HT>(P, ru, v, ip, j, k);
            sh[1].fy[ty][tx] = ymom_flux_y<HT>(P, rv, v, i, j, k);
            if (yedge) sh[1].fy[ty + 1][tx] = ymom_flux_y<HT>(P, rv, v, i, jp, k);
            if (k == k0) zlv = ymom_flux_z<VT>(P, rw, v, i, j, k);
            zhv = ymom_flux_z<VT>(P, rw, v, i, j, k + 1);
        }
        if (zk) {
            sh[2].fx[ty][tx] = zmom_flux_x<HT>(P, ru, w, i, j, k);
            if (xedge) sh[2].fx[ty][tx + 1] = zmom_flux_x<HT>(P, ru, w, ip, j, k);
            sh[2].fy[ty][tx] = zmom_flux_y<HT>(P, rv, w, i, j, k);
            if (yedge) sh[2].fy[ty + 1][tx] = zmom_flux_y<HT>(P, rv, w, i, jp, k);
            if (k == k0 || k == 1) zlw = zmom_flux_z<VT>(P, rw, w, i, j, k);
            zhw = zmom_flux_z<VT>(P, rw, w, i, j, k + 1);
        }
        __syncthreads();
        // ---------------- x-momentum on face i
        if (ok) {
            double rhs = -((sh[0].fx[ty][tx + 1] - sh[0].fx[ty][tx]) * g.dxi * 1.0 +
                           (sh[0].fy[ty + 1][tx] - sh[0].fy[ty][tx]) * g.dyi * 1.0 + (zhu - zlu) * g.dzi);
            zlu = zhu;
            if (P.use_diff)
                rhs -= ((t11[c] - t11[cidx(g, im, j, k)]) * g.dxi * 1.0 + (t12[cidx(g, i, jp, k)] - t12[c]) * g.dyi * 1.0 +
                        (t13[c + g.sk] - t13[c]) * g.dzi);
            double gpx = g.dxi * (pp[c] - pp[cidx(g, im, j, k)]);
            gpx *= 1.0;
            double q = 0.0;
            if (P.moist) q = 0.5 * (prim[4 * N + c] + prim[4 * N + cidx(g, im, j, k)] + prim[5 * N + c] + prim[5 * N + cidx(g, im, j, k)]);
            double src = 0.0;
            if (P.coriolis) {
                double rvl = 0.25 * (rv[cidx(g, i, jp, k)] + rv[c] + rv[cidx(g, im, jp, k)] + rv[cidx(g, im, j, k)]);
                double rwl = 0.25 * (rw[c + g.sk] + rw[c] + rw[cidx(g, i, jm, k + 1)] + rw[cidx(g, i, jm, k)]);
                src += P.cf * (rvl * P.sinphi - rwl * P.cosphi);
            }
            src += 0.5 * (cd[c] + cd[cidx(g, im, j, k)]) * P.geo0;
            rhs += (-gpx - 0.0) / (1.0 + q) + src;
            Fmx[c] = rhs;
        }
        // ---------------- y-momentum on face j
        if (ok) {
            double rhs = -((sh[1].fx[ty][tx + 1] - sh[1].fx[ty][tx]) * g.dxi * 1.0 +
                           (sh[1].fy[ty + 1][tx] - sh[1].fy[ty][tx]) * g.dyi * 1.0 + (zhv - zlv) * g.dzi);
            zlv = zhv;
            if (P.use_diff)
                rhs -= ((t12[cidx(g, ip, j, k)] - t12[c]) * g.dxi * 1.0 + (t22[c] - t22[cidx(g, i, jm, k)]) * g.dyi * 1.0 +
                        (t23[c + g.sk] - t23[c]) * g.dzi);
            double gpy = g.dyi * (pp[c] - pp[cidx(g, i, jm, k)]);
            gpy *= 1.0;
            double q = 0.0;
            if (P.moist) q = 0.5 * (prim[4 * N + c] + prim[4 * N + cidx(g, i, jm, k)] + prim[5 * N + c] + prim[5 * N + cidx(g, i, jm, k)]);
            double src = 0.0;
            if (P.coriolis) {
                double rul = 0.25 * (ru[cidx(g, ip, j, k)] + ru[c] + ru[cidx(g, ip, jm, k)] + ru[cidx(g, i, jm, k)]);
                src += -P.cf * rul * P.sinphi;
            }
            src += 0.5 * (cd[c] + cd[cidx(g, i, jm, k)]) * P.geo1;
            rhs += (-gpy - 0.0) / (1.0 + q) + src;
            Fmy[c] = rhs;
        }
        // ---------------- z-momentum on face k
        if (ok && k == 0) Fmz[c] = 0.0;
        if (zk) {
            double rhs = -((sh[2].fx[ty][tx + 1] - sh[2].fx[ty][tx]) * g.dxi * 1.0 +
                           (sh[2].fy[ty + 1][tx] - sh[2].fy[ty][tx]) * g.dyi * 1.0 + (zhw - zlw) * g.dzi);
            zlw = zhw;
            if (P.use_diff)
                rhs -= ((t13[cidx(g, ip, j, k)] - t13[c]) * g.dxi * 1.0 + (t23[cidx(g, i, jp, k)] - t23[c]) * g.dyi * 1.0 +
                        (t33[c] - t33[c - g.sk]) * g.dzi);
            double b;
            double g2 = -P.gravity;
            if (!P.moist) {
                if (P.buoy_type == 1) {
                    b = g2 * 0.5 * ((cd[c] - P.r0[k + 1]) + (cd[c - g.sk] - P.r0[k]));
                } else {
                    auto T0 = [&](int kk) {
                        double rt0 = eos_rt_given_p(P.p0[kk + 1]);
                        return (rt0 / P.r0[kk + 1]) / pow(p_0 / P.p0[kk + 1], P.rdOcp);
                    };
                    double t0h = T0(k), th_ = eos_T(cd[c], cd[N + c], 0.0);
                    double t0l = T0(k - 1), tl_ = eos_T(cd[c - g.sk], cd[N + c - g.sk], 0.0);
                    double qp_ = (th_ - t0h) / t0h, qm_ = (tl_ - t0l) / t0l;
                    double r0q = 0.5 * (P.r0[k + 1] * qp_ + P.r0[k] * qm_);
                    b = -r0q * g2;
                }
            } else if (P.buoy_type == 1) {
                int nq = P.ncomp - ERF_RHOQ1_COMP;
                double hi = cd[c] + cd[5 * N + c] + cd[6 * N + c] - P.r0[k + 1];
                double lo = cd[c - g.sk] + cd[5 * N + c - g.sk] + cd[6 * N + c - g.sk] - P.r0[k];
                for (int qo = 2; qo < nq; ++qo) { hi += cd[(5 + qo) * N + c]; lo += cd[(5 + qo) * N + c - g.sk]; }
                b = g2 * 0.5 * (hi + lo);
            } else {
                int nq = P.ncomp - ERF_RHOQ1_COMP;
                const double* rd = pavg;
                const double* thd = pavg + g.nz;
                const double* qvd = pavg + 2 * g.nz;
                const double* qcd = pavg + 3 * g.nz;
                const double* qpd = pavg + 4 * g.nz;
                double tp1 = eos_T(rd[k], rd[k] * thd[k], qvd[k]);
                double tm1 = eos_T(rd[k - 1], rd[k - 1] * thd[k - 1], qvd[k - 1]);
                double tp3 = eos_T(cd[c], cd[N + c], cd[5 * N + c] / cd[c]);
                double tm3 = eos_T(cd[c - g.sk], cd[N + c - g.sk], cd[5 * N + c - g.sk] / cd[c - g.sk]);
                double qvp = nq >= 1 ? prim[4 * N + c] : 0.0, qvm = nq >= 1 ? prim[4 * N + c - g.sk] : 0.0;
                double qcp = nq >= 2 ? prim[5 * N + c] : 0.0, qcm = nq >= 2 ? prim[5 * N + c - g.sk] : 0.0;
                double qpp = nq >= 3 ? prim[6 * N + c] : 0.0, qpm = nq >= 3 ? prim[6 * N + c - g.sk] : 0.0;
                double qplus = 0.61 * (qvp - qvd[k]) - (qcp - qcd[k] + qpp - qpd[k]) + (tp3 - tp1) / tp1 * (1.0 + 0.61 * qvd[k] - qcd[k] - qpd[k]);
                double qminus = 0.61 * (qvm - qvd[k - 1]) - (qcm - qcd[k - 1] + qpm - qpd[k - 1]) + (tm3 - tm1) / tm1 * (1.0 + 0.61 * qvd[k - 1] - qcd[k - 1] - qpd[k - 1]);
                double qavg = 0.5 * (qplus + qminus);
                double r0avg = 0.5 * (rd[k] + rd[k - 1]);
                b = -qavg * r0avg * g2;
            }
            double zsrc = b;
            if (P.coriolis) {
                double rul = 0.25 * (ru[cidx(g, ip, j, k)] + ru[c] + ru[cidx(g, ip, j, k - 1)] + ru[c - g.sk]);
                zsrc += P.cf * rul * P.cosphi;
            }
            zsrc += 0.5 * (cd[c] + cd[c - g.sk]) * P.geo2;
            double gpz = g.dzi * (pp[c] - pp[c - g.sk]) / 1.0;
            double q = 0.0;
            if (P.moist) q = 0.5 * (prim[4 * N + c] + prim[4 * N + c - g.sk] + prim[5 * N + c] + prim[5 * N + c - g.sk]);
            rhs += (zsrc - gpz - 0.0) / (1.0 + q);
            Fmz[c] = rhs;
        }
        if (ok && k == g.nz - 1) Fmz[c + g.sk] = 0.0;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host launchers for the tiled kernels: scheme dispatch and grid sizing.
// ---------------------------------------------------------------------------
namespace {

// Levels per block: minimise waves x (levels + 1), the cost of a block being
// its levels plus the extra bottom-face flux evaluation.
template <typename K>
int pick_kz(K kern, const Geo& g) {
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, TTX * TTY, 0) != cudaSuccess || per < 1) per = 1;
    const long cap = (long)per * nsm;
    const long nxy = (long)((g.nx + TTX - 1) / TTX) * ((g.ny + TTY - 1) / TTY);
    int best = g.nz;
    double best_cost = 1e30;
    for (int zb = 1; zb <= g.nz; ++zb) {
        int kz = (g.nz + zb - 1) / zb;
        int zb2 = (g.nz + kz - 1) / kz;
        long waves = (nxy * zb2 + cap - 1) / cap;
        double cost = (double)waves * (kz + 1);
        if (cost < best_cost) { best_cost = cost; best = kz; }
    }
    return best;
}

dim3 tile_grid(const Geo& g, int kz) { return dim3((g.nx + TTX - 1) / TTX, (g.ny + TTY - 1) / TTY, (g.nz + kz - 1) / kz); }

constexpr int U5 = ERF_ADV_UPWIND_5TH, W5 = ERF_ADV_WENO_5;

}  // namespace

using SlowCellK = void (*)(Params, int, StateBuf, StageAux, const double*, double*, double*, double*, double*);
using SlowMomK = void (*)(Params, int, StateBuf, StageAux, const double*, const double*, const double*, const double*,
                          const double*, const double*, const double*, const double*, const double*, const double*,
                          double*, double*, double*);
using PostK = void (*)(Params, int, double, StateBuf, StateBuf, StateBuf, StateBuf, StageAux, StageAux, int,
                       const double*, const double*, const double*, const double*, double*, double*, double*);

static SlowCellK slow_cell_kernel(const Params& P) {
    if (P.dyc_h == U5 && P.dyc_v == U5) return k_slow_cell<U5, U5>;
    if (P.dyc_h == W5 && P.dyc_v == W5) return k_slow_cell<W5, W5>;
    return k_slow_cell<-1, -1>;
}
static SlowMomK slow_mom_kernel(const Params& P) {
    if (P.dyc_h == U5 && P.dyc_v == U5) return k_slow_mom<U5, U5>;
    return k_slow_mom<-1, -1>;
}
static PostK post_kernel(const Params& P) {
    bool dw = P.dry_h == W5 && P.dry_v == W5, du = P.dry_h == U5 && P.dry_v == U5;
    bool mw = P.moi_h == W5 && P.moi_v == W5, mu = P.moi_h == U5 && P.moi_v == U5;
    if (!P.moist) {
        if (dw) return k_post<W5, W5, -1, -1>;
        if (du) return k_post<U5, U5, -1, -1>;
    } else {
        if (dw && mw) return k_post<W5, W5, W5, W5>;
        if (du && mu) return k_post<U5, U5, U5, U5>;
        if (du && mw) return k_post<U5, U5, W5, W5>;
    }
    return k_post<-1, -1, -1, -1>;
}

void tiled_setup(const Params& P, TiledKz* t) {
    t->cell = pick_kz(slow_cell_kernel(P), P.g);
    t->mom = pick_kz(slow_mom_kernel(P), P.g);
    t->post = pick_kz(post_kernel(P), P.g);
}

void launch_slow_cell(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux A, const double* mut,
                      double* Fcons, double* avx, double* avy, double* avz) {
    slow_cell_kernel(P)<<<tile_grid(P.g, t.cell), dim3(TTX, TTY, 1), 0, st>>>(P, t.cell, S, A, mut, Fcons, avx, avy, avz);
}
void launch_slow_mom(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux A, const double* u,
                     const double* v, const double* w, const double* t11, const double* t22, const double* t33,
                     const double* t12, const double* t13, const double* t23, const double* pavg, double* Fmx,
                     double* Fmy, double* Fmz) {
    slow_mom_kernel(P)<<<tile_grid(P.g, t.mom), dim3(TTX, TTY, 1), 0, st>>>(P, t.mom, S, A, u, v, w, t11, t22, t33,
                                                                             t12, t13, t23, pavg, Fmx, Fmy, Fmz);
}
void launch_post(const Params& P, const TiledKz& t, cudaStream_t st, double slow_dt, StateBuf Sold, StateBuf Sst,
                 StateBuf Ssum, StateBuf Snew, StageAux Acur, StageAux Anext, int make_next, const double* mut,
                 const double* avx, const double* avy, const double* avz, double* un, double* vn, double* wn) {
    post_kernel(P)<<<tile_grid(P.g, t.post), dim3(TTX, TTY, 1), 0, st>>>(P, t.post, slow_dt, Sold, Sst, Ssum, Snew,
                                                                          Acur, Anext, make_next, mut, avx, avy, avz,
                                                                          un, vn, wn);
}

}  // namespace erfb
