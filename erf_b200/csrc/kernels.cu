// kernels.cu -- dycore kernels for sm_100a.
//
// Each kernel fuses one or more of the reference's AMReX ParallelFor passes
// (file:line cited per kernel).  Lateral neighbours are addressed through
// periodic index wrapping and vertical ghost values through the wall
// conditions, so no separate ghost-fill pass is launched between stages and
// substeps; the reference's momentum<->velocity round trips at every boundary
// fill (BoundaryConditions/ERF_FillIntermediatePatch.cpp:63-67, 224-236) are
// applied inline where the filled values are next read.
//
// The dycore kernels are templates on R, the type of the bulk arrays (derived
// fields, slow right-hand sides, average momenta, fast coefficients, stresses)
// and of the arithmetic on them: R = double is the plain FP64 form, R = float
// the mixed form.  The prognostic state (conserved variables, momenta,
// between-step velocities), the base state and the equation of state stay
// FP64 in both, and every update of the state is accumulated in FP64.
#include <cfloat>

#include "kernels.cuh"
#include "tiles.cuh"

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
// ---------------------------------------------------------------------------
// MOST ground (ABLMost::compute_most_bcs with moeng_flux, implicit MOST,
// BoundaryConditions/ERF_ABLMost.cpp:289-489, ERF_MOSTStress.H:1395-1555):
// the tangential velocity d levels below the ground is the level-0 value plus
// tau / eta * dz * d, with the Moeng stress from the level-0 velocities, the
// step's plane means and u*, and eta the level-0 eddy viscosity averaged to
// the face (floored at 1e-8).  The stage boundary fills impose it, so the
// readers of stage velocities evaluate it where they reach below the ground.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double most_mu(const Params& P, int64_t c) {
    return P.most_mut_f32 ? double(static_cast<const float*>(P.most_mut)[c])
                          : static_cast<const double*>(P.most_mut)[c];
}
__device__ __forceinline__ double most_ghost_u(const Params& P, const double* __restrict__ u,
                                               const double* __restrict__ v, const double* __restrict__ cons, int i,
                                               int j, int d) {
    const Geo& g = P.g;
    const int im = wrap(i - 1, g.nx), jp = wrap(j + 1, g.ny);
    const double velx = u[cidx(g, i, j, 0)];
    const double vely = 0.25 * (v[cidx(g, i, j, 0)] + v[cidx(g, i, jp, 0)] + v[cidx(g, im, j, 0)] + v[cidx(g, im, jp, 0)]);
    const double rho = 0.5 * (cons[cidx(g, im, j, 0)] + cons[cidx(g, i, j, 0)]);
    const double umean = P.most_avg[0];
    double wsp_mean = 0.5 * (P.most_avg[2] + P.most_avg[2]);
    const double ustar = 0.5 * (P.most_avg[3] + P.most_avg[3]);
    const double wsp = sqrt(velx * velx + vely * vely);
    const double num1 = wsp * umean;
    const double num2 = wsp_mean * (velx - umean);
    const double deltaz = P.most_dz * (0 + d);
    wsp_mean = fmax(wsp_mean, 0.1);
    const double stressx = -rho * ustar * ustar * (num1 + num2) / (wsp_mean * wsp_mean);
    double eta = 0.5 * (most_mu(P, cidx(g, im, j, 0)) + most_mu(P, cidx(g, i, j, 0)));
    eta = fmax(eta, 1e-8);
    return velx + stressx / eta * deltaz;
}
__device__ __forceinline__ double most_ghost_v(const Params& P, const double* __restrict__ u,
                                               const double* __restrict__ v, const double* __restrict__ cons, int i,
                                               int j, int d) {
    const Geo& g = P.g;
    const int jm = wrap(j - 1, g.ny), ip = wrap(i + 1, g.nx);
    const double velx = 0.25 * (u[cidx(g, i, j, 0)] + u[cidx(g, ip, j, 0)] + u[cidx(g, i, jm, 0)] + u[cidx(g, ip, jm, 0)]);
    const double vely = v[cidx(g, i, j, 0)];
    const double rho = 0.5 * (cons[cidx(g, i, jm, 0)] + cons[cidx(g, i, j, 0)]);
    const double vmean = P.most_avg[1];
    double wsp_mean = 0.5 * (P.most_avg[2] + P.most_avg[2]);
    const double ustar = 0.5 * (P.most_avg[3] + P.most_avg[3]);
    const double wsp = sqrt(velx * velx + vely * vely);
    const double num1 = wsp * vmean;
    const double num2 = wsp_mean * (vely - vmean);
    const double deltaz = P.most_dz * (0 + d);
    wsp_mean = fmax(wsp_mean, 0.1);
    const double stressy = -rho * ustar * ustar * (num1 + num2) / (wsp_mean * wsp_mean);
    double eta = 0.5 * (most_mu(P, cidx(g, i, jm, 0)) + most_mu(P, cidx(g, i, j, 0)));
    eta = fmax(eta, 1e-8);
    return vely + stressy / eta * deltaz;
}
// Stage velocities with the MOST ghost rule below the ground: the fields a
// stage reader holds (u, v, cons of the stage), none for the other grounds.
struct MostView {
    const double* u;
    const double* v;
    const double* cons;
};
__device__ __forceinline__ double tang_u(const Params& P, const MostView& m, int i, int j, int k) {
    if (k < 0 && P.most) return most_ghost_u(P, m.u, m.v, m.cons, i, j, -k);
    return tang(m.u, P.g, i, j, k);
}
__device__ __forceinline__ double tang_v(const Params& P, const MostView& m, int i, int j, int k) {
    if (k < 0 && P.most) return most_ghost_v(P, m.u, m.v, m.cons, i, j, -k);
    return tang(m.v, P.g, i, j, k);
}


// ---------------------------------------------------------------------------
// Strain-rate components (Diffusion/ERF_ComputeStrain_N.cpp:28-229) with the
// one-sided wall stencils at no-slip walls.  Edge (i,j,k) of an xy/xz/yz edge
// array sits at the low corner of cell (i,j,k).  Velocities are FP64 state;
// the differences are formed in FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double strain12(const double* u, const double* v, const Geo& g, int i, int j, int k) {
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    return 0.5 * ((__ldg(u + cidx(g, i, j, k)) - __ldg(u + cidx(g, i, jm, k))) * g.dyi +
                  (__ldg(v + cidx(g, i, j, k)) - __ldg(v + cidx(g, im, j, k))) * g.dxi);
}
// Stage strain at the ground face of a MOST ground: the centred difference
// with the MOST ghost velocity below
__device__ __forceinline__ double strain13_most(const Params& P, const MostView& m, const double* w, int i, int j) {
    const Geo& g = P.g;
    int im = wrap(i - 1, g.nx);
    double wx = (__ldg(w + cidx(g, i, j, 0)) - __ldg(w + cidx(g, im, j, 0))) * g.dxi;
    return 0.5 * ((tang_u(P, m, i, j, 0) - tang_u(P, m, i, j, -1)) * g.dzi + wx);
}
__device__ __forceinline__ double strain23_most(const Params& P, const MostView& m, const double* w, int i, int j) {
    const Geo& g = P.g;
    int jm = wrap(j - 1, g.ny);
    double wy = (__ldg(w + cidx(g, i, j, 0)) - __ldg(w + cidx(g, i, jm, 0))) * g.dyi;
    return 0.5 * ((tang_v(P, m, i, j, 0) - tang_v(P, m, i, j, -1)) * g.dzi + wy);
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
// (TimeIntegration/ERF_TI_utils.H:4-45) and p' (ERF_slow_rhs_pre.cpp:337-358),
// evaluated in FP64 from the FP64 state and stored as R.
template <class R>
__device__ __forceinline__ void stage_aux_cell(const Params& P, const double* __restrict__ cons, StageAux<R> A,
                                               int64_t c, int k) {
    const int64_t N = P.g.ncell;
    double rho = cons[c];
    double rt = cons[N + c];
    A.prim[c] = R(rt / rho);
    for (int n = 1; n < P.nprim; ++n) A.prim[n * N + c] = R(cons[(n + 1) * N + c] / rho);
    A.pi[c] = R(eos_exner(rt, P.rdOcp));
    double qv = P.moist ? cons[5 * N + c] / rho : 0.0;
    A.pp[c] = R(eos_p(rt, qv) - (P.ter ? P.p0[c + P.g.sk] : P.p0[k + 1]));
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
template <class R>
__global__ void k_step_begin(Params P, const double* __restrict__ cons, const double* __restrict__ uo,
                             const double* __restrict__ vo, const double* __restrict__ wo, StateBuf S,
                             double* __restrict__ un, double* __restrict__ vn, double* __restrict__ wn,
                             StageAux<R> A, R* __restrict__ mut, TkeBuf<R> tke) {
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
    // a NaN or infinite velocity in the step's input (the state checks of
    // stage_aux_cell cover rho and rho*theta)
    if (!(fabs(uo[c]) <= DBL_MAX) || !(fabs(vo[c]) <= DBL_MAX) || !(fabs(wo[c]) <= DBL_MAX))
        atomicOr(P.status, ST_NAN);
    stage_aux_cell<R>(P, cons, A, c, k);

    if (P.les == ERF_LES_SMAGORINSKY || P.les == ERF_LES_MLP || P.les == ERF_LES_DEARDORFF) {
        int ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
        double s11 = (uo[cidx(g, ip, j, k)] - uo[c]) * g.dxi;
        double s22 = (vo[cidx(g, i, jp, k)] - vo[c]) * g.dyi;
        double s33 = (wo[c + g.sk] - wo[c]) * g.dzi;
        double s12 = 0.25 * (strain12(uo, vo, g, i, j, k) + strain12(uo, vo, g, i, jp, k) +
                             strain12(uo, vo, g, ip, j, k) + strain12(uo, vo, g, ip, jp, k));
        double s13, s23;
        if (P.most && k == 0) {
            // over a MOST ground the ground-face strains are left out and the
            // faces above averaged (ComputeSmnSmn, Diffusion/ERF_EddyViscosity.H:59-77)
            s13 = 0.5 * (strain13(uo, wo, g, i, j, k + 1) + strain13(uo, wo, g, ip, j, k + 1));
            s23 = 0.5 * (strain23(vo, wo, g, i, j, k + 1) + strain23(vo, wo, g, i, jp, k + 1));
        } else {
            s13 = 0.25 * (strain13(uo, wo, g, i, j, k) + strain13(uo, wo, g, i, j, k + 1) +
                          strain13(uo, wo, g, ip, j, k) + strain13(uo, wo, g, ip, j, k + 1));
            s23 = 0.25 * (strain23(vo, wo, g, i, j, k) + strain23(vo, wo, g, i, j, k + 1) +
                          strain23(vo, wo, g, i, jp, k) + strain23(vo, wo, g, i, jp, k + 1));
        }
        double S2 = s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * s12 * s12 + 2.0 * s13 * s13 + 2.0 * s23 * s23;
        if (P.les != ERF_LES_DEARDORFF) {
            mut[c] = R(P.CsDeltaSqr * rho * sqrt(2.0 * S2));
        } else {
            // Deardorff (ERF_ComputeTurbulentViscosity.cpp:129-229, no MOST):
            // SmnSmn for the shear production (formed from the step's
            // velocities, ERF_make_tau_terms.cpp:233-240), K = rho Ck l
            // sqrt(e) with the stratification-limited length, the vertical
            // heat diffusivity (1 + 2 l / Delta) K and the dissipation.
            tke.smn[c] = R(S2);
            const int64_t N = g.ncell;
            const int kp = min(k + 1, g.nz - 1), km = max(k - 1, 0);
            double dtheta_dz;
            if (P.most && k == 0) {
                // one-sided over a MOST ground (ERF_ComputeTurbulentViscosity.cpp:175-188)
                const int64_t c1 = cidx(g, i, j, 1), c2 = cidx(g, i, j, 2);
                dtheta_dz = 0.5 * (-3 * cons[N + c] / cons[c] + 4 * cons[N + c1] / cons[c1] - cons[N + c2] / cons[c2]) * g.dzi;
            } else {
                dtheta_dz = 0.5 * (cons[N + cidx(g, i, j, kp)] / cons[cidx(g, i, j, kp)] -
                                   cons[N + cidx(g, i, j, km)] / cons[cidx(g, i, j, km)]) * g.dzi;
            }
            double E = fmax(cons[2 * N + c] / rho, 0.0);
            double strat = P.g_over_theta0 * dtheta_dz;
            double length;
            if (strat <= 2.220446049250313e-16) {   // DBL_EPSILON
                length = P.Delta;
            } else {
                length = 0.76 * sqrt(E / strat);
                length = fmin(length, P.Delta);
                length = fmax(length, 0.001 * P.Delta);
            }
            double K = rho * P.Ck * length * sqrt(E);
            mut[c] = R(K);
            tke.kthv[c] = R((1. + 2. * length / P.Delta) * K);
            double Ce = ((P.Ce_wall > 0) && (k == 0)) ? P.Ce_wall : 1.9 * P.Ck + P.Ce_lcoeff * length / P.Delta;
            tke.diss[c] = R(rho * Ce * (E * sqrt(E)) / length);
        }
    }
}

// ---------------------------------------------------------------------------
// Stress tensor (erf_make_tau_terms, TimeIntegration/ERF_make_tau_terms.cpp:
// 320-424 with ComputeStress{Cons,Var}Visc_N, Diffusion/ERF_ComputeStress_N.cpp):
// tau_ii at cell centres, tau_12/13/23 on edges.  Strain in FP64 from the
// FP64 velocities, viscosity and stress in R.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_tau(Params P, const double* __restrict__ cons, const double* __restrict__ u,
                      const double* __restrict__ v, const double* __restrict__ w, const R* __restrict__ mut,
                      R* __restrict__ t11, R* __restrict__ t22, R* __restrict__ t33, R* __restrict__ t12,
                      R* __restrict__ t13, R* __restrict__ t23) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny), ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
    int64_t c = cidx(g, i, j, k);
    const R OneThird = R(1. / 3.);
    R s11 = R((u[cidx(g, ip, j, k)] - u[c]) * g.dxi);
    R s22 = R((v[cidx(g, i, jp, k)] - v[c]) * g.dyi);
    R s33 = R((w[c + g.sk] - w[c]) * g.dzi);
    R er = s11 + s22 + s33;
    const R mu_eff = R(P.mu_eff);
    R base = P.use_consA ? R(cons[c]) * mu_eff : mu_eff;
    R m11 = P.use_turb ? base + R(2) * mut[c] : base;
    t11[c] = -m11 * (s11 - OneThird * er);
    t22[c] = -m11 * (s22 - OneThird * er);
    t33[c] = -m11 * (s33 - OneThird * er);
    auto mu = [&](int ii, int jj, int kk) { return __ldg(mut + cidx(g, ii, jj, clampk(kk, g.nz))); };
    auto rho = [&](int ii, int jj, int kk) { return R(__ldg(cons + cidx(g, ii, jj, clampk(kk, g.nz)))); };
    {
        R m = P.use_consA ? R(0.25) * (rho(im, j, k) + rho(i, j, k) + rho(im, jm, k) + rho(i, jm, k)) * mu_eff : mu_eff;
        if (P.use_turb) m = m + R(2) * (R(0.25) * (mu(im, j, k) + mu(i, j, k) + mu(im, jm, k) + mu(i, jm, k)));
        t12[c] = R(strain12(u, v, g, i, j, k)) * -m;
    }
    for (int kk = k; kk <= (k == g.nz - 1 ? g.nz : k); ++kk) {
        int64_t e = cidx(g, i, j, kk);
        R m = P.use_consA ? R(0.25) * (rho(im, j, kk) + rho(i, j, kk) + rho(im, j, kk - 1) + rho(i, j, kk - 1)) * mu_eff : mu_eff;
        if (P.use_turb) m = m + R(2) * (R(0.25) * (mu(im, j, kk) + mu(i, j, kk) + mu(im, j, kk - 1) + mu(i, j, kk - 1)));
        t13[e] = R(strain13(u, w, g, i, j, kk)) * -m;
        R m2 = P.use_consA ? R(0.25) * (rho(i, jm, kk) + rho(i, j, kk) + rho(i, jm, kk - 1) + rho(i, j, kk - 1)) * mu_eff : mu_eff;
        if (P.use_turb) m2 = m2 + R(2) * (R(0.25) * (mu(i, jm, kk) + mu(i, j, kk) + mu(i, jm, kk - 1) + mu(i, j, kk - 1)));
        t23[e] = R(strain23(v, w, g, i, j, kk)) * -m2;
    }
}
// tau_13 / tau_23 on the ground faces of a MOST ground, from the strain with
// the MOST ghost velocities below (run after k_tau, over one plane)
template <class R>
__global__ void k_tau_most_ground(Params P, const double* __restrict__ cons, const double* __restrict__ u,
                                  const double* __restrict__ v, const double* __restrict__ w,
                                  const R* __restrict__ mut, R* __restrict__ t13, R* __restrict__ t23) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    const R mu_eff = R(P.mu_eff);
    auto mu = [&](int ii, int jj, int kk) { return __ldg(mut + cidx(g, ii, jj, clampk(kk, g.nz))); };
    auto rho = [&](int ii, int jj, int kk) { return R(__ldg(cons + cidx(g, ii, jj, clampk(kk, g.nz)))); };
    const MostView mv{u, v, cons};
    const int64_t e = cidx(g, i, j, 0);
    R m = P.use_consA ? R(0.25) * (rho(im, j, 0) + rho(i, j, 0) + rho(im, j, -1) + rho(i, j, -1)) * mu_eff : mu_eff;
    m = m + R(2) * (R(0.25) * (mu(im, j, 0) + mu(i, j, 0) + mu(im, j, -1) + mu(i, j, -1)));
    t13[e] = R(strain13_most(P, mv, w, i, j)) * -m;
    R m2 = P.use_consA ? R(0.25) * (rho(i, jm, 0) + rho(i, j, 0) + rho(i, jm, -1) + rho(i, j, -1)) * mu_eff : mu_eff;
    m2 = m2 + R(2) * (R(0.25) * (mu(i, jm, 0) + mu(i, j, 0) + mu(i, jm, -1) + mu(i, j, -1)));
    t23[e] = R(strain23_most(P, mv, w, i, j)) * -m2;
}

// Stage primitives, Exner function and p' of a state (cons_to_prim,
// ERF_TI_utils.H:4-45), for the per-pass entry points.
template <class R>
__global__ void k_stage_aux(Params P, const double* __restrict__ cons, StageAux<R> A) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    stage_aux_cell<R>(P, cons, A, cidx(g, i, j, k), k);
}

// ---------------------------------------------------------------------------
// Scalar flux helpers
// ---------------------------------------------------------------------------

// Diffusive tendency -div(-rhoAlpha grad phi) (Diffusion/ERF_DiffusionSrcForState_N.cpp:
// 196-667), scalars foextrap at the walls; returns the amount subtracted.
template <class R>
__device__ __forceinline__ R scalar_diff(const Params& P, const double* __restrict__ rhoarr, const R* __restrict__ phi,
                                         const R* __restrict__ mut, double ae_d, double fac_d, int i, int j, int k,
                                         const R* __restrict__ kv = nullptr, R* __restrict__ fz_out = nullptr) {
    const Geo& g = P.g;
    const R ae = R(ae_d), fac = R(fac_d);
    const R dxi = R(g.dxi), dyi = R(g.dyi), dzi = R(g.dzi);
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny), ip = wrap(i + 1, g.nx), jp = wrap(j + 1, g.ny);
    auto ph = [&](int ii, int jj, int kk) { return ccz(phi, g, ii, jj, kk); };
    auto rA = [&](int i0, int j0, int k0, int i1, int j1, int k1) {
        R r = P.use_consA ? R(0.5) * (R(ccz(rhoarr, g, i0, j0, k0)) + R(ccz(rhoarr, g, i1, j1, k1))) * ae : ae;
        if (P.use_turb) r += R(0.5) * (ccz(mut, g, i0, j0, k0) * fac + ccz(mut, g, i1, j1, k1) * fac);
        return r;
    };
    // vertical diffusivity: Deardorff's Theta_v when given
    auto rAz = [&](int k0, int k1) {
        if (kv == nullptr) return rA(i, j, k0, i, j, k1);
        R r = P.use_consA ? R(0.5) * (R(ccz(rhoarr, g, i, j, k0)) + R(ccz(rhoarr, g, i, j, k1))) * ae : ae;
        return r + R(0.5) * (ccz(kv, g, i, j, k0) + ccz(kv, g, i, j, k1));
    };
    R fxl = -rA(i, j, k, im, j, k) * (ph(i, j, k) - ph(im, j, k)) * dxi * R(1);
    R fxh = -rA(ip, j, k, i, j, k) * (ph(ip, j, k) - ph(i, j, k)) * dxi * R(1);
    R fyl = -rA(i, j, k, i, jm, k) * (ph(i, j, k) - ph(i, jm, k)) * dyi * R(1);
    R fyh = -rA(i, jp, k, i, j, k) * (ph(i, jp, k) - ph(i, j, k)) * dyi * R(1);
    R fzl = -rAz(k, k - 1) * (ph(i, j, k) - ph(i, j, k - 1)) * dzi;
    R fzh = -rAz(k + 1, k) * (ph(i, j, k + 1) - ph(i, j, k)) * dzi;
    if (fz_out) {   // the z-face fluxes (hfx_z of ERF_DiffusionSrcForState_N.cpp:422-425)
        fz_out[cidx(g, i, j, k)] = fzl;
        if (k == g.nz - 1) fz_out[cidx(g, i, j, k + 1)] = fzh;
    }
    return (fxh - fxl) * dxi * R(1) + (fyh - fyl) * dyi * R(1) + (fzh - fzl) * dzi;
}

// Horizontal plane averages of rho, theta, qv, qc, qp for buoyancy type 2
// (SourceTerms/ERF_make_buoyancy.cpp:212-249), FP64 sums; also the
// temperature of the mean state of each level.  Each level is split over
// PAVG_PARTS blocks (grid nz x PAVG_PARTS) that write partial sums; the last
// block of a level to finish (counted with an atomic ticket after a memory
// fence) adds the partials in part order and resets the ticket, so the result
// does not depend on which block finishes last.  Buffer layout after the
// 6 nz results: 5 nz PAVG_PARTS partials, then nz tickets (one per double slot).
template <class R>
__global__ void k_plane_avg(Params P, const double* __restrict__ cons, const R* __restrict__ prim,
                            double* __restrict__ avg) {
    const Geo& g = P.g;
    const int k = blockIdx.x, part = blockIdx.y, nz = g.nz;
    const int64_t N = g.ncell;
    double* partial = avg + 6 * nz;
    unsigned int* ticket = reinterpret_cast<unsigned int*>(partial + 5 * nz * PAVG_PARTS);
    double denom = 1.0 / (double)(g.nx * g.ny);
    int nq = P.ncomp - ERF_RHOQ1_COMP;
    const int64_t span = (g.sk + PAVG_PARTS - 1) / PAVG_PARTS;
    const int64_t t0 = part * span, t1 = min(g.sk, t0 + span);
    double acc[5] = {0, 0, 0, 0, 0};
    for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
        int64_t c = g.sk * k + t;
        acc[0] += cons[c] * denom;
        acc[1] += double(prim[c]) * denom;
        if (nq >= 1) acc[2] += double(prim[4 * N + c]) * denom;
        if (nq >= 2) acc[3] += double(prim[5 * N + c]) * denom;
        if (nq >= 3) acc[4] += double(prim[6 * N + c]) * denom;
    }
    __shared__ double sh[5][256];
    __shared__ bool last;
    for (int q = 0; q < 5; ++q) sh[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 5; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int q = 0; q < 5; ++q) partial[(q * nz + k) * PAVG_PARTS + part] = sh[q][0];
        __threadfence();
        last = atomicAdd(&ticket[2 * k], 1u) == PAVG_PARTS - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double m[5];
        for (int q = 0; q < 5; ++q) {
            const volatile double* pq = partial + (q * nz + k) * PAVG_PARTS;
            double sum = 0.0;
            for (int p = 0; p < PAVG_PARTS; ++p) sum += pq[p];
            m[q] = sum;
            avg[q * nz + k] = sum;
        }
        // the plane-mean temperature used by make_buoyancy's type 2
        avg[5 * nz + k] = eos_T(m[0], m[0] * m[1], m[2]);
        ticket[2 * k] = 0u;
    }
}

// Momentum flux helper: vertical stencil of a face velocity (FP64 state) in R
// (ERF_AdvectionSrcForMom_N.H:17-274).
template <int T, class R>
__device__ __forceinline__ R gatherz_tang(const Geo& g, const double* f, int type, R upw, R frac, int i, int j, int k) {
    R s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? R(tang(f, g, i, j, k + off)) : R(0);
    }
    return interp_of<T, R>(type, s, upw, frac);
}
// The same for the stage's u (comp 0) or v (comp 1) over a MOST ground.
template <int T, class R>
__device__ __forceinline__ R gatherz_most(const Params& P, const MostView& mv, int comp, int type, R upw, R frac, int i,
                                          int j, int k) {
    R s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? R(comp == 0 ? tang_u(P, mv, i, j, k + off) : tang_v(P, mv, i, j, k + off))
                                           : R(0);
    }
    return interp_of<T, R>(type, s, upw, frac);
}

// ---------------------------------------------------------------------------
// Acoustic substep, horizontal part (ERF_fast_rhs_N.cpp:115-256): lagged
// d(rho theta) and its forward extrapolation, explicit U'' / V'' update and
// the average-momentum accumulation.  For substeps after the first, the
// previous momenta are first passed through the momentum->velocity->momentum
// round trip of apply_bcs (ERF_TI_fast_rhs_fun.H:183-189).  The increments
// are perturbations about the stage state, formed in FP64 and carried in R;
// the new momenta are accumulated in FP64.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_fast_h(Params P, int step, int nrk, double dtau_d, double facinv, StateBuf Sprev, int prev_rt,
                         StateBuf Sst, StageAux<R> A, const R* __restrict__ Fmx, const R* __restrict__ Fmy,
                         const R* __restrict__ lag_in, R* __restrict__ lag_out, R* __restrict__ avx,
                         R* __restrict__ avy, double* __restrict__ outx, double* __restrict__ outy) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    const int64_t N = g.ncell;
    const R dtau = R(dtau_d);
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    int64_t c = cidx(g, i, j, k), cxm = cidx(g, im, j, k), cym = cidx(g, i, jm, k);
    const R beta_d = R(0.1);
    auto extrap = [&](int64_t cc) {
        R drt = R(Sprev.cons[N + cc] - Sst.cons[N + cc]);
        if (step == 0) return drt;
        return drt + beta_d * (drt - lag_in[cc]);
    };
    R drt_c = R(Sprev.cons[N + c] - Sst.cons[N + c]);
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
    R ndx, ndy;
    if (nrk == 0 && step == 0) {
        ndx = R(px - Sst.mx[c]) + dtau * Fmx[c];
        ndy = R(py - Sst.my[c]) + dtau * Fmy[c];
    } else {
        R ec = extrap(c);
        R gpx = (ec - extrap(cxm)) * R(g.dxi);
        gpx *= R(1);
        R gpy = (ec - extrap(cym)) * R(g.dyi);
        gpy *= R(1);
        if (P.moist) {
            const R* pr = A.prim;
            R qx = R(0.5) * (pr[4 * N + c] + pr[4 * N + cxm] + pr[5 * N + c] + pr[5 * N + cxm]);
            R qy = R(0.5) * (pr[4 * N + c] + pr[4 * N + cym] + pr[5 * N + c] + pr[5 * N + cym]);
            gpx /= (R(1) + qx);
            gpy /= (R(1) + qy);
        }
        R pix = R(0.5) * (A.pi[cxm] + A.pi[c]);
        R piy = R(0.5) * (A.pi[cym] + A.pi[c]);
        R fx = R(-Gamma_ * R_d) * pix * gpx;
        R fy = R(-Gamma_ * R_d) * piy * gpy;
        ndx = R(px - Sst.mx[c]) + dtau * fx + dtau * Fmx[c];
        ndy = R(py - Sst.my[c]) + dtau * fy + dtau * Fmy[c];
    }
    avx[c] += R(facinv) * ndx;
    avy[c] += R(facinv) * ndy;
    outx[c] = Sst.mx[c] + double(ndx);
    outy[c] = Sst.my[c] + double(ndy);
}

// ---------------------------------------------------------------------------
// The stage update without acoustic substepping (no_substep_fun,
// TimeIntegration/ERF_TI_no_substep_fun.H:6-150, fixed or no terrain):
// S_sum = S_old + slow_dt * F_slow for rho, rho*theta and the three momenta,
// accumulated in FP64 from the slow right-hand side (type R).  The boundary
// fill that follows in the reference (apply_bcs of S_sum) is the first of the
// two momentum round trips the slow-post kernels apply on read.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_no_substep(Geo g, double slow_dt, StateBuf Sold, const R* __restrict__ Fcons,
                             const R* __restrict__ Fmx, const R* __restrict__ Fmy, const R* __restrict__ Fmz,
                             StateBuf Ssum) {
    int i, j, k;
    if (!cell_coords(g, i, j, k)) return;
    const int64_t N = g.ncell, c = cidx(g, i, j, k);
    Ssum.cons[c] = Sold.cons[c] + slow_dt * (double(Fcons[c]));
    Ssum.cons[N + c] = Sold.cons[N + c] + slow_dt * (double(Fcons[N + c]));
    Ssum.mx[c] = Sold.mx[c] + slow_dt * double(Fmx[c]);
    Ssum.my[c] = Sold.my[c] + slow_dt * double(Fmy[c]);
    Ssum.mz[c] = Sold.mz[c] + slow_dt * double(Fmz[c]);
    if (k == g.nz - 1) Ssum.mz[c + g.sk] = Sold.mz[c + g.sk] + slow_dt * double(Fmz[c + g.sk]);
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
            // over terrain the fall-flux divergence is per unit computational volume
            // (dJinv, ERF_Kessler.cpp:82-97)
            const double dJinv = P.ter ? 1.0 / P.detJ[cidx(g, i, j, k)] : 1.0;
            double dq_sed = dtn * dJinv * (1.0 / rho) * (fz_hi - fz_lo) / dz;
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
                         int tang_lo_zero, int tang_hi_zero, int wall_w) {
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
            // beyond the walls 0; on the walls 0 without terrain, the stored
            // value (w from Omega = 0) with terrain
            if (k < 0 || k > g.nz || (!wall_w && (k == 0 || k == g.nz))) val = 0.0;
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
// warp from shared memory.  P and Q use the FP64 base and stage state.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_fast_coef(Params P, double D_d, StateBuf Sst, StageAux<R> A, R* __restrict__ cA,
                            R* __restrict__ cInvB, R* __restrict__ cCB, R* __restrict__ cP, R* __restrict__ cQ) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* sm = reinterpret_cast<R*>(sm_raw);
    const Geo& g = P.g;
    Tile t(g);
    const int nz = g.nz, TX = t.tx;
    R* sA = sm;
    R* sB = sA + (nz + 1) * TX;
    R* sC = sB + (nz + 1) * TX;
    const int64_t N = g.ncell;
    const R D = R(D_d), halfg = R(P.halfg);
    const R* th = A.prim;
    if (t.ok) {
        for (int k = 1 + t.w; k <= nz - 1; k += t.nw) {
            int64_t c = cidx(g, t.i, t.j, k), cm = c - g.sk;
            R pi_c = R(0.5) * (A.pi[cm] + A.pi[c]);
            // with terrain (ERF_make_fast_coeffs.cpp:110-140): the 3-D base
            // state, the acoustic terms over detJ at the face and B = detJ + ...
            double dJk = 1.0, inv_dJk = 1.0, r_hi, r_lo, pi_hi, pi_lo;
            if (P.ter) {
                dJk = 0.5 * (P.detJ[c] + P.detJ[cm]);
                inv_dJk = 1. / dJk;
                r_hi = P.r0[c + g.sk]; r_lo = P.r0[c]; pi_hi = P.pi0[c + g.sk]; pi_lo = P.pi0[c];
            } else {
                r_hi = P.r0[k + 1]; r_lo = P.r0[k]; pi_hi = P.pi0[k + 1]; pi_lo = P.pi0[k];
            }
            R P_ = R(-Gamma_ * R_d * g.dzi * inv_dJk + P.halfg * R_d * r_hi / (P.c_v * pi_hi * Sst.cons[N + c]));
            P_ *= pi_c;
            R Q_ = R(Gamma_ * R_d * g.dzi * inv_dJk + P.halfg * R_d * r_lo / (P.c_v * pi_lo * Sst.cons[N + cm]));
            Q_ *= pi_c;
            if (P.moist) {
                R q = R(0.5) * (th[4 * N + c] + th[4 * N + cm] + th[5 * N + c] + th[5 * N + cm]);
                P_ /= (R(1) + q);
                Q_ /= (R(1) + q);
            }
            R tlo = R(0.5) * (th[cidx(g, t.i, t.j, clampk(k - 2, nz))] + th[cm]);
            R tmid = R(0.5) * (th[cm] + th[c]);
            R thi = R(0.5) * (th[c] + th[cidx(g, t.i, t.j, clampk(k + 1, nz))]);
            R a = D * (halfg - Q_ * tlo);
            R cc = D * (-halfg + P_ * thi);
            R b = R(dJk) + D * (Q_ - P_) * tmid;
            sA[k * TX + t.lane] = a; sB[k * TX + t.lane] = b; sC[k * TX + t.lane] = cc;
            cA[c] = a; cP[c] = P_; cQ[c] = Q_;
        }
        if (t.w == 0) {
            for (int k : {0, nz}) {
                sA[k * TX + t.lane] = R(0); sB[k * TX + t.lane] = R(1); sC[k * TX + t.lane] = R(0);
                int64_t f = cidx(g, t.i, t.j, k);
                cA[f] = R(0); cP[f] = R(0); cQ[f] = R(0);
            }
        }
    }
    __syncthreads();
    if (t.w == 0 && t.ok) {
        R bet = sB[t.lane];
        int64_t f0 = cidx(g, t.i, t.j, 0);
        cInvB[f0] = bet;               // B at the bottom row stays uninverted (== 1)
        cCB[f0] = sC[t.lane] * bet;
        for (int k = 1; k <= nz; ++k) {
            R gam = sC[(k - 1) * TX + t.lane] / bet;
            bet = sB[k * TX + t.lane] - sA[k * TX + t.lane] * gam;
            if (!(fabs(double(bet)) > 1e-300)) atomicOr(P.status, ST_BADSTATE);
            R inv = (k < nz) ? R(1) / bet : bet;
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
// because the previous and new states may be the same buffers.  The W''
// system is solved in R; rho, rho*theta and the z-momentum are accumulated
// in FP64.
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(1024) k_fast_vert(Params P, double dtau_d, double facinv, double beta_1d,
                                                    double beta_2d, StateBuf Sprev, int prev_rt, StateBuf Sst,
                                                    StageAux<R> A, const R* __restrict__ Fcons,
                                                    const R* __restrict__ Fmz, const double* __restrict__ newx,
                                                    const double* __restrict__ newy, const R* __restrict__ cA,
                                                    const R* __restrict__ cInvB, const R* __restrict__ cCB,
                                                    const R* __restrict__ cP, const R* __restrict__ cQ,
                                                    R* __restrict__ avz, double* out_cons, double* out_mz) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    R* sm = reinterpret_cast<R*>(sm_raw);
    const Geo& g = P.g;
    Tile t(g);
    const int nz = g.nz, TX = t.tx, L = t.lane;
    R* sT0 = sm;
    R* sT1 = sT0 + nz * TX;
    R* sR = sT1 + nz * TX;
    R* sD = sR + (nz + 1) * TX;
    R* sA = sD + (nz + 1) * TX;
    R* sI = sA + (nz + 1) * TX;
    R* sCB = sI + (nz + 1) * TX;

    const int64_t N = g.ncell;
    const R dxi = R(g.dxi), dyi = R(g.dyi), dzi = R(g.dzi), halfg = R(P.halfg);
    const R dtau = R(dtau_d), beta_1 = R(beta_1d), beta_2 = R(beta_2d);
    const R* th = A.prim;
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
            R xl = R(newx[c] - Sst.mx[c]) / R(1);
            R xh = R(newx[cidx(g, ip, j, k)] - Sst.mx[cidx(g, ip, j, k)]) / R(1);
            R yl = R(newy[c] - Sst.my[c]) / R(1);
            R yh = R(newy[cidx(g, i, jp, k)] - Sst.my[cidx(g, i, jp, k)]) / R(1);
            R mfsq = R(1);
            R tc = th[c];
            sT0[k * TX + L] = (xh - xl) * dxi * mfsq + (yh - yl) * dyi * mfsq;
            sT1[k * TX + L] = ((xh * (tc + th[cidx(g, ip, j, k)]) - xl * (tc + th[cidx(g, im, j, k)])) * dxi * mfsq +
                               (yh * (tc + th[cidx(g, i, jp, k)]) - yl * (tc + th[cidx(g, i, jm, k)])) * dyi * mfsq) * R(0.5);
        }
    }
    __syncthreads();
    // ---- phase 2
    if (t.ok) {
        for (int k = t.w; k <= nz; k += t.nw) {
            int64_t f = cidx(g, i, j, k);
            R Ok = R(prev_mz(k) - Sst.mz[f]);
            sD[k * TX + L] = Ok;
            sA[k * TX + L] = cA[f];
            sI[k * TX + L] = cInvB[f];
            sCB[k * TX + L] = cCB[f];
            R rhs;
            if (k == 0 || k == nz) {
                rhs = Ok + dtau * Fmz[f];
            } else {
                int64_t cm = f - g.sk;
                R Okp1 = R(prev_mz(k + 1) - Sst.mz[f + g.sk]);
                R Okm1 = R(prev_mz(k - 1) - Sst.mz[cm]);
                R cPk = cP[f], cQk = cQ[f];
                R tlo = R(0.5) * (thz(k - 2) + thz(k - 1));
                R tmid = R(0.5) * (thz(k - 1) + thz(k));
                R thi = R(0.5) * (thz(k) + thz(k + 1));
                R drt_k = R(Sprev.cons[N + f] - Sst.cons[N + f]);
                R drt_km = R(Sprev.cons[N + cm] - Sst.cons[N + cm]);
                R odk = R(Sprev.cons[f] - Sst.cons[f]);
                R odkm = R(Sprev.cons[cm] - Sst.cons[cm]);
                R R0 = cPk * drt_k + cQk * drt_km - halfg * (odk + odkm);
                R R1 = halfg * (-Fcons[f] - Fcons[cm] + sT0[k * TX + L] + sT0[(k - 1) * TX + L]) +
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
        R s = sR[L] * sI[L];
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
            R sol = sR[k * TX + L], sol_hi = sR[(k + 1) * TX + L];
            R zl = beta_2 * sol + beta_1 * sD[k * TX + L];
            R zh = beta_2 * sol_hi + beta_1 * sD[(k + 1) * TX + L];
            avz[c] += R(facinv) * zl / (R(1) * R(1));
            if (k == nz - 1) avz[c + g.sk] += R(facinv) * zh / (R(1) * R(1));
            R tc = th[c];
            R t0 = sT0[k * TX + L] + dzi * (zh - zl);
            R t1 = sT1[k * TX + L] + R(0.5) * dzi * (zh * (tc + thz(k + 1)) - zl * (tc + thz(k - 1)));
            double pr = Sprev.cons[c], prt = Sprev.cons[N + c];
            out_cons[c] = pr + double(dtau * (Fcons[c] - t0));
            out_cons[N + c] = prt + double(dtau * (Fcons[N + c] - t1));
            double smz = Sst.mz[c];
            out_mz[c] = smz + double(sol);
            if (k == nz - 1) out_mz[c + g.sk] = Sst.mz[c + g.sk] + double(sol_hi);
        }
    }
}

// ---------------------------------------------------------------------------
// Kessler, one thread per cell: the fall fluxes through the cell's bottom and
// top faces are evaluated from the pre-update neighbours, so cells are
// independent (same arithmetic as k_kessler).  A block holds 32 columns x
// KESS_KB levels: each thread evaluates the fall flux through its bottom face
// and takes its top face's from the thread above through shared memory (the
// block's top level evaluates its own), so each face's flux, with its two
// pow() calls, is formed once.  The pressure is formed once per cell for
// both the temperature and the saturation pressure.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * KESS_KB) k_kessler_cells(Params P, const double* __restrict__ cin,
                                                                double* __restrict__ cout, double dtn, double dz) {
    __shared__ double sfz[KESS_KB][32];
    const Geo& g = P.g;
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y, tz = threadIdx.z;
    const int k = blockIdx.z * KESS_KB + tz;
    const bool live = i < g.nx && k < g.nz;
    const int64_t N = g.ncell;
    const int nz = g.nz;
    const bool rain = P.kessler_rain;
    const bool has_qp = P.ncomp > 7;
    const double fac_cond = lcond / P.c_p;
    const int64_t c = live ? cidx(g, i, j, k) : 0;
    auto qp_of = [&](int64_t cc) { return has_qp ? cin[7 * N + cc] / cin[cc] : 0.0; };
    auto flux = [&](double ra, double qa) {
        qa = fmax(0.0, qa);
        double Vt = 36.34 * pow(ra * 0.001 * qa, 0.1346) * pow(ra / 1.16, -0.5);
        double f = ra * Vt * qa;
        return (fabs(f) < 1e-14) ? 0.0 : f;
    };
    double rho = 1.0, qp = 0.0, fz_lo = 0.0;
    if (live) {
        rho = cin[c];
        qp = qp_of(c);
        if (rain) {
            if (k == 0) fz_lo = flux(rho, qp);
            else fz_lo = flux(0.5 * (cin[c - g.sk] + rho), 0.5 * (qp_of(c - g.sk) + qp));
        }
    }
    sfz[tz][threadIdx.x] = fz_lo;
    __syncthreads();
    if (!live) return;
    double rt = cin[N + c];
    double theta = rt / rho;
    double qv = cin[5 * N + c] / rho;
    double qc = cin[6 * N + c] / rho;
    const double p_pa = eos_p(rt, qv);
    double tabs = p_pa / (R_d * rho * (1.0 + R_v / R_d * qv));   // eos_T(rho, rt, qv) with p formed once
    double pres = p_pa / 100.;
    if (rain) {
        double fz_hi;
        if (k == nz - 1) fz_hi = flux(rho, qp);
        else if (tz + 1 < KESS_KB) fz_hi = sfz[tz + 1][threadIdx.x];
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
        const double dJinv = P.ter ? 1.0 / P.detJ[c] : 1.0;   // ERF_Kessler.cpp:82-97
        double dq_sed = dtn * dJinv * (1.0 / rho) * (fz_hi - fz_lo) / dz;
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


// ---------------------------------------------------------------------------
// Slow RHS for rho and rho*theta (erf_slow_rhs_pre cell part,
// ERF_slow_rhs_pre.cpp:462-526): AdvectionSrcForRho (also initialises the
// average momenta to the stage mass fluxes, ERF_AdvectionSrcForState.cpp:56-71),
// AdvectionSrcForScalars for theta with the dycore scheme
// (ERF_slow_rhs_pre.cpp:139-142, 469-477), DiffusionSrcForState_N for theta.
// ---------------------------------------------------------------------------
template <class R, int TH, int TV>
__global__ void __launch_bounds__(TTX * TTY, ERFB_MINB_CELL) k_slow_cell(Params P, int kz, StateBuf S, StageAux<R> A,
                                                                         const R* __restrict__ mut,
                                                                         const R* __restrict__ hx,
                                                                         const R* __restrict__ hy,
                                                                         const R* __restrict__ hz, TkeBuf<R> tke,
                                                                         R* __restrict__ Fcons, R* __restrict__ avx,
                                                                         R* __restrict__ avy, R* __restrict__ avz) {
    __shared__ FluxTile<R> sh;
    __shared__ Plane<R> pl;
    const Geo& g = P.g;
    const int i = blockIdx.x * TTX + threadIdx.x, j = blockIdx.y * TTY + threadIdx.y;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const int ip = ok ? wrap(i + 1, g.nx) : 0, jp = ok ? wrap(j + 1, g.ny) : 0;
    R zl = R(0), zh = R(0);
    const TileEdge edge = tile_edge(g);
    load_plane(g, pl, A.prim, k0);
    for (int k = k0; k < k1; ++k) {
        plane_wait();
        __syncthreads();
        if (ok)
            tile_put<TH, TV>(g, sh, pl, A.prim, S.mx, S.my, S.mz, P.dyc_h, P.dyc_v, R(P.f_dyc_h), R(P.f_dyc_v), i, j,
                             k, k == k0, zl, zh);
        tile_put_edge<TH>(g, edge, sh, pl, S.mx, S.my, P.dyc_h, R(P.f_dyc_h), k);
        __syncthreads();
        if (k + 1 < k1) load_plane(g, pl, A.prim, k + 1);   // overlaps the update below
        if (ok) {
            R frt = tile_div(g, sh, zl, zh);
            zl = zh;
            int64_t c = cidx(g, i, j, k);
            avx[c] = R(S.mx[c]);
            avy[c] = R(S.my[c]);
            avz[c] = R(S.mz[c]);
            if (k == g.nz - 1) avz[c + g.sk] = R(S.mz[c + g.sk]);
            Fcons[c] = R(-1.0 / 1.0 * ((S.mx[cidx(g, ip, j, k)] - S.mx[c]) * g.dxi +
                                       (S.my[cidx(g, i, jp, k)] - S.my[c]) * g.dyi + (S.mz[c + g.sk] - S.mz[c]) * g.dzi));
            if (P.les == ERF_LES_MLP) {
                // divergence of the learned heat flux rho*q (cell values
                // averaged to faces; no flux through the walls)
                const int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
                auto fz = [&](int kk) {
                    if (kk <= 0 || kk >= g.nz) return R(0);
                    return R(0.5) * (hz[cidx(g, i, j, kk - 1)] + hz[cidx(g, i, j, kk)]);
                };
                R fxl = R(0.5) * (hx[cidx(g, im, j, k)] + hx[c]), fxh = R(0.5) * (hx[c] + hx[cidx(g, ip, j, k)]);
                R fyl = R(0.5) * (hy[cidx(g, i, jm, k)] + hy[c]), fyh = R(0.5) * (hy[c] + hy[cidx(g, i, jp, k)]);
                frt -= (fxh - fxl) * R(g.dxi) + (fyh - fyl) * R(g.dyi) + (fz(k + 1) - fz(k)) * R(g.dzi);
            } else if (P.les == ERF_LES_DEARDORFF) {
                frt -= scalar_diff<R>(P, S.cons, A.prim, mut, P.alphaT_eff, P.invPr, i, j, k, tke.kthv, tke.hfz);
            } else if (P.use_diff) {
                frt -= scalar_diff<R>(P, S.cons, A.prim, mut, P.alphaT_eff, P.invPr, i, j, k);
            }
            Fcons[g.ncell + c] = frt;
        }
        // the next level's first barrier orders the reuse of sh
    }
}

// ---------------------------------------------------------------------------
// Slow RHS post + stage finalisation (erf_slow_rhs_post,
// ERF_slow_rhs_post.cpp:228-531, and post_update = apply_bcs(S_new),
// ERF_TI_slow_rhs_fun.H:284-288):
//   * advection (average momenta) and diffusion of the slow scalars
//     (passive scalar with the dry-scalar scheme; moisture with the moist
//     scheme), S_new = S_old + slow_dt * RHS (FP64), moisture clipped at 0;
//   * rho, rho*theta and the momenta copied from the fast solution, with the
//     momentum/velocity round trips of the two boundary fills;
//   * the stage velocities, and (unless last) the next stage's primitive
//     variables, Exner function and p'.
// ---------------------------------------------------------------------------
// Slow variables, in order: the passive scalar, the moisture species, then
// (Deardorff) rho*KE.  NS is the kernel's capacity: 4 holds the scalar and
// three species, 5 adds KE to them.
template <class R, int DH, int DV, int MH, int MV, int NS>
__global__ void __launch_bounds__(TTX * TTY, ERFB_MINB_POST) k_post(Params P, int kz, double slow_dt, StateBuf Sold,
                                                                    StateBuf Sst, StateBuf Ssum, StateBuf Snew,
                                                                    StageAux<R> Acur, StageAux<R> Anext, int make_next,
                                                                    const R* __restrict__ mut, TkeBuf<R> tke,
                                                                    const R* __restrict__ avx,
                                                                    const R* __restrict__ avy,
                                                                    const R* __restrict__ avz, double* __restrict__ un,
                                                                    double* __restrict__ vn, double* __restrict__ wn) {
    __shared__ FluxTile<R> sh[NS];
    __shared__ Plane<R> pl[NS];
    const Geo& g = P.g;
    const int64_t N = g.ncell;
    const int i = blockIdx.x * TTX + threadIdx.x, j = blockIdx.y * TTY + threadIdx.y;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const int im = ok ? wrap(i - 1, g.nx) : 0, jm = ok ? wrap(j - 1, g.ny) : 0;
    const bool dd = P.les == ERF_LES_DEARDORFF;
    const int nscal = P.moist ? 1 + (P.ncomp - ERF_RHOQ1_COMP) : 1;
    const int nslow = nscal + (dd ? 1 : 0);
    R zl[NS], zh[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) zl[q] = zh[q] = R(0);
    const TileEdge edge = tile_edge(g);
    auto comp_of = [&](int q) {
        return q == 0 ? ERF_RHOSCALAR_COMP : (q < nscal ? ERF_RHOQ1_COMP + q - 1 : ERF_RHOKE_COMP);
    };
    auto slow_phi = [&](int q) { return Acur.prim + (int64_t)(comp_of(q) - 1) * N; };
#pragma unroll
    for (int q = 0; q < NS; ++q)
        if (q < nslow) load_plane(g, pl[q], slow_phi(q), k0);
    for (int k = k0; k < k1; ++k) {
        plane_wait();
        __syncthreads();
        if (ok) {
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                if (q >= nslow) break;
                if (q == 0 || q >= nscal)   // scalar and KE: dry-scalar schemes
                    tile_put<DH, DV>(g, sh[q], pl[q], slow_phi(q), avx, avy, avz, P.dry_h, P.dry_v, R(P.f_dry_h),
                                     R(P.f_dry_v), i, j, k, k == k0, zl[q], zh[q]);
                else
                    tile_put<MH, MV>(g, sh[q], pl[q], slow_phi(q), avx, avy, avz, P.moi_h, P.moi_v, R(P.f_moi_h),
                                     R(P.f_moi_v), i, j, k, k == k0, zl[q], zh[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            if (q >= nslow) break;
            if (q == 0 || q >= nscal)
                tile_put_edge<DH>(g, edge, sh[q], pl[q], avx, avy, P.dry_h, R(P.f_dry_h), k);
            else
                tile_put_edge<MH>(g, edge, sh[q], pl[q], avx, avy, P.moi_h, R(P.f_moi_h), k);
        }
        __syncthreads();
        if (k + 1 < k1) {   // next level's planes arrive during the update below
#pragma unroll
            for (int q = 0; q < NS; ++q)
                if (q < nslow) load_plane(g, pl[q], slow_phi(q), k + 1);
        }
        if (ok) {
            int64_t c = cidx(g, i, j, k);
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                if (q >= nslow) break;
                const int n = comp_of(q);
                R r = tile_div(g, sh[q], zl[q], zh[q]);
                zl[q] = zh[q];
                if (q < nscal) {
                    if (P.use_diff)
                        r -= scalar_diff<R>(P, Sst.cons, Acur.prim + (int64_t)(n - 1) * N, mut, P.alphaC_eff, P.invSc,
                                            i, j, k);
                } else {
                    // KE diffusion (alpha 0, K / sigma_k) and the TKE sources of
                    // ERF_DiffusionSrcForState_N.cpp:681-707: buoyancy, shear
                    // production, dissipation
                    r -= scalar_diff<R>(P, Sst.cons, Acur.prim + (int64_t)(n - 1) * N, mut, 0.0, P.invSigmaK, i, j, k);
                    r += R(P.g_over_theta0) * tke.hfz[c];
                    r += R(2.0) * mut[c] * tke.smn[c];
                    r -= tke.diss[c];
                }
                double v_ = Sold.cons[n * N + c] + slow_dt * double(r);
                Snew.cons[n * N + c] = (q == 0) ? v_ : fmax(v_, q < nscal ? 0.0 : 2.220446049250313e-16);
            }
            Snew.cons[c] = Ssum.cons[c];
            Snew.cons[N + c] = Ssum.cons[N + c];
            if (!dd) Snew.cons[2 * N + c] = Sst.cons[2 * N + c];
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
            if (make_next) stage_aux_cell<R>(P, Snew.cons, Anext, c, k);
        }
        // the next level's first barrier orders the reuse of sh
    }
}

// Momentum fluxes of AdvectionSrcFor{X,Y,Z}Mom_N (ERF_AdvectionSrcForMom_N.H:
// 17-274).  Each is the flux through the low side of the face's control
// volume in one direction; the high side is the same function one index up.
// The x / y stencils of the face velocity come from the level's staged
// plane: column c0 = tx (low face) or tx + 1 (the tile edge's high face),
// row r0 = ty or ty + 1 likewise.
template <int T, class R, class V>
__device__ __forceinline__ R plane_interp_x(const Plane<V>& p, int ty, int c0, int type, R upw, R frac) {
    R s[6];
    const int w = width_of<T>(type);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? R(p.v[ty + PH][c0 + m]) : R(0);
    }
    return interp_of<T, R>(type, s, upw, frac);
}
template <int T, class R, class V>
__device__ __forceinline__ R plane_interp_y(const Plane<V>& p, int r0, int tx, int type, R upw, R frac) {
    R s[6];
    const int w = width_of<T>(type);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? R(p.v[r0 + m][tx + PH]) : R(0);
    }
    return interp_of<T, R>(type, s, upw, frac);
}
template <int HT, class R>
__device__ __forceinline__ R xmom_flux_x(const Params& P, const double* ru, const Plane<double>& pu, int c0, int ty,
                                         int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(ru[cidx(g, wrap(i - 1, g.nx), j, k)]) + R(ru[cidx(g, i, j, k)]));
    return a * plane_interp_x<HT, R>(pu, ty, c0, P.dyc_h, a, R(P.f_dyc_h));
}
template <int HT, class R>
__device__ __forceinline__ R xmom_flux_y(const Params& P, const double* rv, const Plane<double>& pu, int tx, int r0,
                                         int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(rv[cidx(g, i, j, k)]) + R(rv[cidx(g, wrap(i - 1, g.nx), j, k)]));
    return a * plane_interp_y<HT, R>(pu, r0, tx, P.dyc_h, a, R(P.f_dyc_h));
}
template <int VT, class R>
__device__ __forceinline__ R xmom_flux_z(const Params& P, const double* rw, const MostView& mv, int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(rw[cidx(g, i, j, k)]) + R(rw[cidx(g, wrap(i - 1, g.nx), j, k)]));
    if (P.most && k < 3) return a * gatherz_most<VT, R>(P, mv, 0, P.dyc_v, a, R(P.f_dyc_v), i, j, k);
    return a * gatherz_tang<VT, R>(g, mv.u, P.dyc_v, a, R(P.f_dyc_v), i, j, k);
}
template <int HT, class R>
__device__ __forceinline__ R ymom_flux_x(const Params& P, const double* ru, const Plane<double>& pv, int c0, int ty,
                                         int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(ru[cidx(g, i, j, k)]) + R(ru[cidx(g, i, wrap(j - 1, g.ny), k)]));
    return a * plane_interp_x<HT, R>(pv, ty, c0, P.dyc_h, a, R(P.f_dyc_h));
}
template <int HT, class R>
__device__ __forceinline__ R ymom_flux_y(const Params& P, const double* rv, const Plane<double>& pv, int tx, int r0,
                                         int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(rv[cidx(g, i, j, k)]) + R(rv[cidx(g, i, wrap(j - 1, g.ny), k)]));
    return a * plane_interp_y<HT, R>(pv, r0, tx, P.dyc_h, a, R(P.f_dyc_h));
}
template <int VT, class R>
__device__ __forceinline__ R ymom_flux_z(const Params& P, const double* rw, const MostView& mv, int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(rw[cidx(g, i, j, k)]) + R(rw[cidx(g, i, wrap(j - 1, g.ny), k)]));
    if (P.most && k < 3) return a * gatherz_most<VT, R>(P, mv, 1, P.dyc_v, a, R(P.f_dyc_v), i, j, k);
    return a * gatherz_tang<VT, R>(g, mv.v, P.dyc_v, a, R(P.f_dyc_v), i, j, k);
}
template <int HT, class R>
__device__ __forceinline__ R zmom_flux_x(const Params& P, const double* ru, const Plane<double>& pw, int c0, int ty,
                                         int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(ru[cidx(g, i, j, k)]) + R(ru[cidx(g, i, j, k - 1)])) * R(1);
    return a * plane_interp_x<HT, R>(pw, ty, c0, P.dyc_h, a, R(P.f_dyc_h));
}
template <int HT, class R>
__device__ __forceinline__ R zmom_flux_y(const Params& P, const double* rv, const Plane<double>& pw, int tx, int r0,
                                         int i, int j, int k) {
    const Geo& g = P.g;
    R a = R(0.5) * (R(rv[cidx(g, i, j, k)]) + R(rv[cidx(g, i, j, k - 1)])) * R(1);
    return a * plane_interp_y<HT, R>(pw, r0, tx, P.dyc_h, a, R(P.f_dyc_h));
}
// Vertical flux of w between faces kk-1 and kk (the "lo" flux of face kk),
// with the order reduction next to the walls (ERF_AdvectionSrcForMom_N.H:
// 220-265); for kk == nz it is the "hi" flux of the top interior face,
// which the reference takes centred.
template <int VT, class R>
__device__ __forceinline__ R zmom_flux_z(const Params& P, const double* rw, const double* w, int i, int j, int kk) {
    const Geo& g = P.g;
    const int vt = P.dyc_v, lo_z_face = 0, hi_z_face = g.nz;
    const R vf = R(P.f_dyc_v);
    auto wz = [&](int q) { return R(__ldg(w + cidx(g, i, j, q))); };
    auto all = [&](int q, R upw, R frac, int type) {
        R sv[6];
        bool wide = (type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH);
        sv[0] = wide ? wz(q - 3) : R(0);
        sv[1] = (type == ERF_ADV_CENTERED_2ND) ? R(0) : wz(q - 2);
        sv[2] = wz(q - 1);
        sv[3] = wz(q);
        sv[4] = (type == ERF_ADV_CENTERED_2ND) ? R(0) : wz(q + 1);
        sv[5] = wide ? wz(q + 2) : R(0);
        return interp_all<R>(type, sv, upw, frac);
    };
    auto normal = [&](int q, R upw) {
        R sv[6];
        const int wd = width_of<VT>(vt);
        for (int m = 0; m < 6; ++m) {
            int off = m - 3;
            sv[m] = (off >= -wd && off <= wd - 1) ? wz(q + off) : R(0);
        }
        return interp_of<VT, R>(vt, sv, upw, vf);
    };
    R a = R(0.5) * (R(rw[cidx(g, i, j, kk)]) + R(rw[cidx(g, i, j, kk - 1)]));
    R iv;
    if (kk == hi_z_face || kk == lo_z_face + 1) iv = all(kk, a, R(0), ERF_ADV_CENTERED_2ND);
    else if (kk == lo_z_face + 2 || kk == hi_z_face - 1) {
        if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) iv = all(kk, a, R(0), ERF_ADV_CENTERED_4TH);
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
// Buoyancy is evaluated in FP64 from the FP64 state (EOS), the rest in R.
// ---------------------------------------------------------------------------
template <class R, int HT, int VT>
__global__ void __launch_bounds__(TTX * TTY, ERFB_MINB_MOM) k_slow_mom(Params P, int kz, StateBuf S, StageAux<R> A,
                                                                       const double* __restrict__ u,
                                                                       const double* __restrict__ v,
                                                                       const double* __restrict__ w,
                                                                       const R* __restrict__ t11,
                                                                       const R* __restrict__ t22,
                                                                       const R* __restrict__ t33,
                                                                       const R* __restrict__ t12,
                                                                       const R* __restrict__ t13,
                                                                       const R* __restrict__ t23,
                                                                       const double* __restrict__ pavg,
                                                                       R* __restrict__ Fmx, R* __restrict__ Fmy,
                                                                       R* __restrict__ Fmz) {
    __shared__ FluxTile<R> sh[3];
    __shared__ Plane<double> pu, pv, pw;   // face velocities of the level, with halo
    const Geo& g = P.g;
    const int64_t N = g.ncell;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * TTX + tx, j = blockIdx.y * TTY + ty;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const int im = ok ? wrap(i - 1, g.nx) : 0, jm = ok ? wrap(j - 1, g.ny) : 0;
    const int ip = ok ? wrap(i + 1, g.nx) : 0, jp = ok ? wrap(j + 1, g.ny) : 0;
    const TileEdge edge = tile_edge(g);
    const R dxi = R(g.dxi), dyi = R(g.dyi), dzi = R(g.dzi);
    const MostView mv{u, v, S.cons};   // stage velocities (MOST ghosts below a MOST ground)
    const double* ru = S.mx;
    const double* rv = S.my;
    const double* rw = S.mz;
    const double* cd = S.cons;
    const R* prim = A.prim;
    const R* pp = A.pp;
    R zlu = R(0), zhu = R(0), zlv = R(0), zhv = R(0), zlw = R(0), zhw = R(0);
    double t_below = 0.0;   // temperature of the cell below (buoyancy type 2, moist)
    load_plane(g, pu, u, k0);
    load_plane(g, pv, v, k0);
    load_plane(g, pw, w, k0);
    for (int k = k0; k < k1; ++k) {
        const int64_t c = ok ? cidx(g, i, j, k) : 0;
        const bool zk = ok && k >= 1;   // z-momentum on interior faces only
        plane_wait();
        __syncthreads();
        if (ok) {
            sh[0].fx[ty][tx] = xmom_flux_x<HT, R>(P, ru, pu, tx, ty, i, j, k);
            sh[0].fy[ty][tx] = xmom_flux_y<HT, R>(P, rv, pu, tx, ty, i, j, k);
            if (k == k0) zlu = xmom_flux_z<VT, R>(P, rw, mv, i, j, k);
            zhu = xmom_flux_z<VT, R>(P, rw, mv, i, j, k + 1);
            sh[1].fx[ty][tx] = ymom_flux_x<HT, R>(P, ru, pv, tx, ty, i, j, k);
            sh[1].fy[ty][tx] = ymom_flux_y<HT, R>(P, rv, pv, tx, ty, i, j, k);
            if (k == k0) zlv = ymom_flux_z<VT, R>(P, rw, mv, i, j, k);
            zhv = ymom_flux_z<VT, R>(P, rw, mv, i, j, k + 1);
        }
        if (zk) {
            sh[2].fx[ty][tx] = zmom_flux_x<HT, R>(P, ru, pw, tx, ty, i, j, k);
            sh[2].fy[ty][tx] = zmom_flux_y<HT, R>(P, rv, pw, tx, ty, i, j, k);
            if (k == k0 || k == 1) zlw = zmom_flux_z<VT, R>(P, rw, w, i, j, k);
            zhw = zmom_flux_z<VT, R>(P, rw, w, i, j, k + 1);
        }
        // the tile's high-side halo faces (see TileEdge)
        if (edge.row >= 0) {
            const int r = edge.row, ih = wrap(edge.i0 + edge.nvx, g.nx), jr = edge.j0 + r;
            sh[0].fx[r][edge.nvx] = xmom_flux_x<HT, R>(P, ru, pu, edge.nvx, r, ih, jr, k);
            sh[1].fx[r][edge.nvx] = ymom_flux_x<HT, R>(P, ru, pv, edge.nvx, r, ih, jr, k);
            if (k >= 1) sh[2].fx[r][edge.nvx] = zmom_flux_x<HT, R>(P, ru, pw, edge.nvx, r, ih, jr, k);
        }
        if (edge.col >= 0) {
            const int cc = edge.col, ic = edge.i0 + cc, jh = wrap(edge.j0 + edge.nvy, g.ny);
            sh[0].fy[edge.nvy][cc] = xmom_flux_y<HT, R>(P, rv, pu, cc, edge.nvy, ic, jh, k);
            sh[1].fy[edge.nvy][cc] = ymom_flux_y<HT, R>(P, rv, pv, cc, edge.nvy, ic, jh, k);
            if (k >= 1) sh[2].fy[edge.nvy][cc] = zmom_flux_y<HT, R>(P, rv, pw, cc, edge.nvy, ic, jh, k);
        }
        __syncthreads();
        if (k + 1 < k1) {   // next level's planes arrive during the right-hand sides below
            load_plane(g, pu, u, k + 1);
            load_plane(g, pv, v, k + 1);
            load_plane(g, pw, w, k + 1);
        }
        // ---------------- x-momentum on face i
        if (ok) {
            R rhs = -((sh[0].fx[ty][tx + 1] - sh[0].fx[ty][tx]) * dxi * R(1) +
                      (sh[0].fy[ty + 1][tx] - sh[0].fy[ty][tx]) * dyi * R(1) + (zhu - zlu) * dzi);
            zlu = zhu;
            if (P.use_diff)
                rhs -= ((t11[c] - t11[cidx(g, im, j, k)]) * dxi * R(1) + (t12[cidx(g, i, jp, k)] - t12[c]) * dyi * R(1) +
                        (t13[c + g.sk] - t13[c]) * dzi);
            R gpx = dxi * (pp[c] - pp[cidx(g, im, j, k)]);
            gpx *= R(1);
            R q = R(0);
            if (P.moist) q = R(0.5) * (prim[4 * N + c] + prim[4 * N + cidx(g, im, j, k)] + prim[5 * N + c] + prim[5 * N + cidx(g, im, j, k)]);
            R src = R(0);
            if (P.coriolis) {
                R rvl = R(0.25) * (R(rv[cidx(g, i, jp, k)]) + R(rv[c]) + R(rv[cidx(g, im, jp, k)]) + R(rv[cidx(g, im, j, k)]));
                R rwl = R(0.25) * (R(rw[c + g.sk]) + R(rw[c]) + R(rw[cidx(g, i, jm, k + 1)]) + R(rw[cidx(g, i, jm, k)]));
                src += R(P.cf) * (rvl * R(P.sinphi) - rwl * R(P.cosphi));
            }
            src += R(0.5) * (R(cd[c]) + R(cd[cidx(g, im, j, k)])) * R(P.geo0);
            rhs += (-gpx - R(0)) / (R(1) + q) + src;
            Fmx[c] = rhs;
        }
        // ---------------- y-momentum on face j
        if (ok) {
            R rhs = -((sh[1].fx[ty][tx + 1] - sh[1].fx[ty][tx]) * dxi * R(1) +
                      (sh[1].fy[ty + 1][tx] - sh[1].fy[ty][tx]) * dyi * R(1) + (zhv - zlv) * dzi);
            zlv = zhv;
            if (P.use_diff)
                rhs -= ((t12[cidx(g, ip, j, k)] - t12[c]) * dxi * R(1) + (t22[c] - t22[cidx(g, i, jm, k)]) * dyi * R(1) +
                        (t23[c + g.sk] - t23[c]) * dzi);
            R gpy = dyi * (pp[c] - pp[cidx(g, i, jm, k)]);
            gpy *= R(1);
            R q = R(0);
            if (P.moist) q = R(0.5) * (prim[4 * N + c] + prim[4 * N + cidx(g, i, jm, k)] + prim[5 * N + c] + prim[5 * N + cidx(g, i, jm, k)]);
            R src = R(0);
            if (P.coriolis) {
                R rul = R(0.25) * (R(ru[cidx(g, ip, j, k)]) + R(ru[c]) + R(ru[cidx(g, ip, jm, k)]) + R(ru[cidx(g, i, jm, k)]));
                src += -R(P.cf) * rul * R(P.sinphi);
            }
            src += R(0.5) * (R(cd[c]) + R(cd[cidx(g, i, jm, k)])) * R(P.geo1);
            rhs += (-gpy - R(0)) / (R(1) + q) + src;
            Fmy[c] = rhs;
        }
        // ---------------- z-momentum on face k
        if (ok && k == 0) Fmz[c] = R(0);
        if (zk) {
            R rhs = -((sh[2].fx[ty][tx + 1] - sh[2].fx[ty][tx]) * dxi * R(1) +
                      (sh[2].fy[ty + 1][tx] - sh[2].fy[ty][tx]) * dyi * R(1) + (zhw - zlw) * dzi);
            zlw = zhw;
            if (P.use_diff)
                rhs -= ((t13[cidx(g, ip, j, k)] - t13[c]) * dxi * R(1) + (t23[cidx(g, i, jp, k)] - t23[c]) * dyi * R(1) +
                        (t33[c] - t33[c - g.sk]) * dzi);
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
                (void)thd;
                double tp1 = pavg[5 * g.nz + k], tm1 = pavg[5 * g.nz + k - 1];
                // cell temperatures: this level's, and the one below carried
                // up the block's column (evaluated once per cell)
                double tp3 = eos_T(cd[c], cd[N + c], cd[5 * N + c] / cd[c]);
                double tm3 = (k == k0 || k == 1) ? eos_T(cd[c - g.sk], cd[N + c - g.sk], cd[5 * N + c - g.sk] / cd[c - g.sk])
                                       : t_below;
                t_below = tp3;
                double qvp = nq >= 1 ? prim[4 * N + c] : 0.0, qvm = nq >= 1 ? prim[4 * N + c - g.sk] : 0.0;
                double qcp = nq >= 2 ? prim[5 * N + c] : 0.0, qcm = nq >= 2 ? prim[5 * N + c - g.sk] : 0.0;
                double qpp = nq >= 3 ? prim[6 * N + c] : 0.0, qpm = nq >= 3 ? prim[6 * N + c - g.sk] : 0.0;
                double qplus = 0.61 * (qvp - qvd[k]) - (qcp - qcd[k] + qpp - qpd[k]) + (tp3 - tp1) / tp1 * (1.0 + 0.61 * qvd[k] - qcd[k] - qpd[k]);
                double qminus = 0.61 * (qvm - qvd[k - 1]) - (qcm - qcd[k - 1] + qpm - qpd[k - 1]) + (tm3 - tm1) / tm1 * (1.0 + 0.61 * qvd[k - 1] - qcd[k - 1] - qpd[k - 1]);
                double qavg = 0.5 * (qplus + qminus);
                double r0avg = 0.5 * (rd[k] + rd[k - 1]);
                b = -qavg * r0avg * g2;
            }
            R zsrc = R(b);
            if (P.coriolis) {
                R rul = R(0.25) * (R(ru[cidx(g, ip, j, k)]) + R(ru[c]) + R(ru[cidx(g, ip, j, k - 1)]) + R(ru[c - g.sk]));
                zsrc += R(P.cf) * rul * R(P.cosphi);
            }
            zsrc += R(0.5) * (R(cd[c]) + R(cd[c - g.sk])) * R(P.geo2);
            R gpz = dzi * (pp[c] - pp[c - g.sk]) / R(1);
            R q = R(0);
            if (P.moist) q = R(0.5) * (prim[4 * N + c] + prim[4 * N + c - g.sk] + prim[5 * N + c] + prim[5 * N + c - g.sk]);
            rhs += (zsrc - gpz - R(0)) / (R(1) + q);
            Fmz[c] = rhs;
        }
        if (ok && k == g.nz - 1) Fmz[c + g.sk] = R(0);
        // the next level's first barrier orders the reuse of sh
    }
}

// ---------------------------------------------------------------------------
// Host launchers: scheme dispatch, grid sizing and the explicit
// instantiations for the plain (double) and mixed (float) forms.
// ---------------------------------------------------------------------------
namespace {


dim3 cell_block() { return dim3(32, 4, 1); }
dim3 cell_grid(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz); }

constexpr int U5 = ERF_ADV_UPWIND_5TH, W5 = ERF_ADV_WENO_5;

template <class R>
using SlowCellK = void (*)(Params, int, StateBuf, StageAux<R>, const R*, const R*, const R*, const R*, TkeBuf<R>, R*, R*,
                           R*, R*);
template <class R>
using SlowMomK = void (*)(Params, int, StateBuf, StageAux<R>, const double*, const double*, const double*, const R*,
                          const R*, const R*, const R*, const R*, const R*, const double*, R*, R*, R*);
template <class R>
using PostK = void (*)(Params, int, double, StateBuf, StateBuf, StateBuf, StateBuf, StageAux<R>, StageAux<R>, int,
                       const R*, TkeBuf<R>, const R*, const R*, const R*, double*, double*, double*);

template <class R>
SlowCellK<R> slow_cell_kernel(const Params& P) {
    if (P.dyc_h == U5 && P.dyc_v == U5) return k_slow_cell<R, U5, U5>;
    if (P.dyc_h == W5 && P.dyc_v == W5) return k_slow_cell<R, W5, W5>;
    return k_slow_cell<R, -1, -1>;
}
template <class R>
SlowMomK<R> slow_mom_kernel(const Params& P) {
    if (P.dyc_h == U5 && P.dyc_v == U5) return k_slow_mom<R, U5, U5>;
    return k_slow_mom<R, -1, -1>;
}
template <class R>
PostK<R> post_kernel(const Params& P) {
    bool dw = P.dry_h == W5 && P.dry_v == W5, du = P.dry_h == U5 && P.dry_v == U5;
    bool mw = P.moi_h == W5 && P.moi_v == W5, mu = P.moi_h == U5 && P.moi_v == U5;
    const int nslow = (P.moist ? 1 + (P.ncomp - ERF_RHOQ1_COMP) : 1) + (P.les == ERF_LES_DEARDORFF ? 1 : 0);
    if (!P.moist) {
        if (dw) return k_post<R, W5, W5, -1, -1, 4>;
        if (du) return k_post<R, U5, U5, -1, -1, 4>;
    } else if (nslow <= 4) {
        if (dw && mw) return k_post<R, W5, W5, W5, W5, 4>;
        if (du && mu) return k_post<R, U5, U5, U5, U5, 4>;
        if (du && mw) return k_post<R, U5, U5, W5, W5, 4>;
    } else {
        if (dw && mw) return k_post<R, W5, W5, W5, W5, 5>;
        if (du && mu) return k_post<R, U5, U5, U5, U5, 5>;
        if (du && mw) return k_post<R, U5, U5, W5, W5, 5>;
        return k_post<R, -1, -1, -1, -1, 5>;
    }
    return k_post<R, -1, -1, -1, -1, 4>;
}

}  // namespace

template <class R>
void tiled_setup(const Params& P, TiledKz* t) {
    t->cell = pick_kz(slow_cell_kernel<R>(P), P.g);
    t->mom = pick_kz(slow_mom_kernel<R>(P), P.g);
    t->post = pick_kz(post_kernel<R>(P), P.g);
}

// The dynamic shared-memory opt-in is a property of the kernel for the whole
// process, shared by every context: it is raised to the device maximum (the
// size passed at launch still sets each launch's footprint), so that contexts
// of different sizes never lower it below one another's needs.
template <class R>
int vert_setup(size_t vert_smem, size_t coef_smem) {
    int dev = 0, maxopt = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 1;
    if (vert_smem > (size_t)maxopt || coef_smem > (size_t)maxopt) return 1;
    if (cudaFuncSetAttribute(k_fast_vert<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxopt) != cudaSuccess ||
        cudaFuncSetAttribute(k_fast_coef<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxopt) != cudaSuccess)
        return 1;
    return 0;
}

template <class R>
void launch_step_begin(const Params& P, cudaStream_t st, const double* cons, const double* uo, const double* vo,
                       const double* wo, StateBuf S, double* un, double* vn, double* wn, StageAux<R> A, R* mut,
                       TkeBuf<R> tke) {
    k_step_begin<R><<<cell_grid(P.g), cell_block(), 0, st>>>(P, cons, uo, vo, wo, S, un, vn, wn, A, mut, tke);
}
template <class R>
void launch_stage_aux(const Params& P, cudaStream_t st, const double* cons, StageAux<R> A) {
    k_stage_aux<R><<<cell_grid(P.g), cell_block(), 0, st>>>(P, cons, A);
}
template <class R>
void launch_tau(const Params& P, cudaStream_t st, const double* cons, const double* u, const double* v,
                const double* w, const R* mut, R* t11, R* t22, R* t33, R* t12, R* t13, R* t23) {
    k_tau<R><<<cell_grid(P.g), cell_block(), 0, st>>>(P, cons, u, v, w, mut, t11, t22, t33, t12, t13, t23);
    if (P.most)   // the validated MOST configurations carry an eddy-viscosity closure
        k_tau_most_ground<R><<<dim3((P.g.nx + 31) / 32, (P.g.ny + 3) / 4), dim3(32, 4), 0, st>>>(P, cons, u, v, w, mut,
                                                                                               t13, t23);
}
template <class R>
void launch_plane_avg(const Params& P, cudaStream_t st, const double* cons, const R* prim, double* avg) {
    k_plane_avg<R><<<dim3(P.g.nz, PAVG_PARTS), 256, 0, st>>>(P, cons, prim, avg);
}
template <class R>
void launch_fast_h(const Params& P, cudaStream_t st, int step, int nrk, double dtau, double facinv, StateBuf Sprev,
                   int prev_rt, StateBuf Sst, StageAux<R> A, const R* Fmx, const R* Fmy, const R* lag_in, R* lag_out,
                   R* avx, R* avy, double* outx, double* outy) {
    k_fast_h<R><<<cell_grid(P.g), cell_block(), 0, st>>>(P, step, nrk, dtau, facinv, Sprev, prev_rt, Sst, A, Fmx, Fmy,
                                                         lag_in, lag_out, avx, avy, outx, outy);
}
// ABLMost::update_fluxes (BoundaryConditions/ERF_ABLMost.cpp:11-142) on the
// step's old velocities: plane means of u and v on their faces (the periodic
// high face excluded) and of sqrt(uc^2 + vc^2) at the cell centres of level
// most_k (MOSTAverage::compute_plane_averages, ERF_MOSTAverage.cpp:674-940),
// then u* = kappa |U| / ln(z_ref / z0) of the adiabatic surface
// (ERF_MOSTStress.H:89-124).  One block; each thread sums a fixed stride and
// the partial sums are added in a fixed tree, so the result is reproducible.
constexpr int MOST_THREADS = 512;
__global__ void __launch_bounds__(MOST_THREADS) k_most_avg(Params P, const double* __restrict__ u,
                                                           const double* __restrict__ v) {
    __shared__ double red[3][MOST_THREADS];
    const Geo& g = P.g;
    const int k = P.most_k;
    double su = 0.0, sv = 0.0, sm = 0.0;
    for (int64_t q = threadIdx.x; q < g.sk; q += MOST_THREADS) {
        const int i = (int)(q % g.nx), j = (int)(q / g.nx);
        const double uf = u[cidx(g, i, j, k)], vf = v[cidx(g, i, j, k)];
        su += uf;
        sv += vf;
        const double uc = 0.5 * (uf + u[cidx(g, wrap(i + 1, g.nx), j, k)]);
        const double vc = 0.5 * (vf + v[cidx(g, i, wrap(j + 1, g.ny), k)]);
        sm += sqrt(uc * uc + vc * vc + 0.0 * 0.0);
    }
    red[0][threadIdx.x] = su;
    red[1][threadIdx.x] = sv;
    red[2][threadIdx.x] = sm;
    __syncthreads();
    for (int h = MOST_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double denom = 1.0 / (double)g.sk;
        P.most_avg[0] = red[0][0] * denom;
        P.most_avg[1] = red[1][0] * denom;
        P.most_avg[2] = red[2][0] * denom;
        P.most_avg[3] = 0.41 * P.most_avg[2] / log(P.most_zref / P.most_z0);
    }
}
void launch_most_avg(const Params& P, cudaStream_t st, const double* u, const double* v) {
    k_most_avg<<<1, MOST_THREADS, 0, st>>>(P, u, v);
}
template <class R>
void launch_no_substep(const Params& P, cudaStream_t st, double slow_dt, StateBuf Sold, const R* Fcons, const R* Fmx,
                       const R* Fmy, const R* Fmz, StateBuf Ssum) {
    k_no_substep<R><<<cell_grid(P.g), cell_block(), 0, st>>>(P.g, slow_dt, Sold, Fcons, Fmx, Fmy, Fmz, Ssum);
}
template <class R>
void launch_fast_coef(const Params& P, cudaStream_t st, dim3 grid, dim3 block, size_t smem, double D, StateBuf Sst,
                      StageAux<R> A, R* cA, R* cInvB, R* cCB, R* cP, R* cQ) {
    k_fast_coef<R><<<grid, block, smem, st>>>(P, D, Sst, A, cA, cInvB, cCB, cP, cQ);
}
template <class R>
void launch_fast_vert(const Params& P, cudaStream_t st, dim3 grid, dim3 block, size_t smem, double dtau,
                      double facinv, double beta_1, double beta_2, StateBuf Sprev, int prev_rt, StateBuf Sst,
                      StageAux<R> A, const R* Fcons, const R* Fmz, const double* newx, const double* newy,
                      const R* cA, const R* cInvB, const R* cCB, const R* cP, const R* cQ, R* avz, double* out_cons,
                      double* out_mz) {
    k_fast_vert<R><<<grid, block, smem, st>>>(P, dtau, facinv, beta_1, beta_2, Sprev, prev_rt, Sst, A, Fcons, Fmz,
                                              newx, newy, cA, cInvB, cCB, cP, cQ, avz, out_cons, out_mz);
}
template <class R>
void launch_slow_cell(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux<R> A, const R* mut,
                      const R* hx, const R* hy, const R* hz, TkeBuf<R> tke, R* Fcons, R* avx, R* avy, R* avz) {
    slow_cell_kernel<R>(P)<<<tile_grid(P.g, t.cell), dim3(TTX, TTY, 1), 0, st>>>(P, t.cell, S, A, mut, hx, hy, hz,
                                                                                  tke, Fcons, avx, avy, avz);
}
template <class R>
void launch_slow_mom(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux<R> A, const double* u,
                     const double* v, const double* w, const R* t11, const R* t22, const R* t33, const R* t12,
                     const R* t13, const R* t23, const double* pavg, R* Fmx, R* Fmy, R* Fmz) {
    slow_mom_kernel<R>(P)<<<tile_grid(P.g, t.mom), dim3(TTX, TTY, 1), 0, st>>>(P, t.mom, S, A, u, v, w, t11, t22, t33,
                                                                                t12, t13, t23, pavg, Fmx, Fmy, Fmz);
}
template <class R>
void launch_post(const Params& P, const TiledKz& t, cudaStream_t st, double slow_dt, StateBuf Sold, StateBuf Sst,
                 StateBuf Ssum, StateBuf Snew, StageAux<R> Acur, StageAux<R> Anext, int make_next, const R* mut,
                 TkeBuf<R> tke, const R* avx, const R* avy, const R* avz, double* un, double* vn, double* wn) {
    post_kernel<R>(P)<<<tile_grid(P.g, t.post), dim3(TTX, TTY, 1), 0, st>>>(P, t.post, slow_dt, Sold, Sst, Ssum, Snew,
                                                                             Acur, Anext, make_next, mut, tke, avx,
                                                                             avy, avz, un, vn, wn);
}

#define ERFB_INSTANTIATE(R)                                                                                          \
    template void tiled_setup<R>(const Params&, TiledKz*);                                                           \
    template int vert_setup<R>(size_t, size_t);                                                                      \
    template void launch_step_begin<R>(const Params&, cudaStream_t, const double*, const double*, const double*,     \
                                       const double*, StateBuf, double*, double*, double*, StageAux<R>, R*,          \
                                       TkeBuf<R>);                                                                   \
    template void launch_tau<R>(const Params&, cudaStream_t, const double*, const double*, const double*,            \
                                const double*, const R*, R*, R*, R*, R*, R*, R*);                                    \
    template void launch_plane_avg<R>(const Params&, cudaStream_t, const double*, const R*, double*);                \
    template void launch_stage_aux<R>(const Params&, cudaStream_t, const double*, StageAux<R>);                      \
    template void launch_fast_h<R>(const Params&, cudaStream_t, int, int, double, double, StateBuf, int, StateBuf,   \
                                   StageAux<R>, const R*, const R*, const R*, R*, R*, R*, double*, double*);         \
    template void launch_no_substep<R>(const Params&, cudaStream_t, double, StateBuf, const R*, const R*, const R*, \
                                       const R*, StateBuf);                                                          \
    template void launch_fast_coef<R>(const Params&, cudaStream_t, dim3, dim3, size_t, double, StateBuf,             \
                                      StageAux<R>, R*, R*, R*, R*, R*);                                              \
    template void launch_fast_vert<R>(const Params&, cudaStream_t, dim3, dim3, size_t, double, double, double,       \
                                      double, StateBuf, int, StateBuf, StageAux<R>, const R*, const R*,              \
                                      const double*, const double*, const R*, const R*, const R*, const R*,          \
                                      const R*, R*, double*, double*);                                               \
    template void launch_slow_cell<R>(const Params&, const TiledKz&, cudaStream_t, StateBuf, StageAux<R>, const R*,  \
                                      const R*, const R*, const R*, TkeBuf<R>, R*, R*, R*, R*);                      \
    template void launch_slow_mom<R>(const Params&, const TiledKz&, cudaStream_t, StateBuf, StageAux<R>,             \
                                     const double*, const double*, const double*, const R*, const R*, const R*,      \
                                     const R*, const R*, const R*, const double*, R*, R*, R*);                       \
    template void launch_post<R>(const Params&, const TiledKz&, cudaStream_t, double, StateBuf, StateBuf, StateBuf,  \
                                 StateBuf, StageAux<R>, StageAux<R>, int, const R*, TkeBuf<R>, const R*, const R*,   \
                                 const R*, double*, double*, double*);

ERFB_INSTANTIATE(double)
ERFB_INSTANTIATE(float)
#undef ERFB_INSTANTIATE

}  // namespace erfb
