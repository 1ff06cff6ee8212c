// ============================================================================
// erf_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the reference's multirate RK3 dycore step (ERF,
// Source/TimeIntegration/ERF_MRI.H:187-369 and the functions it calls), used as
// the correctness oracle for the CUDA implementation in erf_b200/.  Nothing in
// the product links, imports or executes this file; only tests/, the smoke
// check and bench.py's CPU-baseline leg load the shared library built from it.
//
// Why a restatement: the reference is an AMReX application and AMReX (a git
// submodule, empty in the checkout) plus MPI are absent, so the reference's
// sources cannot be compiled here.  This file follows the reference's loops,
// box extents, ghost-cell fills and operation order line by line, each routine
// citing the reference file:line it restates.  Its own pin is the set of
// reference gold plotfiles checked in tests/test_oracle_gold.py.
//
// Scope (what the C-ABI product supports): one box covering the domain,
// periodic in x and y, SlipWall / NoSlipWall at the bottom and top or a MOST
// ground (flat), flat or static terrain-following grids, map factors 1,
// implicit acoustic substepping or none, Smagorinsky / Deardorff or no LES
// closure, Constant / ConstantAlpha / no molecular diffusion, buoyancy types
// 1-3 (moist over terrain: type 1), Coriolis and geostrophic forcing, Kessler
// microphysics with or without rain.
//
// Layout of the arrays exchanged through the C entry points: dense valid
// regions, i fastest:  cons[ncomp][nz][ny][nx], u[nz][ny][nx+1],
// v[nz][ny+1][nx], w[nz+1][ny][nx]; base state arrays have nz+2 entries
// (index k+1 for cell k).
// ============================================================================

#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <chrono>
#include <memory>

#include "../include/erf_b200.h"

namespace {

// ----------------------------------------------------------------------------
// Physical constants (Source/ERF_Constants.H:10-30, 66-87)
// ----------------------------------------------------------------------------
constexpr double R_d = 287.0;
constexpr double R_v = 461.505;
constexpr double Cp_d = 1004.5;
constexpr double p_0 = 1.0e5;
constexpr double Gamma_ = 1.4;
constexpr double CONST_GRAV = 9.81;
constexpr double ip_0 = 1. / p_0;
constexpr double iR_d = 1. / R_d;
constexpr double iGamma = 1. / Gamma_;
constexpr double L_v = 2.5e6;
constexpr double lcond = 2.501e6;
constexpr double Rd_on_Rv = R_d / R_v;
constexpr double qcw0 = 1.e-3;
constexpr double alphaelq = 1.e-3;

// ----------------------------------------------------------------------------
// Equation of state (Source/Utils/ERF_EOS.H:42-151)
// ----------------------------------------------------------------------------
inline double getPgivenRTh(double rt, double qv = 0.) {
    return p_0 * std::pow(R_d * rt * (1.0 + (R_v / R_d) * qv) * ip_0, Gamma_);
}
inline double getExnergivenRTh(double rt, double rdOcp, double qv = 0.0) {
    return std::pow(R_d * rt * (1.0 + R_v / R_d * qv) * ip_0, Gamma_ * rdOcp);
}
inline double getExnergivenP(double P, double rdOcp) { return std::pow(P * ip_0, rdOcp); }
inline double getRhoThetagivenP(double p, double qv = 0.0) {
    return std::pow(p * std::pow(p_0, Gamma_ - 1), iGamma) * iR_d / (1.0 + R_v / R_d * qv);
}
inline double getTgivenRandRTh(double rho, double rt, double qv = 0.0) {
    double p_loc = p_0 * std::pow(R_d * rt * (1.0 + R_v / R_d * qv) * ip_0, Gamma_);
    return p_loc / (R_d * rho * (1.0 + R_v / R_d * qv));
}
inline double getRhogivenThetaPress(double theta, double p, double rdOcp, double qv = 0.0) {
    return std::pow(p_0, rdOcp) * std::pow(p, iGamma) / (R_d * theta * (1.0 + R_v / R_d * qv));
}

// ----------------------------------------------------------------------------
// Saturation vapour pressure over water: Flatau et al. (1992), Table 4
// polynomials, as used by Source/Utils/ERF_Microphysics_Utils.H:52-160.
// ----------------------------------------------------------------------------
inline double esatw(double t) {
    const double a[9] = {6.11239921, 0.443987641, 0.142986287e-1, 0.264847430e-3,
                         0.302950461e-5, 0.206739458e-7, 0.640689451e-10,
                         -0.952447341e-13, -0.976195544e-15};
    double dtt = std::min(t - 273.16, 70.);
    return a[0] + dtt * (a[1] + dtt * (a[2] + dtt * (a[3] + dtt * (a[4] + dtt * (a[5] + dtt * (a[6] + dtt * (a[7] + a[8] * dtt)))))));
}
inline double dtesatw(double t) {
    const double a[9] = {0.443956472, 0.285976452e-1, 0.794747212e-3, 0.121167162e-4,
                         0.103167413e-6, 0.385208005e-9, -0.604119582e-12,
                         -0.792933209e-14, -0.599634321e-17};
    double dtt = t - 273.16;
    if (dtt >= 70.) return 0.0;
    return a[0] + dtt * (a[1] + dtt * (a[2] + dtt * (a[3] + dtt * (a[4] + dtt * (a[5] + dtt * (a[6] + dtt * (a[7] + a[8] * dtt)))))));
}
inline double qsatw(double t, double p) {
    double es = esatw(t);
    return Rd_on_Rv * es / std::max(es, p - es);
}
inline double dtqsatw(double t, double p) { return Rd_on_Rv * dtesatw(t) / p; }

// ----------------------------------------------------------------------------
// A FAB: box [lo,hi] (inclusive), ncomp components, i fastest.
// ----------------------------------------------------------------------------
struct Fab {
    int lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1}, nc = 0;
    long sj = 0, sk = 0, sn = 0;
    std::vector<double> d;
    Fab() = default;
    Fab(const int l[3], const int h[3], int n, double v = 0.0) { define(l, h, n, v); }
    void define(const int l[3], const int h[3], int n, double v = 0.0) {
        for (int a = 0; a < 3; ++a) { lo[a] = l[a]; hi[a] = h[a]; }
        nc = n;
        sj = hi[0] - lo[0] + 1;
        sk = sj * (hi[1] - lo[1] + 1);
        sn = sk * (hi[2] - lo[2] + 1);
        d.assign((size_t)sn * nc, v);
    }
    inline double& operator()(int i, int j, int k, int n = 0) {
        return d[(i - lo[0]) + (j - lo[1]) * sj + (k - lo[2]) * sk + n * sn];
    }
    inline double operator()(int i, int j, int k, int n = 0) const {
        return d[(i - lo[0]) + (j - lo[1]) * sj + (k - lo[2]) * sk + n * sn];
    }
    void copy_from(const Fab& o) { d = o.d; }
};

struct Bx { int lo[3], hi[3]; };

template <class F>
inline void loop(const Bx& b, F&& f) {
#pragma omp parallel for schedule(static)
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}
template <class F>
inline void loop_serial(const Bx& b, F&& f) {
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}

// Index types: 0 cell, 1 x-face, 2 y-face, 3 z-face
enum { CC = 0, XF = 1, YF = 2, ZF = 3 };

struct Oracle {
    erf_b200_config c;
    int nx, ny, nz, ncomp, nprim;
    int ngc = 4, ngv = 3;
    double dxInv[3];
    double rdOcp;
    bool use_moisture, kessler_rain;
    bool use_diff, use_turb, use_consA;
    bool zlo_noslip, zhi_noslip;
    // MOST surface layer at the ground (BoundaryConditions/ERF_ABLMost.*):
    // Moeng stress, adiabatic surface, constant roughness, plane averages at
    // the reference height snapped to the cell centre of level most_k
    bool most = false;
    int most_k = 0;
    double most_zref = 0.0, most_um = 0.0, most_vm = 0.0, most_umm = 0.0, most_ustar = 0.0;
    // base state, index k+1 for cell k
    std::vector<double> r0, p0, pi0, th0;

    Oracle(const erf_b200_config& cfg) : c(cfg) {
        nx = c.nx; ny = c.ny; nz = c.nz; ncomp = c.ncomp; nprim = ncomp - 1;
        dxInv[0] = 1.0 / c.dx; dxInv[1] = 1.0 / c.dy; dxInv[2] = 1.0 / c.dz;
        rdOcp = R_d / c.c_p;
        use_moisture = (c.moisture != ERF_MOIST_NONE);
        kessler_rain = (c.moisture == ERF_MOIST_KESSLER);
        use_diff = (c.molec_diff_type != ERF_MOLEC_NONE) || (c.les_type != ERF_LES_NONE);
        use_turb = (c.les_type != ERF_LES_NONE);
        use_consA = (c.molec_diff_type == ERF_MOLEC_CONSTANT_ALPHA);
        zlo_noslip = (c.zlo_bc == ERF_BC_NO_SLIP_WALL);
        zhi_noslip = (c.zhi_bc == ERF_BC_NO_SLIP_WALL);
        most = (c.zlo_bc == ERF_BC_MOST);
        if (most) {
            // MOSTAverage::set_k_indices_N (ERF_MOSTAverage.cpp:366-388):
            // the level of z_ref, and z_ref moved to that level's centre
            const double zr = c.most_zref > 0.0 ? c.most_zref : 0.5 * c.dz;
            most_k = static_cast<int>(std::floor(zr / c.dz - 0.5));
            most_zref = (most_k + 0.5) * c.dz;
        }
        r0.assign(nz + 2, 0.); p0.assign(nz + 2, 0.); pi0.assign(nz + 2, 0.); th0.assign(nz + 2, 0.);
    }

    // ------------------------------------------------------------------ boxes
    Bx valid(int t) const {
        Bx b{{0, 0, 0}, {nx - 1, ny - 1, nz - 1}};
        if (t == XF) b.hi[0] = nx;
        if (t == YF) b.hi[1] = ny;
        if (t == ZF) b.hi[2] = nz;
        return b;
    }
    void alloc(Fab& f, int t, int ng, int n) const {
        Bx b = valid(t);
        int l[3], h[3];
        for (int a = 0; a < 3; ++a) { l[a] = b.lo[a] - ng; h[a] = b.hi[a] + ng; }
        f.define(l, h, n, 0.0);
    }
    static Bx grow(Bx b, int gx, int gy, int gz) {
        b.lo[0] -= gx; b.hi[0] += gx; b.lo[1] -= gy; b.hi[1] += gy; b.lo[2] -= gz; b.hi[2] += gz;
        return b;
    }

    // ------------------------------------------------------------------
    // FillBoundary with x/y periodicity: every ghost cell whose periodic
    // image lies in the valid region receives a copy of it, all components.
    // ------------------------------------------------------------------
    void fill_periodic(Fab& f, int t) const {
        Bx v = valid(t);
        int px = nx, py = ny;
        for (int n = 0; n < f.nc; ++n)
            for (int k = f.lo[2]; k <= f.hi[2]; ++k) {
                if (k < v.lo[2] || k > v.hi[2]) continue;
                for (int j = f.lo[1]; j <= f.hi[1]; ++j)
                    for (int i = f.lo[0]; i <= f.hi[0]; ++i) {
                        bool in = (i >= v.lo[0] && i <= v.hi[0] && j >= v.lo[1] && j <= v.hi[1]);
                        if (in) continue;
                        int is = i, js = j;
                        while (is < v.lo[0]) is += px;
                        while (is > v.hi[0]) is -= px;
                        while (js < v.lo[1]) js += py;
                        while (js > v.hi[1]) js -= py;
                        f(i, j, k, n) = f(is, js, k, n);
                    }
            }
    }

    // ERFPhysBCFunct_cons (BoundaryConditions/ERF_PhysBCFunct.cpp:16-75 and
    // ERF_BoundaryConditions_cons.cpp:286-400): FillBoundary, then the vertical
    // foextrap of components [icomp, icomp+ncomp) on the box grown by ng.
    void physbcs_cons(Fab& cons, int icomp, int ncmp, int ng) const {
        fill_periodic(cons, CC);
        Bx b = grow(valid(CC), ng, ng, ng);
        for (int n = icomp; n < icomp + ncmp; ++n)
            for (int k = b.lo[2]; k <= b.hi[2]; ++k) {
                if (k >= 0 && k <= nz - 1) continue;
                int ks = (k < 0) ? 0 : nz - 1;
                for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                    for (int i = b.lo[0]; i <= b.hi[0]; ++i) cons(i, j, k, n) = cons(i, j, ks, n);
            }
    }
    // ERFPhysBCFunct_u / _v (ERF_BoundaryConditions_xvel.cpp:155-230): tangential
    // velocity below/above the walls: ext_dir (no-slip, value 0) or foextrap;
    // below a MOST ground reflect_odd (ERF_init_bcs.cpp:404-410), which the
    // MOST fill of the stage boundary fills then overwrites.
    void physbcs_tangential(Fab& f, int t, int ng) const {
        fill_periodic(f, t);
        Bx b = grow(valid(t), ng, ng, ng);
        for (int k = b.lo[2]; k <= b.hi[2]; ++k) {
            if (k >= 0 && k <= nz - 1) continue;
            bool lo = (k < 0);
            bool noslip = lo ? zlo_noslip : zhi_noslip;
            int ks = lo ? 0 : nz - 1;
            for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
                    if (lo && most) f(i, j, k) = -f(i, j, -1 - k);
                    else f(i, j, k) = noslip ? 0.0 : f(i, j, ks);
                }
        }
    }
    // ERFPhysBCFunct_w (ERF_BoundaryConditions_zvel.cpp:151-227): w = 0 on the
    // bottom and top faces (ext_dir for both wall kinds).
    void physbcs_w(Fab& w, int ng) const {
        fill_periodic(w, ZF);
        Bx b = grow(valid(ZF), ng, ng, 0);
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) { w(i, j, 0) = 0.0; w(i, j, nz) = 0.0; }
    }

    // Utils/ERF_MomentumToVelocity.cpp:25-96 (valid faces only)
    void mom_to_vel(Fab& u, Fab& v, Fab& w, const Fab& cons, const Fab& mx, const Fab& my, const Fab& mz) const {
        loop(valid(XF), [&](int i, int j, int k) { u(i, j, k) = mx(i, j, k) * 2.0 / (cons(i, j, k, 0) + cons(i - 1, j, k, 0)); });
        loop(valid(YF), [&](int i, int j, int k) { v(i, j, k) = my(i, j, k) * 2.0 / (cons(i, j, k, 0) + cons(i, j - 1, k, 0)); });
        loop(valid(ZF), [&](int i, int j, int k) { w(i, j, k) = mz(i, j, k) * 2.0 / (cons(i, j, k, 0) + cons(i, j, k - 1, 0)); });
    }
    // Utils/ERF_VelocityToMomentum.cpp:28-100 on faces grown by (1,1,1)/(1,1,1)/(1,1,0)
    void vel_to_mom(const Fab& u, const Fab& v, const Fab& w, const Fab& cons, Fab& mx, Fab& my, Fab& mz) const {
        loop(grow(valid(XF), 1, 1, 1), [&](int i, int j, int k) { mx(i, j, k) = u(i, j, k) * 0.5 * (cons(i, j, k, 0) + cons(i - 1, j, k, 0)); });
        loop(grow(valid(YF), 1, 1, 1), [&](int i, int j, int k) { my(i, j, k) = v(i, j, k) * 0.5 * (cons(i, j, k, 0) + cons(i, j - 1, k, 0)); });
        loop(grow(valid(ZF), 1, 1, 0), [&](int i, int j, int k) { mz(i, j, k) = w(i, j, k) * 0.5 * (cons(i, j, k, 0) + cons(i, j, k - 1, 0)); });
    }

    struct State { Fab cons, mx, my, mz; };
    struct Vel { Fab u, v, w; };

    void alloc_state(State& s) const {
        alloc(s.cons, CC, ngc, ncomp); alloc(s.mx, XF, ngv, 1); alloc(s.my, YF, ngv, 1); alloc(s.mz, ZF, ngv, 1);
    }
    void alloc_vel(Vel& v) const { alloc(v.u, XF, ngv, 1); alloc(v.v, YF, ngv, 1); alloc(v.w, ZF, ngv, 1); }
    static void copy_state(State& d, const State& s) {
        d.cons.copy_from(s.cons); d.mx.copy_from(s.mx); d.my.copy_from(s.my); d.mz.copy_from(s.mz);
    }

    // FillIntermediatePatch (BoundaryConditions/ERF_FillIntermediatePatch.cpp:32-261), level 0;
    // the MOST ghost velocities are imposed after the physical boundary
    // conditions when allowed (:222-237; apply_bcs allows them outside the
    // acoustic substeps)
    void fill_intermediate(State& S, Vel& V, int ng_cons, int ng_vel, bool cons_only, int icomp, int ncmp,
                           bool allow_most = false) const {
        if (!cons_only) mom_to_vel(V.u, V.v, V.w, S.cons, S.mx, S.my, S.mz);
        physbcs_cons(S.cons, icomp, ncmp, ng_cons);
        if (!cons_only) {
            physbcs_tangential(V.u, XF, ng_vel);
            physbcs_tangential(V.v, YF, ng_vel);
            if (terrain) physbcs_w_T(V.w, V.u, V.v, ng_vel);
            else physbcs_w(V.w, ng_vel);
            if (most && allow_most) impose_most(S.cons, V.u, V.v);
            vel_to_mom(V.u, V.v, V.w, S.cons, S.mx, S.my, S.mz);
        }
        fill_periodic(S.cons, CC); fill_periodic(S.mx, XF); fill_periodic(S.my, YF); fill_periodic(S.mz, ZF);
    }

    // ABLMost::update_fluxes (BoundaryConditions/ERF_ABLMost.cpp:11-142) on
    // the step's old velocities: MOSTAverage::compute_plane_averages
    // (ERF_MOSTAverage.cpp:674-940; policy 0, no interpolation, no time
    // filter) of u and v on their faces (the periodic high face excluded) and
    // of the horizontal speed sqrt(uc^2 + vc^2) at the cell centres of level
    // most_k, then the adiabatic friction velocity of ERF_MOSTStress.H:89-124,
    // u* = kappa umm / ln(z_ref / z0).
    void most_update_fluxes(const Vel& V) {
        const int k = most_k;
        double su = 0.0, sv = 0.0, sm = 0.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                su += V.u(i, j, k);
                sv += V.v(i, j, k);
                double uc = 0.5 * (V.u(i, j, k) + V.u(i + 1, j, k));
                double vc = 0.5 * (V.v(i, j, k) + V.v(i, j + 1, k));
                sm += std::sqrt(uc * uc + vc * vc + 0.0 * 0.0);
            }
        const double denom = 1.0 / (double)(nx * ny);
        most_um = su * denom;
        most_vm = sv * denom;
        most_umm = sm * denom;
        most_ustar = 0.41 * most_umm / std::log(most_zref / c.most_z0);
    }

    // moeng_flux::compute_u_flux / compute_v_flux (ERF_MOSTStress.H:1395-1555)
    // of ABLMost::compute_most_bcs (ERF_ABLMost.cpp:289-489), implicit
    // (not explicit) MOST: every ghost level below the ground gets
    // u(k) = u(0) + tau/eta * dz * (0 - k), with the Moeng stress from the
    // level-0 velocity, the plane means and u*, and eta the eddy viscosity at
    // level 0 averaged to the face (floored at 1e-8).  Index clamps follow
    // the reference's array bounds (velocities 3 ghosts, cons 4, eddy
    // viscosity 2).  The adiabatic surface leaves rho*theta's foextrap ghosts.
    void impose_most(const Fab& cons, Fab& u, Fab& v) const {
        const double WSMIN = 0.1, eta_eps = 1e-8, dz = c.dz;
        const int klo = 0;
        auto clampi = [](int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); };
        // eddy viscosity bounds of a 2-ghost cell array
        const int elx = -2, ehx = nx + 1, ely = -2, ehy = ny + 1;
        auto eta_at = [&](int ie, int je) { return mut(ie, je, klo); };
        for (int k = u.lo[2]; k <= -1; ++k)
            for (int j = u.lo[1]; j <= u.hi[1]; ++j)
                for (int i = u.lo[0]; i <= u.hi[0]; ++i) {
                    int iylo = i <= v.lo[0] ? v.lo[0] : i - 1;
                    int iyhi = i > v.hi[0] ? v.hi[0] : i;
                    int jy = clampi(j, v.lo[1], v.hi[1] - 1);
                    int ic = clampi(i, cons.lo[0] + 1, cons.hi[0]);
                    int jc = clampi(j, cons.lo[1], cons.hi[1]);
                    double velx = u(i, j, klo);
                    double vely = 0.25 * (v(iyhi, jy, klo) + v(iyhi, jy + 1, klo) + v(iylo, jy, klo) + v(iylo, jy + 1, klo));
                    double rho = 0.5 * (cons(ic - 1, jc, klo, 0) + cons(ic, jc, klo, 0));
                    double umean = most_um;
                    double wsp_mean = 0.5 * (most_umm + most_umm);
                    double ustar = 0.5 * (most_ustar + most_ustar);
                    double wsp = std::sqrt(velx * velx + vely * vely);
                    double num1 = wsp * umean;
                    double num2 = wsp_mean * (velx - umean);
                    double deltaz = dz * (klo - k);
                    wsp_mean = std::max(wsp_mean, WSMIN);
                    double stressx = -rho * ustar * ustar * (num1 + num2) / (wsp_mean * wsp_mean);
                    int ie = clampi(i, elx + 1, ehx), je = clampi(j, ely, ehy);
                    double eta = 0.5 * (eta_at(ie - 1, je) + eta_at(ie, je));
                    eta = std::max(eta, eta_eps);
                    u(i, j, k) = u(i, j, klo) + stressx / eta * deltaz;
                }
        for (int k = v.lo[2]; k <= -1; ++k)
            for (int j = v.lo[1]; j <= v.hi[1]; ++j)
                for (int i = v.lo[0]; i <= v.hi[0]; ++i) {
                    int ix = clampi(i, u.lo[0], u.hi[0]);
                    ix = ix > u.hi[0] - 1 ? u.hi[0] - 1 : ix;
                    int jxlo = j <= u.lo[1] ? u.lo[1] : j - 1;
                    int jxhi = j > u.hi[1] ? u.hi[1] : j;
                    int ic = clampi(i, cons.lo[0], cons.hi[0]);
                    int jc = clampi(j, cons.lo[1] + 1, cons.hi[1]);
                    double velx = 0.25 * (u(ix, jxhi, klo) + u(ix + 1, jxhi, klo) + u(ix, jxlo, klo) + u(ix + 1, jxlo, klo));
                    double vely = v(i, j, klo);
                    double rho = 0.5 * (cons(ic, jc - 1, klo, 0) + cons(ic, jc, klo, 0));
                    double vmean = most_vm;
                    double wsp_mean = 0.5 * (most_umm + most_umm);
                    double ustar = 0.5 * (most_ustar + most_ustar);
                    double wsp = std::sqrt(velx * velx + vely * vely);
                    double num1 = wsp * vmean;
                    double num2 = wsp_mean * (vely - vmean);
                    double deltaz = dz * (klo - k);
                    wsp_mean = std::max(wsp_mean, WSMIN);
                    double stressy = -rho * ustar * ustar * (num1 + num2) / (wsp_mean * wsp_mean);
                    int ie = clampi(i, elx, ehx), je = clampi(j, ely + 1, ehy);
                    double eta = 0.5 * (eta_at(ie, je - 1) + eta_at(ie, je));
                    eta = std::max(eta, eta_eps);
                    v(i, j, k) = v(i, j, klo) + stressy / eta * deltaz;
                }
    }

    // apply_bcs (TimeIntegration/ERF_TI_utils.H:53-150)
    void apply_bcs(State& S, Vel& V, int ng_cons, int ng_vel, bool fast_only, bool synced) const {
        int scomp, ncmp, ngu;
        if (!synced) {
            ngu = std::max(ng_cons, ng_vel + 1);
            fill_intermediate(S, V, ngu, 0, true, 0, 1);
        }
        if (synced) {
            scomp = 0; ncmp = fast_only ? 2 : ncomp;
            ngu = std::max(ng_cons, ng_vel + 1);
        } else {
            scomp = 1; ncmp = fast_only ? 1 : ncomp - 1;
            ngu = ng_cons;
        }
        fill_intermediate(S, V, ngu, ng_vel, false, scomp, ncmp, !fast_only);
    }

    // cons_to_prim (TimeIntegration/ERF_TI_utils.H:4-45)
    void cons_to_prim(const Fab& cons, int ng, Fab& prim, Fab& pi_stage) const {
        loop(grow(valid(CC), ng, ng, ng), [&](int i, int j, int k) {
            double rho = cons(i, j, k, 0);
            prim(i, j, k, 0) = cons(i, j, k, 1) / rho;
            for (int n = 1; n < nprim; ++n) prim(i, j, k, n) = cons(i, j, k, 1 + n) / rho;
        });
        loop(grow(valid(CC), 1, 1, 1), [&](int i, int j, int k) { pi_stage(i, j, k) = getExnergivenRTh(cons(i, j, k, 1), rdOcp); });
    }

    // ------------------------------------------------------------------
    // Face interpolants (Source/Utils/ERF_Interpolation_UPW.H, _WENO.H).
    // s[0..5] = phi(-3..+2) relative to the face's high-side cell.
    // ------------------------------------------------------------------
    static double interp(int type, const double s[6], double upw, double upw_frac) {
        const double sm3 = s[0], sm2 = s[1], sm1 = s[2], s0 = s[3], sp1 = s[4], sp2 = s[5];
        const double tol = 1.0e-12, eps = 1.0e-6;
        switch (type) {
        case ERF_ADV_CENTERED_2ND: return 0.5 * (s0 + sm1);
        case ERF_ADV_UPWIND_3RD: {
            if (upw != 0.) upw = (upw > 0) ? 1. : -1.;
            upw *= upw_frac;
            double a1 = s0 + sm1, d1 = s0 - sm1, a2 = sp1 + sm2, d2 = sp1 - sm2;
            return (7.0 / 12.0) * a1 - (1.0 / 12.0) * a2 + upw * (1.0 / 12.0) * (d2 - 3.0 * d1);
        }
        case ERF_ADV_CENTERED_4TH: {
            double a1 = s0 + sm1, a2 = sp1 + sm2;
            return (7.0 / 12.0) * a1 - (1.0 / 12.0) * a2;
        }
        case ERF_ADV_UPWIND_5TH: {
            if (upw != 0.) upw = (upw > 0) ? 1. : -1.;
            upw *= upw_frac;
            double a1 = s0 + sm1, a2 = sp1 + sm2, a3 = sp2 + sm3;
            double d1 = s0 - sm1, d2 = sp1 - sm2, d3 = sp2 - sm3;
            return (37.0 / 60.0) * a1 - (2.0 / 15.0) * a2 + (1.0 / 60.0) * a3 - upw * (1.0 / 60.0) * (d3 - 5.0 * d2 + 10.0 * d1);
        }
        case ERF_ADV_CENTERED_6TH: {
            double a1 = s0 + sm1, a2 = sp1 + sm2, a3 = sp2 + sm3;
            return (37.0 / 60.0) * a1 - (2.0 / 15.0) * a2 + (1.0 / 60.0) * a3;
        }
        case ERF_ADV_WENO_3: {
            auto ev = [&](double a, double b, double cc) {
                double b1 = (b - a) * (b - a), b2 = (cc - b) * (cc - b);
                double w1 = (1.0 / 3.0) / ((eps + b1) * (eps + b1));
                double w2 = (2.0 / 3.0) / ((eps + b2) * (eps + b2));
                double ws = w1 + w2;
                double v1 = -a + 3.0 * b, v2 = b + cc;
                return (w1 * v1 + w2 * v2) / (2.0 * ws);
            };
            if (upw > tol) return ev(sm2, sm1, s0);
            if (upw < -tol) return ev(sp1, s0, sm1);
            return 0.5 * (s0 + sm1);
        }
        case ERF_ADV_WENO_5: {
            auto ev = [&](double a, double b, double cc, double dd, double e) {
                const double c1 = 13.0 / 12.0;
                double b1 = c1 * (a - 2.0 * b + cc) * (a - 2.0 * b + cc) + 0.25 * (a - 4.0 * b + 3.0 * cc) * (a - 4.0 * b + 3.0 * cc);
                double b2 = c1 * (b - 2.0 * cc + dd) * (b - 2.0 * cc + dd) + 0.25 * (b - dd) * (b - dd);
                double b3 = c1 * (cc - 2.0 * dd + e) * (cc - 2.0 * dd + e) + 0.25 * (3.0 * cc - 4.0 * dd + e) * (3.0 * cc - 4.0 * dd + e);
                double w1 = (1.0 / 10.0) / ((eps + b1) * (eps + b1));
                double w2 = (3.0 / 5.0) / ((eps + b2) * (eps + b2));
                double w3 = (3.0 / 10.0) / ((eps + b3) * (eps + b3));
                double ws = w1 + w2 + w3;
                double v1 = 2.0 * a - 7.0 * b + 11.0 * cc;
                double v2 = -b + 5.0 * cc + 2.0 * dd;
                double v3 = 2.0 * cc + 5.0 * dd - e;
                return (w1 * v1 + w2 * v2 + w3 * v3) / (6.0 * ws);
            };
            if (upw > tol) return ev(sm3, sm2, sm1, s0, sp1);
            if (upw < -tol) return ev(sp2, sp1, s0, sm1, sm2);
            return 0.5 * (s0 + sm1);
        }
        default: return NAN;
        }
    }
    // UPWINDALL (ERF_Interpolation_UPW.H:528-611): wall-reduced vertical stencils
    static double interp_all(int type, const double s[6], double upw, double upw_frac) {
        if (type == ERF_ADV_CENTERED_2ND) return 0.5 * (s[3] + s[2]);
        double ss[6] = {s[0], s[1], s[2], s[3], s[4], s[5]};
        if (!(type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH)) { ss[0] = 0.; ss[5] = 0.; }
        if (upw != 0.) upw = (upw > 0) ? 1. : -1.;
        upw *= upw_frac;
        double a1 = ss[3] + ss[2], a2 = ss[4] + ss[1], d1 = ss[3] - ss[2], d2 = ss[4] - ss[1];
        double a3 = ss[5] + ss[0], d3 = ss[5] - ss[0];
        if (type == ERF_ADV_UPWIND_3RD) return (7.0 / 12.0) * a1 - (1.0 / 12.0) * a2 + upw * (1.0 / 12.0) * (d2 - 3.0 * d1);
        if (type == ERF_ADV_CENTERED_4TH) return (7.0 / 12.0) * a1 - (1.0 / 12.0) * a2;
        if (type == ERF_ADV_UPWIND_5TH) return (37.0 / 60.0) * a1 - (2.0 / 15.0) * a2 + (1.0 / 60.0) * a3 - upw * (1.0 / 60.0) * (d3 - 5.0 * d2 + 10.0 * d1);
        if (type == ERF_ADV_CENTERED_6TH) return (37.0 / 60.0) * a1 - (2.0 / 15.0) * a2 + (1.0 / 60.0) * a3;
        return 0.;
    }
    static int stencil_width(int type) {
        switch (type) {
        case ERF_ADV_CENTERED_2ND: return 1;
        case ERF_ADV_UPWIND_3RD: case ERF_ADV_CENTERED_4TH: case ERF_ADV_WENO_3: return 2;
        default: return 3;
        }
    }
    // gather phi(i-3..i+2) along direction dir at component n, only touching
    // entries the scheme reads (others are zero)
    static void gather(const Fab& f, int dir, int i, int j, int k, int n, int type, double s[6]) {
        int w = stencil_width(type);
        for (int m = 0; m < 6; ++m) {
            int off = m - 3;
            bool used = (off >= -w && off <= w - 1);
            if (!used) { s[m] = 0.; continue; }
            int ii = i + (dir == 0 ? off : 0), jj = j + (dir == 1 ? off : 0), kk = k + (dir == 2 ? off : 0);
            s[m] = f(ii, jj, kk, n);
        }
    }

    // ------------------------------------------------------------------
    // ComputeStrain_N (Diffusion/ERF_ComputeStrain_N.cpp:28-229), no map
    // factors, lateral directions periodic, z walls per config.
    // ------------------------------------------------------------------
    void compute_strain(const Bx& bxcc, Bx tbxxy, Bx tbxxz, Bx tbxyz, const Fab& u, const Fab& v, const Fab& w,
                        Fab& s11, Fab& s22, Fab& s33, Fab& s12, Fab& s13, Fab& s23) const {
        const double* di = dxInv;
        bool zl_dir = zlo_noslip && tbxxz.lo[2] == 0;
        bool zh_dir = zhi_noslip && tbxxz.hi[2] == nz;
        if (zl_dir) {
            Bx p = tbxxz; p.hi[2] = p.lo[2];
            loop(p, [&](int i, int j, int k) {
                s13(i, j, k) = 0.5 * ((-(8. / 3.) * u(i, j, k - 1) + 3. * u(i, j, k) - (1. / 3.) * u(i, j, k + 1)) * di[2] + (w(i, j, k) - w(i - 1, j, k)) * di[0]);
            });
            Bx q = tbxyz; q.hi[2] = q.lo[2];
            loop(q, [&](int i, int j, int k) {
                s23(i, j, k) = 0.5 * ((-(8. / 3.) * v(i, j, k - 1) + 3. * v(i, j, k) - (1. / 3.) * v(i, j, k + 1)) * di[2] + (w(i, j, k) - w(i, j - 1, k)) * di[1]);
            });
            tbxxz.lo[2] += 1; tbxyz.lo[2] += 1;
        }
        if (zh_dir) {
            Bx p = tbxxz; p.lo[2] = p.hi[2];
            loop(p, [&](int i, int j, int k) {
                s13(i, j, k) = 0.5 * (-(-(8. / 3.) * u(i, j, k) + 3. * u(i, j, k - 1) - (1. / 3.) * u(i, j, k - 2)) * di[2] + (w(i, j, k) - w(i - 1, j, k)) * di[0]);
            });
            Bx q = tbxyz; q.lo[2] = q.hi[2];
            loop(q, [&](int i, int j, int k) {
                s23(i, j, k) = 0.5 * (-(-(8. / 3.) * v(i, j, k) + 3. * v(i, j, k - 1) - (1. / 3.) * v(i, j, k - 2)) * di[2] + (w(i, j, k) - w(i, j - 1, k)) * di[1]);
            });
            tbxxz.hi[2] -= 1; tbxyz.hi[2] -= 1;
        }
        loop(bxcc, [&](int i, int j, int k) {
            s11(i, j, k) = (u(i + 1, j, k) - u(i, j, k)) * di[0];
            s22(i, j, k) = (v(i, j + 1, k) - v(i, j, k)) * di[1];
            s33(i, j, k) = (w(i, j, k + 1) - w(i, j, k)) * di[2];
        });
        loop(tbxxy, [&](int i, int j, int k) { s12(i, j, k) = 0.5 * ((u(i, j, k) - u(i, j - 1, k)) * di[1] + (v(i, j, k) - v(i - 1, j, k)) * di[0]); });
        loop(tbxxz, [&](int i, int j, int k) { s13(i, j, k) = 0.5 * ((u(i, j, k) - u(i, j, k - 1)) * di[2] + (w(i, j, k) - w(i - 1, j, k)) * di[0]); });
        loop(tbxyz, [&](int i, int j, int k) { s23(i, j, k) = 0.5 * ((v(i, j, k) - v(i, j, k - 1)) * di[2] + (w(i, j, k) - w(i, j - 1, k)) * di[1]); });
    }

    // edge FABs with one lateral ghost layer
    void alloc_edges(Fab& s12, Fab& s13, Fab& s23) const {
        int l12[3] = {-2, -2, 0}, h12[3] = {nx + 2, ny + 2, nz - 1};
        int l13[3] = {-2, -2, 0}, h13[3] = {nx + 2, ny + 1, nz};
        int l23[3] = {-2, -2, 0}, h23[3] = {nx + 1, ny + 2, nz};
        s12.define(l12, h12, 1); s13.define(l13, h13, 1); s23.define(l23, h23, 1);
    }
    void alloc_cc1(Fab& f, int n = 1) const {
        int l[3] = {-2, -2, -1}, h[3] = {nx + 1, ny + 1, nz};
        f.define(l, h, n);
    }

    // ComputeSmnSmn (Diffusion/ERF_EddyViscosity.H:31-83); over a MOST ground
    // (implicit) the level-0 cells leave out the strains on the ground faces
    // and take the one-sided average of the faces above (:59-77)
    static double smnsmn(int i, int j, int k, const Fab& t11, const Fab& t22, const Fab& t33, const Fab& t12, const Fab& t13, const Fab& t23,
                         bool most_k0 = false) {
        double s11 = t11(i, j, k), s22 = t22(i, j, k), s33 = t33(i, j, k);
        double s12 = 0.25 * (t12(i, j, k) + t12(i, j + 1, k) + t12(i + 1, j, k) + t12(i + 1, j + 1, k));
        double s13 = most_k0 ? 0.5 * (t13(i, j, k + 1) + t13(i + 1, j, k + 1))
                             : 0.25 * (t13(i, j, k) + t13(i, j, k + 1) + t13(i + 1, j, k) + t13(i + 1, j, k + 1));
        double s23 = most_k0 ? 0.5 * (t23(i, j, k + 1) + t23(i, j + 1, k + 1))
                             : 0.25 * (t23(i, j, k) + t23(i, j, k + 1) + t23(i, j + 1, k) + t23(i, j + 1, k + 1));
        return s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * s12 * s12 + 2.0 * s13 * s13 + 2.0 * s23 * s23;
    }

    // Step-start strain + ComputeTurbulentViscosityLES (Smagorinsky) with the
    // lateral/periodic/vertical ghost treatment of
    // Diffusion/ERF_ComputeTurbulentViscosity.cpp:54-127, 230-432.
    // mu_t holds EddyDiff::Mom_h (== Mom_v for LES), ghost 1.
    void turbulent_viscosity(const Vel& V, const Fab& cons, Fab& mut) const {
        Fab t11, t22, t33, t12, t13, t23;
        alloc_cc1(t11); alloc_cc1(t22); alloc_cc1(t33); alloc_edges(t12, t13, t23);
        Bx bxcc = grow(valid(CC), 1, 1, 0);
        Bx txy = grow(Bx{{0, 0, 0}, {nx, ny, nz - 1}}, 1, 1, 0);
        Bx txz = grow(Bx{{0, 0, 0}, {nx, ny - 1, nz}}, 1, 1, 0);
        Bx tyz = grow(Bx{{0, 0, 0}, {nx - 1, ny, nz}}, 1, 1, 0);
        if (c.les_type == ERF_LES_DEARDORFF) {
            // ERF_ComputeTurbulentViscosity.cpp:129-229 (no terrain, no MOST)
            const double l_C_k = c.Ck, l_C_e = c.Ce, l_C_e_wall = c.Ce_wall;
            const double Ce_lcoeff = std::max(0.0, l_C_e - 1.9 * l_C_k);
            const double l_abs_g = std::fabs(c.gravity), l_inv_theta0 = 1.0 / c.theta_ref;
            loop(valid(CC), [&](int i, int j, int k) {
                double dzInv = dxInv[2];
                if (terrain) dzInv /= hzeta_cc(i, j, k);   // the grid is deformed in z only
                double cellVolMsf = 1.0 / (dxInv[0] * 1.0 * dxInv[1] * 1.0 * dzInv);
                double DeltaMsf = std::pow(cellVolMsf, 1.0 / 3.0);
                double eps = std::numeric_limits<double>::epsilon();
                double dtheta_dz;
                if (most && k == 0) {
                    // one-sided over a MOST ground (ERF_ComputeTurbulentViscosity.cpp:175-188)
                    dtheta_dz = 0.5 * (-3 * cons(i, j, k, 1) / cons(i, j, k, 0) + 4 * cons(i, j, k + 1, 1) / cons(i, j, k + 1, 0) -
                                       cons(i, j, k + 2, 1) / cons(i, j, k + 2, 0)) * dzInv;
                } else {
                    dtheta_dz = 0.5 * (cons(i, j, k + 1, 1) / cons(i, j, k + 1, 0) -
                                       cons(i, j, k - 1, 1) / cons(i, j, k - 1, 0)) * dzInv;
                }
                double E = std::max(cons(i, j, k, ERF_RHOKE_COMP) / cons(i, j, k, 0), 0.0);
                double stratification = l_abs_g * dtheta_dz * l_inv_theta0;
                double length;
                if (stratification <= eps) {
                    length = DeltaMsf;
                } else {
                    length = 0.76 * std::sqrt(E / stratification);
                    length = std::min(length, DeltaMsf);
                    length = std::max(length, 0.001 * DeltaMsf);
                }
                mut(i, j, k) = cons(i, j, k, 0) * l_C_k * length * std::sqrt(E);
                kthv(i, j, k) = (1. + 2. * length / DeltaMsf) * mut(i, j, k);
                double Ce = ((l_C_e_wall > 0) && (k == 0)) ? l_C_e_wall : 1.9 * l_C_k + Ce_lcoeff * length / DeltaMsf;
                diss(i, j, k) = cons(i, j, k, 0) * Ce * std::pow(E, 1.5) / length;
            });
            fill_periodic(kthv, CC);
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) { kthv(i, j, -1) = kthv(i, j, 0); kthv(i, j, nz) = kthv(i, j, nz - 1); }
        } else {
            if (terrain) {
                Fab t21, t31, t32;
                alloc_edges(t21, t31, t32);
                compute_strain_T(bxcc, txy, txz, tyz, V.u, V.v, V.w, t11, t22, t33, t12, t13, t21, t23, t31, t32);
            } else {
                compute_strain(bxcc, txy, txz, tyz, V.u, V.v, V.w, t11, t22, t33, t12, t13, t23);
            }
            double Cs = c.Cs;
            loop(valid(CC), [&](int i, int j, int k) {
                double S = smnsmn(i, j, k, t11, t22, t33, t12, t13, t23, most && k == 0);
                double dzInv = dxInv[2];
                if (terrain) dzInv /= hzeta_cc(i, j, k);
                double cellVolMsf = 1.0 / (dxInv[0] * 1.0 * dxInv[1] * 1.0 * dzInv);
                double DeltaMsf = std::pow(cellVolMsf, 1.0 / 3.0);
                double CsDeltaSqrMsf = Cs * Cs * DeltaMsf * DeltaMsf;
                mut(i, j, k) = CsDeltaSqrMsf * cons(i, j, k, 0) * std::sqrt(2.0 * S);
            });
        }
        // FillBoundary (periodic) then top/bottom extrapolation
        fill_periodic(mut, CC);
        for (int j = -1; j <= ny; ++j)
            for (int i = -1; i <= nx; ++i) { mut(i, j, -1) = mut(i, j, 0); mut(i, j, nz) = mut(i, j, nz - 1); }
    }

    // Eddy diffusivity of a primitive component (EddyDiff mapping,
    // ERF_ComputeTurbulentViscosity.cpp:323-366): Theta: 1/Pr_t, scalars and
    // moisture: 1/Sc_t.
    double eddy_factor(int prim_index) const {
        if (prim_index == 0) return 1.0 / c.Pr_t;
        if (prim_index == 1 || prim_index == 2) return 1.0 / c.sigma_k;   // KE, QKE
        return 1.0 / c.Sc_t;
    }
    double alpha_eff(int prim_index) const {
        // DiffusionSrcForState_N.cpp:100-165
        if (c.molec_diff_type == ERF_MOLEC_NONE) {
            // rhoAlpha_T/C are still rho0_trans*alpha (0 unless set)
        }
        bool consA = use_consA;
        if (prim_index == 0) return consA ? c.alpha_T : c.rho0_trans * c.alpha_T;
        if (prim_index == 1 || prim_index == 2) return 0.0; // KE, QKE
        return consA ? c.alpha_C : c.rho0_trans * c.alpha_C;
    }

    // DiffusionSrcForState_N (Diffusion/ERF_DiffusionSrcForState_N.cpp:39-667),
    // foextrap scalars at walls, no MOST: adds -div(flux) to rhs comps
    void diffusion_state(int start_comp, int ncmp, const Fab& cell_data, const Fab& prim, Fab& rhs, const Fab& mut) const {
        for (int n = 0; n < ncmp; ++n) {
            int q = start_comp + n, pidx = q - 1;
            double ae = alpha_eff(pidx);
            double fac = eddy_factor(pidx);
            Fab fx, fy, fz;
            alloc(fx, XF, 0, 1); alloc(fy, YF, 0, 1); alloc(fz, ZF, 0, 1);
            auto mu = [&](int i, int j, int k) { return mut(i, j, k) * fac; };
            loop(valid(XF), [&](int i, int j, int k) {
                double rA = use_consA ? 0.5 * (cell_data(i, j, k, 0) + cell_data(i - 1, j, k, 0)) * ae : ae;
                if (use_turb) rA += 0.5 * (mu(i, j, k) + mu(i - 1, j, k));
                fx(i, j, k) = -rA * (prim(i, j, k, pidx) - prim(i - 1, j, k, pidx)) * dxInv[0] * 1.0;
            });
            loop(valid(YF), [&](int i, int j, int k) {
                double rA = use_consA ? 0.5 * (cell_data(i, j, k, 0) + cell_data(i, j - 1, k, 0)) * ae : ae;
                if (use_turb) rA += 0.5 * (mu(i, j, k) + mu(i, j - 1, k));
                fy(i, j, k) = -rA * (prim(i, j, k, pidx) - prim(i, j - 1, k, pidx)) * dxInv[1] * 1.0;
            });
            const bool dd = c.les_type == ERF_LES_DEARDORFF;
            loop(valid(ZF), [&](int i, int j, int k) {
                double rA = use_consA ? 0.5 * (cell_data(i, j, k, 0) + cell_data(i, j, k - 1, 0)) * ae : ae;
                if (use_turb) {
                    // Deardorff's vertical heat diffusivity is EddyDiff::Theta_v
                    if (dd && pidx == 0) rA += 0.5 * (kthv(i, j, k) + kthv(i, j, k - 1));
                    else rA += 0.5 * (mu(i, j, k) + mu(i, j, k - 1));
                }
                fz(i, j, k) = -rA * (prim(i, j, k, pidx) - prim(i, j, k - 1, pidx)) * dxInv[2];
                if (q == ERF_RHOTHETA_COMP) hfz(i, j, k) = fz(i, j, k);   // hfx_z, :422-425
            });
            loop(valid(CC), [&](int i, int j, int k) {
                rhs(i, j, k, q) -= (fx(i + 1, j, k) - fx(i, j, k)) * dxInv[0] * 1.0 + (fy(i, j + 1, k) - fy(i, j, k)) * dxInv[1] * 1.0 + (fz(i, j, k + 1) - fz(i, j, k)) * dxInv[2];
            });
            if (dd && q == ERF_RHOKE_COMP) {
                // TKE sources (:681-707): buoyancy, shear production, dissipation
                const double l_abs_g = std::fabs(c.gravity), l_inv_theta0 = 1.0 / c.theta_ref;
                loop(valid(CC), [&](int i, int j, int k) {
                    rhs(i, j, k, q) += l_abs_g * l_inv_theta0 * hfz(i, j, k);
                    rhs(i, j, k, q) += 2.0 * mut(i, j, k) * smn(i, j, k);
                    rhs(i, j, k, q) -= diss(i, j, k);
                });
            }
        }
    }

    // AdvectionSrcForScalars (Advection/ERF_AdvectionSrcForState.cpp:119-370 and
    // ERF_AdvectionSrcForScalars.H): assigns rhs comps
    void advect_scalars(int icomp, int ncmp, const Fab& ax, const Fab& ay, const Fab& az, const Fab& prim, Fab& rhs,
                        int htype, int vtype, double hfrac, double vfrac) const {
        for (int n = 0; n < ncmp; ++n) {
            int q = icomp + n, pidx = q - 1;
            Fab fx, fy, fz;
            alloc(fx, XF, 0, 1); alloc(fy, YF, 0, 1); alloc(fz, ZF, 0, 1);
            loop(valid(XF), [&](int i, int j, int k) {
                double s[6]; gather(prim, 0, i, j, k, pidx, htype, s);
                fx(i, j, k) = ax(i, j, k) * interp(htype, s, ax(i, j, k), hfrac);
            });
            loop(valid(YF), [&](int i, int j, int k) {
                double s[6]; gather(prim, 1, i, j, k, pidx, htype, s);
                fy(i, j, k) = ay(i, j, k) * interp(htype, s, ay(i, j, k), hfrac);
            });
            loop(valid(ZF), [&](int i, int j, int k) {
                double s[6]; gather(prim, 2, i, j, k, pidx, vtype, s);
                fz(i, j, k) = az(i, j, k) * interp(vtype, s, az(i, j, k), vfrac);
            });
            loop(valid(CC), [&](int i, int j, int k) {
                double invdetJ = terrain ? 1. / detJ(i, j, k) : 1.;
                double mfsq = 1.0;
                rhs(i, j, k, q) = -invdetJ * mfsq * ((fx(i + 1, j, k) - fx(i, j, k)) * dxInv[0] + (fy(i, j + 1, k) - fy(i, j, k)) * dxInv[1] + (fz(i, j, k + 1) - fz(i, j, k)) * dxInv[2]);
            });
        }
    }

    // ------------------------------------------------------------------
    // Everything the integrator keeps across stages.
    // ------------------------------------------------------------------
    State S_old, S_new, S_sum, S_scr, F_slow;
    Vel Vnew;
    Fab prim, pi_stage, mut, fast_coeffs;
    mutable Fab kthv, diss, smn, hfz;   // Deardorff: Theta_v diffusivity, dissipation, SmnSmn, theta's vertical flux
    Fab xsrc, ysrc, zsrc;

    void init_storage() {
        alloc_state(S_old); alloc_state(S_new); alloc_state(S_sum); alloc_state(S_scr); alloc_state(F_slow);
        alloc_vel(Vnew);
        alloc(prim, CC, ngc, nprim);
        alloc(pi_stage, CC, ngc, 1);
        alloc_cc1(mut);
        alloc_cc1(kthv); alloc_cc1(diss); alloc_cc1(smn);
        alloc(hfz, ZF, 0, 1);
        alloc(fast_coeffs, ZF, 0, 5);
        alloc(xsrc, XF, 1, 1); alloc(ysrc, YF, 1, 1); alloc(zsrc, ZF, 1, 1);
    }

    // make_mom_sources + make_buoyancy (SourceTerms/ERF_make_mom_sources.cpp:40-315,
    // SourceTerms/ERF_make_buoyancy.cpp:31-380) on stage data
    void make_mom_sources(const State& S, const Fab& prm) {
        std::fill(xsrc.d.begin(), xsrc.d.end(), 0.0);
        std::fill(ysrc.d.begin(), ysrc.d.end(), 0.0);
        std::fill(zsrc.d.begin(), zsrc.d.end(), 0.0);
        const Fab& cd = S.cons;
        double g2 = -c.gravity;
        Bx tbz_b = valid(ZF); tbz_b.lo[2] = 1; tbz_b.hi[2] = nz - 1;
        if (!use_moisture) {
            if (c.buoyancy_type == 1) {
                loop(tbz_b, [&](int i, int j, int k) {
                    zsrc(i, j, k) = g2 * 0.5 * ((cd(i, j, k, 0) - R0(i, j, k)) + (cd(i, j, k - 1, 0) - R0(i, j, k - 1)));
                });
            } else {
                // dry types 2/3 (T' based) use the base state p0
                loop(tbz_b, [&](int i, int j, int k) {
                    auto T0 = [&](int kk) { double rt0 = getRhoThetagivenP(P0(i, j, kk)); return (rt0 / R0(i, j, kk)) / std::pow(p_0 / P0(i, j, kk), rdOcp); };
                    double t0_hi = T0(k), t_hi = getTgivenRandRTh(cd(i, j, k, 0), cd(i, j, k, 1));
                    double t0_lo = T0(k - 1), t_lo = getTgivenRandRTh(cd(i, j, k - 1, 0), cd(i, j, k - 1, 1));
                    double qplus = (t_hi - t0_hi) / t0_hi, qminus = (t_lo - t0_lo) / t0_lo;
                    double r0_q_avg = 0.5 * (R0(i, j, k) * qplus + R0(i, j, k - 1) * qminus);
                    zsrc(i, j, k) = -r0_q_avg * g2;
                });
            }
        } else if (c.buoyancy_type == 1) {
            int nq = ncomp - ERF_RHOQ1_COMP;
            loop(tbz_b, [&](int i, int j, int k) {
                double hi = cd(i, j, k, 0) + cd(i, j, k, 5) + cd(i, j, k, 6) - R0(i, j, k);
                double lo = cd(i, j, k - 1, 0) + cd(i, j, k - 1, 5) + cd(i, j, k - 1, 6) - R0(i, j, k - 1);
                for (int qo = 2; qo < nq; ++qo) { hi += cd(i, j, k, 5 + qo); lo += cd(i, j, k - 1, 5 + qo); }
                zsrc(i, j, k) = g2 * 0.5 * (hi + lo);
            });
        } else {
            // buoyancy type 2: horizontal plane averages of rho, theta, qv, qc, qp
            int nq = ncomp - ERF_RHOQ1_COMP;
            std::vector<double> rho_d(nz, 0.), th_d(nz, 0.), qv_d(nz, 0.), qc_d(nz, 0.), qp_d(nz, 0.);
            double denom = 1.0 / (double)(nx * ny);
            for (int k = 0; k < nz; ++k)
                for (int j = 0; j < ny; ++j)
                    for (int i = 0; i < nx; ++i) {
                        rho_d[k] += cd(i, j, k, 0) * denom;
                        th_d[k] += prm(i, j, k, 0) * denom;
                        if (nq >= 1) qv_d[k] += prm(i, j, k, 4) * denom;
                        if (nq >= 2) qc_d[k] += prm(i, j, k, 5) * denom;
                        if (nq >= 3) qp_d[k] += prm(i, j, k, 6) * denom;
                    }
            loop(tbz_b, [&](int i, int j, int k) {
                double tp1 = getTgivenRandRTh(rho_d[k], rho_d[k] * th_d[k], qv_d[k]);
                double tm1 = getTgivenRandRTh(rho_d[k - 1], rho_d[k - 1] * th_d[k - 1], qv_d[k - 1]);
                double tp3 = getTgivenRandRTh(cd(i, j, k, 0), cd(i, j, k, 1), cd(i, j, k, 5) / cd(i, j, k, 0));
                double tm3 = getTgivenRandRTh(cd(i, j, k - 1, 0), cd(i, j, k - 1, 1), cd(i, j, k - 1, 5) / cd(i, j, k - 1, 0));
                double qvp = nq >= 1 ? prm(i, j, k, 4) : 0.0, qvm = nq >= 1 ? prm(i, j, k - 1, 4) : 0.0;
                double qcp = nq >= 2 ? prm(i, j, k, 5) : 0.0, qcm = nq >= 2 ? prm(i, j, k - 1, 5) : 0.0;
                double qpp = nq >= 3 ? prm(i, j, k, 6) : 0.0, qpm = nq >= 3 ? prm(i, j, k - 1, 6) : 0.0;
                double qplus = 0.61 * (qvp - qv_d[k]) - (qcp - qc_d[k] + qpp - qp_d[k]) + (tp3 - tp1) / tp1 * (1.0 + 0.61 * qv_d[k] - qc_d[k] - qp_d[k]);
                double qminus = 0.61 * (qvm - qv_d[k - 1]) - (qcm - qc_d[k - 1] + qpm - qp_d[k - 1]) + (tm3 - tm1) / tm1 * (1.0 + 0.61 * qv_d[k - 1] - qc_d[k - 1] - qp_d[k - 1]);
                double qavg = 0.5 * (qplus + qminus);
                double r0avg = 0.5 * (rho_d[k] + rho_d[k - 1]);
                zsrc(i, j, k) = -qavg * r0avg * g2;
            });
        }
        const Fab &ru = S.mx, &rv = S.my, &rw = S.mz;
        Bx tbx = valid(XF), tby = valid(YF), tbz = valid(ZF);
        tbz.hi[2] = nz - 1;
        if (c.use_coriolis) {
            double cf = c.coriolis_factor, sp = c.sinphi, cp = c.cosphi;
            loop(tbx, [&](int i, int j, int k) {
                double rvl = 0.25 * (rv(i, j + 1, k) + rv(i, j, k) + rv(i - 1, j + 1, k) + rv(i - 1, j, k));
                double rwl = 0.25 * (rw(i, j, k + 1) + rw(i, j, k) + rw(i, j - 1, k + 1) + rw(i, j - 1, k));
                xsrc(i, j, k) += cf * (rvl * sp - rwl * cp);
            });
            loop(tby, [&](int i, int j, int k) {
                double rul = 0.25 * (ru(i + 1, j, k) + ru(i, j, k) + ru(i + 1, j - 1, k) + ru(i, j - 1, k));
                ysrc(i, j, k) += -cf * rul * sp;
            });
            loop(tbz, [&](int i, int j, int k) {
                double rul = 0.25 * (ru(i + 1, j, k) + ru(i, j, k) + ru(i + 1, j, k - 1) + ru(i, j, k - 1));
                zsrc(i, j, k) += cf * rul * cp;
            });
        }
        loop(tbx, [&](int i, int j, int k) { xsrc(i, j, k) += 0.5 * (cd(i, j, k, 0) + cd(i - 1, j, k, 0)) * c.abl_geo_forcing[0]; });
        loop(tby, [&](int i, int j, int k) { ysrc(i, j, k) += 0.5 * (cd(i, j, k, 0) + cd(i, j - 1, k, 0)) * c.abl_geo_forcing[1]; });
        loop(tbz, [&](int i, int j, int k) { zsrc(i, j, k) += 0.5 * (cd(i, j, k, 0) + cd(i, j, k - 1, 0)) * c.abl_geo_forcing[2]; });
    }

    // erf_make_tau_terms (TimeIntegration/ERF_make_tau_terms.cpp:320-424), no terrain
    void make_tau(const Vel& V, const State& S, Fab& t11, Fab& t22, Fab& t33, Fab& t12, Fab& t13, Fab& t23) const {
        Fab er; alloc_cc1(er);
        Fab s11, s22, s33, s12, s13, s23;
        alloc_cc1(s11); alloc_cc1(s22); alloc_cc1(s33); alloc_edges(s12, s13, s23);
        Bx bxcc = grow(valid(CC), 1, 1, 0);
        Bx txy = grow(Bx{{0, 0, 0}, {nx, ny, nz - 1}}, 1, 1, 0);
        Bx txz = grow(Bx{{0, 0, 0}, {nx, ny - 1, nz}}, 1, 1, 0);
        Bx tyz = grow(Bx{{0, 0, 0}, {nx - 1, ny, nz}}, 1, 1, 0);
        const Fab &u = V.u, &v = V.v, &w = V.w;
        loop(bxcc, [&](int i, int j, int k) {
            er(i, j, k) = (u(i + 1, j, k) - u(i, j, k)) * dxInv[0] + (v(i, j + 1, k) - v(i, j, k)) * dxInv[1] + (w(i, j, k + 1) - w(i, j, k)) * dxInv[2];
        });
        compute_strain(bxcc, txy, txz, tyz, u, v, w, s11, s22, s33, s12, s13, s23);
        if (c.les_type == ERF_LES_DEARDORFF && tau_nrk == 0) {
            // SmnSmn for the TKE shear production (ERF_make_tau_terms.cpp:233-240)
            Fab& sm = smn;
            loop(valid(CC), [&](int i, int j, int k) { sm(i, j, k) = smnsmn(i, j, k, s11, s22, s33, s12, s13, s23, most && k == 0); });
        }
        double mu_eff = use_consA ? 2.0 * c.dynamic_viscosity / c.rho0_trans : 2.0 * c.dynamic_viscosity;
        const double OneThird = 1. / 3.;
        Bx exy = Bx{{0, 0, 0}, {nx, ny, nz - 1}}, exz = Bx{{0, 0, 0}, {nx, ny - 1, nz}}, eyz = Bx{{0, 0, 0}, {nx - 1, ny, nz}};
        const Fab& cd = S.cons;
        // ComputeStress{Cons,Var}Visc_N (Diffusion/ERF_ComputeStress_N.cpp:23-189)
        loop(bxcc, [&](int i, int j, int k) {
            double m11, m33;
            double base = use_consA ? cd(i, j, k, 0) * mu_eff : mu_eff;
            if (use_turb) { m11 = base + 2.0 * mut(i, j, k); m33 = base + 2.0 * mut(i, j, k); }
            else { m11 = base; m33 = base; }
            t11(i, j, k) = -m11 * (s11(i, j, k) - OneThird * er(i, j, k));
            t22(i, j, k) = -m11 * (s22(i, j, k) - OneThird * er(i, j, k));
            t33(i, j, k) = -m33 * (s33(i, j, k) - OneThird * er(i, j, k));
        });
        loop(exy, [&](int i, int j, int k) {
            double m = use_consA ? 0.25 * (cd(i - 1, j, k, 0) + cd(i, j, k, 0) + cd(i - 1, j - 1, k, 0) + cd(i, j - 1, k, 0)) * mu_eff : mu_eff;
            if (use_turb) m += 2.0 * (0.25 * (mut(i - 1, j, k) + mut(i, j, k) + mut(i - 1, j - 1, k) + mut(i, j - 1, k)));
            t12(i, j, k) = s12(i, j, k) * -m;
        });
        loop(exz, [&](int i, int j, int k) {
            double m = use_consA ? 0.25 * (cd(i - 1, j, k, 0) + cd(i, j, k, 0) + cd(i - 1, j, k - 1, 0) + cd(i, j, k - 1, 0)) * mu_eff : mu_eff;
            if (use_turb) m += 2.0 * (0.25 * (mut(i - 1, j, k) + mut(i, j, k) + mut(i - 1, j, k - 1) + mut(i, j, k - 1)));
            t13(i, j, k) = s13(i, j, k) * -m;
        });
        loop(eyz, [&](int i, int j, int k) {
            double m = use_consA ? 0.25 * (cd(i, j - 1, k, 0) + cd(i, j, k, 0) + cd(i, j - 1, k - 1, 0) + cd(i, j, k - 1, 0)) * mu_eff : mu_eff;
            if (use_turb) m += 2.0 * (0.25 * (mut(i, j - 1, k) + mut(i, j, k) + mut(i, j - 1, k - 1) + mut(i, j, k - 1)));
            t23(i, j, k) = s23(i, j, k) * -m;
        });
    }

    // erf_slow_rhs_pre (TimeIntegration/ERF_slow_rhs_pre.cpp:67-774), no terrain,
    // no anelastic, no mono advection, periodic laterally.
    int tau_nrk = -1;   // stage of the current make_tau call (SmnSmn is formed at stage 0)
    void slow_rhs_pre(int nrk, double dt, State& R, const State& S, State& Scr, const Vel& V) {
        tau_nrk = nrk;
        (void)nrk; (void)dt;
        make_mom_sources(S, prim);
        Fab t11, t22, t33, t12, t13, t23, t21, t31, t32;
        if (use_diff) {
            if (terrain) {
                alloc_tau_T(t11, t22, t33, t12, t13, t21, t23, t31, t32);
                make_tau_T(V, S, t11, t22, t33, t12, t13, t21, t23, t31, t32);
            } else {
                alloc_cc1(t11); alloc_cc1(t22); alloc_cc1(t33); alloc_edges(t12, t13, t23);
                make_tau(V, S, t11, t22, t33, t12, t13, t23);
            }
        }
        std::fill(R.mz.d.begin(), R.mz.d.end(), 0.0);
        const Fab& cd = S.cons;
        // p' on the tile grown by one (z clipped at 0)
        Fab pp; alloc_cc1(pp);
        Bx gbx = grow(valid(CC), 1, 1, 1); gbx.lo[2] = 0;
        loop(gbx, [&](int i, int j, int k) {
            double qv = use_moisture ? cd(i, j, k, ERF_RHOQ1_COMP) / cd(i, j, k, 0) : 0.0;
            pp(i, j, k) = getPgivenRTh(cd(i, j, k, 1), qv) - P0(i, j, k);
        });
        // Contravariant momentum Omega (ERF_slow_rhs_pre.cpp:365-420): rho_w
        // without terrain; with terrain OmegaFromW on the interior faces, 0 at
        // and below the bottom face, rho_w above the top face.
        Fab Om; alloc(Om, ZF, 2, 1);
        loop(grow(valid(ZF), 1, 1, 1), [&](int i, int j, int k) {
            if (!terrain) Om(i, j, k) = S.mz(i, j, k);
            else if (k <= 0) Om(i, j, k) = 0.;
            else if (k >= nz + 1) Om(i, j, k) = S.mz(i, j, k);
            else if (moving)   // the grid's own motion subtracted (rho at the face as in MomentumToVelocity)
                Om(i, j, k) = omega_from_w(i, j, k, S.mz(i, j, k), S.mx, S.my)
                              - 0.5 * (cd(i, j, k, 0) + cd(i, j, k - 1, 0)) * zt(i, j, k);
            else Om(i, j, k) = omega_from_w(i, j, k, S.mz(i, j, k), S.mx, S.my);
        });
        // AdvectionSrcForRho (Advection/ERF_AdvectionSrcForState.cpp:30-93)
        Fab fx, fy, fz;
        alloc(fx, XF, 0, 1); alloc(fy, YF, 0, 1); alloc(fz, ZF, 0, 1);
        loop(valid(XF), [&](int i, int j, int k) { fx(i, j, k) = (terrain ? axA(i, j, k) : 1.0) * S.mx(i, j, k) / 1.0; Scr.mx(i, j, k) = fx(i, j, k); });
        loop(valid(YF), [&](int i, int j, int k) { fy(i, j, k) = (terrain ? ayA(i, j, k) : 1.0) * S.my(i, j, k) / 1.0; Scr.my(i, j, k) = fy(i, j, k); });
        loop(valid(ZF), [&](int i, int j, int k) { fz(i, j, k) = 1.0 * Om(i, j, k) / 1.0; Scr.mz(i, j, k) = fz(i, j, k); });
        loop(valid(CC), [&](int i, int j, int k) {
            R.cons(i, j, k, 0) = -1.0 / (terrain ? detJ(i, j, k) : 1.0) * ((fx(i + 1, j, k) - fx(i, j, k)) * dxInv[0] + (fy(i, j + 1, k) - fy(i, j, k)) * dxInv[1] + (fz(i, j, k + 1) - fz(i, j, k)) * dxInv[2]);
        });
        // rho*theta is advected with the dycore scheme (ERF_slow_rhs_pre.cpp:139-142, 469-477)
        advect_scalars(1, 1, Scr.mx, Scr.my, Scr.mz, prim, R.cons, c.dycore_horiz_adv, c.dycore_vert_adv,
                       c.dycore_horiz_upw_frac, c.dycore_vert_upw_frac);
        if (use_diff) {
            if (terrain) diffusion_state_T(1, 1, cd, prim, R.cons);
            else diffusion_state(1, 1, cd, prim, R.cons, mut);
        }
        // cc_src is zero for the supported configurations; with moving
        // terrain the rho and rho theta right-hand sides carry detJ
        // (ERF_slow_rhs_pre.cpp:528-535)
        if (moving)
            loop(valid(CC), [&](int i, int j, int k) {
                R.cons(i, j, k, 0) *= detJ(i, j, k);
                R.cons(i, j, k, 1) *= detJ(i, j, k);
            });
        if (terrain) {
            advect_mom_T(R, S, V, Om);
            if (use_diff) diffusion_mom_T(R, t11, t22, t33, t12, t13, t21, t23, t31, t32);
            pressure_and_sources(R, pp);
            return;
        }

        advect_mom_N(R, S, V);
        Bx tbx = valid(XF), tby = valid(YF), tbz = valid(ZF);
        tbz.lo[2] = 1; tbz.hi[2] = nz - 1;
        if (use_diff) {
            // DiffusionSrcForMom_N (Diffusion/ERF_DiffusionSrcForMom_N.cpp:25-67)
            loop(tbx, [&](int i, int j, int k) {
                R.mx(i, j, k) -= ((t11(i, j, k) - t11(i - 1, j, k)) * dxInv[0] * 1.0 + (t12(i, j + 1, k) - t12(i, j, k)) * dxInv[1] * 1.0 + (t13(i, j, k + 1) - t13(i, j, k)) * dxInv[2]);
            });
            loop(tby, [&](int i, int j, int k) {
                R.my(i, j, k) -= ((t12(i + 1, j, k) - t12(i, j, k)) * dxInv[0] * 1.0 + (t22(i, j, k) - t22(i, j - 1, k)) * dxInv[1] * 1.0 + (t23(i, j, k + 1) - t23(i, j, k)) * dxInv[2]);
            });
            loop(tbz, [&](int i, int j, int k) {
                R.mz(i, j, k) -= ((t13(i + 1, j, k) - t13(i, j, k)) * dxInv[0] * 1.0 + (t23(i, j + 1, k) - t23(i, j, k)) * dxInv[1] * 1.0 + (t33(i, j, k) - t33(i, j, k - 1)) * dxInv[2]);
            });
        }
        pressure_and_sources(R, pp);
    }

    // AdvectionSrcForMom without terrain (Advection/ERF_AdvectionSrcForMom.cpp:
    // 41-204, ERF_AdvectionSrcForMom_N.H:17-407): assigns R's momentum rhs on
    // x- and y-faces and the interior z-faces.
    void advect_mom_N(State& R, const State& S, const Vel& V) const {
        const Fab &ru = S.mx, &rv = S.my, &rw = S.mz, &u = V.u, &v = V.v, &w = V.w;
        int ht = c.dycore_horiz_adv, vt = c.dycore_vert_adv;
        double hf = c.dycore_horiz_upw_frac, vf = c.dycore_vert_upw_frac;
        bool c2 = (ht == ERF_ADV_CENTERED_2ND && vt == ERF_ADV_CENTERED_2ND);
        auto iX = [&](const Fab& f, int i, int j, int k, double upw) { double s[6]; gather(f, 0, i, j, k, 0, ht, s); return interp(ht, s, upw, hf); };
        auto iY = [&](const Fab& f, int i, int j, int k, double upw) { double s[6]; gather(f, 1, i, j, k, 0, ht, s); return interp(ht, s, upw, hf); };
        auto iZ = [&](const Fab& f, int i, int j, int k, double upw) { double s[6]; gather(f, 2, i, j, k, 0, vt, s); return interp(vt, s, upw, vf); };
        Bx tbx = valid(XF), tby = valid(YF), tbz = valid(ZF);
        tbz.lo[2] = 1; tbz.hi[2] = nz - 1;
        int lo_z_face = 0, hi_z_face = nz;
        loop(tbx, [&](int i, int j, int k) {
            double src;
            if (c2) {
                double xh = 0.25 * (ru(i, j, k) * 1.0 + ru(i + 1, j, k) * 1.0) * (u(i + 1, j, k) + u(i, j, k));
                double xl = 0.25 * (ru(i, j, k) * 1.0 + ru(i - 1, j, k) * 1.0) * (u(i - 1, j, k) + u(i, j, k));
                double yh = 0.25 * (rv(i, j + 1, k) * 1.0 + rv(i - 1, j + 1, k) * 1.0) * (u(i, j + 1, k) + u(i, j, k));
                double yl = 0.25 * (rv(i, j, k) * 1.0 + rv(i - 1, j, k) * 1.0) * (u(i, j - 1, k) + u(i, j, k));
                double zh = 0.25 * (rw(i, j, k + 1) + rw(i - 1, j, k + 1)) * (u(i, j, k + 1) + u(i, j, k));
                double zl = 0.25 * (rw(i, j, k) + rw(i - 1, j, k)) * (u(i, j, k - 1) + u(i, j, k));
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
            } else {
                double a, xh, xl, yh, yl, zh, zl;
                a = 0.5 * (ru(i + 1, j, k) * 1.0 + ru(i, j, k) * 1.0); xh = a * iX(u, i + 1, j, k, a);
                a = 0.5 * (ru(i - 1, j, k) * 1.0 + ru(i, j, k) * 1.0); xl = a * iX(u, i, j, k, a);
                a = 0.5 * (rv(i, j + 1, k) * 1.0 + rv(i - 1, j + 1, k) * 1.0); yh = a * iY(u, i, j + 1, k, a);
                a = 0.5 * (rv(i, j, k) * 1.0 + rv(i - 1, j, k) * 1.0); yl = a * iY(u, i, j, k, a);
                a = 0.5 * (rw(i, j, k + 1) + rw(i - 1, j, k + 1)); zh = a * iZ(u, i, j, k + 1, a);
                a = 0.5 * (rw(i, j, k) + rw(i - 1, j, k)); zl = a * iZ(u, i, j, k, a);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
            }
            R.mx(i, j, k) = -src;
        });
        loop(tby, [&](int i, int j, int k) {
            double src;
            if (c2) {
                double xh = 0.25 * (ru(i + 1, j, k) * 1.0 + ru(i + 1, j - 1, k) * 1.0) * (v(i + 1, j, k) + v(i, j, k));
                double xl = 0.25 * (ru(i, j, k) * 1.0 + ru(i, j - 1, k) * 1.0) * (v(i - 1, j, k) + v(i, j, k));
                double yh = 0.25 * (rv(i, j + 1, k) * 1.0 + rv(i, j, k) * 1.0) * (v(i, j + 1, k) + v(i, j, k));
                double yl = 0.25 * (rv(i, j, k) * 1.0 + rv(i, j - 1, k) * 1.0) * (v(i, j - 1, k) + v(i, j, k));
                double zh = 0.25 * (rw(i, j, k + 1) + rw(i, j - 1, k + 1)) * (v(i, j, k + 1) + v(i, j, k));
                double zl = 0.25 * (rw(i, j, k) + rw(i, j - 1, k)) * (v(i, j, k - 1) + v(i, j, k));
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
            } else {
                double a, xh, xl, yh, yl, zh, zl;
                a = 0.5 * (ru(i + 1, j, k) * 1.0 + ru(i + 1, j - 1, k) * 1.0); xh = a * iX(v, i + 1, j, k, a);
                a = 0.5 * (ru(i, j, k) * 1.0 + ru(i, j - 1, k) * 1.0); xl = a * iX(v, i, j, k, a);
                a = 0.5 * (rv(i, j, k) * 1.0 + rv(i, j + 1, k) * 1.0); yh = a * iY(v, i, j + 1, k, a);
                a = 0.5 * (rv(i, j, k) * 1.0 + rv(i, j - 1, k) * 1.0); yl = a * iY(v, i, j, k, a);
                a = 0.5 * (rw(i, j, k + 1) + rw(i, j - 1, k + 1)); zh = a * iZ(v, i, j, k + 1, a);
                a = 0.5 * (rw(i, j, k) + rw(i, j - 1, k)); zl = a * iZ(v, i, j, k, a);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
            }
            R.my(i, j, k) = -src;
        });
        loop(tbz, [&](int i, int j, int k) {
            double src;
            if (c2) {
                double xh = 0.25 * (ru(i + 1, j, k) + ru(i + 1, j, k - 1)) * 1.0 * (w(i + 1, j, k) + w(i, j, k));
                double xl = 0.25 * (ru(i, j, k) + ru(i, j, k - 1)) * 1.0 * (w(i - 1, j, k) + w(i, j, k));
                double yh = 0.25 * (rv(i, j + 1, k) + rv(i, j + 1, k - 1)) * 1.0 * (w(i, j + 1, k) + w(i, j, k));
                double yl = 0.25 * (rv(i, j, k) + rv(i, j, k - 1)) * 1.0 * (w(i, j - 1, k) + w(i, j, k));
                double zl = 0.25 * (rw(i, j, k) + rw(i, j, k - 1)) * (w(i, j, k) + w(i, j, k - 1));
                double zh = (k == hi_z_face) ? rw(i, j, k) * w(i, j, k) : 0.25 * (rw(i, j, k) + rw(i, j, k + 1)) * (w(i, j, k) + w(i, j, k + 1));
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
            } else {
                double a, xh, xl, yh, yl, zh, zl, ih, il;
                a = 0.5 * (ru(i + 1, j, k) + ru(i + 1, j, k - 1)) * 1.0; xh = a * iX(w, i + 1, j, k, a);
                a = 0.5 * (ru(i, j, k) + ru(i, j, k - 1)) * 1.0; xl = a * iX(w, i, j, k, a);
                a = 0.5 * (rv(i, j + 1, k) + rv(i, j + 1, k - 1)) * 1.0; yh = a * iY(w, i, j + 1, k, a);
                a = 0.5 * (rv(i, j, k) + rv(i, j, k - 1)) * 1.0; yl = a * iY(w, i, j, k, a);
                auto iZall = [&](int kk, double upw, double frac, int type) { double s[6]; gather(w, 2, i, j, kk, 0, (type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH) ? ERF_ADV_UPWIND_5TH : (type == ERF_ADV_CENTERED_2ND ? ERF_ADV_CENTERED_2ND : ERF_ADV_UPWIND_3RD), s); return interp_all(type, s, upw, frac); };
                if (k == hi_z_face) { zh = rw(i, j, k) * w(i, j, k); }
                else {
                    a = 0.5 * (rw(i, j, k) + rw(i, j, k + 1));
                    if (k == hi_z_face - 1) ih = iZall(k + 1, a, 0, ERF_ADV_CENTERED_2ND);
                    else if (k == hi_z_face - 2 || k == lo_z_face + 1) {
                        if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) ih = iZall(k + 1, a, 0, ERF_ADV_CENTERED_4TH);
                        else ih = iZall(k + 1, a, vf, vt);
                    } else ih = iZ(w, i, j, k + 1, a);
                    zh = a * ih;
                }
                if (k == lo_z_face) { zl = rw(i, j, k) * w(i, j, k); }
                else {
                    a = 0.5 * (rw(i, j, k) + rw(i, j, k - 1));
                    if (k == lo_z_face + 1) il = iZall(k, a, 0, ERF_ADV_CENTERED_2ND);
                    else if (k == lo_z_face + 2 || k == hi_z_face - 1) {
                        if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) il = iZall(k, a, 0, ERF_ADV_CENTERED_4TH);
                        else il = iZall(k, a, vf, vt);
                    } else il = iZ(w, i, j, k, a);
                    zl = a * il;
                }
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
            }
            R.mz(i, j, k) = -src;
        });
    }

    // pressure gradient (terrain-corrected with terrain) and momentum sources
    // (ERF_slow_rhs_pre.cpp:594-744)
    void pressure_and_sources(State& R, const Fab& pp) const {
        Bx tbx = valid(XF), tby = valid(YF), tbz = valid(ZF);
        tbz.lo[2] = 1; tbz.hi[2] = nz - 1;
        loop(tbx, [&](int i, int j, int k) {
            double gpx = dxInv[0] * (pp(i, j, k) - pp(i - 1, j, k));
            if (terrain) {
                double mxi = hxi_I(i, j, k), mz = hzeta_I(i, j, k), gz;
                if (k == 0) gz = 0.5 * dxInv[2] * (pp(i - 1, j, k + 1) + pp(i, j, k + 1) - pp(i - 1, j, k) - pp(i, j, k));
                else if (k == nz - 1) gz = 0.5 * dxInv[2] * (pp(i - 1, j, k) + pp(i, j, k) - pp(i - 1, j, k - 1) - pp(i, j, k - 1));
                else gz = 0.25 * dxInv[2] * (pp(i - 1, j, k + 1) + pp(i, j, k + 1) - pp(i - 1, j, k - 1) - pp(i, j, k - 1));
                gpx -= (mxi / mz) * gz;
            }
            gpx *= 1.0;
            double q = 0.0;
            if (use_moisture) q = 0.5 * (prim(i, j, k, 4) + prim(i - 1, j, k, 4) + prim(i, j, k, 5) + prim(i - 1, j, k, 5));
            R.mx(i, j, k) += (-gpx - 0.0) / (1.0 + q) + xsrc(i, j, k);
            if (moving) R.mx(i, j, k) *= hzeta_I(i, j, k);   // ERF_slow_rhs_pre.cpp:633-636
        });
        loop(tby, [&](int i, int j, int k) {
            double gpy = dxInv[1] * (pp(i, j, k) - pp(i, j - 1, k));
            if (terrain) {
                double meta = heta_J(i, j, k), mz = hzeta_J(i, j, k), gz;
                if (k == 0) gz = 0.5 * dxInv[2] * (pp(i, j, k + 1) + pp(i, j - 1, k + 1) - pp(i, j, k) - pp(i, j - 1, k));
                else if (k == nz - 1) gz = 0.5 * dxInv[2] * (pp(i, j, k) + pp(i, j - 1, k) - pp(i, j, k - 1) - pp(i, j - 1, k - 1));
                else gz = 0.25 * dxInv[2] * (pp(i, j, k + 1) + pp(i, j - 1, k + 1) - pp(i, j, k - 1) - pp(i, j - 1, k - 1));
                gpy -= (meta / mz) * gz;
            }
            gpy *= 1.0;
            double q = 0.0;
            if (use_moisture) q = 0.5 * (prim(i, j, k, 4) + prim(i, j - 1, k, 4) + prim(i, j, k, 5) + prim(i, j - 1, k, 5));
            R.my(i, j, k) += (-gpy - 0.0) / (1.0 + q) + ysrc(i, j, k);
            if (moving) R.my(i, j, k) *= hzeta_J(i, j, k);   // :681-684
        });
        loop(tbz, [&](int i, int j, int k) {
            double mz = terrain ? hzeta_K(i, j, k) : 1.0;
            double gpz = dxInv[2] * (pp(i, j, k) - pp(i, j, k - 1)) / mz;
            double q = 0.0;
            if (use_moisture) q = 0.5 * (prim(i, j, k, 4) + prim(i, j, k - 1, 4) + prim(i, j, k, 5) + prim(i, j, k - 1, 5));
            R.mz(i, j, k) += (zsrc(i, j, k) - gpz - 0.0) / (1.0 + q);
            if (moving) R.mz(i, j, k) *= 0.5 * (detJ(i, j, k) + detJ(i, j, k - 1));   // :741-743
        });
    }

    // make_fast_coeffs (TimeIntegration/ERF_make_fast_coeffs.cpp:27-294), no terrain
    void make_fast_coeffs(const State& Sst, double dtau, double beta_s) {
        double beta_2 = 0.5 * (1.0 + beta_s);
        double c_v = c.c_p - R_d;
        double dzi = dxInv[2];
        double halfg = std::abs(0.5 * -c.gravity);
        Fab& fc = fast_coeffs;
        Bx b = valid(CC); b.lo[2] = 1; b.hi[2] = nz - 1;
        loop(b, [&](int i, int j, int k) {
            double rhobar_lo = R0(i, j, k - 1), rhobar_hi = R0(i, j, k), pibar_lo = PI0(i, j, k - 1), pibar_hi = PI0(i, j, k);
            double pi_c = 0.5 * (pi_stage(i, j, k - 1) + pi_stage(i, j, k));
            double cP, cQ, dJk = 1.0;
            if (terrain) {   // ERF_make_fast_coeffs.cpp:110-140
                dJk = 0.5 * (detJ(i, j, k) + detJ(i, j, k - 1));
                double inv_dJk = 1. / dJk;
                cP = -Gamma_ * R_d * dzi * inv_dJk + halfg * R_d * rhobar_hi / (c_v * pibar_hi * Sst.cons(i, j, k, 1));
                cQ = Gamma_ * R_d * dzi * inv_dJk + halfg * R_d * rhobar_lo / (c_v * pibar_lo * Sst.cons(i, j, k - 1, 1));
            } else {
                cP = -Gamma_ * R_d * dzi + halfg * R_d * rhobar_hi / (c_v * pibar_hi * Sst.cons(i, j, k, 1));
                cQ = Gamma_ * R_d * dzi + halfg * R_d * rhobar_lo / (c_v * pibar_lo * Sst.cons(i, j, k - 1, 1));
            }
            cP *= pi_c;
            cQ *= pi_c;
            fc(i, j, k, 3) = cP; fc(i, j, k, 4) = cQ;
            if (use_moisture) {
                double q = 0.5 * (prim(i, j, k, 4) + prim(i, j, k - 1, 4) + prim(i, j, k, 5) + prim(i, j, k - 1, 5));
                cP /= (1.0 + q); cQ /= (1.0 + q);
            }
            double tlo = 0.5 * (prim(i, j, k - 2, 0) + prim(i, j, k - 1, 0));
            double tmid = 0.5 * (prim(i, j, k - 1, 0) + prim(i, j, k, 0));
            double thi = 0.5 * (prim(i, j, k, 0) + prim(i, j, k + 1, 0));
            double D = dtau * dtau * beta_2 * beta_2 * dzi;
            fc(i, j, k, 0) = D * (halfg - cQ * tlo);
            fc(i, j, k, 2) = D * (-halfg + cP * thi);
            fc(i, j, k, 1) = (terrain ? dJk : 1.0) + D * (cQ - cP) * tmid;
        });
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                fc(i, j, 0, 0) = 0.0; fc(i, j, 0, 1) = 1.0; fc(i, j, 0, 2) = 0.0;
                fc(i, j, nz, 0) = 0.0; fc(i, j, nz, 1) = 1.0; fc(i, j, nz, 2) = 0.0;
                double bet = fc(i, j, 0, 1);
                for (int k = 1; k <= nz; ++k) {
                    double gam = fc(i, j, k - 1, 2) / bet;
                    bet = fc(i, j, k, 1) - fc(i, j, k, 0) * gam;
                    fc(i, j, k, 1) = bet;
                }
            }
        loop(b, [&](int i, int j, int k) { fc(i, j, k, 1) = 1.0 / fc(i, j, k, 1); });
    }

    // erf_fast_rhs_N (TimeIntegration/ERF_fast_rhs_N.cpp:36-614), implicit
    void fast_rhs_N(int step, int nrk, const State& Rs, const State& Sprev_in, const State& Sst, State& Sd, State& Scr,
                    double dtau, double beta_s, double facinv) {
        // S_prev may alias S_data: work from a snapshot of the previous values
        State Sprev; alloc_state(Sprev); copy_state(Sprev, Sprev_in);
        double beta_1 = 0.5 * (1.0 - beta_s), beta_2 = 0.5 * (1.0 + beta_s), beta_d = 0.1;
        double dxi = dxInv[0], dyi = dxInv[1], dzi = dxInv[2];
        Fab drt, drw, extrap, trhs, tcx, tcy;
        alloc(drt, CC, 1, 1); alloc(drw, ZF, 1, 1); alloc(extrap, CC, 1, 1); alloc(trhs, CC, 0, 2);
        alloc(tcx, XF, 0, 1); alloc(tcy, YF, 0, 1);
        Fab& lag = Scr.cons;
        loop(grow(valid(CC), 1, 1, 1), [&](int i, int j, int k) {
            drt(i, j, k) = Sprev.cons(i, j, k, 1) - Sst.cons(i, j, k, 1);
            if (step == 0) extrap(i, j, k) = drt(i, j, k);
            else extrap(i, j, k) = drt(i, j, k) + beta_d * (drt(i, j, k) - lag(i, j, k, 1));
            lag(i, j, k, 1) = drt(i, j, k);
        });
        loop(grow(valid(ZF), 1, 1, 0), [&](int i, int j, int k) { drw(i, j, k) = Sprev.mz(i, j, k) - Sst.mz(i, j, k); });
        Fab& ax = Scr.mx; Fab& ay = Scr.my; Fab& az = Scr.mz;
        if (nrk == 0 && step == 0) {
            loop(valid(XF), [&](int i, int j, int k) {
                double nd = Sprev.mx(i, j, k) - Sst.mx(i, j, k) + dtau * Rs.mx(i, j, k);
                ax(i, j, k) += facinv * nd; tcx(i, j, k) = Sst.mx(i, j, k) + nd;
            });
            loop(valid(YF), [&](int i, int j, int k) {
                double nd = Sprev.my(i, j, k) - Sst.my(i, j, k) + dtau * Rs.my(i, j, k);
                ay(i, j, k) += facinv * nd; tcy(i, j, k) = Sst.my(i, j, k) + nd;
            });
        } else {
            loop(valid(XF), [&](int i, int j, int k) {
                double gpx = (extrap(i, j, k) - extrap(i - 1, j, k)) * dxi;
                gpx *= 1.0;
                if (use_moisture) {
                    double q = 0.5 * (prim(i, j, k, 4) + prim(i - 1, j, k, 4) + prim(i, j, k, 5) + prim(i - 1, j, k, 5));
                    gpx /= (1.0 + q);
                }
                double pi_c = 0.5 * (pi_stage(i - 1, j, k) + pi_stage(i, j, k));
                double f = -Gamma_ * R_d * pi_c * gpx;
                double nd = Sprev.mx(i, j, k) - Sst.mx(i, j, k) + dtau * f + dtau * Rs.mx(i, j, k);
                ax(i, j, k) += facinv * nd; tcx(i, j, k) = Sst.mx(i, j, k) + nd;
            });
            loop(valid(YF), [&](int i, int j, int k) {
                double gpy = (extrap(i, j, k) - extrap(i, j - 1, k)) * dyi;
                gpy *= 1.0;
                if (use_moisture) {
                    double q = 0.5 * (prim(i, j, k, 4) + prim(i, j - 1, k, 4) + prim(i, j, k, 5) + prim(i, j - 1, k, 5));
                    gpy /= (1.0 + q);
                }
                double pi_c = 0.5 * (pi_stage(i, j - 1, k) + pi_stage(i, j, k));
                double f = -Gamma_ * R_d * pi_c * gpy;
                double nd = Sprev.my(i, j, k) - Sst.my(i, j, k) + dtau * f + dtau * Rs.my(i, j, k);
                ay(i, j, k) += facinv * nd; tcy(i, j, k) = Sst.my(i, j, k) + nd;
            });
        }
        // horizontal fluxes of rho and rho*theta
        loop(valid(CC), [&](int i, int j, int k) {
            double xl = (tcx(i, j, k) - Sst.mx(i, j, k)) / 1.0, xh = (tcx(i + 1, j, k) - Sst.mx(i + 1, j, k)) / 1.0;
            double yl = (tcy(i, j, k) - Sst.my(i, j, k)) / 1.0, yh = (tcy(i, j + 1, k) - Sst.my(i, j + 1, k)) / 1.0;
            double mfsq = 1.0;
            trhs(i, j, k, 0) = (xh - xl) * dxi * mfsq + (yh - yl) * dyi * mfsq;
            trhs(i, j, k, 1) = ((xh * (prim(i, j, k, 0) + prim(i + 1, j, k, 0)) - xl * (prim(i, j, k, 0) + prim(i - 1, j, k, 0))) * dxi * mfsq +
                                (yh * (prim(i, j, k, 0) + prim(i, j + 1, k, 0)) - yl * (prim(i, j, k, 0) + prim(i, j - 1, k, 0))) * dyi * mfsq) * 0.5;
        });
        double halfg = std::abs(0.5 * -c.gravity);
        Fab RHS, soln; alloc(RHS, ZF, 0, 1); alloc(soln, ZF, 0, 1);
        Bx bs = valid(CC); bs.lo[2] = 1; bs.hi[2] = nz - 1;
        const Fab& fc = fast_coeffs;
        loop(bs, [&](int i, int j, int k) {
            double cP = fc(i, j, k, 3), cQ = fc(i, j, k, 4);
            if (use_moisture) {
                double q = 0.5 * (prim(i, j, k, 4) + prim(i, j, k - 1, 4) + prim(i, j, k, 5) + prim(i, j, k - 1, 5));
                cP /= (1.0 + q); cQ /= (1.0 + q);
            }
            double tlo = 0.5 * (prim(i, j, k - 2, 0) + prim(i, j, k - 1, 0));
            double tmid = 0.5 * (prim(i, j, k - 1, 0) + prim(i, j, k, 0));
            double thi = 0.5 * (prim(i, j, k, 0) + prim(i, j, k + 1, 0));
            double Okp1 = Sprev.mz(i, j, k + 1) - Sst.mz(i, j, k + 1);
            double Ok = Sprev.mz(i, j, k) - Sst.mz(i, j, k);
            double Okm1 = Sprev.mz(i, j, k - 1) - Sst.mz(i, j, k - 1);
            double odk = Sprev.cons(i, j, k, 0) - Sst.cons(i, j, k, 0);
            double odkm1 = Sprev.cons(i, j, k - 1, 0) - Sst.cons(i, j, k - 1, 0);
            double R0 = cP * drt(i, j, k) + cQ * drt(i, j, k - 1) - halfg * (odk + odkm1);
            double R1 = halfg * (-Rs.cons(i, j, k, 0) - Rs.cons(i, j, k - 1, 0) + trhs(i, j, k, 0) + trhs(i, j, k - 1, 0)) +
                        (cP * (Rs.cons(i, j, k, 1) - trhs(i, j, k, 1)) + cQ * (Rs.cons(i, j, k - 1, 1) - trhs(i, j, k - 1, 1)));
            R1 += beta_1 * dzi * ((Okp1 - Okm1) * halfg - (Okp1 * thi - Ok * tmid) * cP - (Ok * tmid - Okm1 * tlo) * cQ);
            RHS(i, j, k) = Ok + dtau * (Rs.mz(i, j, k) + R0 + dtau * beta_2 * R1);
        });
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                RHS(i, j, 0) = Sprev.mz(i, j, 0) - Sst.mz(i, j, 0) + dtau * Rs.mz(i, j, 0);
                RHS(i, j, nz) = Sprev.mz(i, j, nz) - Sst.mz(i, j, nz) + dtau * Rs.mz(i, j, nz);
            }
#pragma omp parallel for
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                soln(i, j, 0) = RHS(i, j, 0) * fc(i, j, 0, 1);
                Sd.mz(i, j, 0) = Sst.mz(i, j, 0) + soln(i, j, 0);
                for (int k = 1; k <= nz; ++k) soln(i, j, k) = (RHS(i, j, k) - fc(i, j, k, 0) * soln(i, j, k - 1)) * fc(i, j, k, 1);
                Sd.mz(i, j, nz) = Sst.mz(i, j, nz) + soln(i, j, nz);
                for (int k = nz - 1; k >= 0; --k) {
                    soln(i, j, k) -= (fc(i, j, k, 2) * fc(i, j, k, 1)) * soln(i, j, k + 1);
                    Sd.mz(i, j, k) = Sst.mz(i, j, k) + soln(i, j, k);
                }
            }
        loop(valid(CC), [&](int i, int j, int k) {
            double zl = beta_2 * soln(i, j, k) + beta_1 * drw(i, j, k);
            double zh = beta_2 * soln(i, j, k + 1) + beta_1 * drw(i, j, k + 1);
            az(i, j, k) += facinv * zl / (1.0 * 1.0);
            if (k == nz - 1) az(i, j, k + 1) += facinv * zh / (1.0 * 1.0);
            trhs(i, j, k, 0) += dzi * (zh - zl);
            trhs(i, j, k, 1) += 0.5 * dzi * (zh * (prim(i, j, k, 0) + prim(i, j, k + 1, 0)) - zl * (prim(i, j, k, 0) + prim(i, j, k - 1, 0)));
        });
        loop(valid(CC), [&](int i, int j, int k) {
            Sd.cons(i, j, k, 0) = Sprev.cons(i, j, k, 0) + dtau * (Rs.cons(i, j, k, 0) - trhs(i, j, k, 0));
            Sd.cons(i, j, k, 1) = Sprev.cons(i, j, k, 1) + dtau * (Rs.cons(i, j, k, 1) - trhs(i, j, k, 1));
        });
        loop(valid(XF), [&](int i, int j, int k) { Sd.mx(i, j, k) = tcx(i, j, k); });
        loop(valid(YF), [&](int i, int j, int k) { Sd.my(i, j, k) = tcy(i, j, k); });
    }

    // erf_slow_rhs_post (TimeIntegration/ERF_slow_rhs_post.cpp:49-559)
    void slow_rhs_post(int nrk, double dt, State& R, const State& Sold, State& Snew, State& Sd, State& Scr) {
        (void)nrk;
        int nsv = ncomp - 2;
        loop(valid(CC), [&](int i, int j, int k) { for (int n = 2; n < 2 + nsv; ++n) Sd.cons(i, j, k, n) = Snew.cons(i, j, k, n); });
        // valid slow variables: RhoScalar always; moisture if present
        auto do_var = [&](int start, int num_adv, int htype, int vtype, double hf, double vf) {
            advect_scalars(start, num_adv, Scr.mx, Scr.my, Scr.mz, prim, R.cons, htype, vtype, hf, vf);
            if (use_diff) {
                if (terrain) diffusion_state_T(start, num_adv, Snew.cons, prim, R.cons);
                else diffusion_state(start, num_adv, Snew.cons, prim, R.cons, mut);
            }
        };
        const bool dd = c.les_type == ERF_LES_DEARDORFF;
        if (dd)   // RhoKE is a slow variable with Deardorff (ERF_slow_rhs_post.cpp:169-172, 366-399)
            do_var(ERF_RHOKE_COMP, 1, c.dryscal_horiz_adv, c.dryscal_vert_adv, c.dryscal_horiz_upw_frac, c.dryscal_vert_upw_frac);
        do_var(ERF_RHOSCALAR_COMP, 1, c.dryscal_horiz_adv, c.dryscal_vert_adv, c.dryscal_horiz_upw_frac, c.dryscal_vert_upw_frac);
        int nq = ncomp - ERF_RHOQ1_COMP;
        if (use_moisture && nq > 0)
            do_var(ERF_RHOQ1_COMP, nq, c.moistscal_horiz_adv, c.moistscal_vert_adv, c.moistscal_horiz_upw_frac, c.moistscal_vert_upw_frac);
        if (moving) {
            // ERF_slow_rhs_post.cpp:467-478: detJ-weighted from the old
            // geometry to the new one; only rho KE (and rho QKE) are clamped
            loop(valid(CC), [&](int i, int j, int k) {
                auto upd = [&](int n) {
                    double tv = detJ(i, j, k) * Sold.cons(i, j, k, n) + dt * detJ(i, j, k) * R.cons(i, j, k, n);
                    Sd.cons(i, j, k, n) = tv / g_new.detJ(i, j, k);
                };
                if (dd) {
                    upd(ERF_RHOKE_COMP);
                    Sd.cons(i, j, k, ERF_RHOKE_COMP) = std::max(Sd.cons(i, j, k, ERF_RHOKE_COMP), std::numeric_limits<double>::epsilon());
                }
                upd(ERF_RHOSCALAR_COMP);
                if (use_moisture)
                    for (int m = ERF_RHOQ1_COMP; m < ncomp; ++m) upd(m);
            });
        } else
        loop(valid(CC), [&](int i, int j, int k) {
            if (dd) {
                int n = ERF_RHOKE_COMP;
                Sd.cons(i, j, k, n) = Sold.cons(i, j, k, n) + dt * R.cons(i, j, k, n);
                Sd.cons(i, j, k, n) = std::max(Sd.cons(i, j, k, n), std::numeric_limits<double>::epsilon());
            }
            int n = ERF_RHOSCALAR_COMP;
            Sd.cons(i, j, k, n) = Sold.cons(i, j, k, n) + dt * R.cons(i, j, k, n);
            if (use_moisture)
                for (int m = ERF_RHOQ1_COMP; m < ncomp; ++m) {
                    Sd.cons(i, j, k, m) = Sold.cons(i, j, k, m) + dt * R.cons(i, j, k, m);
                    Sd.cons(i, j, k, m) = std::max(Sd.cons(i, j, k, m), 0.0);
                }
        });
        loop(valid(CC), [&](int i, int j, int k) { for (int n = 0; n < ncomp; ++n) Snew.cons(i, j, k, n) = Sd.cons(i, j, k, n); });
        loop(valid(XF), [&](int i, int j, int k) { Snew.mx(i, j, k) = Sd.mx(i, j, k); });
        loop(valid(YF), [&](int i, int j, int k) { Snew.my(i, j, k) = Sd.my(i, j, k); });
        loop(valid(ZF), [&](int i, int j, int k) { Snew.mz(i, j, k) = Sd.mz(i, j, k); });
    }

    // Kessler (Microphysics/Kessler/ERF_Kessler.cpp:11-185 with
    // ERF_Init_Kessler.cpp:64-99 and ERF_Update_Kessler.cpp:14-40)
    void kessler(Fab& cons, double dtn) {
        Fab rho, th, qv, qc, qp, tabs, pres, fz;
        alloc(rho, CC, 0, 1); alloc(th, CC, 0, 1); alloc(qv, CC, 0, 1); alloc(qc, CC, 0, 1); alloc(qp, CC, 0, 1);
        alloc(tabs, CC, 0, 1); alloc(pres, CC, 0, 1); alloc(fz, ZF, 0, 1);
        loop(valid(CC), [&](int i, int j, int k) {
            rho(i, j, k) = cons(i, j, k, 0);
            th(i, j, k) = cons(i, j, k, 1) / cons(i, j, k, 0);
            qv(i, j, k) = cons(i, j, k, 5) / cons(i, j, k, 0);
            qc(i, j, k) = cons(i, j, k, 6) / cons(i, j, k, 0);
            qp(i, j, k) = (ncomp > 7) ? cons(i, j, k, 7) / cons(i, j, k, 0) : 0.0;
            tabs(i, j, k) = getTgivenRandRTh(cons(i, j, k, 0), cons(i, j, k, 1), qv(i, j, k));
            pres(i, j, k) = getPgivenRTh(cons(i, j, k, 1), qv(i, j, k)) / 100.;
        });
        double fac_cond = lcond / c.c_p;
        double dz = c.dz;
        if (kessler_rain) {
            loop(valid(ZF), [&](int i, int j, int k) {
                double ra, qa;
                if (k == 0) { ra = rho(i, j, k); qa = qp(i, j, k); }
                else if (k == nz) { ra = rho(i, j, k - 1); qa = qp(i, j, k - 1); }
                else { ra = 0.5 * (rho(i, j, k - 1) + rho(i, j, k)); qa = 0.5 * (qp(i, j, k - 1) + qp(i, j, k)); }
                qa = std::max(0.0, qa);
                double Vt = 36.34 * std::pow(ra * 0.001 * qa, 0.1346) * std::pow(ra / 1.16, -0.5);
                fz(i, j, k) = ra * Vt * qa;
            });
            // the reference zeroes tiny fluxes from inside the cell loop; doing it
            // once beforehand gives the same values
            loop(valid(ZF), [&](int i, int j, int k) { if (std::fabs(fz(i, j, k)) < 1e-14) fz(i, j, k) = 0.0; });
            loop(valid(CC), [&](int i, int j, int k) {
                qv(i, j, k) = std::max(0.0, qv(i, j, k));
                qc(i, j, k) = std::max(0.0, qc(i, j, k));
                qp(i, j, k) = std::max(0.0, qp(i, j, k));
                double p = pres(i, j, k);
                double qs = qsatw(tabs(i, j, k), p), dqs = dtqsatw(tabs(i, j, k), p);
                if (qs <= 0.0) qs = 0.0;
                double d_c2r = 0.0, d_r2v = 0.0, d_v2c = 0.0, d_c2v = 0.0;
                double fac = 1.0 + (L_v / Cp_d) * dqs;
                if (qv(i, j, k) > qs) d_v2c = std::min(qv(i, j, k), (qv(i, j, k) - qs) / (1.0 + fac));
                if (qv(i, j, k) < qs && qc(i, j, k) > 0.0) d_c2v = std::min(qc(i, j, k), (qs - qv(i, j, k)) / (1.0 + fac));
                if (qp(i, j, k) > 0.0 && qv(i, j, k) < qs) {
                    double C = 1.6 + 124.9 * std::pow(0.001 * rho(i, j, k) * qp(i, j, k), 0.2046);
                    d_r2v = 1.0 / (0.001 * rho(i, j, k)) * (1.0 - qv(i, j, k) / qs) * C * std::pow(0.001 * rho(i, j, k) * qp(i, j, k), 0.525) /
                            (5.4e5 + 2.55e6 / (p * qs)) * dtn;
                    d_r2v = std::min(qp(i, j, k), d_r2v);
                }
                if (qc(i, j, k) > 0.0) {
                    double qcc = qc(i, j, k);
                    double auto_r = (qcc > qcw0) ? alphaelq : 0.0;
                    double accrr = 2.2 * std::pow(qp(i, j, k), 0.875);
                    d_c2r = dtn * (accrr * qcc + auto_r * (qcc - qcw0));
                    d_c2r = std::min(d_c2r, qc(i, j, k));
                }
                // over terrain per unit computational volume (ERF_Kessler.cpp:82-97)
                double dJinv = terrain ? 1.0 / detJ(i, j, k) : 1.0;
                double dq_sed = dtn * dJinv * (1.0 / rho(i, j, k)) * (fz(i, j, k + 1) - fz(i, j, k)) / dz;
                if (std::fabs(dq_sed) < 1e-14) dq_sed = 0.0;
                qv(i, j, k) += -d_v2c + d_c2v + d_r2v;
                qc(i, j, k) += d_v2c - d_c2v - d_c2r;
                qp(i, j, k) += dq_sed + d_c2r - d_r2v;
                double tot = th(i, j, k) / tabs(i, j, k);
                th(i, j, k) += tot * fac_cond * (d_v2c - d_c2v - d_r2v);
                qv(i, j, k) = std::max(0.0, qv(i, j, k));
                qc(i, j, k) = std::max(0.0, qc(i, j, k));
                qp(i, j, k) = std::max(0.0, qp(i, j, k));
            });
        } else {
            loop(valid(CC), [&](int i, int j, int k) {
                qc(i, j, k) = std::max(0.0, qc(i, j, k));
                double p = pres(i, j, k);
                double qs = qsatw(tabs(i, j, k), p), dqs = dtqsatw(tabs(i, j, k), p);
                double d_v2c = 0.0, d_c2v = 0.0;
                double fac = 1.0 + (L_v / Cp_d) * dqs;
                if (qv(i, j, k) > qs) d_v2c = std::min(qv(i, j, k), (qv(i, j, k) - qs) / (1.0 + fac));
                if (qv(i, j, k) < qs && qc(i, j, k) > 0.0) d_c2v = std::min(qc(i, j, k), (qs - qv(i, j, k)) / (1.0 + fac));
                qv(i, j, k) += -d_v2c + d_c2v;
                qc(i, j, k) += d_v2c - d_c2v;
                double tot = th(i, j, k) / tabs(i, j, k);
                th(i, j, k) += tot * fac_cond * (d_v2c - d_c2v);
                qv(i, j, k) = std::max(0.0, qv(i, j, k));
                qc(i, j, k) = std::max(0.0, qc(i, j, k));
            });
        }
        loop(valid(CC), [&](int i, int j, int k) {
            cons(i, j, k, 1) = rho(i, j, k) * th(i, j, k);
            cons(i, j, k, 5) = rho(i, j, k) * qv(i, j, k);
            cons(i, j, k, 6) = rho(i, j, k) * qc(i, j, k);
            if (ncomp > 7) cons(i, j, k, 7) = rho(i, j, k) * qp(i, j, k);
        });
        fill_periodic(cons, CC);
    }

    // ------------------------------------------------------------------
    // The stage update without acoustic substepping (no_substep_fun,
    // TimeIntegration/ERF_TI_no_substep_fun.H:6-150, fixed or no terrain):
    // the fast variables (rho, rho*theta and the three momenta) of S_sum are
    // S_old + slow_dt * F_slow over the valid cells and faces.
    // ------------------------------------------------------------------
    void no_substep(State& Ssum, const State& Sold, const State& F, double slow_dt) const {
        loop(valid(CC), [&](int i, int j, int k) {
            for (int n = 0; n < 2; ++n) Ssum.cons(i, j, k, n) = Sold.cons(i, j, k, n) + slow_dt * (F.cons(i, j, k, n));
        });
        loop(valid(XF), [&](int i, int j, int k) { Ssum.mx(i, j, k) = Sold.mx(i, j, k) + slow_dt * F.mx(i, j, k); });
        loop(valid(YF), [&](int i, int j, int k) { Ssum.my(i, j, k) = Sold.my(i, j, k) + slow_dt * F.my(i, j, k); });
        loop(valid(ZF), [&](int i, int j, int k) { Ssum.mz(i, j, k) = Sold.mz(i, j, k) + slow_dt * F.mz(i, j, k); });
    }

    // ------------------------------------------------------------------
    // One full time step: ERF::Advance (TimeIntegration/ERF_Advance.cpp:19-233)
    // -> advance_dycore (ERF_advance_dycore.cpp:37-305) -> MRISplitIntegrator::
    // advance (ERF_MRI.H:187-369) -> advance_microphysics.
    // Persistent state: cons and face velocities (valid + ghosts).
    // ------------------------------------------------------------------
    Fab cons_state;
    Vel vel_state;
    // wall seconds per pass for the CPU baseline's split: 0 closure (strain +
    // eddy viscosity), 1 slow_rhs_pre, 2 fast (coefficients + substeps, or the
    // no-substep update), 3 slow_rhs_post (+ boundary fill), 4 Kessler, 5 rest
    double pass_s[6] = {0, 0, 0, 0, 0, 0};
    std::chrono::steady_clock::time_point tmark;
    void tick() { tmark = std::chrono::steady_clock::now(); }
    void tock(int slot) {
        auto now = std::chrono::steady_clock::now();
        pass_s[slot] += std::chrono::duration<double>(now - tmark).count();
        tmark = now;
    }

    // ==================================================================
    // Static terrain-following grid.  Metric terms of
    // Utils/ERF_TerrainMetrics.H:33-395 and make_J / make_areas / make_zcc
    // (Utils/ERF_TerrainMetrics.cpp:583-715); the _T variants of the slow
    // and fast right-hand sides follow below, each citing its source.
    // z_phys_nd is nodal with 3 lateral ghost nodes and one vertical ghost
    // level on each side; az is 1 everywhere and map factors are 1.
    // ==================================================================
    bool terrain = false;
    Fab znd, detJ, axA, ayA, zcc;
    Fab r0f, p0f, pi0f, th0f;            // base state over the terrain (cell centred)
    double R0(int i, int j, int k) const { return terrain ? r0f(i, j, k) : r0[k + 1]; }
    double P0(int i, int j, int k) const { return terrain ? p0f(i, j, k) : p0[k + 1]; }
    double PI0(int i, int j, int k) const { return terrain ? pi0f(i, j, k) : pi0[k + 1]; }

    // the nodes the metric terms read: the current grid, or another one for
    // the length of an on() call (moving terrain mixes several grids); per
    // thread, since on() runs inside the OpenMP loops
    static inline thread_local const Fab* zsel = nullptr;
    double Z(int i, int j, int k) const { return zsel ? (*zsel)(i, j, k) : znd(i, j, k); }
    template <class F>
    double on(const Fab& zf, F f) {
        const Fab* s = zsel;
        zsel = &zf;
        double r = f();
        zsel = s;
        return r;
    }
    double hzeta_cc(int i, int j, int k) const {
        return 0.25 * dxInv[2] * (Z(i + 1, j, k + 1) + Z(i + 1, j + 1, k + 1) + Z(i, j, k + 1) + Z(i, j + 1, k + 1)
                                  - Z(i + 1, j, k) - Z(i + 1, j + 1, k) - Z(i, j, k) - Z(i, j + 1, k));
    }
    double hxi_cc(int i, int j, int k) const {
        return 0.25 * dxInv[0] * (Z(i + 1, j, k) + Z(i + 1, j + 1, k) + Z(i + 1, j, k + 1) + Z(i + 1, j + 1, k + 1)
                                  - Z(i, j, k) - Z(i, j + 1, k) - Z(i, j, k + 1) - Z(i, j + 1, k + 1));
    }
    double heta_cc(int i, int j, int k) const {
        return 0.25 * dxInv[1] * (Z(i, j + 1, k) + Z(i + 1, j + 1, k) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)
                                  - Z(i, j, k) - Z(i + 1, j, k) - Z(i, j, k + 1) - Z(i + 1, j, k + 1));
    }
    double hzeta_I(int i, int j, int k) const {
        return 0.5 * dxInv[2] * (Z(i, j, k + 1) + Z(i, j + 1, k + 1) - Z(i, j, k) - Z(i, j + 1, k));
    }
    double hxi_I(int i, int j, int k) const {
        return 0.125 * dxInv[0] * (Z(i + 1, j, k) + Z(i + 1, j, k + 1) + Z(i + 1, j + 1, k) + Z(i + 1, j + 1, k + 1)
                                   - Z(i - 1, j, k) - Z(i - 1, j, k + 1) - Z(i - 1, j + 1, k) - Z(i - 1, j + 1, k + 1));
    }
    double heta_I(int i, int j, int k) const {
        return 0.5 * dxInv[1] * (Z(i, j + 1, k) + Z(i, j + 1, k + 1) - Z(i, j, k) - Z(i, j, k + 1));
    }
    double hzeta_J(int i, int j, int k) const {
        return 0.5 * dxInv[2] * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) - Z(i, j, k) - Z(i + 1, j, k));
    }
    double hxi_J(int i, int j, int k) const {
        return 0.5 * dxInv[0] * (Z(i + 1, j, k) + Z(i + 1, j, k + 1) - Z(i, j, k) - Z(i, j, k + 1));
    }
    double heta_J(int i, int j, int k) const {
        return 0.125 * dxInv[1] * (Z(i, j + 1, k) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k) + Z(i + 1, j + 1, k + 1)
                                   - Z(i, j - 1, k) - Z(i, j - 1, k + 1) - Z(i + 1, j - 1, k) - Z(i + 1, j - 1, k + 1));
    }
    double hzeta_K(int i, int j, int k) const {
        return 0.125 * dxInv[2] * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)
                                   - Z(i, j, k - 1) - Z(i + 1, j, k - 1) - Z(i, j + 1, k - 1) - Z(i + 1, j + 1, k - 1));
    }
    double hxi_K(int i, int j, int k) const {
        return 0.5 * dxInv[0] * (Z(i + 1, j, k) + Z(i + 1, j + 1, k) - Z(i, j, k) - Z(i, j + 1, k));
    }
    double heta_K(int i, int j, int k) const {
        return 0.5 * dxInv[1] * (Z(i, j + 1, k) + Z(i + 1, j + 1, k) - Z(i, j, k) - Z(i + 1, j, k));
    }
    // xy-edge (EdgeCenterK), xz-edge (EdgeCenterJ), yz-edge (EdgeCenterI)
    double hzeta_EK(int i, int j, int k) const { return dxInv[2] * (Z(i, j, k + 1) - Z(i, j, k)); }
    double hxi_EK(int i, int j, int k) const {
        return 0.25 * dxInv[0] * (Z(i + 1, j, k) + Z(i + 1, j, k + 1) - Z(i - 1, j, k) - Z(i - 1, j, k + 1));
    }
    double heta_EK(int i, int j, int k) const {
        return 0.25 * dxInv[1] * (Z(i, j + 1, k) + Z(i, j + 1, k + 1) - Z(i, j - 1, k) - Z(i, j - 1, k + 1));
    }
    double hzeta_EJ(int i, int j, int k) const {
        return 0.25 * dxInv[2] * (Z(i, j, k + 1) + Z(i, j + 1, k + 1) - Z(i, j, k - 1) - Z(i, j + 1, k - 1));
    }
    double hxi_EJ(int i, int j, int k) const {
        return 0.25 * dxInv[0] * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i - 1, j + 1, k) - Z(i - 1, j, k));
    }
    double heta_EJ(int i, int j, int k) const { return dxInv[1] * (Z(i, j + 1, k) - Z(i, j, k)); }
    double hzeta_EI(int i, int j, int k) const {
        return 0.25 * dxInv[2] * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) - Z(i, j, k - 1) - Z(i + 1, j, k - 1));
    }
    double hxi_EI(int i, int j, int k) const { return dxInv[0] * (Z(i + 1, j, k) - Z(i, j, k)); }
    double heta_EI(int i, int j, int k) const {
        return 0.25 * dxInv[1] * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j - 1, k) - Z(i, j - 1, k));
    }
    // OmegaFromW / WFromOmega (ERF_TerrainMetrics.H:455-520): metric slopes
    // at the z-face and the face-averaged horizontal velocities (extrapolated
    // to the bottom face).
    void zface_uv(int i, int j, int k, const Fab& ua, const Fab& va, double& u, double& v) const {
        u = (k == 0) ? 1.5 * (0.5 * (ua(i, j, k) + ua(i + 1, j, k))) - 0.5 * (0.5 * (ua(i, j, k + 1) + ua(i + 1, j, k + 1)))
                     : 0.25 * (ua(i, j, k - 1) + ua(i + 1, j, k - 1) + ua(i, j, k) + ua(i + 1, j, k));
        v = (k == 0) ? 1.5 * (0.5 * (va(i, j, k) + va(i, j + 1, k))) - 0.5 * (0.5 * (va(i, j, k + 1) + va(i, j + 1, k + 1)))
                     : 0.25 * (va(i, j, k - 1) + va(i, j + 1, k - 1) + va(i, j, k) + va(i, j + 1, k));
    }
    double zlo_xi(int i, int j, int k) const {
        return 0.5 * dxInv[0] * (Z(i + 1, j + 1, k) + Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i, j, k));
    }
    double zlo_eta(int i, int j, int k) const {
        return 0.5 * dxInv[1] * (Z(i + 1, j + 1, k) + Z(i, j + 1, k) - Z(i + 1, j, k) - Z(i, j, k));
    }
    double omega_from_w(int i, int j, int k, double w, const Fab& ua, const Fab& va) const {
        double mx = zlo_xi(i, j, k), my = zlo_eta(i, j, k), u, v;
        zface_uv(i, j, k, ua, va, u, v);
        return w - mx * u - my * v;
    }
    double w_from_omega(int i, int j, int k, double om, const Fab& ua, const Fab& va) const {
        double mx = zlo_xi(i, j, k), my = zlo_eta(i, j, k), u, v;
        zface_uv(i, j, k, ua, va, u, v);
        return om + mx * u + my * v;
    }

    // Install z_phys_nd (valid nodes, (nz+1)(ny+1)(nx+1), i fastest) and
    // build its ghost nodes the way init_terrain_grid leaves them
    // (Utils/ERF_TerrainMetrics.cpp:88-209, 320-333): lateral ghosts are the
    // periodic images (FillBoundary of nodal data keeps node nx), k = -1 and
    // k = nz+1 are linear extrapolations.  Then detJ, ax, ay, z_cc.
    void set_terrain(const double* z) {
        terrain = true;
        int l[3] = {-3, -3, -1}, h[3] = {nx + 3, ny + 3, nz + 1};
        znd.define(l, h, 1);
        auto wrapn = [](int i, int n) { while (i < 0) i += n; while (i > n) i -= n; return i; };
        for (int k = 0; k <= nz; ++k)
            for (int j = l[1]; j <= h[1]; ++j)
                for (int i = l[0]; i <= h[0]; ++i) {
                    int is = (i >= 0 && i <= nx) ? i : wrapn(i, nx);
                    int js = (j >= 0 && j <= ny) ? j : wrapn(j, ny);
                    if (is == nx && !(i >= 0 && i <= nx)) is = 0;
                    if (js == ny && !(j >= 0 && j <= ny)) js = 0;
                    znd(i, j, k) = z[((size_t)k * (ny + 1) + js) * (nx + 1) + is];
                }
        for (int j = l[1]; j <= h[1]; ++j)
            for (int i = l[0]; i <= h[0]; ++i) {
                znd(i, j, -1) = 2.0 * znd(i, j, 0) - znd(i, j, 1);
                znd(i, j, nz + 1) = 2.0 * znd(i, j, nz) - znd(i, j, nz - 1);
            }
        make_metrics();
    }

    // make_J, make_areas, make_zcc (Utils/ERF_TerrainMetrics.cpp:583-715)
    // from the nodes in znd.
    void make_metrics() {
        int lc[3] = {-2, -2, -1}, hc[3] = {nx + 1, ny + 1, nz};
        detJ.define(lc, hc, 1, 1.0); zcc.define(lc, hc, 1);
        int lx[3] = {-2, -2, -1}, hx[3] = {nx + 2, ny + 1, nz};
        int ly[3] = {-2, -2, -1}, hy[3] = {nx + 1, ny + 2, nz};
        axA.define(lx, hx, 1, 1.0); ayA.define(ly, hy, 1, 1.0);
        const double dzi = dxInv[2];
        for (int k = 0; k <= nz; ++k)
            for (int j = lc[1]; j <= hc[1]; ++j)
                for (int i = lc[0]; i <= hc[0]; ++i) {
                    detJ(i, j, k) = .25 * dzi * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)
                                                 - Z(i, j, k) - Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i + 1, j + 1, k));
                    zcc(i, j, k) = .125 * (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)
                                           + Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1));
                }
        for (int j = lc[1]; j <= hc[1]; ++j)
            for (int i = lc[0]; i <= hc[0]; ++i) { detJ(i, j, -1) = detJ(i, j, 0); zcc(i, j, -1) = zcc(i, j, 0); }
        for (int k = 0; k <= nz; ++k) {
            for (int j = lx[1]; j <= hx[1]; ++j)
                for (int i = lx[0]; i <= hx[0]; ++i)
                    axA(i, j, k) = .5 * dzi * (Z(i, j, k + 1) + Z(i, j + 1, k + 1) - Z(i, j, k) - Z(i, j + 1, k));
            for (int j = ly[1]; j <= hy[1]; ++j)
                for (int i = ly[0]; i <= hy[0]; ++i)
                    ayA(i, j, k) = .5 * dzi * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) - Z(i, j, k) - Z(i + 1, j, k));
        }
    }

    // Base state over the terrain: per column the Newton hydrostatic
    // integration of calc_rho_p (DataStructs/ERF_InputSoundingData.H:176-256)
    // from p_sfc at z = 0 through the column's cell centres z_cc, then
    // erf_enforce_hse with terrain (Initialization/ERF_init1d.cpp:152-241).
    // Outputs (nz+2) planes of ny*nx, plane k+1 for cell level k.
    void make_base_state_terrain(const double* th3, const double* qv3, double th_s, double qv_s, double p_s,
                                 double* rho_o, double* p_o, double* pi_o, double* th_o) const {
        const double tol = 1.0e-12, g = c.gravity;
        std::vector<double> z(nz + 1), th(nz + 1), qv(nz + 1), pm(nz + 1), rd(nz + 1), r(nz + 2), p(nz + 2);
        const size_t plane = (size_t)nx * ny;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                z[0] = 0.; th[0] = th_s; qv[0] = qv_s;
                for (int k = 0; k < nz; ++k) {
                    size_t cix = (size_t)k * plane + (size_t)j * nx + i;
                    z[k + 1] = zcc(i, j, k); th[k + 1] = th3[cix]; qv[k + 1] = qv3[cix];
                }
                pm[0] = p_s;
                rd[0] = getRhogivenThetaPress(th[0], p_s, R_d / Cp_d, qv[0]);
                for (int k = 1; k <= nz; ++k) {
                    double dz = z[k] - z[k - 1];
                    double rlo = rd[k - 1] * (1. + qv[k - 1]);
                    double C = -pm[k - 1] + 0.5 * rlo * g * dz;
                    pm[k] = pm[k - 1];
                    rd[k] = getRhogivenThetaPress(th[k], pm[k], R_d / Cp_d, qv[k]);
                    double rhi = rd[k] * (1. + qv[k]);
                    double F = pm[k] + 0.5 * rhi * g * dz + C;
                    if (std::abs(F) > tol) {
                        int iter = 0;
                        double eps = 1.0e-6, ieps = 1.0e6;
                        do {
                            double hi = getRhogivenThetaPress(th[k], pm[k] + eps, R_d / Cp_d, qv[k]);
                            double lo = getRhogivenThetaPress(th[k], pm[k] - eps, R_d / Cp_d, qv[k]);
                            double dFdp = 1.0 + 0.25 * ieps * (hi - lo) * g * dz;
                            pm[k] -= F / dFdp;
                            rd[k] = getRhogivenThetaPress(th[k], pm[k], R_d / Cp_d, qv[k]);
                            double rt = rd[k] * (1. + qv[k]);
                            F = pm[k] + 0.5 * rt * g * dz + C;
                            ++iter;
                        } while (std::abs(F) > tol && iter < 30);
                    }
                }
                for (int k = 0; k < nz; ++k) r[k + 1] = rd[k + 1];
                r[0] = r[1]; r[nz + 1] = r[nz];
                double hz = zcc(i, j, 0);
                auto put = [&](int kk, double pv) {
                    size_t o = (size_t)kk * plane + (size_t)j * nx + i;
                    rho_o[o] = r[kk]; p_o[o] = pv; pi_o[o] = getExnergivenP(pv, rdOcp);
                    th_o[o] = getRhoThetagivenP(pv) / r[kk];
                };
                p[1] = p_0 - hz * r[1] * g;
                p[0] = p_0 + hz * r[1] * g;
                put(1, p[1]); put(0, p[0]);
                for (int k = 1; k <= nz; ++k) {
                    int kk = k + 1;
                    double dz_loc = zcc(i, j, k) - zcc(i, j, k - 1);
                    double di = 0.5 * (r[kk] + r[kk - 1]);
                    p[kk] = p[kk - 1] - dz_loc * di * g;
                    put(kk, p[kk]);
                }
            }
    }
    // Base state arrays in the (nz+2)-plane layout -> cell-centred Fabs
    // with periodic lateral ghosts.
    void set_base_terrain(const double* rho_b, const double* p_b, const double* pi_b, const double* th_b) {
        int l[3] = {-2, -2, -1}, h[3] = {nx + 1, ny + 1, nz};
        Fab* f[4] = {&r0f, &p0f, &pi0f, &th0f};
        const double* src[4] = {rho_b, p_b, pi_b, th_b};
        for (int a = 0; a < 4; ++a) {
            f[a]->define(l, h, 1);
            for (int k = -1; k <= nz; ++k)
                for (int j = l[1]; j <= h[1]; ++j)
                    for (int i = l[0]; i <= h[0]; ++i) {
                        int is = ((i % nx) + nx) % nx, js = ((j % ny) + ny) % ny;
                        (*f[a])(i, j, k) = src[a][(size_t)(k + 1) * nx * ny + (size_t)js * nx + is];
                    }
        }
    }

    // ==================================================================
    // Moving terrain (terrain_type Moving), no acoustic substepping.
    // The grid is regenerated from the travelling surface wave at every
    // geometry time the reference asks for; the base state evolves by the
    // vertical flux that the moving grid induces.
    // ==================================================================
    bool moving = false;
    double time = 0.0;                   // t_old of the step being taken
    struct Geo { Fab znd, detJ, axA, ayA, zcc; };
    Geo g_old, g_src, g_new;
    Fab r0o, p0o;                        // base_state at the start of the step (r0f / p0f: base_state_new)
    Fab zt;                              // z_t_rk on the z faces

    void save_geo(Geo& g) const { g.znd = znd; g.detJ = detJ; g.axA = axA; g.ayA = ayA; g.zcc = zcc; }
    void load_geo(const Geo& g) { znd = g.znd; detJ = g.detJ; axA = g.axA; ayA = g.ayA; zcc = g.zcc; }

    // Problem::init_custom_terrain (Exec/DevTests/MovingTerrain/ERF_prob.cpp:147-200):
    // the surface h = Ampl sin(kp x - omega t), kp = 2 pi / wavelength,
    // omega = sqrt(g kp); then init_terrain_grid with terrain_smoothing = 2
    // (Utils/ERF_TerrainMetrics.cpp:89-209, 501-536): over the uniform levels
    // z_k = k dz, z(k) = z_k + (1 - z_k / z_top)^3 h, z(-1) = 2 h - z(1);
    // lateral ghosts are the periodic images (FillBoundary), z(nz+1) the
    // linear extrapolation.
    void mt_grid(double t) {
        const double PI = 3.14159265358979323846264338327950288;
        const double kp = 2.0 * PI / c.mt_wavelength, om = std::sqrt(CONST_GRAV * kp);
        const double ztop = nz * c.dz;
        int l[3] = {-3, -3, -1}, h[3] = {nx + 3, ny + 3, nz + 1};
        znd.define(l, h, 1);
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i) {
                const double x = i * c.dx;
                const double hs = c.mt_ampl * std::sin(kp * x - om * t);
                for (int k = 0; k <= nz; ++k) {
                    const double zl = k * c.dz;
                    znd(i, j, k) = zl + std::pow(1. - zl / ztop, 3.0) * hs;
                }
                znd(i, j, 0) = hs;
                znd(i, j, -1) = 2.0 * hs - znd(i, j, 1);
            }
        auto wrapn = [](int i, int n) { while (i < 0) i += n; while (i > n) i -= n; return i; };
        for (int k = -1; k <= nz; ++k)
            for (int j = l[1]; j <= h[1]; ++j)
                for (int i = l[0]; i <= h[0]; ++i) {
                    if (i >= 0 && i <= nx && j >= 0 && j <= ny) continue;
                    int is = (i >= 0 && i <= nx) ? i : wrapn(i, nx);
                    int js = (j >= 0 && j <= ny) ? j : wrapn(j, ny);
                    if (is == nx && !(i >= 0 && i <= nx)) is = 0;
                    if (js == ny && !(j >= 0 && j <= ny)) js = 0;
                    znd(i, j, k) = znd(is, js, k);
                }
        for (int j = l[1]; j <= h[1]; ++j)
            for (int i = l[0]; i <= h[0]; ++i) znd(i, j, nz + 1) = 2.0 * znd(i, j, nz) - znd(i, j, nz - 1);
        make_metrics();
    }

    // slow_rhs_fun_pre, moving terrain (TimeIntegration/ERF_TI_slow_rhs_fun.H:55-107):
    // the geometry at the step's old time, at the stage's source time and
    // at the stage's new time, and z_t = (z_new - z_old) / slow_dt averaged
    // over the four nodes of each z face, on the faces grown by one laterally.
    void mt_stage_geometry(double t_old, double t_src, double t_new, double slow_dt) {
        mt_grid(t_old); save_geo(g_old);
        mt_grid(t_src); save_geo(g_src);
        mt_grid(t_new); save_geo(g_new);
        const double inv_dt = 1. / slow_dt;
        const Fab &zn = g_new.znd, &zo = g_old.znd;
        int l[3] = {-2, -2, 0}, h[3] = {nx + 1, ny + 1, nz};
        zt.define(l, h, 1);
        for (int k = 0; k <= nz; ++k)
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i)
                    zt(i, j, k) = 0.25 * inv_dt * (zn(i + 1, j + 1, k) - zo(i + 1, j + 1, k) + zn(i, j + 1, k) - zo(i, j + 1, k)
                                                   + zn(i + 1, j, k) - zo(i + 1, j, k) + zn(i, j, k) - zo(i, j, k));
    }

    // The base-state update of slow_rhs_fun_pre for moving terrain
    // (ERF_TI_slow_rhs_fun.H:149-210): rho_0 and (rho theta)_0 advanced in
    // flux form by the vertical flux -z_t (face average), detJ-weighted from
    // the step's old base state, and p_0 re-made from (rho theta)_0.  Run
    // after the stage's slow right-hand side, which used the base state of
    // the previous stage.
    void mt_base_state(double dt_base) {
        Fab rt0, rt0n, r0t;
        int l[3] = {-2, -2, -1}, h[3] = {nx + 1, ny + 1, nz};
        rt0.define(l, h, 1); rt0n.define(l, h, 1); r0t.define(l, h, 1);
        for (int k = -1; k <= nz; ++k)
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) {
                    rt0(i, j, k) = getRhoThetagivenP(p0o(i, j, k));
                    rt0n(i, j, k) = getRhoThetagivenP(p0f(i, j, k));
                    r0t(i, j, k) = r0f(i, j, k);
                }
        for (int k = 0; k < nz; ++k)
            for (int j = -1; j <= ny; ++j)
                for (int i = -1; i <= nx; ++i) {
                    double fr_lo = -zt(i, j, k) * 0.5 * (r0t(i, j, k) + r0t(i, j, k - 1));
                    double fr_hi = -zt(i, j, k + 1) * 0.5 * (r0t(i, j, k) + r0t(i, j, k + 1));
                    double frt_lo = fr_lo * 0.5 * (rt0n(i, j, k) / r0t(i, j, k) + rt0n(i, j, k - 1) / r0t(i, j, k - 1));
                    double frt_hi = fr_hi * 0.5 * (rt0n(i, j, k) / r0t(i, j, k) + rt0n(i, j, k + 1) / r0t(i, j, k + 1));
                    double invdetJ = 1.0 / g_src.detJ(i, j, k);
                    double src_r = -invdetJ * (fr_hi - fr_lo) * dxInv[2];
                    double src_rt = -invdetJ * (frt_hi - frt_lo) * dxInv[2];
                    double rho0_new = g_old.detJ(i, j, k) * r0o(i, j, k) + dt_base * g_src.detJ(i, j, k) * src_r;
                    double rt0_new = g_old.detJ(i, j, k) * rt0(i, j, k) + dt_base * g_src.detJ(i, j, k) * src_rt;
                    r0f(i, j, k) = rho0_new / g_new.detJ(i, j, k);
                    rt0_new /= g_new.detJ(i, j, k);
                    p0f(i, j, k) = getPgivenRTh(rt0_new);
                }
        // FillBoundary: lateral ghosts from the periodic images
        for (int k = 0; k < nz; ++k)
            for (int j = l[1]; j <= h[1]; ++j)
                for (int i = l[0]; i <= h[0]; ++i) {
                    if (i >= 0 && i < nx && j >= 0 && j < ny) continue;
                    int is = ((i % nx) + nx) % nx, js = ((j % ny) + ny) % ny;
                    r0f(i, j, k) = r0f(is, js, k);
                    p0f(i, j, k) = p0f(is, js, k);
                }
    }

    // no_substep_fun for moving terrain (TimeIntegration/ERF_TI_no_substep_fun.H:54-109):
    // rho and rho theta advanced detJ-weighted (the slow right-hand side
    // already carries the source geometry's detJ), the horizontal momenta
    // with h_zeta at the faces, rho w with the face detJ; at the moving
    // ground rho w follows the ground: W from Omega = rho z_t on the new grid.
    void no_substep_mt(State& Ssum, const State& Sold, const State& F, double slow_dt) {
        const Fab &dJo = g_old.detJ, &dJn = g_new.detJ, &Zo = g_old.znd, &Zn = g_new.znd;
        auto hzI = [&](const Fab& Zf, int i, int j, int k) {
            return 0.5 * dxInv[2] * (Zf(i, j, k + 1) + Zf(i, j + 1, k + 1) - Zf(i, j, k) - Zf(i, j + 1, k));
        };
        auto hzJ = [&](const Fab& Zf, int i, int j, int k) {
            return 0.5 * dxInv[2] * (Zf(i, j, k + 1) + Zf(i + 1, j, k + 1) - Zf(i, j, k) - Zf(i + 1, j, k));
        };
        loop(valid(CC), [&](int i, int j, int k) {
            for (int n = 0; n < 2; ++n) {
                Ssum.cons(i, j, k, n) = dJo(i, j, k) * Sold.cons(i, j, k, n) + slow_dt * F.cons(i, j, k, n);
                Ssum.cons(i, j, k, n) /= dJn(i, j, k);
            }
        });
        loop(valid(XF), [&](int i, int j, int k) {
            Ssum.mx(i, j, k) = (hzI(Zo, i, j, k) * Sold.mx(i, j, k) + slow_dt * F.mx(i, j, k)) / hzI(Zn, i, j, k);
        });
        loop(valid(YF), [&](int i, int j, int k) {
            Ssum.my(i, j, k) = (hzJ(Zo, i, j, k) * Sold.my(i, j, k) + slow_dt * F.my(i, j, k)) / hzJ(Zn, i, j, k);
        });
        load_geo(g_new);
        loop(valid(ZF), [&](int i, int j, int k) {
            if (k == 0) {
                double rho_on_face = Ssum.cons(i, j, k, 0);
                Ssum.mz(i, j, k) = w_from_omega(i, j, k, rho_on_face * zt(i, j, k), Ssum.mx, Ssum.my);
            } else {
                double ko = 0.5 * (dJo(i, j, k) + dJo(i, j, k - 1));
                double kn = 0.5 * (dJn(i, j, k) + dJn(i, j, k - 1));
                Ssum.mz(i, j, k) = (ko * Sold.mz(i, j, k) + slow_dt * F.mz(i, j, k)) / kn;
            }
        });
    }

    // erf_fast_rhs_MT (TimeIntegration/ERF_fast_rhs_MT.cpp:48-626): one
    // acoustic substep over moving terrain.  Go / Gn: the grids at the
    // substep's old and new times, Gs: the stage's (source) grid; zt: z_t of
    // the stage, zpt: the substep's z_t less it.  The horizontal momenta are
    // advanced h_zeta-weighted, rho w through the column solve on the
    // perturbation of Omega, rho and rho theta detJ-weighted old -> new.
    void fast_rhs_MT(int step, const State& Rs, const State& Sprev_in, const State& Sst, State& Sd, State& Scr,
                     const Geo& Go, const Geo& Gn, const Geo& Gs, const Fab& zpt, double dtau, double beta_s,
                     double facinv) {
        State Sprev; alloc_state(Sprev); copy_state(Sprev, Sprev_in);
        const double beta_1 = 0.5 * (1.0 - beta_s), beta_2 = 0.5 * (1.0 + beta_s), beta_d = 0.1;
        const double dxi = dxInv[0], dyi = dxInv[1], dzi = dxInv[2];
        const bool lagged = c.no_lagged_delta_rt == 0;
        const Fab &dJo = Go.detJ, &dJn = Gn.detJ, &dJs = Gs.detJ;
        Fab extrap, trhs, om;
        alloc(extrap, CC, 1, 1); alloc(trhs, CC, 0, 2); alloc(om, ZF, 0, 1);
        Fab& lag = Scr.cons;
        Fab& cur = Sd.cons;
        loop(grow(valid(CC), 1, 1, 1), [&](int i, int j, int k) {
            if (step == 0) {
                cur(i, j, k, 0) = Sprev.cons(i, j, k, 0);
                cur(i, j, k, 1) = Sprev.cons(i, j, k, 1);
                double d = cur(i, j, k, 1) - Sst.cons(i, j, k, 1);
                extrap(i, j, k) = d;
                lag(i, j, k, 1) = d;
            } else if (lagged) {
                double d = cur(i, j, k, 1) - Sst.cons(i, j, k, 1);
                extrap(i, j, k) = d + beta_d * (d - lag(i, j, k, 1));
                lag(i, j, k, 1) = d;
            } else {
                extrap(i, j, k) = cur(i, j, k, 1) - Sst.cons(i, j, k, 1);
            }
        });
        // horizontal momenta, h_zeta-weighted on the old grid
        loop(valid(XF), [&](int i, int j, int k) {
            double hxi = on(Go.znd, [&] { return hxi_I(i, j, k); }), hz = on(Go.znd, [&] { return hzeta_I(i, j, k); });
            double gp_xi = (extrap(i, j, k) - extrap(i - 1, j, k)) * dxi;
            double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k) - extrap(i, j, k))
                                      : 0.25 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k - 1) - extrap(i, j, k - 1));
            double gpx = hz * gp_xi - hxi * gp_zeta;
            gpx *= 1.0;
            double pi_c = 0.5 * (pi_stage(i - 1, j, k) + pi_stage(i, j, k));
            double f = -Gamma_ * R_d * pi_c * gpx;
            Sd.mx(i, j, k) = hz * Sprev.mx(i, j, k) + dtau * f + dtau * Rs.mx(i, j, k);
        });
        loop(valid(YF), [&](int i, int j, int k) {
            double het = on(Go.znd, [&] { return heta_J(i, j, k); }), hz = on(Go.znd, [&] { return hzeta_J(i, j, k); });
            double gp_eta = (extrap(i, j, k) - extrap(i, j - 1, k)) * dyi;
            double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k) - extrap(i, j - 1, k))
                                      : 0.25 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k - 1) - extrap(i, j - 1, k - 1));
            double gpy = hz * gp_eta - het * gp_zeta;
            gpy *= 1.0;
            double pi_c = 0.5 * (pi_stage(i, j - 1, k) + pi_stage(i, j, k));
            double f = -Gamma_ * R_d * pi_c * gpy;
            Sd.my(i, j, k) = hz * Sprev.my(i, j, k) + dtau * f + dtau * Rs.my(i, j, k);
        });
        // horizontal fluxes of rho and rho theta: the weighted momenta less
        // the stage's on the stage grid
        loop(valid(CC), [&](int i, int j, int k) {
            double hxl = on(Gs.znd, [&] { return hzeta_I(i, j, k); }), hxh = on(Gs.znd, [&] { return hzeta_I(i + 1, j, k); });
            double hyl = on(Gs.znd, [&] { return hzeta_J(i, j, k); }), hyh = on(Gs.znd, [&] { return hzeta_J(i, j + 1, k); });
            double xl = Sd.mx(i, j, k) - Sst.mx(i, j, k) * hxl, xh = Sd.mx(i + 1, j, k) - Sst.mx(i + 1, j, k) * hxh;
            double yl = Sd.my(i, j, k) - Sst.my(i, j, k) * hyl, yh = Sd.my(i, j + 1, k) - Sst.my(i, j + 1, k) * hyh;
            trhs(i, j, k, 0) = (xh - xl) * dxi + (yh - yl) * dyi;
            trhs(i, j, k, 1) = ((xh * (prim(i, j, k, 0) + prim(i + 1, j, k, 0)) - xl * (prim(i, j, k, 0) + prim(i - 1, j, k, 0))) * dxi +
                                (yh * (prim(i, j, k, 0) + prim(i, j + 1, k, 0)) - yl * (prim(i, j, k, 0) + prim(i, j - 1, k, 0))) * dyi) * 0.5;
        });
        // Omega'' of the previous substep on the old grid.  After the first
        // substep the reference passes one state as both the previous and the
        // new one, so the horizontal momenta read here are this substep's
        // (h_zeta-weighted, not yet divided); rho w is still the previous one.
        const Fab& pmx = step == 0 ? Sprev.mx : Sd.mx;
        const Fab& pmy = step == 0 ? Sprev.my : Sd.my;
        loop(valid(ZF), [&](int i, int j, int k) {
            if (k == 0) om(i, j, k) = 0.;
            else if (k == nz) om(i, j, k) = Sprev.mz(i, j, k) - Sst.mz(i, j, k) - zpt(i, j, k);
            else {
                double a = on(Go.znd, [&] { return omega_from_w(i, j, k, Sprev.mz(i, j, k), pmx, pmy); });
                double b = on(Go.znd, [&] { return omega_from_w(i, j, k, Sst.mz(i, j, k), Sst.mx, Sst.my); });
                om(i, j, k) = (a - b) - zpt(i, j, k);
            }
        });
        Fab& avx = Scr.mx; Fab& avy = Scr.my; Fab& avz = Scr.mz;
        loop(valid(XF), [&](int i, int j, int k) {
            Sd.mx(i, j, k) /= on(Gn.znd, [&] { return hzeta_I(i, j, k); });
            avx(i, j, k) += facinv * (Sd.mx(i, j, k) - Sst.mx(i, j, k));
        });
        loop(valid(YF), [&](int i, int j, int k) {
            Sd.my(i, j, k) /= on(Gn.znd, [&] { return hzeta_J(i, j, k); });
            avy(i, j, k) += facinv * (Sd.my(i, j, k) - Sst.my(i, j, k));
        });
        // the column system for the perturbation of Omega
        const double halfg = std::abs(0.5 * -c.gravity);
        const Fab& fc = fast_coeffs;
        Fab RHS, soln; alloc(RHS, ZF, 0, 1); alloc(soln, ZF, 0, 1);
        Bx bs = valid(CC); bs.lo[2] = 1; bs.hi[2] = nz - 1;
        loop(bs, [&](int i, int j, int k) {
            double Jo = 0.5 * (dJo(i, j, k) + dJo(i, j, k - 1));
            double Jn = 0.5 * (dJn(i, j, k) + dJn(i, j, k - 1));
            double Js = 0.5 * (dJs(i, j, k) + dJs(i, j, k - 1));
            double cP = fc(i, j, k, 3), cQ = fc(i, j, k, 4);
            double tlo = 0.5 * (prim(i, j, k - 2, 0) + prim(i, j, k - 1, 0));
            double tmid = 0.5 * (prim(i, j, k - 1, 0) + prim(i, j, k, 0));
            double thi = 0.5 * (prim(i, j, k, 0) + prim(i, j, k + 1, 0));
            double R0t = cP * cur(i, j, k, 1) * Jo + cQ * cur(i, j, k - 1, 1) * Jo
                         - cP * Sst.cons(i, j, k, 1) * Js - cQ * Sst.cons(i, j, k - 1, 1) * Js
                         - halfg * (cur(i, j, k, 0) + cur(i, j, k - 1, 0)) * Jo
                         + halfg * (Sst.cons(i, j, k, 0) + Sst.cons(i, j, k - 1, 0)) * Js;
            double R1t = -halfg * (Rs.cons(i, j, k, 0) + Rs.cons(i, j, k - 1, 0))
                         + (cP * Rs.cons(i, j, k, 1) + cQ * Rs.cons(i, j, k - 1, 1));
            double Okp1 = om(i, j, k + 1), Ok = om(i, j, k), Okm1 = om(i, j, k - 1);
            R1t += (halfg) * (beta_1 * dzi * (Okp1 - Okm1) + trhs(i, j, k, 0) + trhs(i, j, k - 1, 0));
            R1t += -(cP * (beta_1 * dzi * (Okp1 * thi - Ok * tmid) + trhs(i, j, k, 1)) +
                     cQ * (beta_1 * dzi * (Ok * tmid - Okm1 * tlo) + trhs(i, j, k - 1, 1)));
            RHS(i, j, k) = Jo * Sprev.mz(i, j, k) - Js * Sst.mz(i, j, k) + dtau * (Rs.mz(i, j, k) + R0t + dtau * beta_2 * R1t);
            double un = on(Gn.znd, [&] { return omega_from_w(i, j, k, 0., Sd.mx, Sd.my); });
            double us = on(Gs.znd, [&] { return omega_from_w(i, j, k, 0., Sst.mx, Sst.my); });
            double UppVpp = Jn * un - Js * us;
            RHS(i, j, k) += UppVpp;
        });
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double rho_on_bdy = 0.5 * (Sprev.cons(i, j, 0, 0) + Sprev.cons(i, j, -1, 0));
                RHS(i, j, 0) = rho_on_bdy * zpt(i, j, 0);
                soln(i, j, 0) = RHS(i, j, 0) * fc(i, j, 0, 1);
                RHS(i, j, nz) = 0.0;
                for (int k = 1; k <= nz; ++k) soln(i, j, k) = (RHS(i, j, k) - fc(i, j, k, 0) * soln(i, j, k - 1)) * fc(i, j, k, 1);
                for (int k = nz - 1; k >= 0; --k) soln(i, j, k) -= (fc(i, j, k, 2) * fc(i, j, k, 1)) * soln(i, j, k + 1);
                Sd.mz(i, j, nz) = Sst.mz(i, j, nz) + soln(i, j, nz);
            }
        // the new rho w; on the moving ground W from Omega = rho (z_t + z_t'')
        Bx bw = valid(ZF); bw.hi[2] = nz - 1;
        loop(bw, [&](int i, int j, int k) {
            double rho_on_face = 0.5 * (cur(i, j, k, 0) + cur(i, j, k - 1, 0));
            if (k == 0) {
                Sd.mz(i, j, k) = on(Gn.znd, [&] { return w_from_omega(i, j, k, rho_on_face * (zt(i, j, k) + zpt(i, j, k)), Sd.mx, Sd.my); });
                soln(i, j, k) = 0.;
            } else {
                double wn = on(Gn.znd, [&] { return w_from_omega(i, j, k, 0.0, Sd.mx, Sd.my); });
                double ws = on(Gs.znd, [&] { return w_from_omega(i, j, k, 0.0, Sst.mx, Sst.my); });
                double wpp = soln(i, j, k) + (wn - ws);
                double Jo = 0.5 * (dJo(i, j, k) + dJo(i, j, k - 1));
                double Jn = 0.5 * (dJn(i, j, k) + dJn(i, j, k - 1));
                Sd.mz(i, j, k) = Jo * (Sst.mz(i, j, k) + wpp);
                Sd.mz(i, j, k) /= Jn;
                double a = on(Gn.znd, [&] { return omega_from_w(i, j, k, Sd.mz(i, j, k), Sd.mx, Sd.my); });
                double b = on(Gs.znd, [&] { return omega_from_w(i, j, k, Sst.mz(i, j, k), Sst.mx, Sst.my); });
                soln(i, j, k) = a - b;
                soln(i, j, k) -= rho_on_face * zpt(i, j, k);
            }
        });
        // rho and rho theta, detJ-weighted old -> new
        loop(valid(CC), [&](int i, int j, int k) {
            double zl = beta_2 * soln(i, j, k) + beta_1 * om(i, j, k);
            double zh = beta_2 * soln(i, j, k + 1) + beta_1 * om(i, j, k + 1);
            avz(i, j, k) += facinv * zl / (1.0 * 1.0);
            if (k == nz - 1) avz(i, j, k + 1) += facinv * zh / (1.0 * 1.0);
            double frho = -(trhs(i, j, k, 0) + (zh - zl) * dzi);
            double tr = dJo(i, j, k) * cur(i, j, k, 0) + dtau * (Rs.cons(i, j, k, 0) + frho);
            cur(i, j, k, 0) = tr / dJn(i, j, k);
            double frt = -(trhs(i, j, k, 1) + 0.5 * (zh * (prim(i, j, k, 0) + prim(i, j, k + 1, 0)) - zl * (prim(i, j, k, 0) + prim(i, j, k - 1, 0))) * dzi);
            double tt = dJo(i, j, k) * cur(i, j, k, 1) + dtau * (Rs.cons(i, j, k, 1) + frt);
            cur(i, j, k, 1) = tt / dJn(i, j, k);
        });
    }

    // ComputeStrain_T (Diffusion/ERF_ComputeStrain_T.cpp:28-507): z-wall
    // planes first (one-sided derivatives at no-slip walls, GradWz
    // extrapolation otherwise), then the interior.  Periodic laterally, so
    // the x/y Dirichlet planes never apply.
    void compute_strain_T(Bx bxcc, Bx txy, Bx txz, Bx tyz, const Fab& u, const Fab& v, const Fab& w, Fab& s11,
                          Fab& s22, Fab& s33, Fab& s12, Fab& s13, Fab& s21, Fab& s23, Fab& s31, Fab& s32) const {
        const double* di = dxInv;
        const bool zl = zlo_noslip, zh = zhi_noslip;
        if (zl) {
            Bx p = txz; p.hi[2] = p.lo[2]; txz.lo[2] += 1;
            loop(p, [&](int i, int j, int k) {
                double GradWz = 0.5 * di[2] * (w(i, j, k + 1) + w(i - 1, j, k + 1) - w(i, j, k) - w(i - 1, j, k));
                double mxi = hxi_EJ(i, j, k), mz = hzeta_EJ(i, j, k);
                s13(i, j, k) = 0.5 * ((-(8. / 3.) * u(i, j, k - 1) + 3. * u(i, j, k) - (1. / 3.) * u(i, j, k + 1)) * di[2] / mz
                                      + ((w(i, j, k) - w(i - 1, j, k)) * di[0] - (mxi / mz) * GradWz) * 1.0);
                s31(i, j, k) = s13(i, j, k);
            });
        }
        if (zh) {
            Bx p = txz; p.lo[2] = p.hi[2]; txz.hi[2] -= 1;
            loop(p, [&](int i, int j, int k) {
                double mz = hzeta_EJ(i, j, k);
                s13(i, j, k) = 0.5 * (-(-(8. / 3.) * u(i, j, k) + 3. * u(i, j, k - 1) - (1. / 3.) * u(i, j, k - 2)) * di[2] / mz
                                      + (w(i, j, k) - w(i - 1, j, k)) * di[0] * 1.0);
                s31(i, j, k) = s13(i, j, k);
            });
        }
        if (zl) {
            Bx p = tyz; p.hi[2] = p.lo[2]; tyz.lo[2] += 1;
            loop(p, [&](int i, int j, int k) {
                double GradWz = 0.5 * di[2] * (w(i, j, k + 1) + w(i, j - 1, k + 1) - w(i, j, k) - w(i, j - 1, k));
                double meta = heta_EI(i, j, k), mz = hzeta_EI(i, j, k);
                s23(i, j, k) = 0.5 * ((-(8. / 3.) * v(i, j, k - 1) + 3. * v(i, j, k) - (1. / 3.) * v(i, j, k + 1)) * di[2] / mz
                                      + ((w(i, j, k) - w(i, j - 1, k)) * di[1] - (meta / mz) * GradWz) * 1.0);
                s32(i, j, k) = s23(i, j, k);
            });
        }
        if (zh) {
            Bx p = tyz; p.lo[2] = p.hi[2]; tyz.hi[2] -= 1;
            loop(p, [&](int i, int j, int k) {
                double mz = hzeta_EI(i, j, k);
                s23(i, j, k) = 0.5 * (-(-(8. / 3.) * v(i, j, k) + 3. * v(i, j, k - 1) - (1. / 3.) * v(i, j, k - 2)) * di[2] / mz
                                      + (w(i, j, k) - w(i, j - 1, k)) * di[1] * 1.0);
                s32(i, j, k) = s23(i, j, k);
            });
        }
        if (zl) {
            Bx pc = bxcc; pc.hi[2] = pc.lo[2]; bxcc.lo[2] += 1;
            loop(pc, [&](int i, int j, int k) {
                double GradUz = 0.5 * di[2] * ((-(8. / 3.) * u(i, j, k - 1) + 3. * u(i, j, k) - (1. / 3.) * u(i, j, k + 1))
                                               + (-(8. / 3.) * u(i - 1, j, k - 1) + 3. * u(i - 1, j, k) - (1. / 3.) * u(i - 1, j, k + 1)));
                double GradVz = 0.5 * di[2] * ((-(8. / 3.) * v(i, j, k - 1) + 3. * v(i, j, k) - (1. / 3.) * v(i, j, k + 1))
                                               + (-(8. / 3.) * v(i, j - 1, k - 1) + 3. * v(i, j - 1, k) - (1. / 3.) * v(i, j - 1, k + 1)));
                double mxi = hxi_cc(i, j, k), meta = heta_cc(i, j, k), mz = detJ(i, j, k);
                s11(i, j, k) = ((u(i + 1, j, k) / 1.0 - u(i, j, k) / 1.0) * di[0] - (mxi / mz) * GradUz) * 1.0 * 1.0;
                s22(i, j, k) = ((v(i, j + 1, k) / 1.0 - v(i, j, k) / 1.0) * di[1] - (meta / mz) * GradVz) * 1.0 * 1.0;
                s33(i, j, k) = (w(i, j, k + 1) - w(i, j, k)) * di[2] / mz;
            });
            Bx pxy = txy; pxy.hi[2] = pxy.lo[2]; txy.lo[2] += 1;
            loop(pxy, [&](int i, int j, int k) {
                double GradUz = 0.5 * di[2] * ((-(8. / 3.) * u(i, j, k - 1) + 3. * u(i, j, k) - (1. / 3.) * u(i, j, k + 1))
                                               + (-(8. / 3.) * u(i, j - 1, k - 1) + 3. * u(i, j - 1, k) - (1. / 3.) * u(i, j - 1, k + 1)));
                double GradVz = 0.5 * di[2] * ((-(8. / 3.) * v(i, j, k - 1) + 3. * v(i, j, k) - (1. / 3.) * v(i, j, k + 1))
                                               + (-(8. / 3.) * v(i - 1, j, k - 1) + 3. * v(i - 1, j, k) - (1. / 3.) * v(i - 1, j, k + 1)));
                double mxi = hxi_EK(i, j, k), meta = heta_EK(i, j, k), mz = hzeta_EK(i, j, k);
                s12(i, j, k) = 0.5 * ((u(i, j, k) / 1.0 - u(i, j - 1, k) / 1.0) * di[1] + (v(i, j, k) / 1.0 - v(i - 1, j, k) / 1.0) * di[0]
                                      - (meta / mz) * GradUz - (mxi / mz) * GradVz) * 1.0 * 1.0;
                s21(i, j, k) = s12(i, j, k);
            });
        }
        if (!zl && txz.lo[2] == 0) {
            Bx p = txz; p.hi[2] = p.lo[2]; txz.lo[2] += 1;
            loop(p, [&](int i, int j, int k) {
                double GradWz = 0.5 * di[2] * (w(i, j, k + 1) + w(i - 1, j, k + 1) - w(i, j, k) - w(i - 1, j, k));
                double mxi = hxi_EJ(i, j, k), mz = hzeta_EJ(i, j, k);
                s13(i, j, k) = 0.5 * ((u(i, j, k) - u(i, j, k - 1)) * di[2] / mz + ((w(i, j, k) - w(i - 1, j, k)) * di[0] - (mxi / mz) * GradWz) * 1.0);
                s31(i, j, k) = s13(i, j, k);
            });
        }
        if (!zl && tyz.lo[2] == 0) {
            Bx p = tyz; p.hi[2] = p.lo[2]; tyz.lo[2] += 1;
            loop(p, [&](int i, int j, int k) {
                double GradWz = 0.5 * di[2] * (w(i, j, k + 1) + w(i, j - 1, k + 1) - w(i, j, k) - w(i, j - 1, k));
                double meta = heta_EI(i, j, k), mz = hzeta_EI(i, j, k);
                s23(i, j, k) = 0.5 * ((v(i, j, k) - v(i, j, k - 1)) * di[2] / mz + ((w(i, j, k) - w(i, j - 1, k)) * di[1] - (meta / mz) * GradWz) * 1.0);
                s32(i, j, k) = s23(i, j, k);
            });
        }
        if (!zh && txz.hi[2] == nz) {
            Bx p = txz; p.lo[2] = p.hi[2]; txz.hi[2] -= 1;
            loop(p, [&](int i, int j, int k) {
                double mz = hzeta_EJ(i, j, k);
                s13(i, j, k) = 0.5 * ((u(i, j, k) - u(i, j, k - 1)) * di[2] / mz + (w(i, j, k) - w(i - 1, j, k)) * di[0] * 1.0);
                s31(i, j, k) = s13(i, j, k);
            });
        }
        if (!zh && tyz.hi[2] == nz) {
            Bx p = tyz; p.lo[2] = p.hi[2]; tyz.hi[2] -= 1;
            loop(p, [&](int i, int j, int k) {
                double mz = hzeta_EI(i, j, k);
                s23(i, j, k) = 0.5 * ((v(i, j, k) - v(i, j, k - 1)) * di[2] / mz + (w(i, j, k) - w(i, j - 1, k)) * di[1] * 1.0);
                s32(i, j, k) = s23(i, j, k);
            });
        }
        loop(bxcc, [&](int i, int j, int k) {
            double GradUz = 0.25 * di[2] * (u(i, j, k + 1) / 1.0 + u(i - 1, j, k + 1) / 1.0 - u(i, j, k - 1) / 1.0 - u(i - 1, j, k - 1) / 1.0);
            double GradVz = 0.25 * di[2] * (v(i, j, k + 1) / 1.0 + v(i, j - 1, k + 1) / 1.0 - v(i, j, k - 1) / 1.0 - v(i, j - 1, k - 1) / 1.0);
            double mxi = hxi_cc(i, j, k), meta = heta_cc(i, j, k), mz = detJ(i, j, k);
            s11(i, j, k) = ((u(i + 1, j, k) / 1.0 - u(i, j, k) / 1.0) * di[0] - (mxi / mz) * GradUz) * 1.0 * 1.0;
            s22(i, j, k) = ((v(i, j + 1, k) / 1.0 - v(i, j, k) / 1.0) * di[1] - (meta / mz) * GradVz) * 1.0 * 1.0;
            s33(i, j, k) = (w(i, j, k + 1) - w(i, j, k)) * di[2] / mz;
        });
        loop(txy, [&](int i, int j, int k) {
            double GradUz = 0.25 * di[2] * (u(i, j, k + 1) / 1.0 + u(i, j - 1, k + 1) / 1.0 - u(i, j, k - 1) / 1.0 - u(i, j - 1, k - 1) / 1.0);
            double GradVz = 0.25 * di[2] * (v(i, j, k + 1) / 1.0 + v(i - 1, j, k + 1) / 1.0 - v(i, j, k - 1) / 1.0 - v(i - 1, j, k - 1) / 1.0);
            double mxi = hxi_EK(i, j, k), meta = heta_EK(i, j, k), mz = hzeta_EK(i, j, k);
            s12(i, j, k) = 0.5 * ((u(i, j, k) / 1.0 - u(i, j - 1, k) / 1.0) * di[1] + (v(i, j, k) / 1.0 - v(i - 1, j, k) / 1.0) * di[0]
                                  - (meta / mz) * GradUz - (mxi / mz) * GradVz) * 1.0 * 1.0;
            s21(i, j, k) = s12(i, j, k);
        });
        loop(txz, [&](int i, int j, int k) {
            double GradWz = 0.25 * di[2] * (w(i, j, k + 1) + w(i - 1, j, k + 1) - w(i, j, k - 1) - w(i - 1, j, k - 1));
            double mxi = hxi_EJ(i, j, k), mz = hzeta_EJ(i, j, k);
            s13(i, j, k) = 0.5 * ((u(i, j, k) - u(i, j, k - 1)) * di[2] / mz + ((w(i, j, k) - w(i - 1, j, k)) * di[0] - (mxi / mz) * GradWz) * 1.0);
            s31(i, j, k) = s13(i, j, k);
        });
        loop(tyz, [&](int i, int j, int k) {
            double GradWz = 0.25 * di[2] * (w(i, j, k + 1) + w(i, j - 1, k + 1) - w(i, j, k - 1) - w(i, j - 1, k - 1));
            double meta = heta_EI(i, j, k), mz = hzeta_EI(i, j, k);
            s23(i, j, k) = 0.5 * ((v(i, j, k) - v(i, j, k - 1)) * di[2] / mz + ((w(i, j, k) - w(i, j - 1, k)) * di[1] - (meta / mz) * GradWz) * 1.0);
            s32(i, j, k) = s23(i, j, k);
        });
    }

    // The terrain strain boxes of advance_dycore / make_tau_terms: the valid
    // region grown by one laterally (cells and edges).
    void strain_boxes(Bx& bxcc, Bx& txy, Bx& txz, Bx& tyz) const {
        bxcc = grow(valid(CC), 1, 1, 0);
        txy = grow(Bx{{0, 0, 0}, {nx, ny, nz - 1}}, 1, 1, 0);
        txz = grow(Bx{{0, 0, 0}, {nx, ny - 1, nz}}, 1, 1, 0);
        tyz = grow(Bx{{0, 0, 0}, {nx - 1, ny, nz}}, 1, 1, 0);
    }
    void alloc_tau_T(Fab& t11, Fab& t22, Fab& t33, Fab& t12, Fab& t13, Fab& t21, Fab& t23, Fab& t31, Fab& t32) const {
        alloc_cc1(t11); alloc_cc1(t22); alloc_cc1(t33);
        alloc_edges(t12, t13, t23); alloc_edges(t21, t31, t32);
    }

    // make_tau_terms with terrain (TimeIntegration/ERF_make_tau_terms.cpp:
    // 177-317): expansion rate from the contravariant velocity, strain,
    // SmnSmn at stage 0 (Deardorff), then ComputeStressVarVisc_T
    // (Diffusion/ERF_ComputeStress_T.cpp:302-577).
    void make_tau_T(const Vel& V, const State& S, Fab& t11, Fab& t22, Fab& t33, Fab& t12, Fab& t13, Fab& t21,
                    Fab& t23, Fab& t31, Fab& t32) const {
        const Fab &u = V.u, &v = V.v, &w = V.w;
        Bx bxcc, txy, txz, tyz;
        strain_boxes(bxcc, txy, txz, tyz);
        Fab om; alloc(om, ZF, 2, 1);
        Bx ob = grow(valid(ZF), 1, 1, 0);
        loop(ob, [&](int i, int j, int k) { om(i, j, k) = (k == 0) ? 0. : omega_from_w(i, j, k, w(i, j, k), u, v); });
        Fab er; alloc_cc1(er);
        loop(bxcc, [&](int i, int j, int k) {
            double mhi = hzeta_I(i + 1, j, k), mlo = hzeta_I(i, j, k);
            double nhi = hzeta_J(i, j + 1, k), nlo = hzeta_J(i, j, k);
            double rate = (u(i + 1, j, k) / 1.0 * mhi - u(i, j, k) / 1.0 * mlo) * dxInv[0] * 1.0
                          + (v(i, j + 1, k) / 1.0 * nhi - v(i, j, k) / 1.0 * nlo) * dxInv[1] * 1.0
                          + (om(i, j, k + 1) - om(i, j, k)) * dxInv[2];
            er(i, j, k) = rate / detJ(i, j, k);
        });
        compute_strain_T(bxcc, txy, txz, tyz, u, v, w, t11, t22, t33, t12, t13, t21, t23, t31, t32);
        if (c.les_type == ERF_LES_DEARDORFF && tau_nrk == 0) {
            Fab& sm = smn;
            loop(valid(CC), [&](int i, int j, int k) { sm(i, j, k) = smnsmn(i, j, k, t11, t22, t33, t12, t13, t23); });
        }
        // stress on the valid edges, tau_ii on the grown cells
        txy = Bx{{0, 0, 0}, {nx, ny, nz - 1}};
        txz = Bx{{0, 0, 0}, {nx, ny - 1, nz}};
        tyz = Bx{{0, 0, 0}, {nx - 1, ny, nz}};
        const double mu_eff = use_consA ? 2.0 * c.dynamic_viscosity / c.rho0_trans : 2.0 * c.dynamic_viscosity;
        const Fab& cd = S.cons;
        auto rA = [&](int i, int j, int k) { return use_consA ? cd(i, j, k, 0) * mu_eff : mu_eff; };
        auto mt = [&](int i, int j, int k) { return use_turb ? mut(i, j, k) : 0.0; };
        const double OneThird = (1. / 3.);
        loop(bxcc, [&](int i, int j, int k) {
            t11(i, j, k) -= OneThird * er(i, j, k);
            t22(i, j, k) -= OneThird * er(i, j, k);
            t33(i, j, k) -= OneThird * er(i, j, k);
        });
        loop(valid(CC), [&](int i, int j, int k) {
            double mxi = hxi_cc(i, j, k), meta = heta_cc(i, j, k);
            double t31b = 0.25 * (t31(i, j, k) + t31(i + 1, j, k) + t31(i, j, k + 1) + t31(i + 1, j, k + 1));
            double t32b = 0.25 * (t32(i, j, k) + t32(i, j + 1, k) + t32(i, j, k + 1) + t32(i, j + 1, k + 1));
            double mu_tot = rA(i, j, k) + 2.0 * mt(i, j, k);
            t33(i, j, k) -= mxi * t31b + meta * t32b;
            t33(i, j, k) *= -mu_tot;
        });
        auto edge13 = [&](int i, int j, int k, double t11b, double t12b) {
            double mxi = hxi_EJ(i, j, k), meta = heta_EJ(i, j, k), mz = hzeta_EJ(i, j, k);
            double mu_bar = 0.25 * (mt(i - 1, j, k) + mt(i, j, k) + mt(i - 1, j, k - 1) + mt(i, j, k - 1));
            double ra_bar = 0.25 * (rA(i - 1, j, k) + rA(i, j, k) + rA(i - 1, j, k - 1) + rA(i, j, k - 1));
            double mu_tot = ra_bar + 2.0 * mu_bar;
            t13(i, j, k) -= mxi * t11b + meta * t12b;
            t13(i, j, k) *= -mu_tot;
            t31(i, j, k) *= -mu_tot * mz;
        };
        auto edge23 = [&](int i, int j, int k, double t21b, double t22b) {
            double mxi = hxi_EI(i, j, k), meta = heta_EI(i, j, k), mz = hzeta_EI(i, j, k);
            double mu_bar = 0.25 * (mt(i, j - 1, k) + mt(i, j, k) + mt(i, j - 1, k - 1) + mt(i, j, k - 1));
            double ra_bar = 0.25 * (rA(i, j - 1, k) + rA(i, j, k) + rA(i, j - 1, k - 1) + rA(i, j, k - 1));
            double mu_tot = ra_bar + 2.0 * mu_bar;
            t23(i, j, k) -= mxi * t21b + meta * t22b;
            t23(i, j, k) *= -mu_tot;
            t32(i, j, k) *= -mu_tot * mz;
        };
        {   // bottom planes: linear extrapolation of the cell / xy-edge values
            Bx p = txz; p.hi[2] = p.lo[2]; txz.lo[2] += 1;
            loop(p, [&](int i, int j, int k) {
                double a = 0.5 * (t11(i, j, k) + t11(i - 1, j, k)), b = 0.5 * (t11(i, j, k + 1) + t11(i - 1, j, k + 1));
                double t11b = 1.5 * a - 0.5 * b;
                double c1 = 0.5 * (t12(i, j, k) + t12(i, j + 1, k)), d = 0.5 * (t12(i, j, k + 1) + t12(i, j + 1, k + 1));
                double t12b = 1.5 * c1 - 0.5 * d;
                edge13(i, j, k, t11b, t12b);
            });
            Bx q = tyz; q.hi[2] = q.lo[2]; tyz.lo[2] += 1;
            loop(q, [&](int i, int j, int k) {
                double a = 0.5 * (t21(i, j, k) + t21(i + 1, j, k)), b = 0.5 * (t21(i, j, k + 1) + t21(i + 1, j, k + 1));
                double t21b = 1.5 * a - 0.5 * b;
                double c1 = 0.5 * (t22(i, j, k) + t22(i, j - 1, k)), d = 0.5 * (t22(i, j, k + 1) + t22(i, j - 1, k + 1));
                double t22b = 1.5 * c1 - 0.5 * d;
                edge23(i, j, k, t21b, t22b);
            });
        }
        {   // top planes
            Bx p = txz; p.lo[2] = p.hi[2]; txz.hi[2] -= 1;
            loop(p, [&](int i, int j, int k) {
                double lo = 0.5 * (t11(i, j, k - 2) + t11(i - 1, j, k - 2)), hi = 0.5 * (t11(i, j, k - 1) + t11(i - 1, j, k - 1));
                double t11b = 1.5 * hi - 0.5 * lo;
                double lo2 = 0.5 * (t12(i, j, k - 2) + t12(i, j + 1, k - 2)), hi2 = 0.5 * (t12(i, j, k - 1) + t12(i, j + 1, k - 1));
                double t12b = 1.5 * hi2 - 0.5 * lo2;
                edge13(i, j, k, t11b, t12b);
            });
            Bx q = tyz; q.lo[2] = q.hi[2]; tyz.hi[2] -= 1;
            loop(q, [&](int i, int j, int k) {
                double lo = 0.5 * (t21(i, j, k - 2) + t21(i + 1, j, k - 2)), hi = 0.5 * (t21(i, j, k - 1) + t21(i + 1, j, k - 1));
                double t21b = 1.5 * hi - 0.5 * lo;
                double lo2 = 0.5 * (t22(i, j, k - 2) + t22(i, j - 1, k - 2)), hi2 = 0.5 * (t22(i, j, k - 1) + t22(i, j - 1, k - 1));
                double t22b = 1.5 * hi2 - 0.5 * lo2;
                edge23(i, j, k, t21b, t22b);
            });
        }
        loop(txz, [&](int i, int j, int k) {
            double t11b = 0.25 * (t11(i, j, k) + t11(i - 1, j, k) + t11(i, j, k - 1) + t11(i - 1, j, k - 1));
            double t12b = 0.25 * (t12(i, j, k) + t12(i, j + 1, k) + t12(i, j, k - 1) + t12(i, j + 1, k - 1));
            edge13(i, j, k, t11b, t12b);
        });
        loop(tyz, [&](int i, int j, int k) {
            double t21b = 0.25 * (t21(i, j, k) + t21(i + 1, j, k) + t21(i, j, k - 1) + t21(i + 1, j, k - 1));
            double t22b = 0.25 * (t22(i, j, k) + t22(i, j - 1, k) + t22(i, j, k - 1) + t22(i, j - 1, k - 1));
            edge23(i, j, k, t21b, t22b);
        });
        loop(bxcc, [&](int i, int j, int k) {
            double mz = detJ(i, j, k);
            double mu_tot = rA(i, j, k) + 2.0 * mt(i, j, k);
            t11(i, j, k) *= -mu_tot * mz;
            t22(i, j, k) *= -mu_tot * mz;
        });
        loop(txy, [&](int i, int j, int k) {
            double mz = hzeta_EK(i, j, k);
            double mu_bar = 0.25 * (mt(i - 1, j, k) + mt(i, j, k) + mt(i - 1, j - 1, k) + mt(i, j - 1, k));
            double ra_bar = 0.25 * (rA(i - 1, j, k) + rA(i, j, k) + rA(i - 1, j - 1, k) + rA(i, j - 1, k));
            double mu_tot = ra_bar + 2.0 * mu_bar;
            t12(i, j, k) *= -mu_tot * mz;
            t21(i, j, k) *= -mu_tot * mz;
        });
    }

    // DiffusionSrcForMom_T (Diffusion/ERF_DiffusionSrcForMom_T.cpp:31-80)
    void diffusion_mom_T(State& R, const Fab& t11, const Fab& t22, const Fab& t33, const Fab& t12, const Fab& t13,
                         const Fab& t21, const Fab& t23, const Fab& t31, const Fab& t32) const {
        Bx tbx = valid(XF), tby = valid(YF), tbz = valid(ZF);
        tbz.lo[2] = 1; tbz.hi[2] = nz - 1;
        const double dxi = dxInv[0], dyi = dxInv[1], dzi = dxInv[2];
        loop(tbx, [&](int i, int j, int k) {
            double d = ((t11(i, j, k) - t11(i - 1, j, k)) * dxi * 1.0 + (t12(i, j + 1, k) - t12(i, j, k)) * dyi * 1.0
                        + (t13(i, j, k + 1) - t13(i, j, k)) * dzi);
            d /= 0.5 * (detJ(i, j, k) + detJ(i - 1, j, k));
            R.mx(i, j, k) -= d;
        });
        loop(tby, [&](int i, int j, int k) {
            double d = ((t21(i + 1, j, k) - t21(i, j, k)) * dxi * 1.0 + (t22(i, j, k) - t22(i, j - 1, k)) * dyi * 1.0
                        + (t23(i, j, k + 1) - t23(i, j, k)) * dzi);
            d /= 0.5 * (detJ(i, j, k) + detJ(i, j - 1, k));
            R.my(i, j, k) -= d;
        });
        loop(tbz, [&](int i, int j, int k) {
            double d = ((t31(i + 1, j, k) - t31(i, j, k)) * dxi * 1.0 + (t32(i, j + 1, k) - t32(i, j, k)) * dyi * 1.0
                        + (t33(i, j, k) - t33(i, j, k - 1)) * dzi);
            d /= 0.5 * (detJ(i, j, k) + detJ(i, j, k - 1));
            R.mz(i, j, k) -= d;
        });
    }

    // DiffusionSrcForState_T (Diffusion/ERF_DiffusionSrcForState_T.cpp:
    // 207-738) for comps [start_comp, start_comp+ncmp), no MOST, foextrap
    // scalars at the walls: metric-corrected fluxes, the theta z-face flux
    // kept as hfx_z before the cross-term correction, then the divergence
    // over detJ and the Deardorff TKE sources.
    void diffusion_state_T(int start_comp, int ncmp, const Fab& cell_data, const Fab& prm, Fab& rhs) const {
        const bool dd = c.les_type == ERF_LES_DEARDORFF;
        for (int n = 0; n < ncmp; ++n) {
            int q = start_comp + n, pidx = q - 1;
            double ae = alpha_eff(pidx), fac = eddy_factor(pidx);
            Fab fx, fy, fz;
            alloc(fx, XF, 0, 1); alloc(fy, YF, 0, 1); alloc(fz, ZF, 0, 1);
            auto mu = [&](int i, int j, int k) { return mut(i, j, k) * fac; };
            auto rAlpha = [&](double rho_face) { return use_consA ? rho_face * ae : ae; };
            loop(valid(XF), [&](int i, int j, int k) {
                double rA = rAlpha(0.5 * (cell_data(i, j, k, 0) + cell_data(i - 1, j, k, 0)));
                if (use_turb) rA += 0.5 * (mu(i, j, k) + mu(i - 1, j, k));
                double mxi = hxi_I(i, j, k), mz = axA(i, j, k);
                double GradCz = 0.25 * dxInv[2] * (prm(i, j, k + 1, pidx) + prm(i - 1, j, k + 1, pidx) - prm(i, j, k - 1, pidx) - prm(i - 1, j, k - 1, pidx));
                double GradCx = dxInv[0] * (prm(i, j, k, pidx) - prm(i - 1, j, k, pidx));
                fx(i, j, k) = -rA * 1.0 * (GradCx - (mxi / mz) * GradCz);
            });
            loop(valid(YF), [&](int i, int j, int k) {
                double rA = rAlpha(0.5 * (cell_data(i, j, k, 0) + cell_data(i, j - 1, k, 0)));
                if (use_turb) rA += 0.5 * (mu(i, j, k) + mu(i, j - 1, k));
                double meta = heta_J(i, j, k), mz = ayA(i, j, k);
                double GradCz = 0.25 * dxInv[2] * (prm(i, j, k + 1, pidx) + prm(i, j - 1, k + 1, pidx) - prm(i, j, k - 1, pidx) - prm(i, j - 1, k - 1, pidx));
                double GradCy = dxInv[1] * (prm(i, j, k, pidx) - prm(i, j - 1, k, pidx));
                fy(i, j, k) = -rA * 1.0 * (GradCy - (meta / mz) * GradCz);
            });
            loop(valid(ZF), [&](int i, int j, int k) {
                double rA = rAlpha(0.5 * (cell_data(i, j, k, 0) + cell_data(i, j, k - 1, 0)));
                if (use_turb) {
                    if (dd && pidx == 0) rA += 0.5 * (kthv(i, j, k) + kthv(i, j, k - 1));
                    else rA += 0.5 * (mu(i, j, k) + mu(i, j, k - 1));
                }
                double GradCz = dxInv[2] * (prm(i, j, k, pidx) - prm(i, j, k - 1, pidx));
                fz(i, j, k) = -rA * GradCz / 1.0;
                if (q == ERF_RHOTHETA_COMP) hfz(i, j, k) = fz(i, j, k);
            });
            // cross terms on the z-faces: extrapolated at the bottom and top faces
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    {
                        int k = 0;
                        double mxi = hxi_K(i, j, k), meta = heta_K(i, j, k);
                        double xlo = 0.5 * (fx(i, j, k) + fx(i + 1, j, k)), xhi = 0.5 * (fx(i, j, k + 1) + fx(i + 1, j, k + 1));
                        double xb = 1.5 * xlo - 0.5 * xhi;
                        double ylo = 0.5 * (fy(i, j, k) + fy(i, j + 1, k)), yhi = 0.5 * (fy(i, j, k + 1) + fy(i, j + 1, k + 1));
                        double yb = 1.5 * ylo - 0.5 * yhi;
                        fz(i, j, k) -= mxi * xb + meta * yb;
                    }
                    {
                        int k = nz;
                        double mxi = hxi_K(i, j, k), meta = heta_K(i, j, k);
                        double xlo = 0.5 * (fx(i, j, k - 2) + fx(i + 1, j, k - 2)), xhi = 0.5 * (fx(i, j, k - 1) + fx(i + 1, j, k - 1));
                        double xb = 1.5 * xhi - 0.5 * xlo;
                        double ylo = 0.5 * (fy(i, j, k - 2) + fy(i, j + 1, k - 2)), yhi = 0.5 * (fy(i, j, k - 1) + fy(i, j + 1, k - 1));
                        double yb = 1.5 * yhi - 0.5 * ylo;
                        fz(i, j, k) -= mxi * xb + meta * yb;
                    }
                }
            Bx z3 = valid(ZF); z3.lo[2] = 1; z3.hi[2] = nz - 1;
            loop(z3, [&](int i, int j, int k) {
                double mxi = hxi_K(i, j, k), meta = heta_K(i, j, k);
                double xb = 0.25 * (fx(i, j, k) + fx(i + 1, j, k) + fx(i, j, k - 1) + fx(i + 1, j, k - 1));
                double yb = 0.25 * (fy(i, j, k) + fy(i, j + 1, k) + fy(i, j, k - 1) + fy(i, j + 1, k - 1));
                fz(i, j, k) -= mxi * xb + meta * yb;
            });
            loop(valid(XF), [&](int i, int j, int k) { fx(i, j, k) *= hzeta_I(i, j, k); });
            loop(valid(YF), [&](int i, int j, int k) { fy(i, j, k) *= hzeta_J(i, j, k); });
            loop(valid(CC), [&](int i, int j, int k) {
                double s = (fx(i + 1, j, k) - fx(i, j, k)) * dxInv[0] * 1.0 + (fy(i, j + 1, k) - fy(i, j, k)) * dxInv[1] * 1.0
                           + (fz(i, j, k + 1) - fz(i, j, k)) * dxInv[2];
                s /= detJ(i, j, k);
                rhs(i, j, k, q) -= s;
            });
            if (dd && q == ERF_RHOKE_COMP) {
                const double l_abs_g = std::fabs(c.gravity), l_inv_theta0 = 1.0 / c.theta_ref;
                loop(valid(CC), [&](int i, int j, int k) {
                    rhs(i, j, k, q) += l_abs_g * l_inv_theta0 * hfz(i, j, k);
                    rhs(i, j, k, q) += 2.0 * mut(i, j, k) * smn(i, j, k);
                    rhs(i, j, k, q) -= diss(i, j, k);
                });
            }
        }
    }

    // AdvectionSrcForMom with terrain (Advection/ERF_AdvectionSrcForMom.cpp:
    // 208-288 for Centered_2nd, ERF_AdvectionSrcForMom_T.H:17-484 otherwise)
    void advect_mom_T(State& R, const State& S, const Vel& V, const Fab& Om) const {
        const Fab &ru = S.mx, &rv = S.my, &u = V.u, &v = V.v, &w = V.w;
        const Fab &ax = axA, &ay = ayA;
        int ht = c.dycore_horiz_adv, vt = c.dycore_vert_adv;
        double hf = c.dycore_horiz_upw_frac, vf = c.dycore_vert_upw_frac;
        bool c2 = (ht == ERF_ADV_CENTERED_2ND && vt == ERF_ADV_CENTERED_2ND);
        auto iX = [&](const Fab& f, int i, int j, int k, double upw) { double s[6]; gather(f, 0, i, j, k, 0, ht, s); return interp(ht, s, upw, hf); };
        auto iY = [&](const Fab& f, int i, int j, int k, double upw) { double s[6]; gather(f, 1, i, j, k, 0, ht, s); return interp(ht, s, upw, hf); };
        auto iZ = [&](const Fab& f, int i, int j, int k, double upw) { double s[6]; gather(f, 2, i, j, k, 0, vt, s); return interp(vt, s, upw, vf); };
        const double az = 1.0;
        Bx tbx = valid(XF), tby = valid(YF), tbz = valid(ZF);
        tbz.lo[2] = 1; tbz.hi[2] = nz - 1;
        int lo_z_face = 0, hi_z_face = nz;
        loop(tbx, [&](int i, int j, int k) {
            double src;
            if (c2) {
                double xh = 0.25 * (ru(i, j, k) * 1.0 + ru(i + 1, j, k) * 1.0) * (u(i + 1, j, k) + u(i, j, k)) * 0.5 * (ax(i, j, k) + ax(i + 1, j, k));
                double xl = 0.25 * (ru(i, j, k) * 1.0 + ru(i - 1, j, k) * 1.0) * (u(i - 1, j, k) + u(i, j, k)) * 0.5 * (ax(i, j, k) + ax(i - 1, j, k));
                double yh = 0.25 * (rv(i, j + 1, k) * 1.0 + rv(i - 1, j + 1, k) * 1.0) * (u(i, j + 1, k) + u(i, j, k)) * hzeta_EK(i, j + 1, k);
                double yl = 0.25 * (rv(i, j, k) * 1.0 + rv(i - 1, j, k) * 1.0) * (u(i, j - 1, k) + u(i, j, k)) * hzeta_EK(i, j, k);
                double zh = 0.25 * (Om(i, j, k + 1) + Om(i - 1, j, k + 1)) * (u(i, j, k + 1) + u(i, j, k)) * 0.5 * (az + az);
                double zl = 0.25 * (Om(i, j, k) + Om(i - 1, j, k)) * (u(i, j, k - 1) + u(i, j, k)) * 0.5 * (az + az);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
                src = -src / (0.5 * (detJ(i, j, k) + detJ(i - 1, j, k)));
            } else {
                double a, xh, xl, yh, yl, zh, zl;
                a = 0.5 * (ru(i + 1, j, k) * 1.0 + ru(i, j, k) * 1.0); xh = a * iX(u, i + 1, j, k, a) * 0.5 * (ax(i, j, k) + ax(i + 1, j, k));
                a = 0.5 * (ru(i - 1, j, k) * 1.0 + ru(i, j, k) * 1.0); xl = a * iX(u, i, j, k, a) * 0.5 * (ax(i, j, k) + ax(i - 1, j, k));
                a = 0.5 * (rv(i, j + 1, k) * 1.0 + rv(i - 1, j + 1, k) * 1.0); yh = a * iY(u, i, j + 1, k, a) * hzeta_EK(i, j + 1, k);
                a = 0.5 * (rv(i, j, k) * 1.0 + rv(i - 1, j, k) * 1.0); yl = a * iY(u, i, j, k, a) * hzeta_EK(i, j, k);
                a = 0.5 * (Om(i, j, k + 1) + Om(i - 1, j, k + 1)) * 0.5 * (az + az); zh = a * iZ(u, i, j, k + 1, a);
                a = 0.5 * (Om(i, j, k) + Om(i - 1, j, k)) * 0.5 * (az + az); zl = a * iZ(u, i, j, k, a);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
                src /= 0.5 * (detJ(i, j, k) + detJ(i - 1, j, k));
                src = -src;
            }
            R.mx(i, j, k) = src;
        });
        loop(tby, [&](int i, int j, int k) {
            double src;
            if (c2) {
                double xh = 0.25 * (ru(i + 1, j, k) * 1.0 + ru(i + 1, j - 1, k) * 1.0) * (v(i + 1, j, k) + v(i, j, k)) * hzeta_EK(i + 1, j, k);
                double xl = 0.25 * (ru(i, j, k) * 1.0 + ru(i, j - 1, k) * 1.0) * (v(i - 1, j, k) + v(i, j, k)) * hzeta_EK(i, j, k);
                double yh = 0.25 * (rv(i, j + 1, k) * 1.0 + rv(i, j, k) * 1.0) * (v(i, j + 1, k) + v(i, j, k)) * 0.5 * (ay(i, j, k) + ay(i, j + 1, k));
                double yl = 0.25 * (rv(i, j, k) * 1.0 + rv(i, j - 1, k) * 1.0) * (v(i, j - 1, k) + v(i, j, k)) * 0.5 * (ay(i, j, k) + ay(i, j - 1, k));
                double zh = 0.25 * (Om(i, j, k + 1) + Om(i, j - 1, k + 1)) * (v(i, j, k + 1) + v(i, j, k)) * 0.5 * (az + az);
                double zl = 0.25 * (Om(i, j, k) + Om(i, j - 1, k)) * (v(i, j, k - 1) + v(i, j, k)) * 0.5 * (az + az);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
                src = -src / (0.5 * (detJ(i, j, k) + detJ(i, j - 1, k)));
            } else {
                double a, xh, xl, yh, yl, zh, zl;
                a = 0.5 * (ru(i + 1, j, k) * 1.0 + ru(i + 1, j - 1, k) * 1.0); xh = a * iX(v, i + 1, j, k, a) * hzeta_EK(i + 1, j, k);
                a = 0.5 * (ru(i, j, k) * 1.0 + ru(i, j - 1, k) * 1.0); xl = a * iX(v, i, j, k, a) * hzeta_EK(i, j, k);
                a = 0.5 * (rv(i, j, k) * 1.0 + rv(i, j + 1, k) * 1.0); yh = a * 0.5 * (ay(i, j, k) + ay(i, j + 1, k)) * iY(v, i, j + 1, k, a);
                a = 0.5 * (rv(i, j, k) * 1.0 + rv(i, j - 1, k) * 1.0); yl = a * 0.5 * (ay(i, j, k) + ay(i, j - 1, k)) * iY(v, i, j, k, a);
                a = 0.5 * (Om(i, j, k + 1) + Om(i, j - 1, k + 1)) * 0.5 * (az + az); zh = a * iZ(v, i, j, k + 1, a);
                a = 0.5 * (Om(i, j, k) + Om(i, j - 1, k)) * 0.5 * (az + az); zl = a * iZ(v, i, j, k, a);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
                src /= 0.5 * (detJ(i, j, k) + detJ(i, j - 1, k));
                src = -src;
            }
            R.my(i, j, k) = src;
        });
        loop(tbz, [&](int i, int j, int k) {
            double src;
            if (c2) {
                double xh = 0.25 * (ru(i + 1, j, k) + ru(i + 1, j, k - 1)) * 1.0 * (w(i + 1, j, k) + w(i, j, k)) * hzeta_EJ(i + 1, j, k);
                double xl = 0.25 * (ru(i, j, k) + ru(i, j, k - 1)) * 1.0 * (w(i - 1, j, k) + w(i, j, k)) * hzeta_EJ(i, j, k);
                double yh = 0.25 * (rv(i, j + 1, k) + rv(i, j + 1, k - 1)) * 1.0 * (w(i, j + 1, k) + w(i, j, k)) * hzeta_EI(i, j + 1, k);
                double yl = 0.25 * (rv(i, j, k) + rv(i, j, k - 1)) * 1.0 * (w(i, j - 1, k) + w(i, j, k)) * hzeta_EI(i, j, k);
                double zl = 0.25 * (Om(i, j, k) + Om(i, j, k - 1)) * (w(i, j, k) + w(i, j, k - 1));
                double zh = (k == hi_z_face) ? Om(i, j, k) * w(i, j, k) * az
                                             : 0.25 * (Om(i, j, k) + Om(i, j, k + 1)) * (w(i, j, k) + w(i, j, k + 1)) * 0.5 * (az + az);
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
                src = -src / (0.5 * (detJ(i, j, k) + detJ(i, j, k - 1)));
            } else {
                double a, xh, xl, yh, yl, zh, zl, ih = 0, il = 0;
                a = 0.5 * (ru(i + 1, j, k) + ru(i + 1, j, k - 1)) * 1.0; xh = a * iX(w, i + 1, j, k, a) * hzeta_EJ(i + 1, j, k);
                a = 0.5 * (ru(i, j, k) + ru(i, j, k - 1)) * 1.0; xl = a * iX(w, i, j, k, a) * hzeta_EJ(i, j, k);
                a = 0.5 * (rv(i, j + 1, k) + rv(i, j + 1, k - 1)) * 1.0; yh = a * iY(w, i, j + 1, k, a) * hzeta_EI(i, j + 1, k);
                a = 0.5 * (rv(i, j, k) + rv(i, j, k - 1)) * 1.0; yl = a * iY(w, i, j, k, a) * hzeta_EI(i, j, k);
                auto iZall = [&](int kk, double upw, double frac, int type) { double s[6]; gather(w, 2, i, j, kk, 0, (type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH) ? ERF_ADV_UPWIND_5TH : (type == ERF_ADV_CENTERED_2ND ? ERF_ADV_CENTERED_2ND : ERF_ADV_UPWIND_3RD), s); return interp_all(type, s, upw, frac); };
                double Oh = (k == hi_z_face) ? Om(i, j, k) * az : 0.25 * (Om(i, j, k) + Om(i, j, k + 1)) * (az + az);
                if (k == hi_z_face) { zh = Oh * w(i, j, k); }
                else {
                    if (k == hi_z_face - 1) ih = iZall(k + 1, Oh, 0, ERF_ADV_CENTERED_2ND);
                    else if (k == hi_z_face - 2 || k == lo_z_face + 1) {
                        if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) ih = iZall(k + 1, Oh, 0, ERF_ADV_CENTERED_4TH);
                        else ih = iZall(k + 1, Oh, vf, vt);
                    } else ih = iZ(w, i, j, k + 1, Oh);
                    zh = Oh * ih;
                }
                double Ol = (k == 0) ? Om(i, j, k) * az : 0.25 * (Om(i, j, k) + Om(i, j, k - 1)) * (az + az);
                if (k == 0) { zl = Ol * w(i, j, k); }
                else {
                    if (k == lo_z_face + 1) il = iZall(k, Ol, 0, ERF_ADV_CENTERED_2ND);
                    else if (k == lo_z_face + 2 || k == hi_z_face - 1) {
                        if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) il = iZall(k, Ol, 0, ERF_ADV_CENTERED_4TH);
                        else il = iZall(k, Ol, vf, vt);
                    } else il = iZ(w, i, j, k, Ol);
                    zl = Ol * il;
                }
                src = (xh - xl) * dxInv[0] * 1.0 + (yh - yl) * dxInv[1] * 1.0 + (zh - zl) * dxInv[2];
                double denom = 0.5 * (detJ(i, j, k) + detJ(i, j, k - 1));
                src /= denom;
                src = -src;
            }
            R.mz(i, j, k) = src;
        });
    }

    // ERFPhysBCFunct_w::impose_vertical_zvel_bcs with static terrain
    // (BoundaryConditions/ERF_BoundaryConditions_zvel.cpp:200-262): w on the
    // bottom face from Omega = 0; on a wall top likewise.
    void physbcs_w_T(Fab& w, const Fab& u, const Fab& v, int ng) const {
        fill_periodic(w, ZF);
        Bx b = grow(valid(ZF), ng, ng, 0);
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) {
                // a moving ground keeps the w of the update (the moving-terrain
                // branch of impose_vertical_zvel_bcs sets nothing)
                if (!moving) w(i, j, 0) = w_from_omega(i, j, 0, 0.0, u, v);
                w(i, j, nz) = w_from_omega(i, j, nz, 0.0, u, v);
            }
    }

    // erf_fast_rhs_T (TimeIntegration/ERF_fast_rhs_T.cpp:39-704), static
    // terrain, implicit substepping.
    void fast_rhs_T(int step, const State& Rs, const State& Sprev_in, const State& Sst, State& Sd, State& Scr,
                    double dtau, double beta_s, double facinv) {
        State Sprev; alloc_state(Sprev); copy_state(Sprev, Sprev_in);
        double beta_1 = 0.5 * (1.0 - beta_s), beta_2 = 0.5 * (1.0 + beta_s), beta_d = 0.1;
        double dxi = dxInv[0], dyi = dxInv[1], dzi = dxInv[2];
        Fab odr, odrt, extrap, odu, odv, odw, ndu, ndv, trhs, om;
        alloc(odr, CC, 1, 1); alloc(odrt, CC, 1, 1); alloc(extrap, CC, 1, 1);
        alloc(odu, XF, 1, 1); alloc(odv, YF, 1, 1); alloc(odw, ZF, 1, 1);
        alloc(ndu, XF, 1, 1); alloc(ndv, YF, 1, 1); alloc(trhs, CC, 0, 2); alloc(om, ZF, 0, 1);
        Fab& lag = Scr.cons;
        // cur = prev at the first substep (cons comps 0-1, ghosts included)
        Fab& cur = Sd.cons;
        if (step == 0)
            loop(grow(valid(CC), 1, 1, 1), [&](int i, int j, int k) {
                cur(i, j, k, 0) = Sprev.cons(i, j, k, 0); cur(i, j, k, 1) = Sprev.cons(i, j, k, 1);
            });
        loop(grow(valid(XF), 1, 1, 0), [&](int i, int j, int k) {
            odu(i, j, k) = Sprev.mx(i, j, k) - Sst.mx(i, j, k);
            if (k == nz - 1) odu(i, j, k + 1) = odu(i, j, k);
        });
        loop(grow(valid(YF), 1, 1, 0), [&](int i, int j, int k) {
            odv(i, j, k) = Sprev.my(i, j, k) - Sst.my(i, j, k);
            if (k == nz - 1) odv(i, j, k + 1) = odv(i, j, k);
        });
        loop(grow(valid(ZF), 1, 1, 0), [&](int i, int j, int k) { odw(i, j, k) = Sprev.mz(i, j, k) - Sst.mz(i, j, k); });
        loop(grow(valid(CC), 1, 1, 1), [&](int i, int j, int k) {
            odr(i, j, k) = cur(i, j, k, 0) - Sst.cons(i, j, k, 0);
            odrt(i, j, k) = cur(i, j, k, 1) - Sst.cons(i, j, k, 1);
            if (step == 0) extrap(i, j, k) = odrt(i, j, k);
            else extrap(i, j, k) = odrt(i, j, k) + beta_d * (odrt(i, j, k) - lag(i, j, k, 1));
        });
        loop(grow(valid(CC), 1, 1, 1), [&](int i, int j, int k) { lag(i, j, k, 1) = odrt(i, j, k); });
        Fab& avx = Scr.mx; Fab& avy = Scr.my; Fab& avz = Scr.mz;
        loop(valid(XF), [&](int i, int j, int k) {
            double mxi = hxi_I(i, j, k), mz = hzeta_I(i, j, k);
            double gp_xi = (extrap(i, j, k) - extrap(i - 1, j, k)) * dxi;
            double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k) - extrap(i, j, k))
                                      : 0.25 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k - 1) - extrap(i, j, k - 1));
            double gpx = gp_xi - (mxi / mz) * gp_zeta;
            gpx *= 1.0;
            if (use_moisture) {
                double q = 0.5 * (prim(i, j, k, 4) + prim(i - 1, j, k, 4) + prim(i, j, k, 5) + prim(i - 1, j, k, 5));
                gpx /= (1.0 + q);
            }
            double pi_c = 0.5 * (pi_stage(i - 1, j, k) + pi_stage(i, j, k));
            double f = -Gamma_ * R_d * pi_c * gpx;
            ndu(i, j, k) = odu(i, j, k) + dtau * f + dtau * Rs.mx(i, j, k);
            avx(i, j, k) += facinv * ndu(i, j, k);
            Sd.mx(i, j, k) = Sst.mx(i, j, k) + ndu(i, j, k);
        });
        loop(valid(YF), [&](int i, int j, int k) {
            double meta = heta_J(i, j, k), mz = hzeta_J(i, j, k);
            double gp_eta = (extrap(i, j, k) - extrap(i, j - 1, k)) * dyi;
            double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k) - extrap(i, j - 1, k))
                                      : 0.25 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k - 1) - extrap(i, j - 1, k - 1));
            double gpy = gp_eta - (meta / mz) * gp_zeta;
            gpy *= 1.0;
            if (use_moisture) {
                double q = 0.5 * (prim(i, j, k, 4) + prim(i, j - 1, k, 4) + prim(i, j, k, 5) + prim(i, j - 1, k, 5));
                gpy /= (1.0 + q);
            }
            double pi_c = 0.5 * (pi_stage(i, j - 1, k) + pi_stage(i, j, k));
            double f = -Gamma_ * R_d * pi_c * gpy;
            ndv(i, j, k) = odv(i, j, k) + dtau * f + dtau * Rs.my(i, j, k);
            avy(i, j, k) += facinv * ndv(i, j, k);
            Sd.my(i, j, k) = Sst.my(i, j, k) + ndv(i, j, k);
        });
        // horizontal fluxes of rho and rho theta through the sloping faces
        loop(valid(CC), [&](int i, int j, int k) {
            double hxh = 0.5 * dzi * (Z(i + 1, j, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j, k) - Z(i + 1, j + 1, k));
            double hxl = 0.5 * dzi * (Z(i, j, k + 1) + Z(i, j + 1, k + 1) - Z(i, j, k) - Z(i, j + 1, k));
            double hyh = 0.5 * dzi * (Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1) - Z(i, j + 1, k) - Z(i + 1, j + 1, k));
            double hyl = 0.5 * dzi * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) - Z(i, j, k) - Z(i + 1, j, k));
            double xl = ndu(i, j, k) * hxl / 1.0, xh = ndu(i + 1, j, k) * hxh / 1.0;
            double yl = ndv(i, j, k) * hyl / 1.0, yh = ndv(i, j + 1, k) * hyh / 1.0;
            double mfsq = 1.0;
            trhs(i, j, k, 0) = (xh - xl) * dxi * mfsq + (yh - yl) * dyi * mfsq;
            trhs(i, j, k, 1) = ((xh * (prim(i, j, k, 0) + prim(i + 1, j, k, 0)) - xl * (prim(i, j, k, 0) + prim(i - 1, j, k, 0))) * dxi * mfsq +
                                (yh * (prim(i, j, k, 0) + prim(i, j + 1, k, 0)) - yl * (prim(i, j, k, 0) + prim(i, j - 1, k, 0))) * dyi * mfsq) * 0.5;
        });
        // contravariant vertical increment of the previous substep
        loop(valid(ZF), [&](int i, int j, int k) {
            if (k == 0) om(i, j, k) = 0.;
            else if (k == nz) om(i, j, k) = odw(i, j, k);
            else om(i, j, k) = omega_from_w(i, j, k, odw(i, j, k), odu, odv);
        });
        double halfg = std::abs(0.5 * -c.gravity);
        Fab RHS, soln; alloc(RHS, ZF, 0, 1); alloc(soln, ZF, 0, 1);
        Bx bs = valid(CC); bs.lo[2] = 1; bs.hi[2] = nz - 1;
        const Fab& fc = fast_coeffs;
        loop(bs, [&](int i, int j, int k) {
            double dJk = 0.5 * (detJ(i, j, k) + detJ(i, j, k - 1));
            double cP = fc(i, j, k, 3), cQ = fc(i, j, k, 4);
            if (use_moisture) {
                double q = 0.5 * (prim(i, j, k, 4) + prim(i, j, k - 1, 4) + prim(i, j, k, 5) + prim(i, j, k - 1, 5));
                cP /= (1.0 + q); cQ /= (1.0 + q);
            }
            double tlo = 0.5 * (prim(i, j, k - 2, 0) + prim(i, j, k - 1, 0));
            double tmid = 0.5 * (prim(i, j, k - 1, 0) + prim(i, j, k, 0));
            double thi = 0.5 * (prim(i, j, k, 0) + prim(i, j, k + 1, 0));
            double R0t = (-halfg * odr(i, j, k) + cP * odrt(i, j, k)) * detJ(i, j, k)
                         + (-halfg * odr(i, j, k - 1) + cQ * odrt(i, j, k - 1)) * detJ(i, j, k - 1);
            double R1t = -halfg * (Rs.cons(i, j, k, 0) * detJ(i, j, k) + Rs.cons(i, j, k - 1, 0) * detJ(i, j, k - 1))
                         + (cP * Rs.cons(i, j, k, 1) * detJ(i, j, k) + cQ * Rs.cons(i, j, k - 1, 1) * detJ(i, j, k - 1));
            double Okp1 = om(i, j, k + 1), Ok = om(i, j, k), Okm1 = om(i, j, k - 1);
            R1t += (halfg) * (beta_1 * dzi * (Okp1 - Okm1) + trhs(i, j, k, 0) + trhs(i, j, k - 1, 0));
            R1t += -(cP * (beta_1 * dzi * (Okp1 * thi - Ok * tmid) + trhs(i, j, k, 1)) +
                     cQ * (beta_1 * dzi * (Ok * tmid - Okm1 * tlo) + trhs(i, j, k - 1, 1)));
            RHS(i, j, k) = dJk * odw(i, j, k) + dtau * (dJk * Rs.mz(i, j, k) + R0t + dtau * beta_2 * R1t);
            RHS(i, j, k) += dJk * omega_from_w(i, j, k, 0., ndu, ndv);
        });
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                RHS(i, j, 0) = dtau * Rs.mz(i, j, 0);
                RHS(i, j, nz) = dtau * Rs.mz(i, j, nz);
                soln(i, j, 0) = RHS(i, j, 0) * fc(i, j, 0, 1);
                for (int k = 1; k <= nz; ++k) soln(i, j, k) = (RHS(i, j, k) - fc(i, j, k, 0) * soln(i, j, k - 1)) * fc(i, j, k, 1);
                for (int k = nz - 1; k >= 0; --k) soln(i, j, k) -= (fc(i, j, k, 2) * fc(i, j, k, 1)) * soln(i, j, k + 1);
            }
        loop(valid(ZF), [&](int i, int j, int k) {
            Sd.mz(i, j, k) = Sst.mz(i, j, k);
            if (k >= 1 && k <= nz - 1) Sd.mz(i, j, k) += w_from_omega(i, j, k, soln(i, j, k), ndu, ndv);
        });
        loop(valid(CC), [&](int i, int j, int k) {
            double zl = beta_2 * soln(i, j, k) + beta_1 * om(i, j, k);
            double zh = beta_2 * soln(i, j, k + 1) + beta_1 * om(i, j, k + 1);
            avz(i, j, k) += facinv * zl / (1.0 * 1.0);
            if (k == nz - 1) avz(i, j, k + 1) += facinv * zh / (1.0 * 1.0);
            double frho = -(trhs(i, j, k, 0) + (zh - zl) * dzi) / detJ(i, j, k);
            cur(i, j, k, 0) += dtau * (Rs.cons(i, j, k, 0) + frho);
            double frt = -(trhs(i, j, k, 1) + 0.5 * (zh * (prim(i, j, k, 0) + prim(i, j, k + 1, 0)) - zl * (prim(i, j, k, 0) + prim(i, j, k - 1, 0))) * dzi) / detJ(i, j, k);
            cur(i, j, k, 1) += dtau * (Rs.cons(i, j, k, 1) + frt);
        });
    }

    void step(double dt) {
        const double beta_s = 0.1;
        // FillPatch of the old state (ghost cells of cons and velocities)
        tick();
        Fab& Sc = cons_state;
        physbcs_cons(Sc, 0, ncomp, ngc);
        physbcs_tangential(vel_state.u, XF, ngv);
        physbcs_tangential(vel_state.v, YF, ngv);
        if (terrain) physbcs_w_T(vel_state.w, vel_state.u, vel_state.v, ngv);
        else physbcs_w(vel_state.w, ngv);
        // S_old = {cons, V2M(old velocities)}
        S_old.cons.copy_from(Sc);
        if (moving) { r0o = r0f; p0o = p0f; }   // base_state == base_state_new at the step's start
        // turbulent viscosity from the old velocities (strain + Smagorinsky)
        tock(5);
        if (use_turb) turbulent_viscosity(vel_state, S_old.cons, mut);
        tock(0);
        vel_to_mom(vel_state.u, vel_state.v, vel_state.w, S_old.cons, S_old.mx, S_old.my, S_old.mz);
        Vnew.u.copy_from(vel_state.u); Vnew.v.copy_from(vel_state.v); Vnew.w.copy_from(vel_state.w);
        // the MOST fluxes of the step from its old velocities, taken before the
        // prologue fill imposes them (ERF_Advance.cpp:62-86)
        if (most) most_update_fluxes(vel_state);
        apply_bcs(S_old, Vnew, ngc, ngv, false, true);
        cons_to_prim(S_old.cons, ngc, prim, pi_stage);
        // MRISplitIntegrator::advance (ERF_MRI.H:187-324)
        copy_state(S_new, S_old);
        const bool nosub = c.substepping_type == ERF_SUBSTEP_NONE;
        int ratio = c.mri_ratio;
        double sub_dt = nosub ? 0.0 : dt / ratio;
        for (int nrk = 0; nrk < 3; ++nrk) {
            int nsub; double dtau;
            if (nrk == 0) {
                if (c.force_stage1_single_substep || nosub) { nsub = 1; dtau = dt / 3.0; }
                else { nsub = ratio / 3; dtau = sub_dt; }
            } else if (nrk == 1) {
                if (nosub) { nsub = 1; dtau = 0.5 * dt; }
                else { nsub = ratio / 2; dtau = sub_dt; }
            } else {
                if (nosub) { nsub = 1; dtau = dt; }
                else { nsub = ratio; dtau = sub_dt; }
            }
            double slow_dt = (nrk == 0 ? dt / 3.0 : (nrk == 1 ? dt / 2.0 : dt));
            if (nrk > 0) cons_to_prim(S_new.cons, ngc, prim, pi_stage);
            tock(5);
            if (moving) {
                // ERF_MRI.H:245-320 with the moving-terrain branches of
                // slow_rhs_fun_pre / no_substep_fun / slow_rhs_fun_post; the
                // stage times and slow_dt = new stage time - old step time
                double t_so = nrk == 0 ? time : (nrk == 1 ? time + dt / 3.0 : time + dt / 2.0);
                double t_sn = nrk == 0 ? time + dt / 3.0 : (nrk == 1 ? time + dt / 2.0 : time + dt);
                double sdt = t_sn - time;
                mt_stage_geometry(time, t_so, t_sn, sdt);
                load_geo(g_src);
                slow_rhs_pre(nrk, sdt, F_slow, S_new, S_scr, Vnew);
                mt_base_state(sdt);
                if (nosub) {
                    no_substep_mt(S_sum, S_old, F_slow, nsub * dtau);
                    load_geo(g_old);
                    apply_bcs(S_sum, Vnew, ngc, ngv, true, false);
                } else {
                    // fast_rhs_fun, moving terrain (ERF_TI_fast_rhs_fun.H:47-118):
                    // per substep the grids at its old and new times, z_t'' = the
                    // substep's z_t less the stage's, the fast coefficients on the
                    // old grid with the step's old base state, then the boundary
                    // fill on the old grid; the level keeps the last substep's
                    // old grid and the new grid is the last substep's new one.
                    Geo g_stg = g_src, g_so, g_sn;
                    Fab zpt; zpt.define(zt.lo, zt.hi, 1);
                    for (int ks = 0; ks < nsub; ++ks) {
                        mt_grid(time + ks * dtau); save_geo(g_so);
                        mt_grid(time + (ks + 1) * dtau); save_geo(g_sn);
                        const double inv_dt = 1. / dtau;
                        for (int k = 0; k <= nz; ++k)
                            for (int j = -1; j <= ny; ++j)
                                for (int i = -1; i <= nx; ++i) {
                                    const Fab &zn = g_sn.znd, &zo = g_so.znd;
                                    zpt(i, j, k) = 0.25 * inv_dt * (zn(i + 1, j + 1, k) - zo(i + 1, j + 1, k) + zn(i, j + 1, k) - zo(i, j + 1, k)
                                                                    + zn(i + 1, j, k) - zo(i + 1, j, k) + zn(i, j, k) - zo(i, j, k));
                                    zpt(i, j, k) -= zt(i, j, k);
                                }
                        load_geo(g_so);
                        std::swap(r0f, r0o);   // make_fast_coeffs reads base_state, not base_state_new
                        make_fast_coeffs(S_new, dtau, beta_s);
                        std::swap(r0f, r0o);
                        fast_rhs_MT(ks, F_slow, ks == 0 ? S_old : S_sum, S_new, S_sum, S_scr, g_so, g_sn, g_stg, zpt,
                                    dtau, beta_s, 1.0 / (double)nsub);
                        apply_bcs(S_sum, Vnew, 1, 1, true, false);
                    }
                    g_new = g_sn;
                }
                slow_rhs_post(nrk, sdt, F_slow, S_old, S_new, S_sum, S_scr);
                apply_bcs(S_new, Vnew, ngc, ngv, false, false);
                continue;
            }
            slow_rhs_pre(nrk, slow_dt, F_slow, S_new, S_scr, Vnew);
            tock(1);
            double inv_fac = 1.0 / (double)nsub;
            if (nosub) {
                no_substep(S_sum, S_old, F_slow, nsub * dtau);
                apply_bcs(S_sum, Vnew, ngc, ngv, true, false);
            }
            for (int ks = 0; ks < (nosub ? 0 : nsub); ++ks) {
                if (ks == 0) make_fast_coeffs(S_new, dtau, beta_s);
                if (terrain) fast_rhs_T(ks, F_slow, ks == 0 ? S_old : S_sum, S_new, S_sum, S_scr, dtau, beta_s, inv_fac);
                else fast_rhs_N(ks, nrk, F_slow, ks == 0 ? S_old : S_sum, S_new, S_sum, S_scr, dtau, beta_s, inv_fac);
                apply_bcs(S_sum, Vnew, 1, 1, true, false);
            }
            tock(2);
            slow_rhs_post(nrk, slow_dt, F_slow, S_old, S_new, S_sum, S_scr);
            apply_bcs(S_new, Vnew, ngc, ngv, false, false);
            tock(3);
        }
        // post_timestep (ERF.cpp:547-559): the new geometry and base state
        // become the old ones
        if (moving) { load_geo(g_new); time += dt; }
        // new state: cons of S_new, velocities from the last post_update
        Sc.copy_from(S_new.cons);
        vel_state.u.copy_from(Vnew.u); vel_state.v.copy_from(Vnew.v); vel_state.w.copy_from(Vnew.w);
        tock(5);
        if (use_moisture) kessler(Sc, dt);
        tock(4);
    }

    // ------------------------------------------------------------------
    // Hydrostatic base state: InputSoundingData::calc_rho_p
    // (DataStructs/ERF_InputSoundingData.H:176-256) with Newton_Raphson_hse
    // (Utils/ERF_HSE_utils.H:34-72) at cell centres, then erf_enforce_hse
    // (Initialization/ERF_init1d.cpp:152-260).
    // ------------------------------------------------------------------
    void make_base_state(const double* th_cc, const double* qv_cc, double th_s, double qv_s, double p_s,
                         double* rho_o, double* p_o, double* pi_o, double* th_o) const {
        const double tol = 1.0e-12;
        std::vector<double> z(nz + 1), th(nz + 1), qv(nz + 1), pm(nz + 1), rd(nz + 1);
        z[0] = 0.; th[0] = th_s; qv[0] = qv_s;
        for (int k = 0; k < nz; ++k) { z[k + 1] = (k + 0.5) * c.dz; th[k + 1] = th_cc[k]; qv[k + 1] = qv_cc[k]; }
        double g = c.gravity;
        pm[0] = p_s;
        rd[0] = getRhogivenThetaPress(th[0], p_s, R_d / Cp_d, qv[0]);
        for (int k = 1; k <= nz; ++k) {
            double dz = z[k] - z[k - 1];
            double rlo = rd[k - 1] * (1. + qv[k - 1]);
            double C = -pm[k - 1] + 0.5 * rlo * g * dz;
            pm[k] = pm[k - 1];
            rd[k] = getRhogivenThetaPress(th[k], pm[k], R_d / Cp_d, qv[k]);
            double rhi = rd[k] * (1. + qv[k]);
            double F = pm[k] + 0.5 * rhi * g * dz + C;
            if (std::abs(F) > tol) {
                int iter = 0;
                double eps = 1.0e-6, ieps = 1.0e6;
                do {
                    double hi = getRhogivenThetaPress(th[k], pm[k] + eps, R_d / Cp_d, qv[k]);
                    double lo = getRhogivenThetaPress(th[k], pm[k] - eps, R_d / Cp_d, qv[k]);
                    double dFdp = 1.0 + 0.25 * ieps * (hi - lo) * g * dz;
                    pm[k] -= F / dFdp;
                    rd[k] = getRhogivenThetaPress(th[k], pm[k], R_d / Cp_d, qv[k]);
                    double rt = rd[k] * (1. + qv[k]);
                    F = pm[k] + 0.5 * rt * g * dz + C;
                    ++iter;
                } while (std::abs(F) > tol && iter < 30);
            }
        }
        // rho0 at cell centres (dry density), ghosts by foextrap
        for (int k = 0; k < nz; ++k) rho_o[k + 1] = rd[k + 1];
        rho_o[0] = rho_o[1]; rho_o[nz + 1] = rho_o[nz];
        // erf_enforce_hse
        double hz = 0.5 * c.dz;
        p_o[1] = p_0 - hz * rho_o[1] * g;
        pi_o[1] = getExnergivenP(p_o[1], rdOcp);
        th_o[1] = getRhoThetagivenP(p_o[1]) / rho_o[1];
        p_o[0] = p_0 + hz * rho_o[1] * g;
        pi_o[0] = getExnergivenP(p_o[0], rdOcp);
        th_o[0] = getRhoThetagivenP(p_o[0]) / rho_o[0];
        for (int k = 1; k <= nz; ++k) {
            int kk = k + 1;  // k == nz is the top ghost cell
            double di = 0.5 * (rho_o[kk] + rho_o[kk - 1]);
            p_o[kk] = p_o[kk - 1] - c.dz * di * g;
            pi_o[kk] = getExnergivenP(p_o[kk], rdOcp);
            th_o[kk] = getRhoThetagivenP(p_o[kk]) / rho_o[kk];
        }
    }
};

// dense valid-region <-> Fab
void load_cc(Fab& f, const double* a, int nx, int ny, int nz, int nc) {
    for (int n = 0; n < nc; ++n)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) f(i, j, k, n) = a[(((size_t)n * nz + k) * ny + j) * nx + i];
}
void store_cc(const Fab& f, double* a, int nx, int ny, int nz, int nc) {
    for (int n = 0; n < nc; ++n)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) a[(((size_t)n * nz + k) * ny + j) * nx + i] = f(i, j, k, n);
}
void load_box(Fab& f, const double* a, int mx, int my, int mz) {
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j)
            for (int i = 0; i < mx; ++i) f(i, j, k) = a[((size_t)k * my + j) * mx + i];
}
void store_box(const Fab& f, double* a, int mx, int my, int mz) {
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j)
            for (int i = 0; i < mx; ++i) a[((size_t)k * my + j) * mx + i] = f(i, j, k);
}

}  // namespace

// ============================================================================
// C entry points for the test harness (ctypes)
// ============================================================================
extern "C" {

int oracle_make_base_state(const erf_b200_config* cfg, const double* th_cc, const double* qv_cc, double th_s,
                           double qv_s, double p_s, double* rho0, double* p0, double* pi0, double* th0) {
    Oracle o(*cfg);
    o.make_base_state(th_cc, qv_cc, th_s, qv_s, p_s, rho0, p0, pi0, th0);
    return 0;
}

// Advance `nsteps` full steps.  base: rho0,p0,pi0,th0 each nz+2.
int oracle_advance(const erf_b200_config* cfg, const double* rho0, const double* p0, const double* pi0,
                   const double* th0, double* cons, double* u, double* v, double* w, int nsteps) {
    std::unique_ptr<Oracle> o(new Oracle(*cfg));
    int nz = cfg->nz, nx = cfg->nx, ny = cfg->ny;
    for (int k = 0; k < nz + 2; ++k) { o->r0[k] = rho0[k]; o->p0[k] = p0[k]; o->pi0[k] = pi0[k]; o->th0[k] = th0[k]; }
    o->init_storage();
    o->alloc(o->cons_state, CC, o->ngc, o->ncomp);
    o->alloc_vel(o->vel_state);
    load_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    load_box(o->vel_state.u, u, nx + 1, ny, nz);
    load_box(o->vel_state.v, v, nx, ny + 1, nz);
    load_box(o->vel_state.w, w, nx, ny, nz + 1);
    for (int s = 0; s < nsteps; ++s) o->step(cfg->dt);
    store_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    store_box(o->vel_state.u, u, nx + 1, ny, nz);
    store_box(o->vel_state.v, v, nx, ny + 1, nz);
    store_box(o->vel_state.w, w, nx, ny, nz + 1);
    return 0;
}

// oracle_advance with the wall seconds of each pass summed into pass_s[6]
// (closure, slow_rhs_pre, fast, slow_rhs_post, Kessler, rest).
int oracle_advance_timed(const erf_b200_config* cfg, const double* rho0, const double* p0, const double* pi0,
                         const double* th0, double* cons, double* u, double* v, double* w, int nsteps,
                         double* pass_s) {
    std::unique_ptr<Oracle> o(new Oracle(*cfg));
    int nz = cfg->nz, nx = cfg->nx, ny = cfg->ny;
    for (int k = 0; k < nz + 2; ++k) { o->r0[k] = rho0[k]; o->p0[k] = p0[k]; o->pi0[k] = pi0[k]; o->th0[k] = th0[k]; }
    o->init_storage();
    o->alloc(o->cons_state, CC, o->ngc, o->ncomp);
    o->alloc_vel(o->vel_state);
    load_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    load_box(o->vel_state.u, u, nx + 1, ny, nz);
    load_box(o->vel_state.v, v, nx, ny + 1, nz);
    load_box(o->vel_state.w, w, nx, ny, nz + 1);
    for (int s = 0; s < nsteps; ++s) o->step(cfg->dt);
    store_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    store_box(o->vel_state.u, u, nx + 1, ny, nz);
    store_box(o->vel_state.v, v, nx, ny + 1, nz);
    store_box(o->vel_state.w, w, nx, ny, nz + 1);
    for (int q = 0; q < 6; ++q) pass_s[q] = o->pass_s[q];
    return 0;
}

// Base state over terrain.  z_nd: valid nodes (nz+1)(ny+1)(nx+1); th3/qv3:
// nz*ny*nx cell values; outputs (nz+2)*ny*nx, plane k+1 for level k.
int oracle_make_base_state_terrain(const erf_b200_config* cfg, const double* z_nd, const double* th3,
                                   const double* qv3, double th_s, double qv_s, double p_s, double* rho0,
                                   double* p0, double* pi0, double* th0) {
    Oracle o(*cfg);
    o.set_terrain(z_nd);
    o.make_base_state_terrain(th3, qv3, th_s, qv_s, p_s, rho0, p0, pi0, th0);
    return 0;
}

// Metrics of a terrain grid: detJ and z_cc (nz*ny*nx), ax ((nz)(ny)(nx+1)),
// ay ((nz)(ny+1)(nx)), valid region, i fastest.
int oracle_terrain_metrics(const erf_b200_config* cfg, const double* z_nd, double* detJ, double* zcc, double* ax,
                           double* ay) {
    Oracle o(*cfg);
    o.set_terrain(z_nd);
    int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t c = ((size_t)k * ny + j) * nx + i;
                detJ[c] = o.detJ(i, j, k); zcc[c] = o.zcc(i, j, k);
            }
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i) ax[((size_t)k * ny + j) * (nx + 1) + i] = o.axA(i, j, k);
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i < nx; ++i) ay[((size_t)k * (ny + 1) + j) * nx + i] = o.ayA(i, j, k);
    return 0;
}

// Advance over terrain: base state in the (nz+2)-plane layout.
int oracle_advance_terrain(const erf_b200_config* cfg, const double* z_nd, const double* rho0, const double* p0,
                           const double* pi0, const double* th0, double* cons, double* u, double* v, double* w,
                           int nsteps) {
    std::unique_ptr<Oracle> o(new Oracle(*cfg));
    int nz = cfg->nz, nx = cfg->nx, ny = cfg->ny;
    o->set_terrain(z_nd);
    o->set_base_terrain(rho0, p0, pi0, th0);
    o->init_storage();
    o->alloc(o->cons_state, CC, o->ngc, o->ncomp);
    o->alloc_vel(o->vel_state);
    load_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    load_box(o->vel_state.u, u, nx + 1, ny, nz);
    load_box(o->vel_state.v, v, nx, ny + 1, nz);
    load_box(o->vel_state.w, w, nx, ny, nz + 1);
    for (int s = 0; s < nsteps; ++s) o->step(cfg->dt);
    store_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    store_box(o->vel_state.u, u, nx + 1, ny, nz);
    store_box(o->vel_state.v, v, nx, ny + 1, nz);
    store_box(o->vel_state.w, w, nx, ny, nz + 1);
    return 0;
}

// Moving terrain (with or without acoustic substepping): the grid is generated from
// cfg's surface wave at time0 and at every geometry time after it; rho0 ..
// th0 are the initial base state ((nz+2) planes of ny*nx).  On return
// z_nd ((nz+1)(ny+1)(nx+1) valid nodes) holds the grid at the final time and
// rho0_out / p0_out ((nz+2) planes) the evolved base state.
int oracle_advance_moving_terrain(const erf_b200_config* cfg, double time0, const double* rho0, const double* p0,
                                  const double* pi0, const double* th0, double* cons, double* u, double* v,
                                  double* w, int nsteps, double* z_nd, double* rho0_out, double* p0_out) {
    if (!cfg->use_terrain || cfg->terrain_type != ERF_TERRAIN_MOVING) return 1;
    std::unique_ptr<Oracle> o(new Oracle(*cfg));
    int nz = cfg->nz, nx = cfg->nx, ny = cfg->ny;
    o->terrain = true;
    o->moving = true;
    o->time = time0;
    o->mt_grid(time0);
    o->set_base_terrain(rho0, p0, pi0, th0);
    o->init_storage();
    o->alloc(o->cons_state, CC, o->ngc, o->ncomp);
    o->alloc_vel(o->vel_state);
    load_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    load_box(o->vel_state.u, u, nx + 1, ny, nz);
    load_box(o->vel_state.v, v, nx, ny + 1, nz);
    load_box(o->vel_state.w, w, nx, ny, nz + 1);
    for (int s = 0; s < nsteps; ++s) o->step(cfg->dt);
    store_cc(o->cons_state, cons, nx, ny, nz, o->ncomp);
    store_box(o->vel_state.u, u, nx + 1, ny, nz);
    store_box(o->vel_state.v, v, nx, ny + 1, nz);
    store_box(o->vel_state.w, w, nx, ny, nz + 1);
    if (z_nd)
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx; ++i) z_nd[((size_t)k * (ny + 1) + j) * (nx + 1) + i] = o->znd(i, j, k);
    for (int k = -1; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t q = (size_t)(k + 1) * nx * ny + (size_t)j * nx + i;
                if (rho0_out) rho0_out[q] = o->r0f(i, j, k);
                if (p0_out) p0_out[q] = o->p0f(i, j, k);
            }
    return 0;
}

// Kessler alone on a dense valid-region state (cons[ncomp][nz][ny][nx]), as
// ERF::advance_microphysics runs it after the dycore (ERF_Advance.cpp:174 ->
// Kessler::Copy_State_to_Micro, AdvanceKessler, Copy_Micro_to_State).
int oracle_kessler(const erf_b200_config* cfg, double* cons, double dt) {
    if (cfg->moisture != ERF_MOIST_KESSLER && cfg->moisture != ERF_MOIST_KESSLER_NORAIN) return 1;
    std::unique_ptr<Oracle> o(new Oracle(*cfg));
    int nz = cfg->nz, nx = cfg->nx, ny = cfg->ny;
    Fab f;
    o->alloc(f, CC, o->ngc, o->ncomp);
    load_cc(f, cons, nx, ny, nz, o->ncomp);
    o->kessler(f, dt);
    store_cc(f, cons, nx, ny, nz, o->ncomp);
    return 0;
}

// Kessler alone over a terrain grid (z_nd: valid nodes): the sedimentation
// divergence over detJ (ERF_Kessler.cpp:82-97).
int oracle_kessler_terrain(const erf_b200_config* cfg, const double* z_nd, double* cons, double dt) {
    if (cfg->moisture != ERF_MOIST_KESSLER && cfg->moisture != ERF_MOIST_KESSLER_NORAIN) return 1;
    std::unique_ptr<Oracle> o(new Oracle(*cfg));
    o->set_terrain(z_nd);
    int nz = cfg->nz, nx = cfg->nx, ny = cfg->ny;
    Fab f;
    o->alloc(f, CC, o->ngc, o->ncomp);
    load_cc(f, cons, nx, ny, nz, o->ncomp);
    o->kessler(f, dt);
    store_cc(f, cons, nx, ny, nz, o->ncomp);
    return 0;
}

// ----------------------------------------------------------------------------
// Operator hooks: single operators of the restatement on caller arrays, for
// the tests that pin them to the reference's own operator code
// (oracle/ref).  Arrays are the valid box of their index type grown by a
// ghost width g, i fastest, components slowest (a Fab's storage).
// ----------------------------------------------------------------------------
static void fab_in(Fab& f, const double* a) { std::copy(a, a + f.d.size(), f.d.begin()); }
static void fab_out(const Fab& f, double* a) { std::copy(f.d.begin(), f.d.end(), a); }
static void fab_sub_in(Fab& f, const double* a, const int l[3], const int h[3], int nc) {
    // copy a smaller box [l, h] x nc (i fastest) into f
    long sx = h[0] - l[0] + 1, sy = h[1] - l[1] + 1, sz = h[2] - l[2] + 1;
    for (int n = 0; n < nc; ++n)
        for (int k = l[2]; k <= h[2]; ++k)
            for (int j = l[1]; j <= h[1]; ++j)
                for (int i = l[0]; i <= h[0]; ++i)
                    f(i, j, k, n) = a[(i - l[0]) + (j - l[1]) * sx + (k - l[2]) * sx * sy + n * sx * sy * sz];
}
static void fab_sub_out(const Fab& f, double* a, const int l[3], const int h[3], int nc) {
    long sx = h[0] - l[0] + 1, sy = h[1] - l[1] + 1, sz = h[2] - l[2] + 1;
    for (int n = 0; n < nc; ++n)
        for (int k = l[2]; k <= h[2]; ++k)
            for (int j = l[1]; j <= h[1]; ++j)
                for (int i = l[0]; i <= h[0]; ++i)
                    a[(i - l[0]) + (j - l[1]) * sx + (k - l[2]) * sx * sy + n * sx * sy * sz] = f(i, j, k, n);
}

// AdvectionSrcForScalars of comps icomp..icomp+ncomp-1: avg momenta on faces
// (g = 0), primitives (nprim comps, g = 3), rhs (ncons comps, g = 0).
int oracle_op_advect_scalars(const erf_b200_config* cfg, int icomp, int ncomp, int htype, int vtype, double hfrac,
                             double vfrac, const double* avx, const double* avy, const double* avz,
                             const double* prim, int nprim, double* rhs, int ncons) {
    Oracle o(*cfg);
    Fab ax, ay, az, pr, r;
    o.alloc(ax, XF, 0, 1); o.alloc(ay, YF, 0, 1); o.alloc(az, ZF, 0, 1);
    o.alloc(pr, CC, 3, nprim); o.alloc(r, CC, 0, ncons);
    fab_in(ax, avx); fab_in(ay, avy); fab_in(az, avz); fab_in(pr, prim); fab_in(r, rhs);
    o.advect_scalars(icomp, ncomp, ax, ay, az, pr, r, htype, vtype, hfrac, vfrac);
    fab_out(r, rhs);
    return 0;
}

// Strain of advance_dycore's prologue on its boxes: velocities with g = 2;
// outputs on the cell box grown by one (s11, s22, s33) and the same extent
// nodal in x, y and z (s12, s13, s23), i.e. (nx+2)(ny+2)(nz+2) and
// (nx+3)(ny+3)(nz+3) values from index -1.
int oracle_op_strain(const erf_b200_config* cfg, const double* u, const double* v, const double* w, double* s11,
                     double* s22, double* s33, double* s12, double* s13, double* s23) {
    Oracle o(*cfg);
    int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    Fab U, V, W;
    o.alloc(U, XF, 2, 1); o.alloc(V, YF, 2, 1); o.alloc(W, ZF, 2, 1);
    fab_in(U, u); fab_in(V, v); fab_in(W, w);
    int lc[3] = {-1, -1, -1}, hc[3] = {nx, ny, nz}, he[3] = {nx + 1, ny + 1, nz + 1};
    Fab a11(lc, hc, 1), a22(lc, hc, 1), a33(lc, hc, 1), a12(lc, he, 1), a13(lc, he, 1), a23(lc, he, 1);
    Bx bxcc = Oracle::grow(o.valid(CC), 1, 1, 0);
    Bx txy = Oracle::grow(Bx{{0, 0, 0}, {nx, ny, nz - 1}}, 1, 1, 0);
    Bx txz = Oracle::grow(Bx{{0, 0, 0}, {nx, ny - 1, nz}}, 1, 1, 0);
    Bx tyz = Oracle::grow(Bx{{0, 0, 0}, {nx - 1, ny, nz}}, 1, 1, 0);
    o.compute_strain(bxcc, txy, txz, tyz, U, V, W, a11, a22, a33, a12, a13, a23);
    fab_out(a11, s11); fab_out(a22, s22); fab_out(a33, s33); fab_out(a12, s12); fab_out(a13, s13); fab_out(a23, s23);
    return 0;
}

// The terrain strain on the same boxes (z_nd: valid nodes, the oracle adds
// its ghost nodes); also returns the ghosted node heights (nodes -3..n+3
// laterally, -1..nz+1 vertically) and detJ (cells -2..n+1 laterally,
// -1..nz vertically) the oracle derived, for the reference run.
int oracle_op_strain_T(const erf_b200_config* cfg, const double* z_valid, const double* u, const double* v,
                       const double* w, double* z_g1, double* detJ_g1, double* s11, double* s22, double* s33,
                       double* s12, double* s13, double* s21, double* s23, double* s31, double* s32) {
    Oracle o(*cfg);
    int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    o.set_terrain(z_valid);
    Fab U, V, W;
    o.alloc(U, XF, 2, 1); o.alloc(V, YF, 2, 1); o.alloc(W, ZF, 2, 1);
    fab_in(U, u); fab_in(V, v); fab_in(W, w);
    int lc[3] = {-1, -1, -1}, hc[3] = {nx, ny, nz}, he[3] = {nx + 1, ny + 1, nz + 1};
    Fab a11(lc, hc, 1), a22(lc, hc, 1), a33(lc, hc, 1), a12(lc, he, 1), a13(lc, he, 1), a21(lc, he, 1), a23(lc, he, 1),
        a31(lc, he, 1), a32(lc, he, 1);
    Bx bxcc = Oracle::grow(o.valid(CC), 1, 1, 0);
    Bx txy = Oracle::grow(Bx{{0, 0, 0}, {nx, ny, nz - 1}}, 1, 1, 0);
    Bx txz = Oracle::grow(Bx{{0, 0, 0}, {nx, ny - 1, nz}}, 1, 1, 0);
    Bx tyz = Oracle::grow(Bx{{0, 0, 0}, {nx - 1, ny, nz}}, 1, 1, 0);
    o.compute_strain_T(bxcc, txy, txz, tyz, U, V, W, a11, a22, a33, a12, a13, a21, a23, a31, a32);
    fab_out(a11, s11); fab_out(a22, s22); fab_out(a33, s33); fab_out(a12, s12); fab_out(a13, s13); fab_out(a21, s21);
    fab_out(a23, s23); fab_out(a31, s31); fab_out(a32, s32);
    fab_out(o.znd, z_g1);      // nodes -3..n+3 laterally, -1..nz+1 vertically
    fab_out(o.detJ, detJ_g1);  // cells -2..n+1 laterally, -1..nz vertically
    return 0;
}

// Eddy viscosity of the step prologue (Smagorinsky or Deardorff by
// cfg->les_type): velocities g = 2, cons (ncomp) g = 1; outputs g = 1:
// mu_t, the Deardorff vertical heat diffusivity and the dissipation.
int oracle_op_eddy_viscosity(const erf_b200_config* cfg, const double* u, const double* v, const double* w,
                             const double* cons, double* mut_out, double* kthv_out, double* diss_out) {
    Oracle o(*cfg);
    int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    o.init_storage();
    Oracle::Vel V;
    o.alloc_vel(V);
    int lx[3] = {-2, -2, -2}, hx[3] = {nx + 2, ny + 1, nz + 1};
    int ly[3] = {-2, -2, -2}, hy[3] = {nx + 1, ny + 2, nz + 1};
    int lz[3] = {-2, -2, -2}, hz[3] = {nx + 1, ny + 1, nz + 2};
    fab_sub_in(V.u, u, lx, hx, 1); fab_sub_in(V.v, v, ly, hy, 1); fab_sub_in(V.w, w, lz, hz, 1);
    Fab C;
    o.alloc(C, CC, o.ngc, o.ncomp);
    int lc[3] = {-1, -1, -1}, hc[3] = {nx, ny, nz};
    fab_sub_in(C, cons, lc, hc, o.ncomp);
    o.turbulent_viscosity(V, C, o.mut);
    fab_sub_out(o.mut, mut_out, lc, hc, 1);
    fab_sub_out(o.kthv, kthv_out, lc, hc, 1);
    fab_sub_out(o.diss, diss_out, lc, hc, 1);
    return 0;
}

// Momentum advection without terrain (AdvectionSrcForMom): momenta and
// velocities as faces with g = 3; rhs outputs as faces with g = 0 (z-faces
// written for k = 1..nz-1).
int oracle_op_advect_mom(const erf_b200_config* cfg, const double* ru, const double* rv, const double* rw,
                         const double* u, const double* v, const double* w, double* rx, double* ry, double* rz) {
    Oracle o(*cfg);
    Oracle::State S, R;
    Oracle::Vel V;
    o.alloc(S.cons, CC, 1, o.ncomp);
    o.alloc(S.mx, XF, 3, 1); o.alloc(S.my, YF, 3, 1); o.alloc(S.mz, ZF, 3, 1);
    o.alloc(V.u, XF, 3, 1); o.alloc(V.v, YF, 3, 1); o.alloc(V.w, ZF, 3, 1);
    o.alloc(R.mx, XF, 0, 1); o.alloc(R.my, YF, 0, 1); o.alloc(R.mz, ZF, 0, 1);
    fab_in(S.mx, ru); fab_in(S.my, rv); fab_in(S.mz, rw); fab_in(V.u, u); fab_in(V.v, v); fab_in(V.w, w);
    o.advect_mom_N(R, S, V);
    fab_out(R.mx, rx); fab_out(R.my, ry); fab_out(R.mz, rz);
    return 0;
}

// Interpolant known-answer hook: evaluates one face interpolant.
double oracle_interp(int type, const double* s6, double upw, double frac) { return Oracle::interp(type, s6, upw, frac); }

// Saturation mixing ratio over water (hPa input), for known-answer tests.
double oracle_qsatw(double t, double p_hpa) { return qsatw(t, p_hpa); }

}  // extern "C"
