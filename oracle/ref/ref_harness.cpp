// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points that run the reference's own hot-path leaf operators
// (compiled unmodified from ERF's Source/ tree against the single-box AMReX
// stand-in in shim/) on caller-supplied arrays, so the tests can pin the
// oracle's restatement of each operator to the reference's code:
//
//   ref_interp            UPWIND3/5, CENTERED2/4/6, WENO3/5 face interpolants
//                         (Utils/ERF_Interpolation_UPW.H, _WENO.H)
//   ref_advect_scalars    AdvectionSrcForScalars (Advection/ERF_AdvectionSrcForState.cpp:119-395)
//   ref_strain_N          ComputeStrain_N (Diffusion/ERF_ComputeStrain_N.cpp:28-229)
//   ref_strain_T          ComputeStrain_T (Diffusion/ERF_ComputeStrain_T.cpp)
//   ref_eddy_viscosity    ComputeStrain_N on advance_dycore's boxes + ComputeTurbulentViscosity
//                         (Smagorinsky / Deardorff; ERF_advance_dycore.cpp:114-223,
//                         Diffusion/ERF_ComputeTurbulentViscosity.cpp:32-521)
//   ref_kessler           Kessler::Init / Copy_State_to_Micro / AdvanceKessler /
//                         Copy_Micro_to_State (Microphysics/Kessler/*)
//   ref_qsatw             erf_qsatw (Utils/ERF_Microphysics_Utils.H)
//
// Arrays follow one convention on both sides (oracle hooks and this file):
// the valid box of the array's index type (cell, x-, y- or z-face; faces are
// nodal in their direction) grown by a ghost width g on every side, i
// fastest, components slowest.
#include <AMReX_MultiFab.H>

#include "ERF_Advection.H"
#include "ERF_Diffusion.H"
#include "ERF_EddyViscosity.H"
#include "ERF_EOS.H"
#include "ERF_Interpolation.H"
#include "ERF_Kessler.H"
#include "ERF_Microphysics_Utils.H"

using namespace amrex;

namespace {

// valid box of index type t (0 cell, 1 x-face, 2 y-face, 3 z-face)
Box vbox(int nx, int ny, int nz, int t) {
    Box b(IntVect(0, 0, 0), IntVect(nx - 1, ny - 1, nz - 1));
    if (t >= 1) b.surroundingNodes(t - 1);
    return b;
}
template <class T>
Array4<T> view(T* p, Box b, int nc) {
    return Array4<T>(p, b.lo.dim3(), (b.hi + 1).dim3(), nc);
}
Array4<const Real> cview(const double* p, int nx, int ny, int nz, int t, int g, int nc) {
    return view<const Real>(p, grow(vbox(nx, ny, nz, t), g), nc);
}
Array4<Real> mview(double* p, int nx, int ny, int nz, int t, int g, int nc) {
    return view<Real>(p, grow(vbox(nx, ny, nz, t), g), nc);
}
// boundary records: periodic laterally, walls below / above
std::vector<BCRec> wall_bcs(int zlo_noslip, int zhi_noslip) {
    std::vector<BCRec> bcs(BCVars::NumTypes);
    for (auto& b : bcs) {
        for (int d = 0; d < 2; ++d) { b.setLo(d, ERFBCType::int_dir); b.setHi(d, ERFBCType::int_dir); }
        b.setLo(2, ERFBCType::foextrap);
        b.setHi(2, ERFBCType::foextrap);
    }
    bcs[BCVars::xvel_bc].setLo(2, zlo_noslip ? ERFBCType::ext_dir : ERFBCType::foextrap);
    bcs[BCVars::yvel_bc].setLo(2, zlo_noslip ? ERFBCType::ext_dir : ERFBCType::foextrap);
    bcs[BCVars::xvel_bc].setHi(2, zhi_noslip ? ERFBCType::ext_dir : ERFBCType::foextrap);
    bcs[BCVars::yvel_bc].setHi(2, zhi_noslip ? ERFBCType::ext_dir : ERFBCType::foextrap);
    bcs[BCVars::zvel_bc].setLo(2, ERFBCType::ext_dir);
    bcs[BCVars::zvel_bc].setHi(2, ERFBCType::ext_dir);
    return bcs;
}
void set_domain(int nx, int ny, int nz) {
    ShimDomain::domain = vbox(nx, ny, nz, 0);
    ShimDomain::periodic[0] = ShimDomain::periodic[1] = 1;
    ShimDomain::periodic[2] = 0;
}
Geometry geometry(int nx, int ny, int nz, double dx, double dy, double dz) {
    Geometry g;
    g.g.domain = vbox(nx, ny, nz, 0);
    g.g.dx[0] = dx; g.g.dx[1] = dy; g.g.dx[2] = dz;
    g.g.is_periodic[0] = g.g.is_periodic[1] = 1;
    return g;
}
// a one-box MultiFab of index type t with ghost g, filled from / copied to a flat array
MultiFab make_mf(int nx, int ny, int nz, int t, int g, int nc, const double* src = nullptr) {
    MultiFab m(BoxArray(vbox(nx, ny, nz, t)), DistributionMapping(), nc, g);
    if (src) std::copy(src, src + m.fab.bx.numPts() * nc, m.fab.p);
    return m;
}

}  // namespace

extern "C" {

// One face value from a 6-point stencil s6 = phi at offsets -3..+2 from the
// face's high-side cell, through the reference's interpolant struct.
double ref_interp(int type, const double* s6, double upw, double frac) {
    Real buf[6];
    for (int q = 0; q < 6; ++q) buf[q] = s6[q];
    Array4<const Real> a(buf, Dim3{-3, 0, 0}, Dim3{3, 1, 1}, 1);
    Real v = 0.0;
    switch (type) {
    case 101: CENTERED2(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    case 102: UPWIND3(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    case 103: CENTERED4(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    case 104: UPWIND5(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    case 105: CENTERED6(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    case 106: WENO3(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    case 108: WENO5(a).InterpolateInX(0, 0, 0, 0, v, upw, frac); break;
    default: return std::nan("");
    }
    return v;
}

// AdvectionSrcForScalars on the valid box: avg momenta on faces (g = 0),
// primitives (nprim comps, g = 3), rhs (ncons comps, g = 0; comps
// icomp..icomp+ncomp-1 are written).
int ref_advect_scalars(int nx, int ny, int nz, double dx, double dy, double dz, int icomp, int ncomp, int htype,
                       int vtype, double hfrac, double vfrac, const double* avx, const double* avy, const double* avz,
                       const double* prim, int nprim, double* rhs, int ncons) {
    set_domain(nx, ny, nz);
    Box bx = vbox(nx, ny, nz, 0);
    auto ax = cview(avx, nx, ny, nz, 1, 0, 1), ay = cview(avy, nx, ny, nz, 2, 0, 1), az = cview(avz, nx, ny, nz, 3, 0, 1);
    auto pr = cview(prim, nx, ny, nz, 0, 3, nprim);
    auto r = mview(rhs, nx, ny, nz, 0, 0, ncons);
    std::vector<Real> ones((size_t)nx * ny * nz, 1.0), cons((size_t)nx * ny * nz * ncons, 0.0);
    auto detJ = cview(ones.data(), nx, ny, nz, 0, 0, 1);
    auto mf = view<const Real>(ones.data(), Box(IntVect(0, 0, 0), IntVect(nx - 1, ny - 1, 0)), 1);
    auto cur = cview(cons.data(), nx, ny, nz, 0, 0, ncons);
    std::vector<Real> fx((size_t)(nx + 1) * ny * nz * ncons), fy((size_t)nx * (ny + 1) * nz * ncons),
        fz((size_t)nx * ny * (nz + 1) * ncons);
    GpuArray<const Array4<Real>, 3> flx{{mview(fx.data(), nx, ny, nz, 1, 0, ncons), mview(fy.data(), nx, ny, nz, 2, 0, ncons),
                                         mview(fz.data(), nx, ny, nz, 3, 0, ncons)}};
    GpuArray<Array4<Real>, 3> tmp{{Array4<Real>(), Array4<Real>(), Array4<Real>()}};
    GpuArray<Real, 3> dxi{{1.0 / dx, 1.0 / dy, 1.0 / dz}};
    auto bcs = wall_bcs(0, 0);
    AdvectionSrcForScalars(0.0, bx, icomp, ncomp, ax, ay, az, cur, pr, r, false, nullptr, nullptr, detJ, dxi, mf,
                           AdvType(htype), AdvType(vtype), hfrac, vfrac, flx, tmp, bx, bcs.data());
    return 0;
}

// AdvectionSrcForMom without terrain on erf_slow_rhs_pre's boxes (x/y faces;
// interior z faces): momenta and velocities with g = 3, rhs with g = 0.
int ref_advect_mom(int nx, int ny, int nz, double dx, double dy, double dz, int htype, int vtype, double hfrac,
                   double vfrac, const double* ru, const double* rv, const double* rw, const double* u,
                   const double* v, const double* w, double* rx, double* ry, double* rz) {
    set_domain(nx, ny, nz);
    Box bx = vbox(nx, ny, nz, 0);
    Box bxx = vbox(nx, ny, nz, 1), bxy = vbox(nx, ny, nz, 2), bxz = vbox(nx, ny, nz, 3);
    bxz.growLo(2, -1);
    bxz.growHi(2, -1);
    auto RU = cview(ru, nx, ny, nz, 1, 3, 1), RV = cview(rv, nx, ny, nz, 2, 3, 1), RW = cview(rw, nx, ny, nz, 3, 3, 1);
    auto U = cview(u, nx, ny, nz, 1, 3, 1), V = cview(v, nx, ny, nz, 2, 3, 1), W = cview(w, nx, ny, nz, 3, 3, 1);
    auto X = mview(rx, nx, ny, nz, 1, 0, 1), Y = mview(ry, nx, ny, nz, 2, 0, 1), Z = mview(rz, nx, ny, nz, 3, 0, 1);
    Box big = grow(convert(vbox(nx, ny, nz, 0), IntVect(1, 1, 1)), 4);
    std::vector<Real> ones((size_t)big.numPts(), 1.0);
    auto one3 = view<const Real>(ones.data(), big, 1);
    auto mf = view<const Real>(ones.data(), Box(IntVect(-4, -4, 0), IntVect(nx + 4, ny + 4, 0)), 1);
    std::vector<Real> cons((size_t)grow(bx, 1).numPts(), 1.0);
    auto cd = view<const Real>(cons.data(), grow(bx, 1), 1);
    GpuArray<Real, 3> dxi{{1.0 / dx, 1.0 / dy, 1.0 / dz}};
    auto bcs = wall_bcs(0, 0);
    AdvectionSrcForMom(bx, bxx, bxy, bxz, X, Y, Z, cd, U, V, W, RU, RV, RW, one3, one3, one3, one3, one3, dxi, mf, mf,
                       mf, AdvType(htype), AdvType(vtype), hfrac, vfrac, false, 0, nz, bx, bcs.data());
    return 0;
}

// ComputeStrain_N over the boxes advance_dycore uses (cells and edges grown by
// one laterally): velocities with g = 2, outputs on the cell box grown by one
// in every direction (tau11/22/33 as cells, tau12/13/23 as the same box
// extent nodal in their two directions).
int ref_strain_N(int nx, int ny, int nz, double dx, double dy, double dz, int zlo_noslip, int zhi_noslip,
                 const double* u, const double* v, const double* w, double* t11, double* t22, double* t33,
                 double* t12, double* t13, double* t23) {
    set_domain(nx, ny, nz);
    Box dom = vbox(nx, ny, nz, 0);
    Box bxcc = grow(dom, IntVect(1, 1, 0));
    Box txy = grow(convert(dom, IntVect(1, 1, 0)), IntVect(1, 1, 0));
    Box txz = grow(convert(dom, IntVect(1, 0, 1)), IntVect(1, 1, 0));
    Box tyz = grow(convert(dom, IntVect(0, 1, 1)), IntVect(1, 1, 0));
    auto U = cview(u, nx, ny, nz, 1, 2, 1), V = cview(v, nx, ny, nz, 2, 2, 1), W = cview(w, nx, ny, nz, 3, 2, 1);
    Box out = grow(dom, 1);
    Box oe(out.lo, out.hi + 1);   // common extent of the edge outputs
    auto a11 = view<Real>(t11, out, 1), a22 = view<Real>(t22, out, 1), a33 = view<Real>(t33, out, 1);
    auto a12 = view<Real>(t12, oe, 1), a13 = view<Real>(t13, oe, 1), a23 = view<Real>(t23, oe, 1);
    std::vector<Real> ones((size_t)(nx + 8) * (ny + 8), 1.0);
    auto mf = view<const Real>(ones.data(), Box(IntVect(-4, -4, 0), IntVect(nx + 3, ny + 3, 0)), 1);
    GpuArray<Real, 3> dxi{{1.0 / dx, 1.0 / dy, 1.0 / dz}};
    auto bcs = wall_bcs(zlo_noslip, zhi_noslip);
    ComputeStrain_N(bxcc, txy, txz, tyz, dom, U, V, W, a11, a22, a33, a12, a13, a23, bcs.data(), dxi, mf, mf, mf);
    return 0;
}

// ComputeStrain_T on the same boxes, with z_phys_nd (nodes -3..n+3
// laterally, -1..nz+1 vertically) and detJ (cells -2..n+1 laterally,
// -1..nz vertically); tau21, tau31 and tau32 are returned beside the others.
int ref_strain_T(int nx, int ny, int nz, double dx, double dy, double dz, int zlo_noslip, int zhi_noslip,
                 const double* u, const double* v, const double* w, const double* z_nd, const double* detJ,
                 double* t11, double* t22, double* t33, double* t12, double* t13, double* t21, double* t23,
                 double* t31, double* t32) {
    set_domain(nx, ny, nz);
    Box dom = vbox(nx, ny, nz, 0);
    Box bxcc = grow(dom, IntVect(1, 1, 0));
    Box txy = grow(convert(dom, IntVect(1, 1, 0)), IntVect(1, 1, 0));
    Box txz = grow(convert(dom, IntVect(1, 0, 1)), IntVect(1, 1, 0));
    Box tyz = grow(convert(dom, IntVect(0, 1, 1)), IntVect(1, 1, 0));
    auto U = cview(u, nx, ny, nz, 1, 2, 1), V = cview(v, nx, ny, nz, 2, 2, 1), W = cview(w, nx, ny, nz, 3, 2, 1);
    Box nodes = grow(convert(dom, IntVect(1, 1, 1)), IntVect(3, 3, 1));
    auto Z = view<const Real>(z_nd, nodes, 1);
    auto J = view<const Real>(detJ, Box(IntVect(-2, -2, -1), IntVect(nx + 1, ny + 1, nz)), 1);
    Box out = grow(dom, 1);
    Box oe(out.lo, out.hi + 1);
    auto a11 = view<Real>(t11, out, 1), a22 = view<Real>(t22, out, 1), a33 = view<Real>(t33, out, 1);
    auto a12 = view<Real>(t12, oe, 1), a13 = view<Real>(t13, oe, 1), a21 = view<Real>(t21, oe, 1);
    auto a23 = view<Real>(t23, oe, 1), a31 = view<Real>(t31, oe, 1), a32 = view<Real>(t32, oe, 1);
    std::vector<Real> ones((size_t)(nx + 8) * (ny + 8), 1.0);
    auto mf = view<const Real>(ones.data(), Box(IntVect(-4, -4, 0), IntVect(nx + 3, ny + 3, 0)), 1);
    GpuArray<Real, 3> dxi{{1.0 / dx, 1.0 / dy, 1.0 / dz}};
    auto bcs = wall_bcs(zlo_noslip, zhi_noslip);
    ComputeStrain_T(bxcc, txy, txz, tyz, dom, U, V, W, a11, a22, a33, a12, a13, a21, a23, a31, a32, Z, J, bcs.data(),
                    dxi, mf, mf, mf);
    return 0;
}

// Eddy viscosity of advance_dycore (ERF_advance_dycore.cpp:114-223): the
// strain of the old velocities (g = 2) on advance_dycore's boxes, then
// ComputeTurbulentViscosity with les_type 1 (Smagorinsky: Cs) or 2
// (Deardorff: Ck, Ce, Ce_wall, theta_ref, sigma_k).  cons: ncons comps, g = 1.
// Outputs (cells, g = 1): the EddyDiff components Mom_h, Theta_v and the
// dissipation (Deardorff).
int ref_eddy_viscosity(int nx, int ny, int nz, double dx, double dy, double dz, int zlo_noslip, int zhi_noslip,
                       int les, double Cs, double Pr_t, double Sc_t, double Ck, double Ce, double Ce_wall,
                       double theta_ref, double sigma_k, double gravity, const double* u, const double* v,
                       const double* w, const double* cons, int ncons, double* mut, double* kthv, double* diss) {
    set_domain(nx, ny, nz);
    Box dom = vbox(nx, ny, nz, 0);
    MultiFab xv = make_mf(nx, ny, nz, 1, 2, 1, u), yv = make_mf(nx, ny, nz, 2, 2, 1, v), zv = make_mf(nx, ny, nz, 3, 2, 1, w);
    MultiFab T11 = make_mf(nx, ny, nz, 0, 1, 1), T22 = make_mf(nx, ny, nz, 0, 1, 1), T33 = make_mf(nx, ny, nz, 0, 1, 1);
    MultiFab T12(BoxArray(convert(dom, IntVect(1, 1, 0))), DistributionMapping(), 1, 1);
    MultiFab T13(BoxArray(convert(dom, IntVect(1, 0, 1))), DistributionMapping(), 1, 1);
    MultiFab T23(BoxArray(convert(dom, IntVect(0, 1, 1))), DistributionMapping(), 1, 1);
    MultiFab C = make_mf(nx, ny, nz, 0, 1, ncons, cons);
    MultiFab eddy = make_mf(nx, ny, nz, 0, 1, EddyDiff::NumDiffs);
    MultiFab H1 = make_mf(nx, ny, nz, 0, 0, 1), H2 = make_mf(nx, ny, nz, 0, 0, 1), H3 = make_mf(nx, ny, nz, 0, 0, 1);
    MultiFab D = make_mf(nx, ny, nz, 0, 1, 1);   // the dissipation, valid cells written
    MultiFab mfu = make_mf(nx, ny, nz, 1, 3, 1), mfv = make_mf(nx, ny, nz, 2, 3, 1);
    mfu.setVal(1.0); mfv.setVal(1.0);
    std::vector<Real> ones((size_t)(nx + 8) * (ny + 8), 1.0);
    auto mf = view<const Real>(ones.data(), Box(IntVect(-4, -4, 0), IntVect(nx + 3, ny + 3, 0)), 1);
    GpuArray<Real, 3> dxi{{1.0 / dx, 1.0 / dy, 1.0 / dz}};
    auto bcs = wall_bcs(zlo_noslip, zhi_noslip);
    if (les == 1) {
        // strain only for the Smagorinsky closure (the Deardorff length scale
        // reads the state; advance_dycore forms the strain with any diffusion)
        MFIter mfi(C);
        Box bxcc = grow(dom, IntVect(1, 1, 0));
        Box txy = grow(convert(dom, IntVect(1, 1, 0)), IntVect(1, 1, 0));
        Box txz = grow(convert(dom, IntVect(1, 0, 1)), IntVect(1, 1, 0));
        Box tyz = grow(convert(dom, IntVect(0, 1, 1)), IntVect(1, 1, 0));
        auto a11 = T11.array(mfi), a22 = T22.array(mfi), a33 = T33.array(mfi);
        auto a12 = T12.array(mfi), a13 = T13.array(mfi), a23 = T23.array(mfi);
        ComputeStrain_N(bxcc, txy, txz, tyz, dom, xv.const_array(mfi), yv.const_array(mfi), zv.const_array(mfi), a11,
                        a22, a33, a12, a13, a23, bcs.data(), dxi, mf, mf, mf);
    }
    SolverChoice sc;
    sc.turbChoice.resize(1);
    TurbChoice& tc = sc.turbChoice[0];
    tc.les_type = les == 1 ? LESType::Smagorinsky : LESType::Deardorff;
    tc.pbl_type = PBLType::None;
    tc.Cs = Cs; tc.Pr_t = Pr_t; tc.Pr_t_inv = 1.0 / Pr_t; tc.Sc_t = Sc_t; tc.Sc_t_inv = 1.0 / Sc_t;
    tc.Ck = Ck; tc.Ce = Ce; tc.Ce_wall = Ce_wall; tc.theta_ref = theta_ref; tc.sigma_k = sigma_k;
    sc.gravity = gravity;
    sc.use_terrain = false;
    Geometry geom = geometry(nx, ny, nz, dx, dy, dz);
    std::unique_ptr<MultiFab> no_z;
    std::unique_ptr<ABLMost> most;
    ComputeTurbulentViscosity(xv, yv, T11, T22, T33, T12, T13, T23, C, eddy, H1, H2, H3, D, geom, mfu, mfv, no_z, sc,
                              most, false, false, 0, bcs.data(), false);
    const Long n = eddy.fab.bx.numPts();
    std::copy(eddy.fab.p + EddyDiff::Mom_h * n, eddy.fab.p + (EddyDiff::Mom_h + 1) * n, mut);
    std::copy(eddy.fab.p + EddyDiff::Theta_v * n, eddy.fab.p + (EddyDiff::Theta_v + 1) * n, kthv);
    std::copy(D.fab.p, D.fab.p + D.fab.bx.numPts(), diss);
    return 0;
}

// One Kessler step on cons (g = 0), as ERF::advance_microphysics runs it:
// Update_Micro_Vars, Advance, Update_State_Vars.  The reference's Kessler
// carries three moisture species with or without rain (its state always has
// 8 components, and Copy_State_to_Micro / Copy_Micro_to_State touch all
// three), so ncons must be 8.
int ref_kessler(int nx, int ny, int nz, double dx, double dy, double dz, int rain, double c_p, double dt,
                double* cons, int ncons) {
    if (ncons != 8) return 1;
    set_domain(nx, ny, nz);
    MultiFab C = make_mf(nx, ny, nz, 0, 0, ncons, cons);
    SolverChoice sc;
    sc.moisture_type = rain ? MoistureType::Kessler : MoistureType::Kessler_NoRain;
    sc.do_cloud = true;
    sc.do_precip = rain != 0;
    sc.c_p = c_p;
    sc.ave_plane = 2;
    sc.use_terrain = false;
    Geometry geom = geometry(nx, ny, nz, dx, dy, dz);
    Kessler k;
    k.Define(sc);
    std::unique_ptr<MultiFab> no_z, no_j;
    k.Init(C, C.boxArray(), geom, dt, no_z, no_j);
    k.Update_Micro_Vars(C);
    k.Advance(dt, sc);
    k.Update_State_Vars(C);
    std::copy(C.fab.p, C.fab.p + C.fab.bx.numPts() * ncons, cons);
    return 0;
}

double ref_qsatw(double t, double p_hpa) {
    Real q = 0.0;
    erf_qsatw(t, p_hpa, q);
    return q;
}

}  // extern "C"
