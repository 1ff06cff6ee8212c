// terrain.cu -- static terrain-following grid: metrics, per-column base state
// and the terrain (_T) variants of the dycore passes.
//
// The grid is the reference's z_phys_nd (Utils/ERF_TerrainMetrics.cpp:88-335)
// stored as (nz+3) planes of nx*ny nodes (plane k+1 holds node level k, so
// the extrapolated levels -1 and nz+1 are included); the terrain must be
// periodic (node nx equal to node 0), so lateral node indices wrap like the
// cell indices.  Arithmetic is FP64 throughout; the bulk arrays (right-hand
// sides, stresses, averaged momenta, primitives) are stored in R.
//
// Passes (each one thread per cell, face or column, reading neighbours
// directly):
//   k_ter_metrics     make_J / make_zcc (ERF_TerrainMetrics.cpp:583-715)
//   k_ter_base_state  calc_rho_p + erf_enforce_hse per column
//   k_ter_step_begin  old-state boundary round trip, w from Omega = 0 at the
//                     ground and the lid, cons_to_prim, eddy viscosity
//   k_ter_strain /    make_tau_terms with terrain (ERF_make_tau_terms.cpp:
//   k_ter_stress      177-317, ComputeStrain_T, ComputeStressVarVisc_T)
//   k_ter_rawflux     raw diffusive face fluxes (shared by the cross terms)
//   k_ter_slow_cell   rho / rho*theta slow RHS with face areas and detJ
//   k_ter_slow_mom    AdvectionSrcForMom_T, DiffusionSrcForMom_T, terrain
//                     pressure gradient, sources
//   k_ter_fast_h,     erf_fast_rhs_T (TimeIntegration/ERF_fast_rhs_T.cpp)
//   k_ter_fv_bnd,
//   k_ter_fast_vert
//   k_ter_post        erf_slow_rhs_post with terrain and the stage's
//                     boundary round trips
#include <cfloat>

#include "kernels.cuh"
#include "tiles.cuh"

// The library compiles this file twice so that the two halves build side by
// side: as terrain.cu (ERFB_TER_F32 0: every non-template definition and the
// FP64 instantiations) and through terrain_f32.cu (ERFB_TER_F32 1: the FP32
// instantiations only).  Kernels that are not templates are static, so each
// half may hold its own copy of those it launches.
#ifndef ERFB_TER_F32
#define ERFB_TER_F32 0
#endif

namespace erfb {
namespace {

// Resident blocks of 128 threads per SM asked of the compiler for the
// heavy one-thread-per-cell passes (register caps 128 / 64): above their
// natural register counts these kernels are latency-bound at 3-5 blocks.
#define TER_MINB_SLOW_CELL 4
#define TER_MINB_STRAIN 8
#define TER_MINB_POST 4   // the tiled post pass: 256-thread blocks
#define TER_MINB_SLOW_MOM 8
#define TER_MINB_STRESS 8
constexpr int TU5 = ERF_ADV_UPWIND_5TH, TW5 = ERF_ADV_WENO_5;   // compile-time scheme codes

// ---------------------------------------------------------------------------
// Metric terms (Utils/ERF_TerrainMetrics.H:33-395), same operand order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double Zn(const Params& P, int i, int j, int k) {
    const Geo& g = P.g;
    return __ldg(P.znd + (int64_t)(k + 1) * g.sk + (int64_t)wrap(j, g.ny) * g.nx + wrap(i, g.nx));
}
#define ZN(a, b, c) Zn(P, a, b, c)
__device__ __forceinline__ double detJ_at(const Params& P, int i, int j, int k) {
    const Geo& g = P.g;
    return __ldg(P.detJ + cidx(g, wrap(i, g.nx), wrap(j, g.ny), clampk(k, g.nz)));
}
__device__ __forceinline__ double hzeta_cc_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dzi * (ZN(i + 1, j, k + 1) + ZN(i + 1, j + 1, k + 1) + ZN(i, j, k + 1) + ZN(i, j + 1, k + 1)
                             - ZN(i + 1, j, k) - ZN(i + 1, j + 1, k) - ZN(i, j, k) - ZN(i, j + 1, k));
}
__device__ __forceinline__ double hxi_cc_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dxi * (ZN(i + 1, j, k) + ZN(i + 1, j + 1, k) + ZN(i + 1, j, k + 1) + ZN(i + 1, j + 1, k + 1)
                             - ZN(i, j, k) - ZN(i, j + 1, k) - ZN(i, j, k + 1) - ZN(i, j + 1, k + 1));
}
__device__ __forceinline__ double heta_cc_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dyi * (ZN(i, j + 1, k) + ZN(i + 1, j + 1, k) + ZN(i, j + 1, k + 1) + ZN(i + 1, j + 1, k + 1)
                             - ZN(i, j, k) - ZN(i + 1, j, k) - ZN(i, j, k + 1) - ZN(i + 1, j, k + 1));
}
// x faces (also ax) and y faces (also ay)
__device__ __forceinline__ double hzeta_I_fn(const Params& P, int i, int j, int k) {
    return 0.5 * P.g.dzi * (ZN(i, j, k + 1) + ZN(i, j + 1, k + 1) - ZN(i, j, k) - ZN(i, j + 1, k));
}
__device__ __forceinline__ double hxi_I_fn(const Params& P, int i, int j, int k) {
    return 0.125 * P.g.dxi * (ZN(i + 1, j, k) + ZN(i + 1, j, k + 1) + ZN(i + 1, j + 1, k) + ZN(i + 1, j + 1, k + 1)
                              - ZN(i - 1, j, k) - ZN(i - 1, j, k + 1) - ZN(i - 1, j + 1, k) - ZN(i - 1, j + 1, k + 1));
}
__device__ __forceinline__ double hzeta_J_fn(const Params& P, int i, int j, int k) {
    return 0.5 * P.g.dzi * (ZN(i, j, k + 1) + ZN(i + 1, j, k + 1) - ZN(i, j, k) - ZN(i + 1, j, k));
}
__device__ __forceinline__ double heta_J_fn(const Params& P, int i, int j, int k) {
    return 0.125 * P.g.dyi * (ZN(i, j + 1, k) + ZN(i, j + 1, k + 1) + ZN(i + 1, j + 1, k) + ZN(i + 1, j + 1, k + 1)
                              - ZN(i, j - 1, k) - ZN(i, j - 1, k + 1) - ZN(i + 1, j - 1, k) - ZN(i + 1, j - 1, k + 1));
}
// z faces
__device__ __forceinline__ double hzeta_K_fn(const Params& P, int i, int j, int k) {
    return 0.125 * P.g.dzi * (ZN(i, j, k + 1) + ZN(i + 1, j, k + 1) + ZN(i, j + 1, k + 1) + ZN(i + 1, j + 1, k + 1)
                              - ZN(i, j, k - 1) - ZN(i + 1, j, k - 1) - ZN(i, j + 1, k - 1) - ZN(i + 1, j + 1, k - 1));
}
__device__ __forceinline__ double hxi_K_fn(const Params& P, int i, int j, int k) {
    return 0.5 * P.g.dxi * (ZN(i + 1, j, k) + ZN(i + 1, j + 1, k) - ZN(i, j, k) - ZN(i, j + 1, k));
}
__device__ __forceinline__ double heta_K_fn(const Params& P, int i, int j, int k) {
    return 0.5 * P.g.dyi * (ZN(i, j + 1, k) + ZN(i + 1, j + 1, k) - ZN(i, j, k) - ZN(i + 1, j, k));
}
// xy edges (EdgeCenterK), xz edges (EdgeCenterJ), yz edges (EdgeCenterI)
__device__ __forceinline__ double hzeta_EK_fn(const Params& P, int i, int j, int k) { return P.g.dzi * (ZN(i, j, k + 1) - ZN(i, j, k)); }
__device__ __forceinline__ double hxi_EK_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dxi * (ZN(i + 1, j, k) + ZN(i + 1, j, k + 1) - ZN(i - 1, j, k) - ZN(i - 1, j, k + 1));
}
__device__ __forceinline__ double heta_EK_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dyi * (ZN(i, j + 1, k) + ZN(i, j + 1, k + 1) - ZN(i, j - 1, k) - ZN(i, j - 1, k + 1));
}
__device__ __forceinline__ double hzeta_EJ_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dzi * (ZN(i, j, k + 1) + ZN(i, j + 1, k + 1) - ZN(i, j, k - 1) - ZN(i, j + 1, k - 1));
}
__device__ __forceinline__ double hxi_EJ_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dxi * (ZN(i + 1, j + 1, k) + ZN(i + 1, j, k) - ZN(i - 1, j + 1, k) - ZN(i - 1, j, k));
}
__device__ __forceinline__ double heta_EJ_fn(const Params& P, int i, int j, int k) { return P.g.dyi * (ZN(i, j + 1, k) - ZN(i, j, k)); }
__device__ __forceinline__ double hzeta_EI_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dzi * (ZN(i, j, k + 1) + ZN(i + 1, j, k + 1) - ZN(i, j, k - 1) - ZN(i + 1, j, k - 1));
}
__device__ __forceinline__ double hxi_EI_fn(const Params& P, int i, int j, int k) { return P.g.dxi * (ZN(i + 1, j, k) - ZN(i, j, k)); }
__device__ __forceinline__ double heta_EI_fn(const Params& P, int i, int j, int k) {
    return 0.25 * P.g.dyi * (ZN(i + 1, j + 1, k) + ZN(i, j + 1, k) - ZN(i + 1, j - 1, k) - ZN(i, j - 1, k));
}
// slopes of a z-face (OmegaFromW / WFromOmega, ERF_TerrainMetrics.H:455-520)
__device__ __forceinline__ double zlo_xi_fn(const Params& P, int i, int j, int k) {
    return 0.5 * P.g.dxi * (ZN(i + 1, j + 1, k) + ZN(i + 1, j, k) - ZN(i, j + 1, k) - ZN(i, j, k));
}
__device__ __forceinline__ double zlo_eta_fn(const Params& P, int i, int j, int k) {
    return 0.5 * P.g.dyi * (ZN(i + 1, j + 1, k) + ZN(i, j + 1, k) - ZN(i + 1, j, k) - ZN(i, j, k));
}
#undef ZN

// Static-terrain metric tables: the metric terms the passes read,
// evaluated once per cell / face / edge by the functions above (so bit-identical to
// evaluating them in place) and stored as TER_NMET planes of (nz+1) x ny x
// nx values, k in [0, nz].  A pass reads one value instead of re-deriving it
// from four to eight nodes of z_phys_nd; outside [0, nz] the function runs.
enum { MT_HZETA_I, MT_HXI_I, MT_HZETA_J, MT_HETA_J, MT_HXI_K, MT_HETA_K, MT_HZETA_EK, MT_HZETA_EJ, MT_HZETA_EI,
       MT_ZLO_XI, MT_ZLO_ETA, MT_HZETA_CC, MT_HXI_CC, MT_HETA_CC, MT_HZETA_K, MT_HXI_EK, MT_HETA_EK, MT_HXI_EJ,
       MT_HETA_EJ, MT_HXI_EI, MT_HETA_EI, MT_COUNT };
static_assert(MT_COUNT == TER_NMET, "metric table count");
__device__ __forceinline__ double mt_at(const Params& P, int q, int i, int j, int k) {
    const Geo& g = P.g;
    return __ldg(P.met + (int64_t)q * g.nzf + cidx(g, wrap(i, g.nx), wrap(j, g.ny), k));
}
#define ERFB_MT(name, q)                                                           \
    __device__ __forceinline__ double name(const Params& P, int i, int j, int k) { \
        if (k >= 0 && k <= P.g.nz) return mt_at(P, q, i, j, k);                   \
        return name##_fn(P, i, j, k);                                              \
    }
ERFB_MT(hzeta_I, MT_HZETA_I)
ERFB_MT(hxi_I, MT_HXI_I)
ERFB_MT(hzeta_J, MT_HZETA_J)
ERFB_MT(heta_J, MT_HETA_J)
ERFB_MT(hxi_K, MT_HXI_K)
ERFB_MT(heta_K, MT_HETA_K)
ERFB_MT(hzeta_EK, MT_HZETA_EK)
ERFB_MT(hzeta_EJ, MT_HZETA_EJ)
ERFB_MT(hzeta_EI, MT_HZETA_EI)
ERFB_MT(zlo_xi, MT_ZLO_XI)
ERFB_MT(zlo_eta, MT_ZLO_ETA)
ERFB_MT(hzeta_cc, MT_HZETA_CC)
ERFB_MT(hxi_cc, MT_HXI_CC)
ERFB_MT(heta_cc, MT_HETA_CC)
ERFB_MT(hzeta_K, MT_HZETA_K)
ERFB_MT(hxi_EK, MT_HXI_EK)
ERFB_MT(heta_EK, MT_HETA_EK)
ERFB_MT(hxi_EJ, MT_HXI_EJ)
ERFB_MT(heta_EJ, MT_HETA_EJ)
ERFB_MT(hxi_EI, MT_HXI_EI)
ERFB_MT(heta_EI, MT_HETA_EI)
#undef ERFB_MT

// Face-averaged horizontal components at z-face (i,j,k) of x/y-face arrays
// given as accessors (extrapolated to the bottom face).
template <class FU, class FV>
__device__ __forceinline__ void zface_uv(int i, int j, int k, FU ua, FV va, double& u, double& v) {
    if (k == 0) {
        u = 1.5 * (0.5 * (ua(i, j, k) + ua(i + 1, j, k))) - 0.5 * (0.5 * (ua(i, j, k + 1) + ua(i + 1, j, k + 1)));
        v = 1.5 * (0.5 * (va(i, j, k) + va(i, j + 1, k))) - 0.5 * (0.5 * (va(i, j, k + 1) + va(i, j + 1, k + 1)));
    } else {
        u = 0.25 * (ua(i, j, k - 1) + ua(i + 1, j, k - 1) + ua(i, j, k) + ua(i + 1, j, k));
        v = 0.25 * (va(i, j, k - 1) + va(i, j + 1, k - 1) + va(i, j, k) + va(i, j + 1, k));
    }
}
template <class FU, class FV>
__device__ __forceinline__ double omega_from_w(const Params& P, int i, int j, int k, double w, FU ua, FV va) {
    double mx = zlo_xi(P, i, j, k), my = zlo_eta(P, i, j, k), u, v;
    zface_uv(i, j, k, ua, va, u, v);
    return w - mx * u - my * v;
}
template <class FU, class FV>
__device__ __forceinline__ double w_from_omega(const Params& P, int i, int j, int k, double om, FU ua, FV va) {
    double mx = zlo_xi(P, i, j, k), my = zlo_eta(P, i, j, k), u, v;
    zface_uv(i, j, k, ua, va, u, v);
    return om + mx * u + my * v;
}

// qv + qc averaged over two cells (the moist pressure-gradient factor
// 1 + q of ERF_slow_rhs_pre.cpp:594-744 and ERF_fast_rhs_T.cpp:230-300);
// 0 for a dry state.
template <class R>
__device__ __forceinline__ double moist_q(const Params& P, const R* prim, int64_t a, int64_t b) {
    if (!P.moist) return 0.0;
    const int64_t N = P.g.ncell;
    return 0.5 * (double(prim[4 * N + a]) + double(prim[4 * N + b]) + double(prim[5 * N + a]) + double(prim[5 * N + b]));
}

// Base state at (i,j,k), k in [-1, nz].
__device__ __forceinline__ double bs(const double* f, const Geo& g, int i, int j, int k) {
    return __ldg(f + (int64_t)(k + 1) * g.sk + (int64_t)j * g.nx + i);
}

// Horizontal momentum after the M -> V -> M round trip of a boundary fill
// (face (i,j,k) wrapped laterally, k in [0, nz)) and the velocity it gives.
__device__ __forceinline__ double rt_u(const Geo& g, const double* cons, const double* mx, int i, int j, int k) {
    i = wrap(i, g.nx); j = wrap(j, g.ny);
    double rs = cons[cidx(g, i, j, k)] + cons[cidx(g, wrap(i - 1, g.nx), j, k)];
    return (mx[cidx(g, i, j, k)] * 2.0) / rs;
}
__device__ __forceinline__ double rt_v(const Geo& g, const double* cons, const double* my, int i, int j, int k) {
    i = wrap(i, g.nx); j = wrap(j, g.ny);
    double rs = cons[cidx(g, i, j, k)] + cons[cidx(g, i, wrap(j - 1, g.ny), k)];
    return (my[cidx(g, i, j, k)] * 2.0) / rs;
}

// Tangential velocity with its wall ghost (ext_dir 0 or foextrap), lateral
// indices wrapped here.
__device__ __forceinline__ double tvel(const double* f, const Geo& g, int i, int j, int k) {
    i = wrap(i, g.nx); j = wrap(j, g.ny);
    if (k < 0) return g.zlo_noslip ? 0.0 : __ldg(f + cidx(g, i, j, 0));
    if (k >= g.nz) return g.zhi_noslip ? 0.0 : __ldg(f + cidx(g, i, j, g.nz - 1));
    return __ldg(f + cidx(g, i, j, k));
}
// w at z-face k in [0, nz], lateral wrap
__device__ __forceinline__ double wvel(const double* f, const Geo& g, int i, int j, int k) {
    i = wrap(i, g.nx); j = wrap(j, g.ny);
    k = k < 0 ? 0 : (k > g.nz ? g.nz : k);
    return __ldg(f + cidx(g, i, j, k));
}
// cell-centred value with lateral wrap and foextrap in z
template <class V>
__device__ __forceinline__ double ccw(const V* f, const Geo& g, int i, int j, int k) {
    return double(__ldg(f + cidx(g, wrap(i, g.nx), wrap(j, g.ny), clampk(k, g.nz))));
}

__device__ __forceinline__ bool cell_ij(const Geo& g, int& i, int& j, int& k) {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y * blockDim.y + threadIdx.y;
    k = blockIdx.z;
    return i < g.nx && j < g.ny && k < g.nz;
}
dim3 ter_block() { return dim3(32, 4, 1); }
dim3 ter_grid(const Geo& g, int nk) { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, nk); }

}  // namespace

// ---------------------------------------------------------------------------
// Metrics: detJ per cell and z at cell centres (levels 0..nz, the top one
// from the extrapolated node level).
// ---------------------------------------------------------------------------
static __global__ void k_ter_metrics(Params P, double* __restrict__ detJ, double* __restrict__ zcc) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    auto Z = [&](int a, int b, int c) { return Zn(P, a, b, c); };
    if (k < g.nz)
        detJ[cidx(g, i, j, k)] = .25 * g.dzi * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)
                                                - Z(i, j, k) - Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i + 1, j + 1, k));
    zcc[cidx(g, i, j, k)] = .125 * (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k)
                                    + Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1));
}
// The metric tables (k in [0, nz] for every plane)
static __global__ void k_ter_met_tables(Params P, double* __restrict__ met) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    double* m = met + cidx(g, i, j, k);
    const int64_t s = g.nzf;
    m[MT_HZETA_I * s] = hzeta_I_fn(P, i, j, k);
    m[MT_HXI_I * s] = hxi_I_fn(P, i, j, k);
    m[MT_HZETA_J * s] = hzeta_J_fn(P, i, j, k);
    m[MT_HETA_J * s] = heta_J_fn(P, i, j, k);
    m[MT_HXI_K * s] = hxi_K_fn(P, i, j, k);
    m[MT_HETA_K * s] = heta_K_fn(P, i, j, k);
    m[MT_HZETA_EK * s] = hzeta_EK_fn(P, i, j, k);
    m[MT_HZETA_EJ * s] = hzeta_EJ_fn(P, i, j, k);
    m[MT_HZETA_EI * s] = hzeta_EI_fn(P, i, j, k);
    m[MT_ZLO_XI * s] = zlo_xi_fn(P, i, j, k);
    m[MT_ZLO_ETA * s] = zlo_eta_fn(P, i, j, k);
    m[MT_HZETA_CC * s] = hzeta_cc_fn(P, i, j, k);
    m[MT_HXI_CC * s] = hxi_cc_fn(P, i, j, k);
    m[MT_HETA_CC * s] = heta_cc_fn(P, i, j, k);
    m[MT_HZETA_K * s] = hzeta_K_fn(P, i, j, k);
    m[MT_HXI_EK * s] = hxi_EK_fn(P, i, j, k);
    m[MT_HETA_EK * s] = heta_EK_fn(P, i, j, k);
    m[MT_HXI_EJ * s] = hxi_EJ_fn(P, i, j, k);
    m[MT_HETA_EJ * s] = heta_EJ_fn(P, i, j, k);
    m[MT_HXI_EI * s] = hxi_EI_fn(P, i, j, k);
    m[MT_HETA_EI * s] = heta_EI_fn(P, i, j, k);
}
#if !ERFB_TER_F32
void launch_ter_metrics(const Params& P, cudaStream_t st, double* detJ, double* zcc) {
    k_ter_metrics<<<ter_grid(P.g, P.g.nz + 1), ter_block(), 0, st>>>(P, detJ, zcc);
    k_ter_met_tables<<<ter_grid(P.g, P.g.nz + 1), ter_block(), 0, st>>>(P, const_cast<double*>(P.met));
}
#endif

// ---------------------------------------------------------------------------
// Moving terrain (terrain_type Moving), without acoustic substepping.  The
// grid is regenerated on the device at every geometry time of the stage
// (the step's old time, the stage's source and new times) from the device
// copy of the step's old time, so that the step graph replays unchanged.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mt_time_at(double T, double dt, int tsel) {
    return tsel == 0 ? T : (tsel == 1 ? T + dt / 3.0 : (tsel == 2 ? T + dt / 2.0 : T + dt));
}
// node (i,j,k) of a grid in the znd layout ((nz+3) planes, lateral periodic)
__device__ __forceinline__ double znode(const double* z, const Geo& g, int i, int j, int k) {
    return __ldg(z + (int64_t)(k + 1) * g.sk + (int64_t)wrap(j, g.ny) * g.nx + wrap(i, g.nx));
}
// make_J of one cell from the nodes (Utils/ERF_TerrainMetrics.cpp:583-640);
// k = -1 takes level 0 (the grid's ghost level mirrors the first cell)
__device__ __forceinline__ double mt_detj(const double* z, const Geo& g, int i, int j, int k) {
    if (k < 0) k = 0;
    auto Z = [&](int a, int b, int c) { return znode(z, g, a, b, c); };
    return .25 * g.dzi * (Z(i, j, k + 1) + Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)
                          - Z(i, j, k) - Z(i + 1, j, k) - Z(i, j + 1, k) - Z(i + 1, j + 1, k));
}

// Problem::init_custom_terrain of the travelling wave
// (Exec/DevTests/MovingTerrain/ERF_prob.cpp:147-200) and init_terrain_grid
// with terrain_smoothing = 2 (Utils/ERF_TerrainMetrics.cpp:501-536, 320-333):
// z(k) = z_k + (1 - z_k / z_top)^3 h over z_k = k dz, z(0) = h,
// z(-1) = 2 h - z(1), z(nz+1) = 2 z(nz) - z(nz-1).  One thread per column.
static __global__ void k_mt_grid(Params P, const double* __restrict__ tdev, double dt, int tsel, double* __restrict__ z) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    // tsel >= 0: a stage point; tsel < 0: substep -1 - tsel of length dt, T + ks dt
    const double t = tsel >= 0 ? mt_time_at(*tdev, dt, tsel) : *tdev + (-1 - tsel) * dt;
    const double x = i * P.mt_dx;
    // products and sums rounded one at a time, as the host C++ of the
    // reference forms them (no fused multiply-add): the grid's node heights
    // enter z_t through differences over a substep, which magnify any change
    const double hs = __dmul_rn(P.mt_ampl, sin(__dsub_rn(__dmul_rn(P.mt_kp, x), __dmul_rn(P.mt_om, t))));
    const int nz = g.nz;
    double* col = z + (int64_t)j * g.nx + i;
    double zk1 = 0.0, zkm1 = 0.0, zk = hs;
    for (int k = 0; k <= nz; ++k) {
        const double zl = k * P.mt_dz;
        double v = __dadd_rn(zl, __dmul_rn(P.mt_fac[k], hs));
        if (k == 0) v = hs;
        col[(int64_t)(k + 1) * g.sk] = v;
        if (k == 1) zk1 = v;
        if (k == nz - 1) zkm1 = v;
        if (k == nz) zk = v;
    }
    col[0] = 2.0 * hs - zk1;
    col[(int64_t)(nz + 2) * g.sk] = 2.0 * zk - zkm1;
}
#if !ERFB_TER_F32
void launch_mt_grid(const Params& P, cudaStream_t st, const double* tdev, double dt, int tsel, double* z) {
    k_mt_grid<<<ter_grid(P.g, 1), ter_block(), 0, st>>>(P, tdev, dt, tsel, z);
}
#endif

// z_t of the stage (ERF_TI_slow_rhs_fun.H:84-107): (z_new - z_old) / slow_dt
// averaged over the four nodes of each z face, slow_dt = new stage time - T.
static __global__ void k_mt_zt(Params P, const double* __restrict__ zo, const double* __restrict__ zn,
                        const double* __restrict__ tdev, double dt, int tsel_new, double* __restrict__ zt) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    const double T = *tdev;
    const double inv_dt = 1. / (mt_time_at(T, dt, tsel_new) - T);
    auto N = [&](int a, int b) { return znode(zn, g, a, b, k); };
    auto O = [&](int a, int b) { return znode(zo, g, a, b, k); };
    zt[cidx(g, i, j, k)] = 0.25 * inv_dt * (N(i + 1, j + 1) - O(i + 1, j + 1) + N(i, j + 1) - O(i, j + 1)
                                            + N(i + 1, j) - O(i + 1, j) + N(i, j) - O(i, j));
}
#if !ERFB_TER_F32
void launch_mt_zt(const Params& P, cudaStream_t st, const double* zo, const double* zn, const double* tdev,
                  double dt, int tsel_new, double* zt) {
    k_mt_zt<<<ter_grid(P.g, P.g.nz + 1), ter_block(), 0, st>>>(P, zo, zn, tdev, dt, tsel_new, zt);
}
#endif

// The base-state update of a moving-terrain stage (ERF_TI_slow_rhs_fun.H:149-210):
// rho_0 and (rho theta)_0 advanced from the step's old base state by the
// vertical flux -z_t (face averages of the previous stage's new base state),
// detJ-weighted old -> source -> new; p_0 from (rho theta)_0.  One thread
// per column walks up the levels, keeping the level below (already
// overwritten) in registers; the ghost levels are not updated.
static __global__ void k_mt_base_state(Params P, const double* __restrict__ r0o, const double* __restrict__ p0o,
                                const double* __restrict__ zo, const double* __restrict__ zs,
                                const double* __restrict__ zn, const double* __restrict__ tdev, double dt,
                                int tsel_new, double* __restrict__ r0n, double* __restrict__ p0n) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const double T = *tdev;
    const double dt_base = mt_time_at(T, dt, tsel_new) - T;
    const double* zt = P.mt_zt;
    auto at = [&](int k) { return (int64_t)(k + 1) * g.sk + (int64_t)j * g.nx + i; };
    double r_m = r0n[at(-1)], rt_m = eos_rt_given_p(p0n[at(-1)]);
    double r_c = r0n[at(0)], rt_c = eos_rt_given_p(p0n[at(0)]);
    for (int k = 0; k < g.nz; ++k) {
        const double r_p = r0n[at(k + 1)], rt_p = eos_rt_given_p(p0n[at(k + 1)]);
        const double zl = zt[cidx(g, i, j, k)], zh = zt[cidx(g, i, j, k + 1)];
        double fr_lo = -zl * 0.5 * (r_c + r_m);
        double fr_hi = -zh * 0.5 * (r_c + r_p);
        double frt_lo = fr_lo * 0.5 * (rt_c / r_c + rt_m / r_m);
        double frt_hi = fr_hi * 0.5 * (rt_c / r_c + rt_p / r_p);
        const double Js = mt_detj(zs, g, i, j, k), Jo = mt_detj(zo, g, i, j, k), Jn = mt_detj(zn, g, i, j, k);
        double invdetJ = 1.0 / Js;
        double src_r = -invdetJ * (fr_hi - fr_lo) * g.dzi;
        double src_rt = -invdetJ * (frt_hi - frt_lo) * g.dzi;
        double rho0_new = Jo * r0o[at(k)] + dt_base * Js * src_r;
        double rt0_new = Jo * eos_rt_given_p(p0o[at(k)]) + dt_base * Js * src_rt;
        r0n[at(k)] = rho0_new / Jn;
        rt0_new /= Jn;
        p0n[at(k)] = eos_p(rt0_new, 0.0);
        r_m = r_c; rt_m = rt_c; r_c = r_p; rt_c = rt_p;
    }
}
#if !ERFB_TER_F32
void launch_mt_base_state(const Params& P, cudaStream_t st, const double* r0o, const double* p0o, const double* zo,
                          const double* zs, const double* zn, const double* tdev, double dt, int tsel_new,
                          double* r0n, double* p0n) {
    k_mt_base_state<<<ter_grid(P.g, 1), ter_block(), 0, st>>>(P, r0o, p0o, zo, zs, zn, tdev, dt, tsel_new, r0n, p0n);
}
#endif

// no_substep_fun for moving terrain (TimeIntegration/ERF_TI_no_substep_fun.H:54-109),
// part 1: rho and rho theta detJ-weighted old -> new, the horizontal
// momenta with h_zeta of their faces (the slow right-hand sides already
// carry the source geometry's factors).
__device__ __forceinline__ double mt_hzI(const double* z, const Geo& g, int i, int j, int k) {
    return 0.5 * g.dzi * (znode(z, g, i, j, k + 1) + znode(z, g, i, j + 1, k + 1) - znode(z, g, i, j, k) - znode(z, g, i, j + 1, k));
}
__device__ __forceinline__ double mt_hzJ(const double* z, const Geo& g, int i, int j, int k) {
    return 0.5 * g.dzi * (znode(z, g, i, j, k + 1) + znode(z, g, i + 1, j, k + 1) - znode(z, g, i, j, k) - znode(z, g, i + 1, j, k));
}
template <class R>
__global__ void k_mt_no_substep_h(Params P, double slow_dt, StateBuf Sold, const R* __restrict__ Fcons,
                                  const R* __restrict__ Fmx, const R* __restrict__ Fmy, const double* __restrict__ zo,
                                  const double* __restrict__ zn, StateBuf Ssum) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int64_t c = cidx(g, i, j, k), N = g.ncell;
    const double Jo = mt_detj(zo, g, i, j, k), Jn = mt_detj(zn, g, i, j, k);
    for (int n = 0; n < 2; ++n) {
        double v = Jo * Sold.cons[n * N + c] + slow_dt * double(Fcons[n * N + c]);
        Ssum.cons[n * N + c] = v / Jn;
    }
    Ssum.mx[c] = (mt_hzI(zo, g, i, j, k) * Sold.mx[c] + slow_dt * double(Fmx[c])) / mt_hzI(zn, g, i, j, k);
    Ssum.my[c] = (mt_hzJ(zo, g, i, j, k) * Sold.my[c] + slow_dt * double(Fmy[c])) / mt_hzJ(zn, g, i, j, k);
}
// part 2: rho w with the face detJ; on the moving ground W from Omega =
// rho z_t on the new grid with the new horizontal momenta.
template <class R>
__global__ void k_mt_no_substep_w(Params P, double slow_dt, StateBuf Sold, const R* __restrict__ Fmz,
                                  const double* __restrict__ zo, const double* __restrict__ zn, StateBuf Ssum) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    const int64_t c = cidx(g, i, j, k);
    if (k == 0) {
        Params Pn = P;
        Pn.znd = zn;
        auto MX = [&](int a, int b, int kk) { return Ssum.mx[cidx(g, wrap(a, g.nx), wrap(b, g.ny), kk)]; };
        auto MY = [&](int a, int b, int kk) { return Ssum.my[cidx(g, wrap(a, g.nx), wrap(b, g.ny), kk)]; };
        double mx = zlo_xi_fn(Pn, i, j, 0), my = zlo_eta_fn(Pn, i, j, 0), u, v;
        zface_uv(i, j, 0, MX, MY, u, v);
        const double rho_on_face = Ssum.cons[c];
        Ssum.mz[c] = rho_on_face * P.mt_zt[c] + mx * u + my * v;
    } else {
        double ko = 0.5 * (mt_detj(zo, g, i, j, k) + mt_detj(zo, g, i, j, k - 1));
        double kn = 0.5 * (mt_detj(zn, g, i, j, k) + mt_detj(zn, g, i, j, k - 1));
        Ssum.mz[c] = (ko * Sold.mz[c] + slow_dt * double(Fmz[c])) / kn;
    }
}
template <class R>
void launch_mt_no_substep(const Params& P, cudaStream_t st, double slow_dt, StateBuf Sold, const R* Fcons,
                          const R* Fmx, const R* Fmy, const R* Fmz, const double* zo, const double* zn, StateBuf Ssum) {
    k_mt_no_substep_h<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, slow_dt, Sold, Fcons, Fmx, Fmy, zo, zn, Ssum);
    k_mt_no_substep_w<R><<<ter_grid(P.g, P.g.nz + 1), ter_block(), 0, st>>>(P, slow_dt, Sold, Fmz, zo, zn, Ssum);
}
#if !ERFB_TER_F32
template void launch_mt_no_substep<double>(const Params&, cudaStream_t, double, StateBuf, const double*, const double*,
                                           const double*, const double*, const double*, const double*, StateBuf);
#else
template void launch_mt_no_substep<float>(const Params&, cudaStream_t, double, StateBuf, const float*, const float*,
                                          const float*, const float*, const double*, const double*, StateBuf);
#endif

// ---------------------------------------------------------------------------
// Acoustic substeps over moving terrain (erf_fast_rhs_MT,
// TimeIntegration/ERF_fast_rhs_MT.cpp:48-626).  zo / zn: the grids at the
// substep's old and new times, zs: the stage's; zpt: the substep's z_t less
// the stage's.  The new state's horizontal momenta are formed h_zeta-weighted
// in place, read that way by the flux and Omega'' kernels, then divided by
// the new grid's h_zeta; one thread per column solves for Omega'' and
// updates rho w, rho and rho theta.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void mt_slopes(const double* z, const Geo& g, int i, int j, int k, double& sx, double& sy) {
    sx = 0.5 * g.dxi * (znode(z, g, i + 1, j + 1, k) + znode(z, g, i + 1, j, k) - znode(z, g, i, j + 1, k) - znode(z, g, i, j, k));
    sy = 0.5 * g.dyi * (znode(z, g, i + 1, j + 1, k) + znode(z, g, i, j + 1, k) - znode(z, g, i + 1, j, k) - znode(z, g, i, j, k));
}
__device__ __forceinline__ double mt_hxI(const double* z, const Geo& g, int i, int j, int k) {
    auto Z = [&](int a, int b, int c) { return znode(z, g, a, b, c); };
    return 0.125 * g.dxi * (Z(i + 1, j, k) + Z(i + 1, j, k + 1) + Z(i + 1, j + 1, k) + Z(i + 1, j + 1, k + 1)
                            - Z(i - 1, j, k) - Z(i - 1, j, k + 1) - Z(i - 1, j + 1, k) - Z(i - 1, j + 1, k + 1));
}
__device__ __forceinline__ double mt_hetaJ(const double* z, const Geo& g, int i, int j, int k) {
    auto Z = [&](int a, int b, int c) { return znode(z, g, a, b, c); };
    return 0.125 * g.dyi * (Z(i, j + 1, k) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k) + Z(i + 1, j + 1, k + 1)
                            - Z(i, j - 1, k) - Z(i, j - 1, k + 1) - Z(i + 1, j - 1, k) - Z(i + 1, j - 1, k + 1));
}
// OmegaFromW of face (i,j,k) on grid z, horizontal momenta mx / my
__device__ __forceinline__ double mt_omega(const double* z, const Geo& g, int i, int j, int k, double w,
                                           const double* mx, const double* my) {
    auto U = [&](int a, int b, int c) { return mx[cidx(g, wrap(a, g.nx), wrap(b, g.ny), c)]; };
    auto V = [&](int a, int b, int c) { return my[cidx(g, wrap(a, g.nx), wrap(b, g.ny), c)]; };
    double sx, sy, u, v;
    mt_slopes(z, g, i, j, k, sx, sy);
    zface_uv(i, j, k, U, V, u, v);
    return w - sx * u - sy * v;
}
__device__ __forceinline__ double mt_wfrom(const double* z, const Geo& g, int i, int j, int k, double om,
                                           const double* mx, const double* my) {
    auto U = [&](int a, int b, int c) { return mx[cidx(g, wrap(a, g.nx), wrap(b, g.ny), c)]; };
    auto V = [&](int a, int b, int c) { return my[cidx(g, wrap(a, g.nx), wrap(b, g.ny), c)]; };
    double sx, sy, u, v;
    mt_slopes(z, g, i, j, k, sx, sy);
    zface_uv(i, j, k, U, V, u, v);
    return om + sx * u + sy * v;
}

// the substep's z_t less the stage's (ERF_TI_fast_rhs_fun.H:66-90)
static __global__ void k_mt_zpt(Params P, const double* __restrict__ zo, const double* __restrict__ zn, double inv_dt,
                         double* __restrict__ zpt) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    auto N = [&](int a, int b) { return znode(zn, g, a, b, k); };
    auto O = [&](int a, int b) { return znode(zo, g, a, b, k); };
    const int64_t f = cidx(g, i, j, k);
    double v = 0.25 * inv_dt * (N(i + 1, j + 1) - O(i + 1, j + 1) + N(i, j + 1) - O(i, j + 1) + N(i + 1, j) - O(i + 1, j) + N(i, j) - O(i, j));
    zpt[f] = v - P.mt_zt[f];
}
// detJ of a grid's cells (make_J)
static __global__ void k_mt_detj(Params P, const double* __restrict__ z, double* __restrict__ detJ) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    detJ[cidx(g, i, j, k)] = mt_detj(z, g, i, j, k);
}

// x / y momenta of the substep, h_zeta-weighted on the old grid
// (ERF_fast_rhs_MT.cpp:197-273); d(rho theta) extrapolated with or without
// the lagged correction; the new lag.
template <class R>
__global__ void k_mt_fast_h(Params P, int step, int lagged, double dtau, StateBuf Sprev, StateBuf Sst, StageAux<R> A,
                            const R* __restrict__ Fmx, const R* __restrict__ Fmy, const R* __restrict__ lag_in,
                            R* __restrict__ lag_out, const double* __restrict__ zo, StateBuf Ssum) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    const int64_t N = g.ncell;
    const int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    const int64_t c = cidx(g, i, j, k), cxm = cidx(g, im, j, k), cym = cidx(g, i, jm, k);
    const double beta_d = 0.1, dxi = g.dxi, dyi = g.dyi, dzi = g.dzi;
    auto extrap = [&](int ii, int jj, int kk) {
        int64_t e = cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), clampk(kk, nz));
        double d = Sprev.cons[N + e] - Sst.cons[N + e];
        if (step == 0 || !lagged) return d;
        return d + beta_d * (d - double(lag_in[e]));
    };
    if (step == 0 || lagged) lag_out[c] = R(Sprev.cons[N + c] - Sst.cons[N + c]);
    double mx, my;
    {
        double hxi = mt_hxI(zo, g, i, j, k), hz = mt_hzI(zo, g, i, j, k);
        double gp_xi = (extrap(i, j, k) - extrap(i - 1, j, k)) * dxi;
        double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k) - extrap(i, j, k))
                                  : 0.25 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k - 1) - extrap(i, j, k - 1));
        double gpx = hz * gp_xi - hxi * gp_zeta;
        gpx *= 1.0;
        double pi_c = 0.5 * (double(A.pi[cxm]) + double(A.pi[c]));
        double f = -Gamma_ * R_d * pi_c * gpx;
        mx = hz * Sprev.mx[c] + dtau * f + dtau * double(Fmx[c]);
    }
    {
        double het = mt_hetaJ(zo, g, i, j, k), hz = mt_hzJ(zo, g, i, j, k);
        double gp_eta = (extrap(i, j, k) - extrap(i, j - 1, k)) * dyi;
        double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k) - extrap(i, j - 1, k))
                                  : 0.25 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k - 1) - extrap(i, j - 1, k - 1));
        double gpy = hz * gp_eta - het * gp_zeta;
        gpy *= 1.0;
        double pi_c = 0.5 * (double(A.pi[cym]) + double(A.pi[c]));
        double f = -Gamma_ * R_d * pi_c * gpy;
        my = hz * Sprev.my[c] + dtau * f + dtau * double(Fmy[c]);
    }
    Ssum.mx[c] = mx;
    Ssum.my[c] = my;
}

// horizontal fluxes of rho and rho theta (the weighted momenta less the
// stage's on the stage grid) and Omega'' of the previous substep on the old
// grid (ERF_fast_rhs_MT.cpp:283-340).  After the first substep the previous
// and new states are one, so Omega'' reads the weighted momenta, as the
// reference's aliased arrays do.
template <class R>
__global__ void k_mt_fast_flux(Params P, StateBuf Sprev, StateBuf Sst, StageAux<R> A, StateBuf Ssum,
                               const double* __restrict__ zo, const double* __restrict__ zs,
                               const double* __restrict__ zpt, double* __restrict__ trhs, double* __restrict__ om) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    const int nz = g.nz;
    const int64_t N = g.ncell, f = cidx(g, i, j, k);
    if (k < nz) {
        const int ip = wrap(i + 1, g.nx), im = wrap(i - 1, g.nx), jp = wrap(j + 1, g.ny), jm = wrap(j - 1, g.ny);
        const int64_t cxp = cidx(g, ip, j, k), cyp = cidx(g, i, jp, k);
        double xl = Ssum.mx[f] - Sst.mx[f] * mt_hzI(zs, g, i, j, k), xh = Ssum.mx[cxp] - Sst.mx[cxp] * mt_hzI(zs, g, i + 1, j, k);
        double yl = Ssum.my[f] - Sst.my[f] * mt_hzJ(zs, g, i, j, k), yh = Ssum.my[cyp] - Sst.my[cyp] * mt_hzJ(zs, g, i, j + 1, k);
        auto th = [&](int a, int b) { return double(A.prim[cidx(g, a, b, k)]); };
        const double t0 = th(i, j);
        trhs[f] = (xh - xl) * g.dxi + (yh - yl) * g.dyi;
        trhs[N + f] = ((xh * (t0 + th(ip, j)) - xl * (t0 + th(im, j))) * g.dxi +
                       (yh * (t0 + th(i, jp)) - yl * (t0 + th(i, jm))) * g.dyi) * 0.5;
    }
    double o;
    if (k == 0) o = 0.;
    else if (k == nz) o = Sprev.mz[f] - Sst.mz[f] - zpt[f];
    else {
        double a = mt_omega(zo, g, i, j, k, Sprev.mz[f], Sprev.mx, Sprev.my);
        double b = mt_omega(zo, g, i, j, k, Sst.mz[f], Sst.mx, Sst.my);
        o = (a - b) - zpt[f];
    }
    om[f] = o;
}

// the horizontal momenta divided by the new grid's h_zeta; their average
template <class R>
__global__ void k_mt_fast_div(Params P, double facinv, StateBuf Sst, const double* __restrict__ zn, StateBuf Ssum,
                              R* __restrict__ avx, R* __restrict__ avy) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int64_t c = cidx(g, i, j, k);
    double mx = Ssum.mx[c] / mt_hzI(zn, g, i, j, k);
    double my = Ssum.my[c] / mt_hzJ(zn, g, i, j, k);
    Ssum.mx[c] = mx;
    Ssum.my[c] = my;
    avx[c] += R(facinv * (mx - Sst.mx[c]));
    avy[c] += R(facinv * (my - Sst.my[c]));
}

// The Omega'' column system (ERF_fast_rhs_MT.cpp:375-600) in four kernels:
// its right-hand side (one thread per z face: the old / new / stage face
// detJ, the stage's coefficients made on the substep's old grid), the
// Thomas sweep (one thread per column, the only serial part), rho w from
// Omega'' with the ground at W from Omega = rho (z_t + z_t'') (one thread
// per face), then the vertical fluxes, the average contravariant momentum
// and rho / rho theta detJ-weighted old -> new (one thread per cell).
// soln: the right-hand side, then the solution, then the new Omega''.
template <class R>
__global__ void k_mt_col_rhs(Params P, double dtau, double beta_1, double beta_2, StateBuf Sprev, StateBuf Sst,
                             StageAux<R> A, const R* __restrict__ Fcons, const R* __restrict__ Fmz,
                             const R* __restrict__ cP, const R* __restrict__ cQ, const double* __restrict__ zo,
                             const double* __restrict__ zn, const double* __restrict__ zs,
                             const double* __restrict__ zpt, const double* __restrict__ om,
                             const double* __restrict__ trhs, StateBuf Ssum, double* __restrict__ soln) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    const int nz = g.nz;
    const int64_t N = g.ncell;
    auto C = [&](int kk) { return cidx(g, i, j, kk); };
    const int64_t a = C(k);
    if (k == 0) {
        const double rho_on_bdy = 0.5 * (Sprev.cons[a] + Sprev.cons[a]);
        soln[a] = rho_on_bdy * zpt[a];
        return;
    }
    if (k == nz) {
        soln[a] = 0.0;
        return;
    }
    const double dzi = g.dzi, halfg = fabs(0.5 * -P.gravity);
    auto th = [&](int kk) { return double(A.prim[C(clampk(kk, nz))]); };
    auto fJ = [&](const double* z) { return 0.5 * (mt_detj(z, g, i, j, k) + mt_detj(z, g, i, j, k - 1)); };
    const double Jo = fJ(zo), Jn = fJ(zn), Js = fJ(zs);
    const double cp = double(cP[a]), cq = double(cQ[a]);
    const double tlo = 0.5 * (th(k - 2) + th(k - 1)), tmid = 0.5 * (th(k - 1) + th(k)), thi = 0.5 * (th(k) + th(k + 1));
    const int64_t b = C(k - 1);
    double R0t = cp * Sprev.cons[N + a] * Jo + cq * Sprev.cons[N + b] * Jo
                 - cp * Sst.cons[N + a] * Js - cq * Sst.cons[N + b] * Js
                 - halfg * (Sprev.cons[a] + Sprev.cons[b]) * Jo
                 + halfg * (Sst.cons[a] + Sst.cons[b]) * Js;
    double R1t = -halfg * (double(Fcons[a]) + double(Fcons[b])) + (cp * double(Fcons[N + a]) + cq * double(Fcons[N + b]));
    const double Okp1 = om[C(k + 1)], Ok = om[a], Okm1 = om[b];
    R1t += (halfg) * (beta_1 * dzi * (Okp1 - Okm1) + trhs[a] + trhs[b]);
    R1t += -(cp * (beta_1 * dzi * (Okp1 * thi - Ok * tmid) + trhs[N + a]) +
             cq * (beta_1 * dzi * (Ok * tmid - Okm1 * tlo) + trhs[N + b]));
    double rhs = Jo * Sprev.mz[a] - Js * Sst.mz[a] + dtau * (double(Fmz[a]) + R0t + dtau * beta_2 * R1t);
    double un = mt_omega(zn, g, i, j, k, 0., Ssum.mx, Ssum.my);
    double us = mt_omega(zs, g, i, j, k, 0., Sst.mx, Sst.my);
    rhs += Jn * un - Js * us;
    soln[a] = rhs;
}
template <class R>
__global__ void k_mt_col_sweep(Params P, StateBuf Sst, const R* __restrict__ cA, const R* __restrict__ cInvB,
                               const R* __restrict__ cCB, StateBuf Ssum, double* __restrict__ soln) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int nz = g.nz;
    auto C = [&](int kk) { return cidx(g, i, j, kk); };
    double s = soln[C(0)] * double(cInvB[C(0)]);
    soln[C(0)] = s;
    for (int k = 1; k <= nz; ++k) {
        s = (soln[C(k)] - double(cA[C(k)]) * s) * double(cInvB[C(k)]);
        soln[C(k)] = s;
    }
    Ssum.mz[C(nz)] = Sst.mz[C(nz)] + s;
    for (int k = nz - 1; k >= 0; --k) {
        s = soln[C(k)] - double(cCB[C(k)]) * s;
        soln[C(k)] = s;
    }
}
template <class R>
__global__ void k_mt_col_w(Params P, StateBuf Sprev, StateBuf Sst, const double* __restrict__ zo,
                           const double* __restrict__ zn, const double* __restrict__ zs,
                           const double* __restrict__ zpt, StateBuf Ssum, double* __restrict__ soln) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    const int64_t a = cidx(g, i, j, k);
    const double rho_on_face = 0.5 * (Sprev.cons[a] + Sprev.cons[cidx(g, i, j, k > 0 ? k - 1 : 0)]);
    if (k == 0) {
        Ssum.mz[a] = mt_wfrom(zn, g, i, j, 0, rho_on_face * (P.mt_zt[a] + zpt[a]), Ssum.mx, Ssum.my);
        soln[a] = 0.;
        return;
    }
    auto fJ = [&](const double* z) { return 0.5 * (mt_detj(z, g, i, j, k) + mt_detj(z, g, i, j, k - 1)); };
    double wn = mt_wfrom(zn, g, i, j, k, 0.0, Ssum.mx, Ssum.my);
    double ws = mt_wfrom(zs, g, i, j, k, 0.0, Sst.mx, Sst.my);
    double wpp = soln[a] + (wn - ws);
    double m = fJ(zo) * (Sst.mz[a] + wpp);
    m /= fJ(zn);
    Ssum.mz[a] = m;
    double o1 = mt_omega(zn, g, i, j, k, m, Ssum.mx, Ssum.my);
    double o2 = mt_omega(zs, g, i, j, k, Sst.mz[a], Sst.mx, Sst.my);
    double sv = o1 - o2;
    sv -= rho_on_face * zpt[a];
    soln[a] = sv;
}
template <class R>
__global__ void k_mt_col_cons(Params P, double dtau, double beta_1, double beta_2, double facinv, StateBuf Sprev,
                              StageAux<R> A, const R* __restrict__ Fcons, const double* __restrict__ zo,
                              const double* __restrict__ zn, const double* __restrict__ om,
                              const double* __restrict__ trhs, const double* __restrict__ soln,
                              R* __restrict__ avz, StateBuf Ssum) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    const int64_t N = g.ncell, a = cidx(g, i, j, k), ah = cidx(g, i, j, k + 1);
    auto th = [&](int kk) { return double(A.prim[cidx(g, i, j, clampk(kk, nz))]); };
    double zl = beta_2 * soln[a] + beta_1 * om[a];
    double zh = beta_2 * soln[ah] + beta_1 * om[ah];
    avz[a] += R(facinv * zl / (1.0 * 1.0));
    if (k == nz - 1) avz[ah] += R(facinv * zh / (1.0 * 1.0));
    const double Jo = mt_detj(zo, g, i, j, k), Jn = mt_detj(zn, g, i, j, k);
    double frho = -(trhs[a] + (zh - zl) * g.dzi);
    double tr = Jo * Sprev.cons[a] + dtau * (double(Fcons[a]) + frho);
    double frt = -(trhs[N + a] + 0.5 * (zh * (th(k) + th(k + 1)) - zl * (th(k) + th(k - 1))) * g.dzi);
    double tt = Jo * Sprev.cons[N + a] + dtau * (double(Fcons[N + a]) + frt);
    Ssum.cons[a] = tr / Jn;
    Ssum.cons[N + a] = tt / Jn;
}

// the boundary fill after a substep (apply_bcs, fast variables): the
// momenta through M -> V -> M with the walls' density ghosts; w on the flat
// lid from Omega = 0, the moving ground untouched but round-tripped
static __global__ void k_mt_fast_bc(Params P, StateBuf Ssum) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    const int nz = g.nz;
    const int64_t f = cidx(g, i, j, k);
    if (k < nz) {
        double rs = Ssum.cons[f] + Ssum.cons[cidx(g, wrap(i - 1, g.nx), j, k)];
        double u = (Ssum.mx[f] * 2.0) / rs;
        Ssum.mx[f] = (u * 0.5) * rs;
        rs = Ssum.cons[f] + Ssum.cons[cidx(g, i, wrap(j - 1, g.ny), k)];
        double v = (Ssum.my[f] * 2.0) / rs;
        Ssum.my[f] = (v * 0.5) * rs;
    }
    if (k == nz) {
        Ssum.mz[f] = 0.0;   // W from Omega = 0 on the flat lid
    } else {
        double rs = Ssum.cons[f] + Ssum.cons[k > 0 ? f - g.sk : f];
        double w = (Ssum.mz[f] * 2.0) / rs;
        Ssum.mz[f] = (w * 0.5) * rs;
    }
}

#if !ERFB_TER_F32
void launch_mt_grid_sub(const Params& P, cudaStream_t st, const double* tdev, double dtau, int ks, double* z) {
    k_mt_grid<<<ter_grid(P.g, 1), ter_block(), 0, st>>>(P, tdev, dtau, -1 - ks, z);
}
#endif
#if !ERFB_TER_F32
void launch_mt_zpt(const Params& P, cudaStream_t st, const double* zo, const double* zn, double dtau, double* zpt) {
    k_mt_zpt<<<ter_grid(P.g, P.g.nz + 1), ter_block(), 0, st>>>(P, zo, zn, 1. / dtau, zpt);
}
#endif
#if !ERFB_TER_F32
void launch_mt_detj(const Params& P, cudaStream_t st, const double* z, double* detJ) {
    k_mt_detj<<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, z, detJ);
}
#endif
template <class R>
void launch_mt_fast(const Params& P, cudaStream_t st, int step, int lagged, double dtau, double beta_s, double facinv,
                    StateBuf Sprev, StateBuf Sst, StageAux<R> A, const R* Fcons, const R* Fmx, const R* Fmy,
                    const R* Fmz, const R* lag_in, R* lag_out, const R* cA, const R* cInvB, const R* cCB, const R* cP,
                    const R* cQ, const double* zo, const double* zn, const double* zs, const double* zpt,
                    double* trhs, double* om, double* soln, R* avx, R* avy, R* avz, StateBuf Ssum, int last) {
    const Geo& g = P.g;
    const double beta_1 = 0.5 * (1.0 - beta_s), beta_2 = 0.5 * (1.0 + beta_s);
    k_mt_fast_h<R><<<ter_grid(g, g.nz), ter_block(), 0, st>>>(P, step, lagged, dtau, Sprev, Sst, A, Fmx, Fmy, lag_in,
                                                              lag_out, zo, Ssum);
    k_mt_fast_flux<R><<<ter_grid(g, g.nz + 1), ter_block(), 0, st>>>(P, Sprev, Sst, A, Ssum, zo, zs, zpt, trhs, om);
    k_mt_fast_div<R><<<ter_grid(g, g.nz), ter_block(), 0, st>>>(P, facinv, Sst, zn, Ssum, avx, avy);
    k_mt_col_rhs<R><<<ter_grid(g, g.nz + 1), ter_block(), 0, st>>>(P, dtau, beta_1, beta_2, Sprev, Sst, A, Fcons, Fmz,
                                                                  cP, cQ, zo, zn, zs, zpt, om, trhs, Ssum, soln);
    k_mt_col_sweep<R><<<ter_grid(g, 1), ter_block(), 0, st>>>(P, Sst, cA, cInvB, cCB, Ssum, soln);
    k_mt_col_w<R><<<ter_grid(g, g.nz), ter_block(), 0, st>>>(P, Sprev, Sst, zo, zn, zs, zpt, Ssum, soln);
    k_mt_col_cons<R><<<ter_grid(g, g.nz), ter_block(), 0, st>>>(P, dtau, beta_1, beta_2, facinv, Sprev, A, Fcons, zo, zn,
                                                                om, trhs, soln, avz, Ssum);
    if (!last) k_mt_fast_bc<<<ter_grid(g, g.nz + 1), ter_block(), 0, st>>>(P, Ssum);
}
#if !ERFB_TER_F32
template void launch_mt_fast<double>(const Params&, cudaStream_t, int, int, double, double, double, StateBuf, StateBuf,
                                     StageAux<double>, const double*, const double*, const double*, const double*,
                                     const double*, double*, const double*, const double*, const double*,
                                     const double*, const double*, const double*, const double*, const double*,
                                     const double*, double*, double*, double*, double*, double*, double*, StateBuf, int);
#else
template void launch_mt_fast<float>(const Params&, cudaStream_t, int, int, double, double, double, StateBuf, StateBuf,
                                    StageAux<float>, const float*, const float*, const float*, const float*,
                                    const float*, float*, const float*, const float*, const float*, const float*,
                                    const float*, const double*, const double*, const double*, const double*, double*,
                                    double*, double*, float*, float*, float*, StateBuf, int);
#endif

// ---------------------------------------------------------------------------
// Step diagnostics of a resident state (sum_integrated_quantities /
// volWgtSumMF, IO/ERF_WriteScalarProfiles.cpp:14-60, 378-420): the
// integrals of rho and rho theta over the physical volume (dx dy dz detJ per
// cell; detJ from P.detJ with static terrain, from the nodes of zgrid with
// moving terrain, 1 without terrain) and max |w| over the z faces.
// Fixed-order two-pass reduction, so the result does not depend on
// scheduling.
// ---------------------------------------------------------------------------
constexpr int DIAG_BLOCKS = 592, DIAG_THREADS = 256;
static __global__ void __launch_bounds__(DIAG_THREADS) k_diag_partial(Params P, const double* __restrict__ cons,
                                                               const double* __restrict__ w,
                                                               const double* __restrict__ zgrid,
                                                               double* __restrict__ part) {
    const Geo& g = P.g;
    __shared__ double sm[3][DIAG_THREADS];
    double m = 0.0, rt = 0.0, wm = 0.0;
    const int64_t N = g.ncell, stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += stride) {
        double J = 1.0;
        if (zgrid) {
            const int k = (int)(c / g.sk), r = (int)(c - (int64_t)k * g.sk), j = r / g.nx, i = r - j * g.nx;
            J = mt_detj(zgrid, g, i, j, k);
        } else if (P.ter) {
            J = P.detJ[c];
        }
        m += cons[c] * J;
        rt += cons[N + c] * J;
    }
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < g.nzf; f += stride) wm = fmax(wm, fabs(w[f]));
    sm[0][threadIdx.x] = m; sm[1][threadIdx.x] = rt; sm[2][threadIdx.x] = wm;
    __syncthreads();
    for (int h = DIAG_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            sm[0][threadIdx.x] += sm[0][threadIdx.x + h];
            sm[1][threadIdx.x] += sm[1][threadIdx.x + h];
            sm[2][threadIdx.x] = fmax(sm[2][threadIdx.x], sm[2][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = sm[0][0]; part[3 * blockIdx.x + 1] = sm[1][0]; part[3 * blockIdx.x + 2] = sm[2][0];
    }
}
static __global__ void k_diag_final(Params P, const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double m = 0.0, rt = 0.0, wm = 0.0;
    for (int b = 0; b < nb; ++b) { m += part[3 * b]; rt += part[3 * b + 1]; wm = fmax(wm, part[3 * b + 2]); }
    const double vol = 1.0 / (P.g.dxi * P.g.dyi * P.g.dzi);
    out[0] = m * vol; out[1] = rt * vol; out[2] = wm;
}
#if !ERFB_TER_F32
void launch_diagnostics(const Params& P, cudaStream_t st, const double* cons, const double* w, const double* zgrid,
                        double* part, double* out) {
    k_diag_partial<<<DIAG_BLOCKS, DIAG_THREADS, 0, st>>>(P, cons, w, zgrid, part);
    k_diag_final<<<1, 32, 0, st>>>(P, part, DIAG_BLOCKS, out);
}
#endif
#if !ERFB_TER_F32
int diagnostics_scratch_doubles() { return 3 * DIAG_BLOCKS + 3; }
#endif

// post_timestep's clock (ERF.cpp:547-559 with t_new = t_old + dt)
static __global__ void k_mt_advance_time(double* t, double dt) { *t = *t + dt; }
#if !ERFB_TER_F32
void launch_mt_advance_time(cudaStream_t st, double* tdev, double dt) { k_mt_advance_time<<<1, 1, 0, st>>>(tdev, dt); }
#endif

// ---------------------------------------------------------------------------
// Base state over the terrain, one thread per column: calc_rho_p Newton
// integration from p_sfc at z = 0 through the column's cell centres
// (ERF_InputSoundingData.H:176-256), then erf_enforce_hse with terrain
// (ERF_init1d.cpp:152-241).  Output (nz+2) planes, plane k+1 for level k.
// ---------------------------------------------------------------------------
static __global__ void k_ter_base_state(Params P, const double* __restrict__ zcc, const double* __restrict__ th3,
                                 const double* __restrict__ qv3, double th_s, double qv_s, double p_s,
                                 double* __restrict__ rho0, double* __restrict__ p0o, double* __restrict__ pi0o,
                                 double* __restrict__ th0o) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const double tol = 1.0e-12, grav = P.gravity, rdOcp = P.rdOcp;
    const double RdOCp = R_d / Cp_d;
    const int64_t col = (int64_t)j * g.nx + i, sk = g.sk;
    const int nz = g.nz;
    double pm = p_s;
    double rd = eos_rho_given_theta_p(th_s, p_s, RdOCp, qv_s);
    double zprev = 0.0, qprev = qv_s;
    for (int k = 1; k <= nz; ++k) {
        int64_t c = (int64_t)(k - 1) * sk + col;
        double z = zcc[c];
        double th = th3[c], qv = qv3[c];
        double dzl = z - zprev;
        double rlo = rd * (1. + qprev);
        double C = -pm + 0.5 * rlo * grav * dzl;
        double pk = pm;
        double rk = eos_rho_given_theta_p(th, pk, RdOCp, qv);
        double rhi = rk * (1. + qv);
        double F = pk + 0.5 * rhi * grav * dzl + C;
        if (fabs(F) > tol) {
            int iter = 0;
            double eps = 1.0e-6, ieps = 1.0e6;
            do {
                double hi = eos_rho_given_theta_p(th, pk + eps, RdOCp, qv);
                double lo = eos_rho_given_theta_p(th, pk - eps, RdOCp, qv);
                double dFdp = 1.0 + 0.25 * ieps * (hi - lo) * grav * dzl;
                pk -= F / dFdp;
                rk = eos_rho_given_theta_p(th, pk, RdOCp, qv);
                double rt = rk * (1. + qv);
                F = pk + 0.5 * rt * grav * dzl + C;
                ++iter;
            } while (fabs(F) > tol && iter < 30);
        }
        rho0[(int64_t)k * sk + col] = rk;
        pm = pk; rd = rk; zprev = z; qprev = qv;
    }
    rho0[col] = rho0[sk + col];
    rho0[(int64_t)(nz + 1) * sk + col] = rho0[(int64_t)nz * sk + col];
    auto put = [&](int kk, double pv) {
        int64_t o = (int64_t)kk * sk + col;
        p0o[o] = pv;
        pi0o[o] = eos_exner_p(pv, rdOcp);
        th0o[o] = eos_rt_given_p(pv) / rho0[o];
    };
    double hz = zcc[col];
    double r1 = rho0[sk + col];
    double pprev = p_0 - hz * r1 * grav;
    put(1, pprev);
    put(0, p_0 + hz * r1 * grav);
    for (int k = 1; k <= nz; ++k) {
        int kk = k + 1;
        double dz_loc = zcc[(int64_t)k * sk + col] - zcc[(int64_t)(k - 1) * sk + col];
        double di = 0.5 * (rho0[(int64_t)kk * sk + col] + rho0[(int64_t)(kk - 1) * sk + col]);
        pprev = pprev - dz_loc * di * grav;
        put(kk, pprev);
    }
}
#if !ERFB_TER_F32
void launch_ter_base_state(const Params& P, cudaStream_t st, const double* zcc, const double* th3, const double* qv3,
                           double th_s, double qv_s, double p_s, double* rho0, double* p0, double* pi0, double* th0) {
    dim3 b(32, 4, 1), gr((P.g.nx + 31) / 32, (P.g.ny + 3) / 4, 1);
    k_ter_base_state<<<gr, b, 0, st>>>(P, zcc, th3, qv3, th_s, qv_s, p_s, rho0, p0, pi0, th0);
}
#endif


namespace {

// ---------------------------------------------------------------------------
// Strain rates with terrain (ComputeStrain_T, Diffusion/ERF_ComputeStrain_T.cpp:
// 268-505) at one cell / edge, for velocity accessors U(i,j,k), V, W that
// supply the wall ghosts.  k ranges: cells [0,nz), xy edges [0,nz), xz / yz
// edges [0,nz].
// ---------------------------------------------------------------------------
template <class FU, class FV, class FW>
__device__ __forceinline__ void strain_cc_T(const Params& P, int i, int j, int k, FU U, FV V, FW W, double& s11, double& s22,
                            double& s33) {
    const double dxi = P.g.dxi, dyi = P.g.dyi, dzi = P.g.dzi;
    double GradUz, GradVz;
    if (k == 0 && P.g.zlo_noslip) {
        GradUz = 0.5 * dzi * ((-(8. / 3.) * U(i, j, k - 1) + 3. * U(i, j, k) - (1. / 3.) * U(i, j, k + 1))
                              + (-(8. / 3.) * U(i - 1, j, k - 1) + 3. * U(i - 1, j, k) - (1. / 3.) * U(i - 1, j, k + 1)));
        GradVz = 0.5 * dzi * ((-(8. / 3.) * V(i, j, k - 1) + 3. * V(i, j, k) - (1. / 3.) * V(i, j, k + 1))
                              + (-(8. / 3.) * V(i, j - 1, k - 1) + 3. * V(i, j - 1, k) - (1. / 3.) * V(i, j - 1, k + 1)));
    } else {
        GradUz = 0.25 * dzi * (U(i, j, k + 1) / 1.0 + U(i - 1, j, k + 1) / 1.0 - U(i, j, k - 1) / 1.0 - U(i - 1, j, k - 1) / 1.0);
        GradVz = 0.25 * dzi * (V(i, j, k + 1) / 1.0 + V(i, j - 1, k + 1) / 1.0 - V(i, j, k - 1) / 1.0 - V(i, j - 1, k - 1) / 1.0);
    }
    double mxi = hxi_cc(P, i, j, k), meta = heta_cc(P, i, j, k), mz = detJ_at(P, i, j, k);
    s11 = ((U(i + 1, j, k) / 1.0 - U(i, j, k) / 1.0) * dxi - (mxi / mz) * GradUz) * 1.0 * 1.0;
    s22 = ((V(i, j + 1, k) / 1.0 - V(i, j, k) / 1.0) * dyi - (meta / mz) * GradVz) * 1.0 * 1.0;
    s33 = (W(i, j, k + 1) - W(i, j, k)) * dzi / mz;
}
template <class FU, class FV>
__device__ __forceinline__ double strain12_T(const Params& P, int i, int j, int k, FU U, FV V) {
    const double dxi = P.g.dxi, dyi = P.g.dyi, dzi = P.g.dzi;
    double GradUz, GradVz;
    if (k == 0 && P.g.zlo_noslip) {
        GradUz = 0.5 * dzi * ((-(8. / 3.) * U(i, j, k - 1) + 3. * U(i, j, k) - (1. / 3.) * U(i, j, k + 1))
                              + (-(8. / 3.) * U(i, j - 1, k - 1) + 3. * U(i, j - 1, k) - (1. / 3.) * U(i, j - 1, k + 1)));
        GradVz = 0.5 * dzi * ((-(8. / 3.) * V(i, j, k - 1) + 3. * V(i, j, k) - (1. / 3.) * V(i, j, k + 1))
                              + (-(8. / 3.) * V(i - 1, j, k - 1) + 3. * V(i - 1, j, k) - (1. / 3.) * V(i - 1, j, k + 1)));
    } else {
        GradUz = 0.25 * dzi * (U(i, j, k + 1) / 1.0 + U(i, j - 1, k + 1) / 1.0 - U(i, j, k - 1) / 1.0 - U(i, j - 1, k - 1) / 1.0);
        GradVz = 0.25 * dzi * (V(i, j, k + 1) / 1.0 + V(i - 1, j, k + 1) / 1.0 - V(i, j, k - 1) / 1.0 - V(i - 1, j, k - 1) / 1.0);
    }
    double mxi = hxi_EK(P, i, j, k), meta = heta_EK(P, i, j, k), mz = hzeta_EK(P, i, j, k);
    return 0.5 * ((U(i, j, k) / 1.0 - U(i, j - 1, k) / 1.0) * dyi + (V(i, j, k) / 1.0 - V(i - 1, j, k) / 1.0) * dxi
                  - (meta / mz) * GradUz - (mxi / mz) * GradVz) * 1.0 * 1.0;
}
template <class FU, class FW>
__device__ __forceinline__ double strain13_T(const Params& P, int i, int j, int k, FU U, FW W) {
    const double dxi = P.g.dxi, dzi = P.g.dzi;
    const int nz = P.g.nz;
    double mz = hzeta_EJ(P, i, j, k);
    if (k == 0) {
        double GradWz = 0.5 * dzi * (W(i, j, k + 1) + W(i - 1, j, k + 1) - W(i, j, k) - W(i - 1, j, k));
        double mxi = hxi_EJ(P, i, j, k);
        if (P.g.zlo_noslip)
            return 0.5 * ((-(8. / 3.) * U(i, j, k - 1) + 3. * U(i, j, k) - (1. / 3.) * U(i, j, k + 1)) * dzi / mz
                          + ((W(i, j, k) - W(i - 1, j, k)) * dxi - (mxi / mz) * GradWz) * 1.0);
        return 0.5 * ((U(i, j, k) - U(i, j, k - 1)) * dzi / mz + ((W(i, j, k) - W(i - 1, j, k)) * dxi - (mxi / mz) * GradWz) * 1.0);
    }
    if (k == nz) {
        if (P.g.zhi_noslip)
            return 0.5 * (-(-(8. / 3.) * U(i, j, k) + 3. * U(i, j, k - 1) - (1. / 3.) * U(i, j, k - 2)) * dzi / mz
                          + (W(i, j, k) - W(i - 1, j, k)) * dxi * 1.0);
        return 0.5 * ((U(i, j, k) - U(i, j, k - 1)) * dzi / mz + (W(i, j, k) - W(i - 1, j, k)) * dxi * 1.0);
    }
    double GradWz = 0.25 * dzi * (W(i, j, k + 1) + W(i - 1, j, k + 1) - W(i, j, k - 1) - W(i - 1, j, k - 1));
    double mxi = hxi_EJ(P, i, j, k);
    return 0.5 * ((U(i, j, k) - U(i, j, k - 1)) * dzi / mz + ((W(i, j, k) - W(i - 1, j, k)) * dxi - (mxi / mz) * GradWz) * 1.0);
}
template <class FV, class FW>
__device__ __forceinline__ double strain23_T(const Params& P, int i, int j, int k, FV V, FW W) {
    const double dyi = P.g.dyi, dzi = P.g.dzi;
    const int nz = P.g.nz;
    double mz = hzeta_EI(P, i, j, k);
    if (k == 0) {
        double GradWz = 0.5 * dzi * (W(i, j, k + 1) + W(i, j - 1, k + 1) - W(i, j, k) - W(i, j - 1, k));
        double meta = heta_EI(P, i, j, k);
        if (P.g.zlo_noslip)
            return 0.5 * ((-(8. / 3.) * V(i, j, k - 1) + 3. * V(i, j, k) - (1. / 3.) * V(i, j, k + 1)) * dzi / mz
                          + ((W(i, j, k) - W(i, j - 1, k)) * dyi - (meta / mz) * GradWz) * 1.0);
        return 0.5 * ((V(i, j, k) - V(i, j, k - 1)) * dzi / mz + ((W(i, j, k) - W(i, j - 1, k)) * dyi - (meta / mz) * GradWz) * 1.0);
    }
    if (k == nz) {
        if (P.g.zhi_noslip)
            return 0.5 * (-(-(8. / 3.) * V(i, j, k) + 3. * V(i, j, k - 1) - (1. / 3.) * V(i, j, k - 2)) * dzi / mz
                          + (W(i, j, k) - W(i, j - 1, k)) * dyi * 1.0);
        return 0.5 * ((V(i, j, k) - V(i, j, k - 1)) * dzi / mz + (W(i, j, k) - W(i, j - 1, k)) * dyi * 1.0);
    }
    double GradWz = 0.25 * dzi * (W(i, j, k + 1) + W(i, j - 1, k + 1) - W(i, j, k - 1) - W(i, j - 1, k - 1));
    double meta = heta_EI(P, i, j, k);
    return 0.5 * ((V(i, j, k) - V(i, j, k - 1)) * dzi / mz + ((W(i, j, k) - W(i, j - 1, k)) * dyi - (meta / mz) * GradWz) * 1.0);
}
// ComputeSmnSmn (Diffusion/ERF_EddyViscosity.H:31-83) from the terrain strains
template <class FU, class FV, class FW>
__device__ __forceinline__ double smnsmn_T(const Params& P, int i, int j, int k, FU U, FV V, FW W) {
    double s11, s22, s33;
    strain_cc_T(P, i, j, k, U, V, W, s11, s22, s33);
    double s12 = 0.25 * (strain12_T(P, i, j, k, U, V) + strain12_T(P, i, j + 1, k, U, V) + strain12_T(P, i + 1, j, k, U, V)
                         + strain12_T(P, i + 1, j + 1, k, U, V));
    double s13 = 0.25 * (strain13_T(P, i, j, k, U, W) + strain13_T(P, i, j, k + 1, U, W) + strain13_T(P, i + 1, j, k, U, W)
                         + strain13_T(P, i + 1, j, k + 1, U, W));
    double s23 = 0.25 * (strain23_T(P, i, j, k, V, W) + strain23_T(P, i, j, k + 1, V, W) + strain23_T(P, i, j + 1, k, V, W)
                         + strain23_T(P, i, j + 1, k + 1, V, W));
    return s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * s12 * s12 + 2.0 * s13 * s13 + 2.0 * s23 * s23;
}

// Base-state pressure at the cell of linear index c (level k) with terrain.
__device__ __forceinline__ double p0_at(const Params& P, int64_t c, int k) {
    return P.ter ? P.p0[c + P.g.sk] : P.p0[k + 1];
}
template <class R>
__device__ __forceinline__ void stage_aux_ter(const Params& P, const double* __restrict__ cons, StageAux<R> A,
                                              int64_t c, int k) {
    const int64_t N = P.g.ncell;
    double rho = cons[c];
    double rt = cons[N + c];
    A.prim[c] = R(rt / rho);
    for (int n = 1; n < P.nprim; ++n) A.prim[n * N + c] = R(cons[(n + 1) * N + c] / rho);
    A.pi[c] = R(eos_exner(rt, P.rdOcp));
    double qv = P.moist ? cons[5 * N + c] / rho : 0.0;
    A.pp[c] = R(eos_p(rt, qv) - p0_at(P, c, k));
    if (!(rt > 0.0) || !(rho > 0.0)) atomicOr(P.status, ST_BADSTATE);
}

}  // namespace

// ---------------------------------------------------------------------------
// Step prologue with terrain.  The old velocities give the momenta through
// the V -> M -> V -> M round trip of apply_bcs(state_old) (as without
// terrain); w on the ground and on the lid is WFromOmega(Omega = 0) of the
// round-tripped u, v (ERF_BoundaryConditions_zvel.cpp:200-262).  The eddy
// viscosity uses the input velocities with w from the same condition, the
// terrain strain and a local filter width (dz / h_zeta;
// ERF_ComputeTurbulentViscosity.cpp:85-229).
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_ter_step_begin(Params P, const double* __restrict__ cons, const double* __restrict__ uo,
                                 const double* __restrict__ vo, const double* __restrict__ wo, StateBuf S,
                                 double* __restrict__ un, double* __restrict__ vn, double* __restrict__ wn,
                                 StageAux<R> A, R* __restrict__ mut, TkeBuf<R> tke) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    int64_t c = cidx(g, i, j, k);
    double rho = cons[c];
    // round-tripped old velocity at a face (the value apply_bcs leaves), with
    // the wall ghost
    auto urt = [&](int ii, int jj, int kk) {
        ii = wrap(ii, g.nx); jj = wrap(jj, g.ny);
        int kc = clampk(kk, nz);
        if ((kk < 0 && g.zlo_noslip) || (kk >= nz && g.zhi_noslip)) return 0.0;
        double rs = cons[cidx(g, ii, jj, kc)] + cons[cidx(g, wrap(ii - 1, g.nx), jj, kc)];
        double m0 = (uo[cidx(g, ii, jj, kc)] * 0.5) * rs;
        return (m0 * 2.0) / rs;
    };
    auto vrt = [&](int ii, int jj, int kk) {
        ii = wrap(ii, g.nx); jj = wrap(jj, g.ny);
        int kc = clampk(kk, nz);
        if ((kk < 0 && g.zlo_noslip) || (kk >= nz && g.zhi_noslip)) return 0.0;
        double rs = cons[cidx(g, ii, jj, kc)] + cons[cidx(g, ii, wrap(jj - 1, g.ny), kc)];
        double m0 = (vo[cidx(g, ii, jj, kc)] * 0.5) * rs;
        return (m0 * 2.0) / rs;
    };
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
    if (k == 0 && !P.mt_zt) {
        double wb = w_from_omega(P, i, j, 0, 0.0, urt, vrt);
        S.mz[c] = (wb * 0.5) * (rho + rho); wn[c] = wb;
    } else {
        // (a moving ground keeps its w: the moving-terrain branch of
        // impose_vertical_zvel_bcs sets nothing; rho below the ground is
        // the foextrap ghost)
        double rs = rho + (k == 0 ? rho : cons[c - g.sk]);
        double m0 = (wo[c] * 0.5) * rs, w1 = (m0 * 2.0) / rs;
        S.mz[c] = (w1 * 0.5) * rs; wn[c] = w1;
    }
    if (k == nz - 1) {
        double wt = w_from_omega(P, i, j, nz, 0.0, urt, vrt);
        S.mz[c + g.sk] = (wt * 0.5) * (rho + rho); wn[c + g.sk] = wt;
    }
    if (!(fabs(uo[c]) <= DBL_MAX) || !(fabs(vo[c]) <= DBL_MAX) || !(fabs(wo[c]) <= DBL_MAX))
        atomicOr(P.status, ST_NAN);
    stage_aux_ter<R>(P, cons, A, c, k);

    if (P.les == ERF_LES_NONE) return;
    // input velocities with their wall ghosts; w on the walls from Omega = 0
    auto U = [&](int ii, int jj, int kk) { return tvel(uo, g, ii, jj, kk); };
    auto V = [&](int ii, int jj, int kk) { return tvel(vo, g, ii, jj, kk); };
    auto W = [&](int ii, int jj, int kk) {
        if (kk <= 0 || kk >= nz) return w_from_omega(P, ii, jj, kk <= 0 ? 0 : nz, 0.0, U, V);
        return wvel(wo, g, ii, jj, kk);
    };
    double dzInv = g.dzi / hzeta_cc(P, i, j, k);
    double cellVolMsf = 1.0 / (g.dxi * 1.0 * g.dyi * 1.0 * dzInv);
    double DeltaMsf = pow(cellVolMsf, 1.0 / 3.0);
    if (P.les == ERF_LES_SMAGORINSKY) {
        double S2 = smnsmn_T(P, i, j, k, U, V, W);
        double CsDeltaSqrMsf = P.Cs * P.Cs * DeltaMsf * DeltaMsf;
        mut[c] = R(CsDeltaSqrMsf * rho * sqrt(2.0 * S2));
    } else if (P.les == ERF_LES_DEARDORFF) {
        const int64_t N = g.ncell;
        const int kp = min(k + 1, nz - 1), km = max(k - 1, 0);
        double dtheta_dz = 0.5 * (cons[N + cidx(g, i, j, kp)] / cons[cidx(g, i, j, kp)] -
                                  cons[N + cidx(g, i, j, km)] / cons[cidx(g, i, j, km)]) * dzInv;
        double E = fmax(cons[2 * N + c] / rho, 0.0);
        double strat = P.g_over_theta0 * dtheta_dz;
        double length;
        if (strat <= 2.220446049250313e-16) {
            length = DeltaMsf;
        } else {
            length = 0.76 * sqrt(E / strat);
            length = fmin(length, DeltaMsf);
            length = fmax(length, 0.001 * DeltaMsf);
        }
        double K = rho * P.Ck * length * sqrt(E);
        mut[c] = R(K);
        tke.kthv[c] = R((1. + 2. * length / DeltaMsf) * K);
        double Ce = ((P.Ce_wall > 0) && (k == 0)) ? P.Ce_wall : 1.9 * P.Ck + P.Ce_lcoeff * length / DeltaMsf;
        tke.diss[c] = R(rho * Ce * (E * sqrt(E)) / length);
    }
}

// ---------------------------------------------------------------------------
// make_tau_terms with terrain, pass 1: strain rates of the stage velocities,
// tau_ii less a third of the expansion rate (from the contravariant
// velocity, ERF_make_tau_terms.cpp:185-216), S12 / S13 / S23 on the edges,
// and SmnSmn of the first stage for the Deardorff shear production.
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(128, TER_MINB_STRAIN) k_ter_strain(Params P, int nrk, const double* __restrict__ u, const double* __restrict__ v,
                             const double* __restrict__ w, TerBuf<R> T, TkeBuf<R> tke) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    int64_t c = cidx(g, i, j, k);
    auto U = [&](int ii, int jj, int kk) { return tvel(u, g, ii, jj, kk); };
    auto V = [&](int ii, int jj, int kk) { return tvel(v, g, ii, jj, kk); };
    auto W = [&](int ii, int jj, int kk) { return wvel(w, g, ii, jj, kk); };
    auto om = [&](int kk) { return (kk == 0) ? 0. : omega_from_w(P, i, j, kk, W(i, j, kk), U, V); };
    double mhi = hzeta_I(P, i + 1, j, k), mlo = hzeta_I(P, i, j, k);
    double nhi = hzeta_J(P, i, j + 1, k), nlo = hzeta_J(P, i, j, k);
    double rate = (U(i + 1, j, k) / 1.0 * mhi - U(i, j, k) / 1.0 * mlo) * g.dxi * 1.0
                  + (V(i, j + 1, k) / 1.0 * nhi - V(i, j, k) / 1.0 * nlo) * g.dyi * 1.0
                  + (om(k + 1) - om(k)) * g.dzi;
    double er = rate / detJ_at(P, i, j, k);
    double s11, s22, s33;
    strain_cc_T(P, i, j, k, U, V, W, s11, s22, s33);
    const double OneThird = (1. / 3.);
    T.s11[c] = R(s11 - OneThird * er);
    T.s22[c] = R(s22 - OneThird * er);
    T.s33[c] = R(s33 - OneThird * er);
    T.s12[c] = R(strain12_T(P, i, j, k, U, V));
    T.s13[c] = R(strain13_T(P, i, j, k, U, W));
    T.s23[c] = R(strain23_T(P, i, j, k, V, W));
    if (k == nz - 1) {
        T.s13[c + g.sk] = R(strain13_T(P, i, j, nz, U, W));
        T.s23[c + g.sk] = R(strain23_T(P, i, j, nz, V, W));
    }
    if (P.les == ERF_LES_DEARDORFF && nrk == 0) tke.smn[c] = R(smnsmn_T(P, i, j, k, U, V, W));
}

// ---------------------------------------------------------------------------
// Pass 2: ComputeStressVarVisc_T (Diffusion/ERF_ComputeStress_T.cpp:302-577).
// tau33 takes the raw S31 / S32 cross terms; tau13 / tau23 the tau11 / tau12
// (tau21 / tau22) averages, linearly extrapolated to the bottom and top
// faces; tau31 = -mu h_zeta S13, tau32 likewise; tau11, tau22 and tau12
// (= tau21) carry h_zeta.
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(128, TER_MINB_STRESS) k_ter_stress(Params P, const double* __restrict__ cons, const R* __restrict__ mut, TerBuf<R> T,
                             R* __restrict__ t11, R* __restrict__ t22, R* __restrict__ t33, R* __restrict__ t12,
                             R* __restrict__ t13, R* __restrict__ t23) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    int64_t c = cidx(g, i, j, k);
    const double mu_eff = P.mu_eff;
    auto rA = [&](int ii, int jj, int kk) { return P.use_consA ? ccw(cons, g, ii, jj, kk) * mu_eff : mu_eff; };
    auto mt = [&](int ii, int jj, int kk) { return P.use_turb ? ccw(mut, g, ii, jj, kk) : 0.0; };
    auto S11 = [&](int ii, int jj, int kk) { return ccw(T.s11, g, ii, jj, kk); };
    auto S22 = [&](int ii, int jj, int kk) { return ccw(T.s22, g, ii, jj, kk); };
    auto E12 = [&](int ii, int jj, int kk) { return double(T.s12[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), clampk(kk, nz))]); };
    auto E13 = [&](int ii, int jj, int kk) { return double(T.s13[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    auto E23 = [&](int ii, int jj, int kk) { return double(T.s23[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    {   // tau33
        double mxi = hxi_cc(P, i, j, k), meta = heta_cc(P, i, j, k);
        double t31b = 0.25 * (E13(i, j, k) + E13(i + 1, j, k) + E13(i, j, k + 1) + E13(i + 1, j, k + 1));
        double t32b = 0.25 * (E23(i, j, k) + E23(i, j + 1, k) + E23(i, j, k + 1) + E23(i, j + 1, k + 1));
        double mu_tot = rA(i, j, k) + 2.0 * mt(i, j, k);
        double v33 = double(T.s33[c]);
        v33 -= mxi * t31b + meta * t32b;
        v33 *= -mu_tot;
        t33[c] = R(v33);
        double mz = detJ_at(P, i, j, k);
        t11[c] = R(double(T.s11[c]) * (-mu_tot * mz));
        t22[c] = R(double(T.s22[c]) * (-mu_tot * mz));
    }
    {   // tau12 (= tau21) on the xy edge (i,j,k)
        double mz = hzeta_EK(P, i, j, k);
        double mu_bar = 0.25 * (mt(i - 1, j, k) + mt(i, j, k) + mt(i - 1, j - 1, k) + mt(i, j - 1, k));
        double ra_bar = 0.25 * (rA(i - 1, j, k) + rA(i, j, k) + rA(i - 1, j - 1, k) + rA(i, j - 1, k));
        double mu_tot = ra_bar + 2.0 * mu_bar;
        t12[c] = R(double(T.s12[c]) * (-mu_tot * mz));
    }
    for (int kk = k; kk <= (k == nz - 1 ? nz : k); ++kk) {
        int64_t e = cidx(g, i, j, kk);
        double t11b, t12b, t21b, t22b;
        if (kk == 0) {
            double a = 0.5 * (S11(i, j, kk) + S11(i - 1, j, kk)), b = 0.5 * (S11(i, j, kk + 1) + S11(i - 1, j, kk + 1));
            t11b = 1.5 * a - 0.5 * b;
            double c1 = 0.5 * (E12(i, j, kk) + E12(i, j + 1, kk)), d = 0.5 * (E12(i, j, kk + 1) + E12(i, j + 1, kk + 1));
            t12b = 1.5 * c1 - 0.5 * d;
            double a2 = 0.5 * (E12(i, j, kk) + E12(i + 1, j, kk)), b2 = 0.5 * (E12(i, j, kk + 1) + E12(i + 1, j, kk + 1));
            t21b = 1.5 * a2 - 0.5 * b2;
            double c2 = 0.5 * (S22(i, j, kk) + S22(i, j - 1, kk)), d2 = 0.5 * (S22(i, j, kk + 1) + S22(i, j - 1, kk + 1));
            t22b = 1.5 * c2 - 0.5 * d2;
        } else if (kk == nz) {
            double lo = 0.5 * (S11(i, j, kk - 2) + S11(i - 1, j, kk - 2)), hi = 0.5 * (S11(i, j, kk - 1) + S11(i - 1, j, kk - 1));
            t11b = 1.5 * hi - 0.5 * lo;
            double lo2 = 0.5 * (E12(i, j, kk - 2) + E12(i, j + 1, kk - 2)), hi2 = 0.5 * (E12(i, j, kk - 1) + E12(i, j + 1, kk - 1));
            t12b = 1.5 * hi2 - 0.5 * lo2;
            double lo3 = 0.5 * (E12(i, j, kk - 2) + E12(i + 1, j, kk - 2)), hi3 = 0.5 * (E12(i, j, kk - 1) + E12(i + 1, j, kk - 1));
            t21b = 1.5 * hi3 - 0.5 * lo3;
            double lo4 = 0.5 * (S22(i, j, kk - 2) + S22(i, j - 1, kk - 2)), hi4 = 0.5 * (S22(i, j, kk - 1) + S22(i, j - 1, kk - 1));
            t22b = 1.5 * hi4 - 0.5 * lo4;
        } else {
            t11b = 0.25 * (S11(i, j, kk) + S11(i - 1, j, kk) + S11(i, j, kk - 1) + S11(i - 1, j, kk - 1));
            t12b = 0.25 * (E12(i, j, kk) + E12(i, j + 1, kk) + E12(i, j, kk - 1) + E12(i, j + 1, kk - 1));
            t21b = 0.25 * (E12(i, j, kk) + E12(i + 1, j, kk) + E12(i, j, kk - 1) + E12(i + 1, j, kk - 1));
            t22b = 0.25 * (S22(i, j, kk) + S22(i, j - 1, kk) + S22(i, j, kk - 1) + S22(i, j - 1, kk - 1));
        }
        {
            double mxi = hxi_EJ(P, i, j, kk), meta = heta_EJ(P, i, j, kk), mz = hzeta_EJ(P, i, j, kk);
            double mu_bar = 0.25 * (mt(i - 1, j, kk) + mt(i, j, kk) + mt(i - 1, j, kk - 1) + mt(i, j, kk - 1));
            double ra_bar = 0.25 * (rA(i - 1, j, kk) + rA(i, j, kk) + rA(i - 1, j, kk - 1) + rA(i, j, kk - 1));
            double mu_tot = ra_bar + 2.0 * mu_bar;
            double s13 = double(T.s13[e]);
            double v13 = s13;
            v13 -= mxi * t11b + meta * t12b;
            v13 *= -mu_tot;
            t13[e] = R(v13);
            T.t31[e] = R(s13 * (-mu_tot * mz));
        }
        {
            double mxi = hxi_EI(P, i, j, kk), meta = heta_EI(P, i, j, kk), mz = hzeta_EI(P, i, j, kk);
            double mu_bar = 0.25 * (mt(i, j - 1, kk) + mt(i, j, kk) + mt(i, j - 1, kk - 1) + mt(i, j, kk - 1));
            double ra_bar = 0.25 * (rA(i, j - 1, kk) + rA(i, j, kk) + rA(i, j - 1, kk - 1) + rA(i, j, kk - 1));
            double mu_tot = ra_bar + 2.0 * mu_bar;
            double s23 = double(T.s23[e]);
            double v23 = s23;
            v23 -= mxi * t21b + meta * t22b;
            v23 *= -mu_tot;
            t23[e] = R(v23);
            T.t32[e] = R(s23 * (-mu_tot * mz));
        }
    }
}

namespace {
// Scalar diffusion with terrain (DiffusionSrcForState_T,
// Diffusion/ERF_DiffusionSrcForState_T.cpp:207-738) for one primitive field:
// metric-corrected x / y fluxes, z fluxes with the cross terms (extrapolated
// at the bottom and top faces), x / y fluxes scaled by h_zeta, divergence
// over detJ.  kv, when given, is the vertical diffusivity (Deardorff Theta_v).
template <class R>
struct DiffT {
    const Params& P;
    const double* rho;
    const R* phi;
    const R* mut;
    const R* kv;
    double ae, fac;
    const R* fxr = nullptr;   // raw face fluxes from k_ter_rawflux, when given
    const R* fyr = nullptr;
    __device__ __forceinline__ double p(int i, int j, int k) const { return ccw(phi, P.g, i, j, k); }
    __device__ __forceinline__ double mu(int i, int j, int k) const { return ccw(mut, P.g, i, j, k) * fac; }
    __device__ __forceinline__ double xraw(int i, int j, int k) const {
        const Geo& g = P.g;
        double rA = P.use_consA ? (0.5 * (ccw(rho, g, i, j, k) + ccw(rho, g, i - 1, j, k))) * ae : ae;
        if (P.use_turb) rA += 0.5 * (mu(i, j, k) + mu(i - 1, j, k));
        double mxi = hxi_I(P, i, j, k), mz = hzeta_I(P, i, j, k);
        double GradCz = 0.25 * g.dzi * (p(i, j, k + 1) + p(i - 1, j, k + 1) - p(i, j, k - 1) - p(i - 1, j, k - 1));
        double GradCx = g.dxi * (p(i, j, k) - p(i - 1, j, k));
        return -rA * 1.0 * (GradCx - (mxi / mz) * GradCz);
    }
    __device__ __forceinline__ double yraw(int i, int j, int k) const {
        const Geo& g = P.g;
        double rA = P.use_consA ? (0.5 * (ccw(rho, g, i, j, k) + ccw(rho, g, i, j - 1, k))) * ae : ae;
        if (P.use_turb) rA += 0.5 * (mu(i, j, k) + mu(i, j - 1, k));
        double meta = heta_J(P, i, j, k), mz = hzeta_J(P, i, j, k);
        double GradCz = 0.25 * g.dzi * (p(i, j, k + 1) + p(i, j - 1, k + 1) - p(i, j, k - 1) - p(i, j - 1, k - 1));
        double GradCy = g.dyi * (p(i, j, k) - p(i, j - 1, k));
        return -rA * 1.0 * (GradCy - (meta / mz) * GradCz);
    }
    __device__ __forceinline__ double xr(int i, int j, int k) const {
        if (fxr) return double(fxr[cidx(P.g, wrap(i, P.g.nx), wrap(j, P.g.ny), k)]);
        return xraw(i, j, k);
    }
    __device__ __forceinline__ double yr(int i, int j, int k) const {
        if (fyr) return double(fyr[cidx(P.g, wrap(i, P.g.nx), wrap(j, P.g.ny), k)]);
        return yraw(i, j, k);
    }
    // z-face flux (k in [0, nz]); raw receives the flux before the cross terms
    __device__ __forceinline__ double zflux(int i, int j, int k, double& raw) const {
        const Geo& g = P.g;
        const int nz = g.nz;
        double rA = P.use_consA ? (0.5 * (ccw(rho, g, i, j, k) + ccw(rho, g, i, j, k - 1))) * ae : ae;
        if (P.use_turb) {
            if (kv) rA += 0.5 * (ccw(kv, g, i, j, k) + ccw(kv, g, i, j, k - 1));
            else rA += 0.5 * (mu(i, j, k) + mu(i, j, k - 1));
        }
        double GradCz = g.dzi * (p(i, j, k) - p(i, j, k - 1));
        double fz = -rA * GradCz / 1.0;
        raw = fz;
        double mxi = hxi_K(P, i, j, k), meta = heta_K(P, i, j, k), xb, yb;
        if (k == 0) {
            double xlo = 0.5 * (xr(i, j, k) + xr(i + 1, j, k)), xhi = 0.5 * (xr(i, j, k + 1) + xr(i + 1, j, k + 1));
            xb = 1.5 * xlo - 0.5 * xhi;
            double ylo = 0.5 * (yr(i, j, k) + yr(i, j + 1, k)), yhi = 0.5 * (yr(i, j, k + 1) + yr(i, j + 1, k + 1));
            yb = 1.5 * ylo - 0.5 * yhi;
        } else if (k == nz) {
            double xlo = 0.5 * (xr(i, j, k - 2) + xr(i + 1, j, k - 2)), xhi = 0.5 * (xr(i, j, k - 1) + xr(i + 1, j, k - 1));
            xb = 1.5 * xhi - 0.5 * xlo;
            double ylo = 0.5 * (yr(i, j, k - 2) + yr(i, j + 1, k - 2)), yhi = 0.5 * (yr(i, j, k - 1) + yr(i, j + 1, k - 1));
            yb = 1.5 * yhi - 0.5 * ylo;
        } else {
            xb = 0.25 * (xr(i, j, k) + xr(i + 1, j, k) + xr(i, j, k - 1) + xr(i + 1, j, k - 1));
            yb = 0.25 * (yr(i, j, k) + yr(i, j + 1, k) + yr(i, j, k - 1) + yr(i, j + 1, k - 1));
        }
        fz -= mxi * xb + meta * yb;
        return fz;
    }
    // divergence over detJ (the amount the reference subtracts from the RHS)
    __device__ __forceinline__ double div(int i, int j, int k, double& raw_lo, double& raw_hi) const {
        const Geo& g = P.g;
        double fxl = xr(i, j, k) * hzeta_I(P, i, j, k), fxh = xr(i + 1, j, k) * hzeta_I(P, i + 1, j, k);
        double fyl = yr(i, j, k) * hzeta_J(P, i, j, k), fyh = yr(i, j + 1, k) * hzeta_J(P, i, j + 1, k);
        double fzl = zflux(i, j, k, raw_lo), fzh = zflux(i, j, k + 1, raw_hi);
        double s = (fxh - fxl) * g.dxi * 1.0 + (fyh - fyl) * g.dyi * 1.0 + (fzh - fzl) * g.dzi;
        return s / detJ_at(P, i, j, k);
    }
};

// Contravariant momentum Omega at z-face (i,j,k) of a state whose face
// velocities are u, v (for the momentum ghost above the lid):
// 0 at the ground, OmegaFromW inside and at the lid (ERF_slow_rhs_pre.cpp:365-420).
__device__ __forceinline__ double omega_mom(const Params& P, StateBuf S, const double* u, const double* v, int i, int j, int k) {
    const Geo& g = P.g;
    if (k <= 0) return 0.;
    auto MX = [&](int ii, int jj, int kk) {
        ii = wrap(ii, g.nx); jj = wrap(jj, g.ny);
        if (kk < g.nz) return S.mx[cidx(g, ii, jj, kk)];
        // momentum ghost above the lid: V2M of the tangential ghost velocity
        int kt = g.nz - 1;
        double rs = S.cons[cidx(g, ii, jj, kt)] + S.cons[cidx(g, wrap(ii - 1, g.nx), jj, kt)];
        return tvel(u, g, ii, jj, g.nz) * 0.5 * rs;
    };
    auto MY = [&](int ii, int jj, int kk) {
        ii = wrap(ii, g.nx); jj = wrap(jj, g.ny);
        if (kk < g.nz) return S.my[cidx(g, ii, jj, kk)];
        int kt = g.nz - 1;
        double rs = S.cons[cidx(g, ii, jj, kt)] + S.cons[cidx(g, ii, wrap(jj - 1, g.ny), kt)];
        return tvel(v, g, ii, jj, g.nz) * 0.5 * rs;
    };
    double rw = S.mz[cidx(g, wrap(i, g.nx), wrap(j, g.ny), k)];
    double om = omega_from_w(P, i, j, k, rw, MX, MY);
    if (P.mt_zt && k < g.nz) {   // the grid's own motion (ERF_slow_rhs_pre.cpp:389-398); z_t = 0 at the lid
        const int ii = wrap(i, g.nx), jj = wrap(j, g.ny);
        const double rho_at_face = 0.5 * (S.cons[cidx(g, ii, jj, k)] + S.cons[cidx(g, ii, jj, k - 1)]);
        om -= rho_at_face * P.mt_zt[cidx(g, ii, jj, k)];
    }
    return om;
}

// Face interpolation of a cell field along x / y / z (the stencil's unused
// entries are zero); upw the advecting flux.  TS >= 0 fixes the scheme at
// compile time, TS < 0 takes it from `type` at run time (same arithmetic).
template <int TS, class FP>
__device__ __forceinline__ double interp_dir(int dir, int i, int j, int k, FP phi, int type, double upw, double frac) {
    double s[6];
    const int w = width_of<TS>(type);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        bool used = (off >= -w && off <= w - 1);
        s[m] = used ? phi(i + (dir == 0 ? off : 0), j + (dir == 1 ? off : 0), k + (dir == 2 ? off : 0)) : 0.0;
    }
    return interp_of<TS, double>(type, s, upw, frac);
}
}  // namespace

// ---------------------------------------------------------------------------
// Raw diffusive face fluxes of DiffusionSrcForState_T (before the cross
// terms and the h_zeta scaling) for up to two fields, one thread per cell
// writing its low x and y faces, so that the z-face cross terms read them
// instead of re-evaluating them.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_ter_rawflux(Params P, const double* __restrict__ rho, const R* __restrict__ mut,
                              const R* __restrict__ phiA, double aeA, double facA, R* __restrict__ fxA,
                              R* __restrict__ fyA, const R* __restrict__ phiB, double aeB, double facB,
                              R* __restrict__ fxB, R* __restrict__ fyB) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    int64_t c = cidx(g, i, j, k);
    DiffT<R> A{P, rho, phiA, mut, nullptr, aeA, facA};
    fxA[c] = R(A.xraw(i, j, k));
    fyA[c] = R(A.yraw(i, j, k));
    if (phiB) {
        DiffT<R> B{P, rho, phiB, mut, nullptr, aeB, facB};
        fxB[c] = R(B.xraw(i, j, k));
        fyB[c] = R(B.yraw(i, j, k));
    }
}

// ---------------------------------------------------------------------------
// Slow RHS of rho and rho*theta with terrain (ERF_slow_rhs_pre.cpp:365-500):
// Omega, AdvectionSrcForRho with the face areas (ax = h_zeta at x faces,
// ay likewise, az = 1) over detJ, the average momenta, theta advection with
// the dycore scheme, DiffusionSrcForState_T and hfx_z.
// ---------------------------------------------------------------------------
template <class R, int HT, int VT>
__global__ void __launch_bounds__(128, TER_MINB_SLOW_CELL) k_ter_slow_cell(Params P, StateBuf S, StageAux<R> A, const double* __restrict__ u,
                                const double* __restrict__ v, const R* __restrict__ mut, TkeBuf<R> tke, TerBuf<R> T,
                                R* __restrict__ Fcons, R* __restrict__ avx, R* __restrict__ avy, R* __restrict__ avz) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    const int64_t N = g.ncell;
    int64_t c = cidx(g, i, j, k);
    auto fxm = [&](int ii, int jj, int kk) {   // ax * rho_u
        return hzeta_I(P, ii, jj, kk) * S.mx[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)] / 1.0;
    };
    auto fym = [&](int ii, int jj, int kk) {
        return hzeta_J(P, ii, jj, kk) * S.my[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)] / 1.0;
    };
    auto fzm = [&](int ii, int jj, int kk) { return 1.0 * omega_mom(P, S, u, v, ii, jj, kk) / 1.0; };
    double fxl = fxm(i, j, k), fxh = fxm(i + 1, j, k), fyl = fym(i, j, k), fyh = fym(i, j + 1, k);
    double fzl = fzm(i, j, k), fzh = fzm(i, j, k + 1);
    avx[c] = R(fxl); avy[c] = R(fyl); avz[c] = R(fzl);
    if (k == nz - 1) avz[c + g.sk] = R(fzh);
    const double Jc = detJ_at(P, i, j, k);
    double frho = -1.0 / Jc * ((fxh - fxl) * g.dxi + (fyh - fyl) * g.dyi + (fzh - fzl) * g.dzi);
    // theta with the dycore scheme, advected by the average momenta
    auto th = [&](int ii, int jj, int kk) { return ccw(A.prim, g, ii, jj, kk); };
    const int ht = P.dyc_h, vt = P.dyc_v;
    const double hf = P.f_dyc_h, vf = P.f_dyc_v;
    double tx_l = fxl * interp_dir<HT>(0, i, j, k, th, ht, fxl, hf), tx_h = fxh * interp_dir<HT>(0, i + 1, j, k, th, ht, fxh, hf);
    double ty_l = fyl * interp_dir<HT>(1, i, j, k, th, ht, fyl, hf), ty_h = fyh * interp_dir<HT>(1, i, j + 1, k, th, ht, fyh, hf);
    double tz_l = fzl * interp_dir<VT>(2, i, j, k, th, vt, fzl, vf), tz_h = fzh * interp_dir<VT>(2, i, j, k + 1, th, vt, fzh, vf);
    double invdetJ = 1. / Jc;
    double frt = -invdetJ * 1.0 * ((tx_h - tx_l) * g.dxi + (ty_h - ty_l) * g.dyi + (tz_h - tz_l) * g.dzi);
    if (P.use_diff) {
        const bool dd = P.les == ERF_LES_DEARDORFF;
        DiffT<R> D{P, S.cons, A.prim, mut, dd ? tke.kthv : nullptr, P.alphaT_eff, P.invPr, T.fx[0], T.fy[0]};
        double rlo, rhi;
        frt -= D.div(i, j, k, rlo, rhi);
        if (dd) {
            tke.hfz[c] = R(rlo);
            if (k == nz - 1) tke.hfz[c + g.sk] = R(rhi);
        }
    }
    if (P.mt_zt) {   // moving terrain: the rho and rho theta RHS carry detJ (ERF_slow_rhs_pre.cpp:528-535)
        frho *= Jc;
        frt *= Jc;
    }
    Fcons[c] = R(frho);
    Fcons[N + c] = R(frt);
}

// ---------------------------------------------------------------------------
// Slow RHS of the momenta with terrain (ERF_slow_rhs_pre.cpp:556-744):
// AdvectionSrcForMom (terrain; Centered_2nd inline or the
// ERF_AdvectionSrcForMom_T.H templates), DiffusionSrcForMom_T, the pressure
// gradient with the terrain correction, buoyancy about the 3-D base state,
// Coriolis and geostrophic forcing.  One thread per cell handles the x, y
// and (k >= 1) z faces at (i,j,k).  Omega is the stage's, left in avz by
// k_ter_slow_cell.
// ---------------------------------------------------------------------------
template <class R, int HT, int VT>
__global__ void __launch_bounds__(128, TER_MINB_SLOW_MOM) k_ter_slow_mom(Params P, StateBuf S, StageAux<R> A, const double* __restrict__ u,
                               const double* __restrict__ v, const double* __restrict__ w, const R* __restrict__ t11,
                               const R* __restrict__ t22, const R* __restrict__ t33, const R* __restrict__ t12,
                               const R* __restrict__ t13, const R* __restrict__ t23, TerBuf<R> T,
                               const R* __restrict__ Om_in, R* __restrict__ Fmx, R* __restrict__ Fmy,
                               R* __restrict__ Fmz) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    const int64_t N = g.ncell;
    int64_t c = cidx(g, i, j, k);
    const double dxi = g.dxi, dyi = g.dyi, dzi = g.dzi;
    auto RU = [&](int ii, int jj, int kk) { return S.mx[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)] * 1.0; };
    auto RV = [&](int ii, int jj, int kk) { return S.my[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)] * 1.0; };
    auto Om = [&](int ii, int jj, int kk) { return double(Om_in[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    auto U = [&](int ii, int jj, int kk) { return tvel(u, g, ii, jj, kk); };
    auto V = [&](int ii, int jj, int kk) { return tvel(v, g, ii, jj, kk); };
    auto W = [&](int ii, int jj, int kk) { return wvel(w, g, ii, jj, kk); };
    auto Jt = [&](int ii, int jj, int kk) { return detJ_at(P, ii, jj, kk); };
    auto pp = [&](int ii, int jj, int kk) { return ccw(A.pp, g, ii, jj, kk); };
    const int ht = P.dyc_h, vt = P.dyc_v;
    const double hf = P.f_dyc_h, vf = P.f_dyc_v;
    const bool c2 = (ht == ERF_ADV_CENTERED_2ND && vt == ERF_ADV_CENTERED_2ND);
    const double az = 1.0;
    const double g2 = -P.gravity;
    // ---------------- x-momentum at face (i,j,k)
    {
        double src;
        if (c2) {
            double xh = 0.25 * (RU(i, j, k) * 1.0 + RU(i + 1, j, k) * 1.0) * (U(i + 1, j, k) + U(i, j, k)) * 0.5 * (hzeta_I(P, i, j, k) + hzeta_I(P, i + 1, j, k));
            double xl = 0.25 * (RU(i, j, k) * 1.0 + RU(i - 1, j, k) * 1.0) * (U(i - 1, j, k) + U(i, j, k)) * 0.5 * (hzeta_I(P, i, j, k) + hzeta_I(P, i - 1, j, k));
            double yh = 0.25 * (RV(i, j + 1, k) * 1.0 + RV(i - 1, j + 1, k) * 1.0) * (U(i, j + 1, k) + U(i, j, k)) * hzeta_EK(P, i, j + 1, k);
            double yl = 0.25 * (RV(i, j, k) * 1.0 + RV(i - 1, j, k) * 1.0) * (U(i, j - 1, k) + U(i, j, k)) * hzeta_EK(P, i, j, k);
            double zh = 0.25 * (Om(i, j, k + 1) + Om(i - 1, j, k + 1)) * (U(i, j, k + 1) + U(i, j, k)) * 0.5 * (az + az);
            double zl = 0.25 * (Om(i, j, k) + Om(i - 1, j, k)) * (U(i, j, k - 1) + U(i, j, k)) * 0.5 * (az + az);
            src = (xh - xl) * dxi * 1.0 + (yh - yl) * dyi * 1.0 + (zh - zl) * dzi;
            src = -src / (0.5 * (Jt(i, j, k) + Jt(i - 1, j, k)));
        } else {
            double a, xh, xl, yh, yl, zh, zl;
            a = 0.5 * (RU(i + 1, j, k) * 1.0 + RU(i, j, k) * 1.0); xh = a * interp_dir<HT>(0, i + 1, j, k, U, ht, a, hf) * 0.5 * (hzeta_I(P, i, j, k) + hzeta_I(P, i + 1, j, k));
            a = 0.5 * (RU(i - 1, j, k) * 1.0 + RU(i, j, k) * 1.0); xl = a * interp_dir<HT>(0, i, j, k, U, ht, a, hf) * 0.5 * (hzeta_I(P, i, j, k) + hzeta_I(P, i - 1, j, k));
            a = 0.5 * (RV(i, j + 1, k) * 1.0 + RV(i - 1, j + 1, k) * 1.0); yh = a * interp_dir<HT>(1, i, j + 1, k, U, ht, a, hf) * hzeta_EK(P, i, j + 1, k);
            a = 0.5 * (RV(i, j, k) * 1.0 + RV(i - 1, j, k) * 1.0); yl = a * interp_dir<HT>(1, i, j, k, U, ht, a, hf) * hzeta_EK(P, i, j, k);
            a = 0.5 * (Om(i, j, k + 1) + Om(i - 1, j, k + 1)) * 0.5 * (az + az); zh = a * interp_dir<VT>(2, i, j, k + 1, U, vt, a, vf);
            a = 0.5 * (Om(i, j, k) + Om(i - 1, j, k)) * 0.5 * (az + az); zl = a * interp_dir<VT>(2, i, j, k, U, vt, a, vf);
            src = (xh - xl) * dxi * 1.0 + (yh - yl) * dyi * 1.0 + (zh - zl) * dzi;
            src /= 0.5 * (Jt(i, j, k) + Jt(i - 1, j, k));
            src = -src;
        }
        double r = src;
        if (P.use_diff) {
            auto T11 = [&](int ii) { return double(t11[cidx(g, wrap(ii, g.nx), j, k)]); };
            double d = ((T11(i) - T11(i - 1)) * dxi * 1.0 + (double(t12[cidx(g, i, wrap(j + 1, g.ny), k)]) - double(t12[c])) * dyi * 1.0
                        + (double(t13[c + g.sk]) - double(t13[c])) * dzi);
            d /= 0.5 * (Jt(i, j, k) + Jt(i - 1, j, k));
            r -= d;
        }
        double gpx = dxi * (pp(i, j, k) - pp(i - 1, j, k));
        {
            double mxi = hxi_I(P, i, j, k), mz = hzeta_I(P, i, j, k), gz;
            if (k == 0) gz = 0.5 * dzi * (pp(i - 1, j, k + 1) + pp(i, j, k + 1) - pp(i - 1, j, k) - pp(i, j, k));
            else if (k == nz - 1) gz = 0.5 * dzi * (pp(i - 1, j, k) + pp(i, j, k) - pp(i - 1, j, k - 1) - pp(i, j, k - 1));
            else gz = 0.25 * dzi * (pp(i - 1, j, k + 1) + pp(i, j, k + 1) - pp(i - 1, j, k - 1) - pp(i, j, k - 1));
            gpx -= (mxi / mz) * gz;
        }
        gpx *= 1.0;
        double xsrc = 0.0;
        if (P.coriolis) {
            double rvl = 0.25 * (RV(i, j + 1, k) + RV(i, j, k) + RV(i - 1, j + 1, k) + RV(i - 1, j, k));
            double rwl = 0.25 * (S.mz[cidx(g, i, j, k + 1)] + S.mz[c] + S.mz[cidx(g, i, wrap(j - 1, g.ny), k + 1)] + S.mz[cidx(g, i, wrap(j - 1, g.ny), k)]);
            xsrc += P.cf * (rvl * P.sinphi - rwl * P.cosphi);
        }
        xsrc += 0.5 * (S.cons[c] + S.cons[cidx(g, wrap(i - 1, g.nx), j, k)]) * P.geo0;
        r += (-gpx - 0.0) / (1.0 + moist_q(P, A.prim, c, cidx(g, wrap(i - 1, g.nx), j, k))) + xsrc;
        if (P.mt_zt) r *= hzeta_I(P, i, j, k);   // moving terrain (ERF_slow_rhs_pre.cpp:633-636)
        Fmx[c] = R(r);
    }
    // ---------------- y-momentum at face (i,j,k)
    {
        double src;
        if (c2) {
            double xh = 0.25 * (RU(i + 1, j, k) * 1.0 + RU(i + 1, j - 1, k) * 1.0) * (V(i + 1, j, k) + V(i, j, k)) * hzeta_EK(P, i + 1, j, k);
            double xl = 0.25 * (RU(i, j, k) * 1.0 + RU(i, j - 1, k) * 1.0) * (V(i - 1, j, k) + V(i, j, k)) * hzeta_EK(P, i, j, k);
            double yh = 0.25 * (RV(i, j + 1, k) * 1.0 + RV(i, j, k) * 1.0) * (V(i, j + 1, k) + V(i, j, k)) * 0.5 * (hzeta_J(P, i, j, k) + hzeta_J(P, i, j + 1, k));
            double yl = 0.25 * (RV(i, j, k) * 1.0 + RV(i, j - 1, k) * 1.0) * (V(i, j - 1, k) + V(i, j, k)) * 0.5 * (hzeta_J(P, i, j, k) + hzeta_J(P, i, j - 1, k));
            double zh = 0.25 * (Om(i, j, k + 1) + Om(i, j - 1, k + 1)) * (V(i, j, k + 1) + V(i, j, k)) * 0.5 * (az + az);
            double zl = 0.25 * (Om(i, j, k) + Om(i, j - 1, k)) * (V(i, j, k - 1) + V(i, j, k)) * 0.5 * (az + az);
            src = (xh - xl) * dxi * 1.0 + (yh - yl) * dyi * 1.0 + (zh - zl) * dzi;
            src = -src / (0.5 * (Jt(i, j, k) + Jt(i, j - 1, k)));
        } else {
            double a, xh, xl, yh, yl, zh, zl;
            a = 0.5 * (RU(i + 1, j, k) * 1.0 + RU(i + 1, j - 1, k) * 1.0); xh = a * interp_dir<HT>(0, i + 1, j, k, V, ht, a, hf) * hzeta_EK(P, i + 1, j, k);
            a = 0.5 * (RU(i, j, k) * 1.0 + RU(i, j - 1, k) * 1.0); xl = a * interp_dir<HT>(0, i, j, k, V, ht, a, hf) * hzeta_EK(P, i, j, k);
            a = 0.5 * (RV(i, j, k) * 1.0 + RV(i, j + 1, k) * 1.0); yh = a * 0.5 * (hzeta_J(P, i, j, k) + hzeta_J(P, i, j + 1, k)) * interp_dir<HT>(1, i, j + 1, k, V, ht, a, hf);
            a = 0.5 * (RV(i, j, k) * 1.0 + RV(i, j - 1, k) * 1.0); yl = a * 0.5 * (hzeta_J(P, i, j, k) + hzeta_J(P, i, j - 1, k)) * interp_dir<HT>(1, i, j, k, V, ht, a, hf);
            a = 0.5 * (Om(i, j, k + 1) + Om(i, j - 1, k + 1)) * 0.5 * (az + az); zh = a * interp_dir<VT>(2, i, j, k + 1, V, vt, a, vf);
            a = 0.5 * (Om(i, j, k) + Om(i, j - 1, k)) * 0.5 * (az + az); zl = a * interp_dir<VT>(2, i, j, k, V, vt, a, vf);
            src = (xh - xl) * dxi * 1.0 + (yh - yl) * dyi * 1.0 + (zh - zl) * dzi;
            src /= 0.5 * (Jt(i, j, k) + Jt(i, j - 1, k));
            src = -src;
        }
        double r = src;
        if (P.use_diff) {
            auto T22 = [&](int jj) { return double(t22[cidx(g, i, wrap(jj, g.ny), k)]); };
            double d = ((double(t12[cidx(g, wrap(i + 1, g.nx), j, k)]) - double(t12[c])) * dxi * 1.0 + (T22(j) - T22(j - 1)) * dyi * 1.0
                        + (double(t23[c + g.sk]) - double(t23[c])) * dzi);
            d /= 0.5 * (Jt(i, j, k) + Jt(i, j - 1, k));
            r -= d;
        }
        double gpy = dyi * (pp(i, j, k) - pp(i, j - 1, k));
        {
            double meta = heta_J(P, i, j, k), mz = hzeta_J(P, i, j, k), gz;
            if (k == 0) gz = 0.5 * dzi * (pp(i, j, k + 1) + pp(i, j - 1, k + 1) - pp(i, j, k) - pp(i, j - 1, k));
            else if (k == nz - 1) gz = 0.5 * dzi * (pp(i, j, k) + pp(i, j - 1, k) - pp(i, j, k - 1) - pp(i, j - 1, k - 1));
            else gz = 0.25 * dzi * (pp(i, j, k + 1) + pp(i, j - 1, k + 1) - pp(i, j, k - 1) - pp(i, j - 1, k - 1));
            gpy -= (meta / mz) * gz;
        }
        gpy *= 1.0;
        double ysrc = 0.0;
        if (P.coriolis) {
            double rul = 0.25 * (RU(i + 1, j, k) + RU(i, j, k) + RU(i + 1, j - 1, k) + RU(i, j - 1, k));
            ysrc += -P.cf * rul * P.sinphi;
        }
        ysrc += 0.5 * (S.cons[c] + S.cons[cidx(g, i, wrap(j - 1, g.ny), k)]) * P.geo1;
        r += (-gpy - 0.0) / (1.0 + moist_q(P, A.prim, c, cidx(g, i, wrap(j - 1, g.ny), k))) + ysrc;
        if (P.mt_zt) r *= hzeta_J(P, i, j, k);   // :681-684
        Fmy[c] = R(r);
    }
    // ---------------- z-momentum at face (i,j,k), 1 <= k <= nz-1
    if (k == 0) {
        Fmz[c] = R(0);
        if (nz == 1) Fmz[c + g.sk] = R(0);
        return;
    }
    {
        const int lo_z_face = 0, hi_z_face = nz;
        double src;
        if (c2) {
            double xh = 0.25 * (RU(i + 1, j, k) + RU(i + 1, j, k - 1)) * 1.0 * (W(i + 1, j, k) + W(i, j, k)) * hzeta_EJ(P, i + 1, j, k);
            double xl = 0.25 * (RU(i, j, k) + RU(i, j, k - 1)) * 1.0 * (W(i - 1, j, k) + W(i, j, k)) * hzeta_EJ(P, i, j, k);
            double yh = 0.25 * (RV(i, j + 1, k) + RV(i, j + 1, k - 1)) * 1.0 * (W(i, j + 1, k) + W(i, j, k)) * hzeta_EI(P, i, j + 1, k);
            double yl = 0.25 * (RV(i, j, k) + RV(i, j, k - 1)) * 1.0 * (W(i, j - 1, k) + W(i, j, k)) * hzeta_EI(P, i, j, k);
            double zl = 0.25 * (Om(i, j, k) + Om(i, j, k - 1)) * (W(i, j, k) + W(i, j, k - 1));
            double zh = (k == hi_z_face) ? Om(i, j, k) * W(i, j, k) * az
                                         : 0.25 * (Om(i, j, k) + Om(i, j, k + 1)) * (W(i, j, k) + W(i, j, k + 1)) * 0.5 * (az + az);
            src = (xh - xl) * dxi * 1.0 + (yh - yl) * dyi * 1.0 + (zh - zl) * dzi;
            src = -src / (0.5 * (Jt(i, j, k) + Jt(i, j, k - 1)));
        } else {
            double a, xh, xl, yh, yl, zh, zl;
            a = 0.5 * (RU(i + 1, j, k) + RU(i + 1, j, k - 1)) * 1.0; xh = a * interp_dir<HT>(0, i + 1, j, k, W, ht, a, hf) * hzeta_EJ(P, i + 1, j, k);
            a = 0.5 * (RU(i, j, k) + RU(i, j, k - 1)) * 1.0; xl = a * interp_dir<HT>(0, i, j, k, W, ht, a, hf) * hzeta_EJ(P, i, j, k);
            a = 0.5 * (RV(i, j + 1, k) + RV(i, j + 1, k - 1)) * 1.0; yh = a * interp_dir<HT>(1, i, j + 1, k, W, ht, a, hf) * hzeta_EI(P, i, j + 1, k);
            a = 0.5 * (RV(i, j, k) + RV(i, j, k - 1)) * 1.0; yl = a * interp_dir<HT>(1, i, j, k, W, ht, a, hf) * hzeta_EI(P, i, j, k);
            auto iZall = [&](int kk, double upw, double frac, int type) {
                int gt = (type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH) ? ERF_ADV_UPWIND_5TH
                         : (type == ERF_ADV_CENTERED_2ND ? ERF_ADV_CENTERED_2ND : ERF_ADV_UPWIND_3RD);
                double s[6];
                const int wd = stencil_width(gt);
                for (int m = 0; m < 6; ++m) {
                    int off = m - 3;
                    s[m] = (off >= -wd && off <= wd - 1) ? W(i, j, kk + off) : 0.0;
                }
                return interp_all<double>(type, s, upw, frac);
            };
            double Oh = (k == hi_z_face) ? Om(i, j, k) * az : 0.25 * (Om(i, j, k) + Om(i, j, k + 1)) * (az + az);
            double ih, il;
            if (k == hi_z_face - 1) ih = iZall(k + 1, Oh, 0, ERF_ADV_CENTERED_2ND);
            else if (k == hi_z_face - 2 || k == lo_z_face + 1) {
                if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) ih = iZall(k + 1, Oh, 0, ERF_ADV_CENTERED_4TH);
                else ih = iZall(k + 1, Oh, vf, vt);
            } else ih = interp_dir<VT>(2, i, j, k + 1, W, vt, Oh, vf);
            zh = Oh * ih;
            double Ol = 0.25 * (Om(i, j, k) + Om(i, j, k - 1)) * (az + az);
            if (k == lo_z_face + 1) il = iZall(k, Ol, 0, ERF_ADV_CENTERED_2ND);
            else if (k == lo_z_face + 2 || k == hi_z_face - 1) {
                if (vt != ERF_ADV_CENTERED_2ND && vt != ERF_ADV_UPWIND_3RD) il = iZall(k, Ol, 0, ERF_ADV_CENTERED_4TH);
                else il = iZall(k, Ol, vf, vt);
            } else il = interp_dir<VT>(2, i, j, k, W, vt, Ol, vf);
            zl = Ol * il;
            src = (xh - xl) * dxi * 1.0 + (yh - yl) * dyi * 1.0 + (zh - zl) * dzi;
            double denom = 0.5 * (Jt(i, j, k) + Jt(i, j, k - 1));
            src /= denom;
            src = -src;
        }
        double r = src;
        if (P.use_diff) {
            double d = ((double(T.t31[cidx(g, wrap(i + 1, g.nx), j, k)]) - double(T.t31[c])) * dxi * 1.0
                        + (double(T.t32[cidx(g, i, wrap(j + 1, g.ny), k)]) - double(T.t32[c])) * dyi * 1.0
                        + (double(t33[c]) - double(t33[c - g.sk])) * dzi);
            d /= 0.5 * (Jt(i, j, k) + Jt(i, j, k - 1));
            r -= d;
        }
        double mz = hzeta_K(P, i, j, k);
        double gpz = dzi * (pp(i, j, k) - pp(i, j, k - 1)) / mz;
        double zsrc = 0.0;
        if (P.buoy_type == 1 && P.moist) {
            // total density of air and water (make_buoyancy, ERF_make_buoyancy.cpp:92-130)
            const int nq = P.ncomp - ERF_RHOQ1_COMP;
            double hi = S.cons[c] + S.cons[5 * N + c] + S.cons[6 * N + c] - bs(P.r0, g, i, j, k);
            double lo = S.cons[c - g.sk] + S.cons[5 * N + c - g.sk] + S.cons[6 * N + c - g.sk] - bs(P.r0, g, i, j, k - 1);
            for (int qo = 2; qo < nq; ++qo) { hi += S.cons[(5 + qo) * N + c]; lo += S.cons[(5 + qo) * N + c - g.sk]; }
            zsrc = g2 * 0.5 * (hi + lo);
        } else if (P.buoy_type == 1) {
            zsrc = g2 * 0.5 * ((S.cons[c] - bs(P.r0, g, i, j, k)) + (S.cons[c - g.sk] - bs(P.r0, g, i, j, k - 1)));
        } else {
            auto T0 = [&](int kk) {
                double p0v = bs(P.p0, g, i, j, kk);
                double rt0 = eos_rt_given_p(p0v);
                return (rt0 / bs(P.r0, g, i, j, kk)) / pow(p_0 / p0v, P.rdOcp);
            };
            double t0_hi = T0(k), t_hi = eos_T(S.cons[c], S.cons[N + c], 0.0);
            double t0_lo = T0(k - 1), t_lo = eos_T(S.cons[c - g.sk], S.cons[N + c - g.sk], 0.0);
            double qplus = (t_hi - t0_hi) / t0_hi, qminus = (t_lo - t0_lo) / t0_lo;
            double r0_q_avg = 0.5 * (bs(P.r0, g, i, j, k) * qplus + bs(P.r0, g, i, j, k - 1) * qminus);
            zsrc = -r0_q_avg * g2;
        }
        if (P.coriolis) {
            double rul = 0.25 * (RU(i + 1, j, k) + RU(i, j, k) + RU(i + 1, j, k - 1) + RU(i, j, k - 1));
            zsrc += P.cf * rul * P.cosphi;
        }
        zsrc += 0.5 * (S.cons[c] + S.cons[c - g.sk]) * P.geo2;
        r += (zsrc - gpz - 0.0) / (1.0 + moist_q(P, A.prim, c, c - g.sk));
        if (P.mt_zt) r *= 0.5 * (Jt(i, j, k) + Jt(i, j, k - 1));   // :741-743
        Fmz[c] = R(r);
        if (k == nz - 1) Fmz[c + g.sk] = R(0);
    }
}

// ---------------------------------------------------------------------------
// Acoustic substep with terrain, horizontal part (ERF_fast_rhs_T.cpp:130-320):
// lagged d(rho theta) and its extrapolation, U'' / V'' with the
// terrain-corrected gradient of the extrapolated d(rho theta); the old and
// new increments are kept for the vertical part.
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_ter_fast_h(Params P, int step, double dtau, double facinv, StateBuf Sprev, int prev_rt,
                             StateBuf Sst, StageAux<R> A, const R* __restrict__ Fmx, const R* __restrict__ Fmy,
                             const R* __restrict__ lag_in, R* __restrict__ lag_out, TerBuf<R> T, R* __restrict__ avx,
                             R* __restrict__ avy, double* __restrict__ outx, double* __restrict__ outy) {
    const Geo& g = P.g;
    int i, j, k;
    if (!cell_ij(g, i, j, k)) return;
    const int nz = g.nz;
    const int64_t N = g.ncell;
    int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    int64_t c = cidx(g, i, j, k), cxm = cidx(g, im, j, k), cym = cidx(g, i, jm, k);
    const double beta_d = 0.1, dxi = g.dxi, dyi = g.dyi, dzi = g.dzi;
    auto extrap = [&](int ii, int jj, int kk) {
        int64_t e = cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), clampk(kk, nz));
        double drt = Sprev.cons[N + e] - Sst.cons[N + e];
        if (step == 0) return drt;
        return drt + beta_d * (drt - double(lag_in[e]));
    };
    lag_out[c] = R(Sprev.cons[N + c] - Sst.cons[N + c]);
    double px = Sprev.mx[c], py = Sprev.my[c];
    if (prev_rt) {
        double rs = Sprev.cons[c] + Sprev.cons[cxm];
        double ut = (px * 2.0) / rs;
        px = (ut * 0.5) * rs;
        rs = Sprev.cons[c] + Sprev.cons[cym];
        double vt = (py * 2.0) / rs;
        py = (vt * 0.5) * rs;
    }
    double odu = px - Sst.mx[c], odv = py - Sst.my[c];
    double gpx, gpy;
    {
        double mxi = hxi_I(P, i, j, k), mz = hzeta_I(P, i, j, k);
        double gp_xi = (extrap(i, j, k) - extrap(i - 1, j, k)) * dxi;
        double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k) - extrap(i, j, k))
                                  : 0.25 * dzi * (extrap(i - 1, j, k + 1) + extrap(i, j, k + 1) - extrap(i - 1, j, k - 1) - extrap(i, j, k - 1));
        gpx = gp_xi - (mxi / mz) * gp_zeta;
        gpx *= 1.0;
        gpx /= (1.0 + moist_q(P, A.prim, c, cxm));
    }
    {
        double meta = heta_J(P, i, j, k), mz = hzeta_J(P, i, j, k);
        double gp_eta = (extrap(i, j, k) - extrap(i, j - 1, k)) * dyi;
        double gp_zeta = (k == 0) ? 0.5 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k) - extrap(i, j - 1, k))
                                  : 0.25 * dzi * (extrap(i, j, k + 1) + extrap(i, j - 1, k + 1) - extrap(i, j, k - 1) - extrap(i, j - 1, k - 1));
        gpy = gp_eta - (meta / mz) * gp_zeta;
        gpy *= 1.0;
        gpy /= (1.0 + moist_q(P, A.prim, c, cym));
    }
    double pix = 0.5 * (double(A.pi[cxm]) + double(A.pi[c]));
    double piy = 0.5 * (double(A.pi[cym]) + double(A.pi[c]));
    double fx = -Gamma_ * R_d * pix * gpx;
    double fy = -Gamma_ * R_d * piy * gpy;
    double ndu = odu + dtau * fx + dtau * double(Fmx[c]);
    double ndv = odv + dtau * fy + dtau * double(Fmy[c]);
    T.ndu[c] = R(ndu); T.ndv[c] = R(ndv);
    T.odu[c] = R(odu); T.odv[c] = R(odv);
    avx[c] += R(facinv * ndu);
    avy[c] += R(facinv * ndv);
    outx[c] = Sst.mx[c] + ndu;
    outy[c] = Sst.my[c] + ndv;
}

// ---------------------------------------------------------------------------
// Acoustic substep with terrain, vertical part (ERF_fast_rhs_T.cpp:320-680):
// horizontal rho / rho*theta fluxes through the sloping faces, Omega of the
// previous increments, the detJ-weighted right-hand side of the Omega''
// system, the Thomas sweep on the stage's coefficients, then w'' from
// Omega'', the vertical fluxes, the average contravariant momentum, rho and
// rho*theta (k_ter_fast_vert below).
// ---------------------------------------------------------------------------
namespace {
template <class R>
__device__ __forceinline__ double prev_mz_ter(const Params& P, StateBuf Sprev, int prev_rt, int i, int j, int k) {
    const Geo& g = P.g;
    const int nz = g.nz;
    int64_t f = cidx(g, i, j, k);
    double m = Sprev.mz[f];
    if (!prev_rt) return m;
    if (k == 0 || k == nz) {
        auto U1 = [&](int ii, int jj, int kk) {
            if (kk >= nz) {
                if (g.zhi_noslip) return 0.0;
                kk = nz - 1;
            }
            return rt_u(g, Sprev.cons, Sprev.mx, ii, jj, kk);
        };
        auto V1 = [&](int ii, int jj, int kk) {
            if (kk >= nz) {
                if (g.zhi_noslip) return 0.0;
                kk = nz - 1;
            }
            return rt_v(g, Sprev.cons, Sprev.my, ii, jj, kk);
        };
        int kc = (k == 0) ? 0 : nz - 1;
        double r = Sprev.cons[cidx(g, i, j, kc)];
        double wb = w_from_omega(P, i, j, k, 0.0, U1, V1);
        return (wb * 0.5) * (r + r);
    }
    double rs = Sprev.cons[f] + Sprev.cons[f - g.sk];
    double wt = (m * 2.0) / rs;
    return (wt * 0.5) * rs;
}
}  // namespace

// The same vertical part as one pass per column tile (the layout of
// k_fast_vert: TX columns of a row j, the block's warps spread over the
// levels, the column arrays in shared memory), so that the horizontal
// fluxes, Omega of the old increments, the right-hand side and the solution
// never leave the SM; one warp runs the Thomas sweep.  The momentum of the
// previous substep on the ground and lid faces (w from Omega = 0 of its
// round-tripped u, v) reads neighbouring columns of a state the update
// overwrites in place, so k_ter_fv_bnd forms it first.
template <class R>
__global__ void k_ter_fv_bnd(Params P, StateBuf Sprev, TerBuf<R> T) {
    const Geo& g = P.g;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int64_t col = (int64_t)j * g.nx + i;
    T.bnd[col] = prev_mz_ter<R>(P, Sprev, 1, i, j, 0);
    T.bnd[g.sk + col] = prev_mz_ter<R>(P, Sprev, 1, i, j, g.nz);
}

template <class R>
__global__ void __launch_bounds__(1024) k_ter_fast_vert(Params P, double dtau, double facinv, double beta_1,
                                                        double beta_2, StateBuf Sprev, int prev_rt, StateBuf Sst,
                                                        StageAux<R> A, const R* __restrict__ Fcons,
                                                        const R* __restrict__ Fmz, TerBuf<R> T,
                                                        const R* __restrict__ cA, const R* __restrict__ cInvB,
                                                        const R* __restrict__ cCB, const R* __restrict__ cP,
                                                        const R* __restrict__ cQ, R* __restrict__ avz,
                                                        double* out_cons, double* out_mz) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    double* sm = reinterpret_cast<double*>(sm_raw);
    const Geo& g = P.g;
    const int nz = g.nz, TX = blockDim.x, L = threadIdx.x, w0 = threadIdx.y, nw = blockDim.y;
    const int i = blockIdx.x * TX + L, j = blockIdx.y;
    const bool ok = i < g.nx;
    double* sT0 = sm;                   // horizontal rho flux divergence (cells)
    double* sT1 = sT0 + nz * TX;        // horizontal rho*theta flux divergence (cells)
    double* sO = sT1 + nz * TX;         // Omega of the old increments (faces)
    double* sR = sO + (nz + 1) * TX;    // right-hand side, then the solution (faces)
    double* sA = sR + (nz + 1) * TX;
    double* sI = sA + (nz + 1) * TX;
    double* sCB = sI + (nz + 1) * TX;
    const int64_t N = g.ncell, sk = g.sk;
    const double dxi = g.dxi, dyi = g.dyi, dzi = g.dzi, halfg = P.halfg;
    auto th = [&](int ii, int jj, int kk) { return ccw(A.prim, g, ii, jj, kk); };
    auto NDU = [&](int ii, int jj, int kk) { return double(T.ndu[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    auto NDV = [&](int ii, int jj, int kk) { return double(T.ndv[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    auto ODU = [&](int ii, int jj, int kk) { return double(T.odu[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    auto ODV = [&](int ii, int jj, int kk) { return double(T.odv[cidx(g, wrap(ii, g.nx), wrap(jj, g.ny), kk)]); };
    auto prev_mz = [&](int k) {
        if (prev_rt && (k == 0 || k == nz)) return T.bnd[(k == 0 ? 0 : sk) + (int64_t)j * g.nx + i];
        return prev_mz_ter<R>(P, Sprev, prev_rt, i, j, k);
    };
    // ---- phase 1: horizontal fluxes (cells), Omega'' of the old increments and the coefficients (faces)
    if (ok) {
        for (int k = w0; k <= nz; k += nw) {
            const int64_t f = cidx(g, i, j, k);
            if (k < nz) {
                double hxh = hzeta_I(P, i + 1, j, k), hxl = hzeta_I(P, i, j, k);
                double hyh = hzeta_J(P, i, j + 1, k), hyl = hzeta_J(P, i, j, k);
                double xl = NDU(i, j, k) * hxl / 1.0, xh = NDU(i + 1, j, k) * hxh / 1.0;
                double yl = NDV(i, j, k) * hyl / 1.0, yh = NDV(i, j + 1, k) * hyh / 1.0;
                double mfsq = 1.0;
                double tc = th(i, j, k);
                sT0[k * TX + L] = (xh - xl) * dxi * mfsq + (yh - yl) * dyi * mfsq;
                sT1[k * TX + L] = ((xh * (tc + th(i + 1, j, k)) - xl * (tc + th(i - 1, j, k))) * dxi * mfsq +
                                   (yh * (tc + th(i, j + 1, k)) - yl * (tc + th(i, j - 1, k))) * dyi * mfsq) * 0.5;
            }
            double odw = prev_mz(k) - Sst.mz[f];
            double om;
            if (k == 0) om = 0.;
            else if (k == nz) om = odw;
            else om = omega_from_w(P, i, j, k, odw, ODU, ODV);
            sO[k * TX + L] = om;
            sA[k * TX + L] = double(cA[f]);
            sI[k * TX + L] = double(cInvB[f]);
            sCB[k * TX + L] = double(cCB[f]);
        }
    }
    __syncthreads();
    // ---- phase 2: the detJ-weighted right-hand side of the Omega'' system (faces)
    if (ok) {
        for (int k = w0; k <= nz; k += nw) {
            const int64_t f = cidx(g, i, j, k);
            if (k == 0 || k == nz) {
                sR[k * TX + L] = dtau * double(Fmz[f]);
                continue;
            }
            int64_t cm = f - sk;
            double Jk = detJ_at(P, i, j, k), Jkm = detJ_at(P, i, j, k - 1);
            double dJk = 0.5 * (Jk + Jkm);
            double cPk = double(cP[f]), cQk = double(cQ[f]);
            double tlo = 0.5 * (th(i, j, k - 2) + th(i, j, k - 1));
            double tmid = 0.5 * (th(i, j, k - 1) + th(i, j, k));
            double thi = 0.5 * (th(i, j, k) + th(i, j, k + 1));
            double odr_k = Sprev.cons[f] - Sst.cons[f], odr_km = Sprev.cons[cm] - Sst.cons[cm];
            double odrt_k = Sprev.cons[N + f] - Sst.cons[N + f], odrt_km = Sprev.cons[N + cm] - Sst.cons[N + cm];
            double R0t = (-halfg * odr_k + cPk * odrt_k) * Jk + (-halfg * odr_km + cQk * odrt_km) * Jkm;
            double R1t = -halfg * (double(Fcons[f]) * Jk + double(Fcons[cm]) * Jkm)
                         + (cPk * double(Fcons[N + f]) * Jk + cQk * double(Fcons[N + cm]) * Jkm);
            double Okp1 = sO[(k + 1) * TX + L], Ok = sO[k * TX + L], Okm1 = sO[(k - 1) * TX + L];
            R1t += (halfg) * (beta_1 * dzi * (Okp1 - Okm1) + sT0[k * TX + L] + sT0[(k - 1) * TX + L]);
            R1t += -(cPk * (beta_1 * dzi * (Okp1 * thi - Ok * tmid) + sT1[k * TX + L]) +
                     cQk * (beta_1 * dzi * (Ok * tmid - Okm1 * tlo) + sT1[(k - 1) * TX + L]));
            double odw = prev_mz(k) - Sst.mz[f];
            double rhs = dJk * odw + dtau * (dJk * double(Fmz[f]) + R0t + dtau * beta_2 * R1t);
            rhs += dJk * omega_from_w(P, i, j, k, 0., NDU, NDV);
            sR[k * TX + L] = rhs;
        }
    }
    __syncthreads();
    // ---- phase 3: forward elimination / back substitution, one warp
    if (w0 == 0 && ok) {
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
    // ---- phase 4: w'' from Omega'', vertical fluxes, average Omega, rho and rho*theta
    if (ok) {
        for (int k = w0; k <= nz; k += nw) {
            const int64_t f = cidx(g, i, j, k);
            double m = Sst.mz[f];
            if (k >= 1 && k <= nz - 1) m += w_from_omega(P, i, j, k, sR[k * TX + L], NDU, NDV);
            out_mz[f] = m;
            if (k == nz) continue;
            const int64_t c = f;
            double zl = beta_2 * sR[k * TX + L] + beta_1 * sO[k * TX + L];
            double zh = beta_2 * sR[(k + 1) * TX + L] + beta_1 * sO[(k + 1) * TX + L];
            avz[c] += R(facinv * zl / (1.0 * 1.0));
            if (k == nz - 1) avz[c + sk] += R(facinv * zh / (1.0 * 1.0));
            double Jc = detJ_at(P, i, j, k);
            double tc = th(i, j, k);
            double frho = -(sT0[k * TX + L] + (zh - zl) * dzi) / Jc;
            double frt = -(sT1[k * TX + L] + 0.5 * (zh * (tc + th(i, j, k + 1)) - zl * (tc + th(i, j, k - 1))) * dzi) / Jc;
            double pr = Sprev.cons[c], prt = Sprev.cons[N + c];
            out_cons[c] = pr + dtau * (double(Fcons[c]) + frho);
            out_cons[N + c] = prt + dtau * (double(Fcons[N + c]) + frt);
        }
    }
}

// ---------------------------------------------------------------------------
// Slow RHS of the slow variables with terrain and the stage update
// (ERF_slow_rhs_post.cpp:169-530): passive scalar and (Deardorff) rho*KE
// advected with the average momenta (over detJ), DiffusionSrcForState_T with
// the TKE sources, S_new = S_old + dt RHS (KE clipped at DBL_EPSILON); rho,
// rho*theta and the momenta from the fast solution through the two boundary
// round trips, w on the ground and the lid from Omega = 0 of the new u, v;
// the next stage's primitives.
// ---------------------------------------------------------------------------
template <class R, int DH, int DV, int MH, int MV, int NS, bool MT = false>
__global__ void __launch_bounds__(TTX * TTY, TER_MINB_POST) k_ter_post(Params P, int kz, double slow_dt, StateBuf Sold,
                                                                       StateBuf Sst, StateBuf Ssum, StateBuf Snew,
                                                                       StageAux<R> Acur, StageAux<R> Anext,
                                                                       int make_next, const R* __restrict__ mut,
                                                                       TkeBuf<R> tke, TerBuf<R> T,
                                                                       const R* __restrict__ avx,
                                                                       const R* __restrict__ avy,
                                                                       const R* __restrict__ avz, double* __restrict__ un,
                                                                       double* __restrict__ vn, double* __restrict__ wn) {
    __shared__ FluxTile<R> sh[NS];
    __shared__ Plane<R> pl[NS];
    const Geo& g = P.g;
    const int nz = g.nz;
    const int64_t N = g.ncell;
    const int i = blockIdx.x * TTX + threadIdx.x, j = blockIdx.y * TTY + threadIdx.y;
    const bool ok = i < g.nx && j < g.ny;
    const int k0 = blockIdx.z * kz, k1 = min(k0 + kz, g.nz);
    const bool dd = P.les == ERF_LES_DEARDORFF;
    // slow variables: the passive scalar, the moisture species, then (Deardorff) rho*KE
    const int nscal = P.moist ? 1 + (P.ncomp - ERF_RHOQ1_COMP) : 1;
    const int nslow = nscal + (dd ? 1 : 0);
    R zl[NS], zh[NS];
    double dz_lo[NS];   // diffusive z flux through the cell's bottom face, carried up the column
#pragma unroll
    for (int q = 0; q < NS; ++q) { zl[q] = zh[q] = R(0); dz_lo[q] = 0.0; }
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
        // advective fluxes with the average (area-weighted, contravariant) momenta
        if (ok) {
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                if (q >= nslow) break;
                if (q == 0 || q >= nscal)
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
        if (!ok) continue;   // the next level's first barrier orders the reuse of sh
        const int64_t c = cidx(g, i, j, k);
        const double invdetJ = 1. / detJ_at(P, i, j, k);
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            if (q >= nslow) break;
            const bool ke = q >= nscal, species = q > 0 && q < nscal;
            const int n = comp_of(q);
            // -div over detJ; (-S) invdetJ equals the reference's -invdetJ S bit for bit
            double r = double(tile_div(g, sh[q], zl[q], zh[q])) * invdetJ;
            zl[q] = zh[q];
            if (P.use_diff) {
                // DiffT::div with the z-face flux carried from the level below:
                // raw x / y fluxes precomputed for the scalar and KE, the species' formed here
                const R* phi = slow_phi(q);
                DiffT<R> D{P, Sst.cons, phi, mut, nullptr, ke ? 0.0 : P.alphaC_eff, ke ? P.invSigmaK : P.invSc,
                           species ? nullptr : T.fx[ke ? 1 : 0], species ? nullptr : T.fy[ke ? 1 : 0]};
                double raw;
                double fxl = D.xr(i, j, k) * hzeta_I(P, i, j, k), fxh = D.xr(i + 1, j, k) * hzeta_I(P, i + 1, j, k);
                double fyl = D.yr(i, j, k) * hzeta_J(P, i, j, k), fyh = D.yr(i, j + 1, k) * hzeta_J(P, i, j + 1, k);
                double fzl = (k == k0) ? D.zflux(i, j, k, raw) : dz_lo[q];
                double fzh = D.zflux(i, j, k + 1, raw);
                dz_lo[q] = fzh;
                double sd = (fxh - fxl) * g.dxi * 1.0 + (fyh - fyl) * g.dyi * 1.0 + (fzh - fzl) * g.dzi;
                r -= sd / detJ_at(P, i, j, k);
            }
            if (ke) {
                r += P.g_over_theta0 * double(tke.hfz[c]);
                r += 2.0 * double(mut[c]) * double(tke.smn[c]);
                r -= double(tke.diss[c]);
            }
            if (MT) {
                // moving terrain (ERF_slow_rhs_post.cpp:467-478): detJ-weighted
                // old -> new; only rho KE is clamped
                const double Jo = detJ_at(P, i, j, k), Jn = mt_detj(P.mt_znew, g, i, j, k);
                double tv = Jo * Sold.cons[n * N + c] + slow_dt * Jo * r;
                tv /= Jn;
                Snew.cons[n * N + c] = ke ? fmax(tv, 2.220446049250313e-16) : tv;
                continue;
            }
            double v_ = Sold.cons[n * N + c] + slow_dt * r;
            Snew.cons[n * N + c] = (q == 0) ? v_ : fmax(v_, species ? 0.0 : 2.220446049250313e-16);
        }
        Snew.cons[c] = Ssum.cons[c];
        Snew.cons[N + c] = Ssum.cons[N + c];
        if (!dd) Snew.cons[2 * N + c] = Sst.cons[2 * N + c];
        Snew.cons[3 * N + c] = Sst.cons[3 * N + c];
        double rho = Ssum.cons[c];
        // horizontal momenta through the two round trips; velocity u2
        auto u2f = [&](int ii, int jj, int kk) {
            if (kk < 0 || kk >= nz) {
                if ((kk < 0 && g.zlo_noslip) || (kk >= nz && g.zhi_noslip)) return 0.0;
                kk = kk < 0 ? 0 : nz - 1;
            }
            ii = wrap(ii, g.nx); jj = wrap(jj, g.ny);
            int64_t e = cidx(g, ii, jj, kk);
            double rs = Ssum.cons[e] + Ssum.cons[cidx(g, wrap(ii - 1, g.nx), jj, kk)];
            double m = Ssum.mx[e];
            double u1 = (m * 2.0) / rs; m = (u1 * 0.5) * rs;
            return (m * 2.0) / rs;
        };
        auto v2f = [&](int ii, int jj, int kk) {
            if (kk < 0 || kk >= nz) {
                if ((kk < 0 && g.zlo_noslip) || (kk >= nz && g.zhi_noslip)) return 0.0;
                kk = kk < 0 ? 0 : nz - 1;
            }
            ii = wrap(ii, g.nx); jj = wrap(jj, g.ny);
            int64_t e = cidx(g, ii, jj, kk);
            double rs = Ssum.cons[e] + Ssum.cons[cidx(g, ii, wrap(jj - 1, g.ny), kk)];
            double m = Ssum.my[e];
            double v1 = (m * 2.0) / rs; m = (v1 * 0.5) * rs;
            return (m * 2.0) / rs;
        };
        {
            double rs = rho + Ssum.cons[cidx(g, wrap(i - 1, g.nx), j, k)];
            double u2 = u2f(i, j, k);
            Snew.mx[c] = (u2 * 0.5) * rs; un[c] = u2;
        }
        {
            double rs = rho + Ssum.cons[cidx(g, i, wrap(j - 1, g.ny), k)];
            double v2 = v2f(i, j, k);
            Snew.my[c] = (v2 * 0.5) * rs; vn[c] = v2;
        }
        if (k == 0 && !MT) {
            double wb = w_from_omega(P, i, j, 0, 0.0, u2f, v2f);
            Snew.mz[c] = (wb * 0.5) * (rho + rho); wn[c] = wb;
        } else {
            // (on a moving ground the w of the update, through the two round trips)
            double rs = rho + (k == 0 ? rho : Ssum.cons[c - g.sk]);
            double m = Ssum.mz[c];
            double w1 = (m * 2.0) / rs; m = (w1 * 0.5) * rs;
            double w2 = (m * 2.0) / rs; m = (w2 * 0.5) * rs;
            Snew.mz[c] = m; wn[c] = w2;
        }
        if (k == nz - 1) {
            double wt = w_from_omega(P, i, j, nz, 0.0, u2f, v2f);
            Snew.mz[c + g.sk] = (wt * 0.5) * (rho + rho); wn[c + g.sk] = wt;
        }
        if (make_next) stage_aux_ter<R>(P, Snew.cons, Anext, c, k);
    }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <class R>
void launch_ter_step_begin(const Params& P, cudaStream_t st, const double* cons, const double* uo, const double* vo,
                           const double* wo, StateBuf S, double* un, double* vn, double* wn, StageAux<R> A, R* mut,
                           TkeBuf<R> tke) {
    k_ter_step_begin<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, cons, uo, vo, wo, S, un, vn, wn, A, mut, tke);
}
template <class R>
void launch_ter_tau(const Params& P, cudaStream_t st, int nrk, const double* cons, const double* u, const double* v,
                    const double* w, const R* mut, TerBuf<R> T, TkeBuf<R> tke, R* t11, R* t22, R* t33, R* t12, R* t13,
                    R* t23) {
    k_ter_strain<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, nrk, u, v, w, T, tke);
    k_ter_stress<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, cons, mut, T, t11, t22, t33, t12, t13, t23);
}
template <class R>
void launch_ter_slow_cell(const Params& P, cudaStream_t st, StateBuf S, StageAux<R> A, const double* u,
                          const double* v, const R* mut, TkeBuf<R> tke, TerBuf<R> T, R* Fcons, R* avx, R* avy,
                          R* avz) {
    if (P.use_diff)
        k_ter_rawflux<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, S.cons, mut, A.prim, P.alphaT_eff, P.invPr,
                                                                        T.fx[0], T.fy[0], nullptr, 0.0, 0.0, nullptr,
                                                                        nullptr);
    const bool u5 = P.dyc_h == TU5 && P.dyc_v == TU5;
    (u5 ? k_ter_slow_cell<R, TU5, TU5> : k_ter_slow_cell<R, -1, -1>)<<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(
        P, S, A, u, v, mut, tke, T, Fcons, avx, avy, avz);
}
template <class R>
void launch_ter_slow_mom(const Params& P, cudaStream_t st, StateBuf S, StageAux<R> A, const double* u,
                         const double* v, const double* w, const R* t11, const R* t22, const R* t33, const R* t12,
                         const R* t13, const R* t23, TerBuf<R> T, const R* Om, R* Fmx, R* Fmy, R* Fmz) {
    const bool u5 = P.dyc_h == TU5 && P.dyc_v == TU5;
    (u5 ? k_ter_slow_mom<R, TU5, TU5> : k_ter_slow_mom<R, -1, -1>)<<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(
        P, S, A, u, v, w, t11, t22, t33, t12, t13, t23, T, Om, Fmx, Fmy, Fmz);
}
template <class R>
void launch_ter_fast_h(const Params& P, cudaStream_t st, int step, double dtau, double facinv, StateBuf Sprev,
                       int prev_rt, StateBuf Sst, StageAux<R> A, const R* Fmx, const R* Fmy, const R* lag_in,
                       R* lag_out, TerBuf<R> T, R* avx, R* avy, double* outx, double* outy) {
    k_ter_fast_h<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(P, step, dtau, facinv, Sprev, prev_rt, Sst, A, Fmx,
                                                                   Fmy, lag_in, lag_out, T, avx, avy, outx, outy);
}
template <class R>
void launch_ter_fast_vert(const Params& P, cudaStream_t st, int tx, size_t smem, double dtau, double facinv,
                          double beta_1, double beta_2, StateBuf Sprev, int prev_rt, StateBuf Sst, StageAux<R> A,
                          const R* Fcons, const R* Fmz, TerBuf<R> T, const R* cA, const R* cInvB, const R* cCB,
                          const R* cP, const R* cQ, R* avz, double* out_cons, double* out_mz) {
    if (prev_rt)
        k_ter_fv_bnd<R><<<dim3((P.g.nx + 31) / 32, (P.g.ny + 3) / 4, 1), ter_block(), 0, st>>>(P, Sprev, T);
    dim3 grid((P.g.nx + tx - 1) / tx, P.g.ny, 1), block(tx, 1024 / tx, 1);
    k_ter_fast_vert<R><<<grid, block, smem, st>>>(P, dtau, facinv, beta_1, beta_2, Sprev, prev_rt, Sst, A, Fcons, Fmz,
                                                  T, cA, cInvB, cCB, cP, cQ, avz, out_cons, out_mz);
}
// Columns per block of k_ter_fast_vert (the widest power of two up to 32 whose
// FP64 column arrays fit) and its shared memory; 0 columns if none fits.
template <class R>
void ter_vert_attr(size_t smem) {
    cudaFuncSetAttribute(k_ter_fast_vert<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}
#if !ERFB_TER_F32
extern template void ter_vert_attr<float>(size_t);
void ter_vert_shape(int nz, int* tx, size_t* smem) {
    int dev = 0, maxopt = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxopt, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int t = 32;
    while (t >= 1 && (size_t)(7 * nz + 5) * t * sizeof(double) > (size_t)maxopt) t /= 2;
    *tx = t;
    *smem = t >= 1 ? (size_t)(7 * nz + 5) * t * sizeof(double) : 0;
    if (t >= 1) {
        ter_vert_attr<double>(*smem);
        ter_vert_attr<float>(*smem);
    }
}
#endif
namespace {
// The tiled post pass per scheme: dry scalars (and KE) and moisture
// species compile-time Upwind5 / WENO5 where the configuration has them,
// the run-time dispatch otherwise; NS = 2 holds the scalar and KE of a dry
// state, 5 the scalar, three species and KE.
template <class R>
using TerPostK = void (*)(Params, int, double, StateBuf, StateBuf, StateBuf, StateBuf, StageAux<R>, StageAux<R>, int,
                          const R*, TkeBuf<R>, TerBuf<R>, const R*, const R*, const R*, double*, double*, double*);
template <class R>
TerPostK<R> ter_post_kernel(const Params& P) {
    const bool du = P.dry_h == TU5 && P.dry_v == TU5, mw = P.moi_h == TW5 && P.moi_v == TW5;
    if (P.mt_znew) return k_ter_post<R, -1, -1, -1, -1, 2, true>;   // moving terrain: dry
    if (!P.moist) return du ? k_ter_post<R, TU5, TU5, -1, -1, 2> : k_ter_post<R, -1, -1, -1, -1, 2>;
    if (du && mw) return k_ter_post<R, TU5, TU5, TW5, TW5, 5>;
    return k_ter_post<R, -1, -1, -1, -1, 5>;
}
}  // namespace

template <class R>
void launch_ter_post(const Params& P, cudaStream_t st, int kz, double slow_dt, StateBuf Sold, StateBuf Sst,
                     StateBuf Ssum, StateBuf Snew, StageAux<R> Acur, StageAux<R> Anext, int make_next, const R* mut,
                     TkeBuf<R> tke, TerBuf<R> T, const R* avx, const R* avy, const R* avz, double* un, double* vn,
                     double* wn) {
    if (P.use_diff) {
        const int64_t N = P.g.ncell;
        const bool dd = P.les == ERF_LES_DEARDORFF;
        k_ter_rawflux<R><<<ter_grid(P.g, P.g.nz), ter_block(), 0, st>>>(
            P, Sst.cons, mut, Acur.prim + (int64_t)(ERF_RHOSCALAR_COMP - 1) * N, P.alphaC_eff, P.invSc, T.fx[0],
            T.fy[0], dd ? Acur.prim + (int64_t)(ERF_RHOKE_COMP - 1) * N : nullptr, 0.0, P.invSigmaK, T.fx[1],
            T.fy[1]);
    }
    ter_post_kernel<R>(P)<<<tile_grid(P.g, kz), dim3(TTX, TTY, 1), 0, st>>>(P, kz, slow_dt, Sold, Sst, Ssum, Snew,
                                                                            Acur, Anext, make_next, mut, tke, T, avx,
                                                                            avy, avz, un, vn, wn);
}
template <class R>
int ter_post_kz(const Params& P) {
    return pick_kz(ter_post_kernel<R>(P), P.g);
}

#define ERFB_TER_INSTANTIATE(R)                                                                                     \
    template void launch_ter_step_begin<R>(const Params&, cudaStream_t, const double*, const double*, const double*, \
                                           const double*, StateBuf, double*, double*, double*, StageAux<R>, R*,      \
                                           TkeBuf<R>);                                                               \
    template void launch_ter_tau<R>(const Params&, cudaStream_t, int, const double*, const double*, const double*,   \
                                    const double*, const R*, TerBuf<R>, TkeBuf<R>, R*, R*, R*, R*, R*, R*);          \
    template void launch_ter_slow_cell<R>(const Params&, cudaStream_t, StateBuf, StageAux<R>, const double*,         \
                                          const double*, const R*, TkeBuf<R>, TerBuf<R>, R*, R*, R*, R*);            \
    template void launch_ter_slow_mom<R>(const Params&, cudaStream_t, StateBuf, StageAux<R>, const double*,          \
                                         const double*, const double*, const R*, const R*, const R*, const R*,       \
                                         const R*, const R*, TerBuf<R>, const R*, R*, R*, R*);                       \
    template void launch_ter_fast_h<R>(const Params&, cudaStream_t, int, double, double, StateBuf, int, StateBuf,    \
                                       StageAux<R>, const R*, const R*, const R*, R*, TerBuf<R>, R*, R*, double*,    \
                                       double*);                                                                     \
    template void launch_ter_fast_vert<R>(const Params&, cudaStream_t, int, size_t, double, double, double, double, \
                                          StateBuf, int, StateBuf, StageAux<R>, const R*, const R*, TerBuf<R>,       \
                                          const R*, const R*, const R*, const R*, const R*, R*, double*, double*);   \
    template void launch_ter_post<R>(const Params&, cudaStream_t, int, double, StateBuf, StateBuf, StateBuf,         \
                                     StateBuf, StageAux<R>, StageAux<R>, int, const R*, TkeBuf<R>, TerBuf<R>,        \
                                     const R*, const R*, const R*, double*, double*, double*);                       \
    template int ter_post_kz<R>(const Params&);                                                                      \
    template void ter_vert_attr<R>(size_t);

#if !ERFB_TER_F32
ERFB_TER_INSTANTIATE(double)
#else
ERFB_TER_INSTANTIATE(float)
#endif
#undef ERFB_TER_INSTANTIATE

}  // namespace erfb
