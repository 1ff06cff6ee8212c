// api.cu -- host side of the C-ABI: context, device buffers, the multirate RK3
// step sequence (MRISplitIntegrator::advance, TimeIntegration/ERF_MRI.H:187-369)
// and its CUDA-graph replay.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kernels.cuh"
#include "mlp.cuh"

// NVTX range for the length of a scope (an entry point or a step's launch)
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace erfb {
__global__ void k_kessler(Params P, double* cons, double dtn, double dz);
__global__ void k_kessler_cells(Params P, const double* cin, double* cout, double dtn, double dz);
__global__ void k_base_state(int nz, double dz, double g, double rdOcp, const double* th_cc, const double* qv_cc,
                             double th_s, double qv_s, double p_s, double* rho0, double* p0o, double* pi0o,
                             double* th0o);
__global__ void k_pack(Geo g, erf_b200_fab f, int kind, int ncomp, double* dst);
__global__ void k_unpack(Geo g, erf_b200_fab f, int kind, int ncomp, const double* src, int tang_lo_zero,
                         int tang_hi_zero, int wall_w);
}  // namespace erfb

using namespace erfb;

// Bulk arrays of a context (type R: double plain, float mixed).
template <class R>
struct Bulk {
    R *Fcons, *Fmx, *Fmy, *Fmz;   // slow right-hand sides
    R *avx, *avy, *avz;           // average momenta of the substeps
    R* lag[2];                    // lagged d(rho theta), ping-pong
    StageAux<R> aux[2];           // stage primitives, Exner, p'
    R* mut;                       // eddy viscosity
    R *t11, *t22, *t33, *t12, *t13, *t23;
    R *cA, *cInvB, *cCB, *cP, *cQ;  // fast coefficients of the current stage
    R *c12 = nullptr, *c13 = nullptr, *c23 = nullptr;  // learned closure: cell-centred off-diagonal stresses
    R *hx = nullptr, *hy = nullptr, *hz = nullptr;     // learned closure: rho * heat flux
    TkeBuf<R> tke{nullptr, nullptr, nullptr, nullptr}; // Deardorff closure arrays
    TerBuf<R> ter{};                                    // static terrain scratch
};

// Threads per block of the vertical acoustic kernel (columns x level groups).
#ifndef ERFB_VERT_THREADS
#define ERFB_VERT_THREADS 1024
#endif

struct erf_b200_ctx {
    erf_b200_config cfg;
    Params P;
    Geo g;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // side branch of a stage: the plane averages and the fast coefficients
    // depend only on the stage state, so they run beside tau / slow_cell /
    // slow_mom (forked and joined with events; captured into the graphs)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_pavg = nullptr, ev_coef = nullptr;
    int device = 0;
    size_t bytes = 0;
    std::vector<void*> allocs;

    StateBuf S[4];            // [0],[1] alternate old/new, [2] second stage buffer, [3] fast sum
    double* vel[2][3];        // alternating old/new face velocities (FP64 prognostic)
    double* pavg;
    double* most_avg;         // MOST plane means {u, v, |U|, u*} of the step
    bool most_set = false;    // per-pass entries: most_avg made by erf_b200_most_update_fluxes
    Bulk<double> bd;          // bulk arrays of the plain form
    Bulk<float> bf;           // bulk arrays of the mixed form
    bool mixed = false;
    const erf_b200_mlp* net = nullptr;   // learned closure (les_type ERF_LES_MLP)
    unsigned int* fallback = nullptr;    // cells that fell back to Smagorinsky
    int closure_grid = 1;
    double* feat_theta = nullptr;        // feature extraction scratch
    float* feat_out = nullptr;
    int tile_tx = 32, vert_warps = 32, coef_warps = 8;
    TiledKz tkz{1, 1, 1};
    size_t vert_smem = 0, coef_smem = 0;
    double *r0, *p0, *pi0, *th0;   // nz+2 values, or (nz+2) planes with terrain
    double *znd = nullptr, *detJ = nullptr, *zcc = nullptr;   // static terrain
    double* met = nullptr;                                    // its metric tables
    // moving terrain: the grids at the step's old time (z[0] = znd, with
    // met / detJ / zcc) and at the stage's source (z[1], with met1 / detJ1 /
    // zcc1) and new (z[2]) times; z_t; the step's old base state; the clock
    struct MovingTerrain {
        double* z[5];                  // + the substep's old and new grids
        double *met1, *detJ1, *zcc1;
        double* zt;
        double *r0o, *p0o;
        double* time;
        double *detJso, *zpt, *trhs, *om, *soln;   // acoustic substeps
        double* fac;                              // Sullivan's factor per level
    } mt{};
    int ter_tx = 0;                                           // k_ter_fast_vert columns per block
    size_t ter_smem = 0;                                      // and its shared memory
    bool ter_set = false;
    int last = -1;               // state slot of the latest state (erf_b200_diagnostics)
    double* diag = nullptr;      // its scratch (partials, result)
    double *h_stage;          // device staging buffers for the host-array entry point
    int* status;
    bool base_set = false;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaGraph_t graph_raw[2] = {nullptr, nullptr};   // kept for ensemble graphs
    int lag_parity_per_step = 0;
    int cur = -1;             // slot of the resident state (-1: none loaded)
};

namespace {

thread_local cudaError_t g_last_cuda_error = cudaSuccess;   // for erf_b200_last_cuda_error

int cuda_fail(cudaError_t e) {
    if (e == cudaSuccess) return ERF_B200_OK;
    g_last_cuda_error = e;
    return e == cudaErrorMemoryAllocation ? ERF_B200_ENOMEM : ERF_B200_ECUDA;
}
#define CK(x)                                   \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return cuda_fail(e_); \
    } while (0)

template <class T>
int dalloc(erf_b200_ctx* c, T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(e);
    cudaMemsetAsync(q, 0, n * sizeof(T), c->stream);
    c->allocs.push_back(q);
    c->bytes += n * sizeof(T);
    *p = (T*)q;
    return ERF_B200_OK;
}

bool adv_supported(int t) {
    return t == ERF_ADV_CENTERED_2ND || t == ERF_ADV_UPWIND_3RD || t == ERF_ADV_CENTERED_4TH ||
           t == ERF_ADV_UPWIND_5TH || t == ERF_ADV_CENTERED_6TH || t == ERF_ADV_WENO_3 || t == ERF_ADV_WENO_5;
}

// The MOST reference height snapped to the cell centre of its level
// (MOSTAverage::set_z_positions, ERF_MOSTAverage.cpp:257-300, no
// interpolation); 0 means the first cell centre.
void most_reference_level(const erf_b200_config& c, int& k, double& zref) {
    const double zr = c.most_zref > 0.0 ? c.most_zref : 0.5 * c.dz;
    k = static_cast<int>(std::floor(zr / c.dz - 0.5));
    zref = (k + 0.5) * c.dz;
}

int validate(const erf_b200_config* c) {
    if (!c) return ERF_B200_EINVAL;
    if (c->nx < 4 || c->ny < 4 || c->nz < 4) return ERF_B200_ECONFIG;
    if (!(c->dx > 0 && c->dy > 0 && c->dz > 0 && c->dt > 0)) return ERF_B200_ECONFIG;
    if (c->substepping_type != ERF_SUBSTEP_IMPLICIT && c->substepping_type != ERF_SUBSTEP_NONE) return ERF_B200_ECONFIG;
    // the substep ratio matters with substepping only (ERF_MRI.H:202-204)
    if (c->substepping_type == ERF_SUBSTEP_IMPLICIT && (c->mri_ratio < 2 || (c->mri_ratio % 2) != 0))
        return ERF_B200_ECONFIG;
    if (c->zlo_bc != ERF_BC_NO_SLIP_WALL && c->zlo_bc != ERF_BC_SLIP_WALL && c->zlo_bc != ERF_BC_MOST)
        return ERF_B200_ECONFIG;
    if (c->zhi_bc != ERF_BC_NO_SLIP_WALL && c->zhi_bc != ERF_BC_SLIP_WALL) return ERF_B200_ECONFIG;
    if (c->zlo_bc == ERF_BC_MOST) {
        // MOST ground: flat, under an eddy-viscosity closure (eta of the ghost
        // rule), z0 below the snapped reference height; with moisture the
        // adiabatic ground adds no moisture flux (the reference computes one
        // for its CUSTOM flux type only, ERF_ABLMost.cpp:413-433)
        if (c->use_terrain) return ERF_B200_ECONFIG;
        if (c->les_type != ERF_LES_SMAGORINSKY && c->les_type != ERF_LES_DEARDORFF) return ERF_B200_ECONFIG;
        if (!(c->most_z0 > 0.0) || !(c->most_zref >= 0.0) || !(c->most_zref < c->nz * c->dz)) return ERF_B200_ECONFIG;
        int k;
        double zr;
        most_reference_level(*c, k, zr);
        if (k < 0 || k >= c->nz || !(zr > c->most_z0)) return ERF_B200_ECONFIG;
    }
    // the vertical momentum stencils reduce order near walls only for the
    // Upwind/Centered family (ERF_AdvectionSrcForMom_N.H:225-265)
    if (!adv_supported(c->dycore_horiz_adv) || !adv_supported(c->dycore_vert_adv)) return ERF_B200_ECONFIG;
    if (c->dycore_horiz_adv == ERF_ADV_WENO_3 || c->dycore_horiz_adv == ERF_ADV_WENO_5) return ERF_B200_ECONFIG;
    if (c->dycore_vert_adv == ERF_ADV_WENO_3 || c->dycore_vert_adv == ERF_ADV_WENO_5) return ERF_B200_ECONFIG;
    // Centered_2nd in both directions takes AdvectionSrcForMom's simplified
    // form (ERF_AdvectionSrcForMom.cpp:95-110, 205-215), built on the terrain path
    if (!c->use_terrain && c->dycore_horiz_adv == ERF_ADV_CENTERED_2ND && c->dycore_vert_adv == ERF_ADV_CENTERED_2ND)
        return ERF_B200_ECONFIG;
    if (!adv_supported(c->dryscal_horiz_adv) || !adv_supported(c->dryscal_vert_adv)) return ERF_B200_ECONFIG;
    if (!adv_supported(c->moistscal_horiz_adv) || !adv_supported(c->moistscal_vert_adv)) return ERF_B200_ECONFIG;
    if (c->les_type != ERF_LES_NONE && c->les_type != ERF_LES_SMAGORINSKY && c->les_type != ERF_LES_DEARDORFF &&
        c->les_type != ERF_LES_MLP)
        return ERF_B200_ECONFIG;
    if (c->les_type == ERF_LES_DEARDORFF && (!(c->theta_ref > 0.0) || !(c->sigma_k > 0.0) || !(c->Ck > 0.0)))
        return ERF_B200_ECONFIG;
    if (c->les_type == ERF_LES_MLP && c->molec_diff_type != ERF_MOLEC_NONE) return ERF_B200_ECONFIG;
    if (c->use_terrain != 0 && c->use_terrain != 1) return ERF_B200_ECONFIG;
    if (c->terrain_type != ERF_TERRAIN_STATIC && c->terrain_type != ERF_TERRAIN_MOVING) return ERF_B200_ECONFIG;
    if (c->terrain_type == ERF_TERRAIN_MOVING) {
        // moving terrain: the reference's MovingTerrain setting -- dry,
        // Centered_2nd dycore (asserted by slow_rhs_fun_pre), no diffusion,
        // buoyancy type 1, slip walls
        if (!c->use_terrain) return ERF_B200_ECONFIG;
        if (c->moisture != ERF_MOIST_NONE || c->les_type != ERF_LES_NONE || c->molec_diff_type != ERF_MOLEC_NONE)
            return ERF_B200_ECONFIG;
        if (c->dycore_horiz_adv != ERF_ADV_CENTERED_2ND || c->dycore_vert_adv != ERF_ADV_CENTERED_2ND)
            return ERF_B200_ECONFIG;
        if (c->buoyancy_type != 1 || c->zlo_bc != ERF_BC_SLIP_WALL || c->zhi_bc != ERF_BC_SLIP_WALL)
            return ERF_B200_ECONFIG;
        if (!(c->mt_wavelength > 0.0) || !(std::fabs(c->mt_ampl) < 0.5 * c->nz * c->dz)) return ERF_B200_ECONFIG;
    } else if (c->no_lagged_delta_rt) {
        return ERF_B200_ECONFIG;   // the reference allows it for moving terrain only (ERF_DataStruct.H:389)
    }
    if (c->use_terrain) {
        // terrain path: LES closure (or no diffusion), explicit closures only;
        // with moisture, buoyancy type 1 (total density against the 3-D base state)
        if (c->les_type == ERF_LES_MLP) return ERF_B200_ECONFIG;
        if (c->les_type == ERF_LES_NONE && c->molec_diff_type != ERF_MOLEC_NONE) return ERF_B200_ECONFIG;
        if (c->moisture != ERF_MOIST_NONE && c->buoyancy_type != 1) return ERF_B200_ECONFIG;
    }
    if (c->molec_diff_type < 0 || c->molec_diff_type > 2) return ERF_B200_ECONFIG;
    if (c->moisture == ERF_MOIST_NONE) {
        if (c->ncomp != 5) return ERF_B200_ECONFIG;
    } else if (c->moisture == ERF_MOIST_KESSLER) {
        if (c->ncomp != 8) return ERF_B200_ECONFIG;
    } else if (c->moisture == ERF_MOIST_KESSLER_NORAIN) {
        if (c->ncomp != 7 || c->buoyancy_type != 1) return ERF_B200_ECONFIG;
    } else {
        return ERF_B200_ECONFIG;
    }
    if (c->buoyancy_type != 1 && c->buoyancy_type != 2 && c->buoyancy_type != 3) return ERF_B200_ECONFIG;
    if (c->precision != ERF_PREC_FP64 && c->precision != ERF_PREC_MIXED) return ERF_B200_ECONFIG;
    return ERF_B200_OK;
}

void make_params(erf_b200_ctx* c) {
    const erf_b200_config& f = c->cfg;
    Geo& g = c->g;
    g.nx = f.nx; g.ny = f.ny; g.nz = f.nz;
    g.sk = (int64_t)f.nx * f.ny;
    g.ncell = g.sk * f.nz;
    g.nzf = g.sk * (f.nz + 1);
    g.dxi = 1.0 / f.dx; g.dyi = 1.0 / f.dy; g.dzi = 1.0 / f.dz;
    g.zlo_noslip = f.zlo_bc == ERF_BC_NO_SLIP_WALL;
    g.zhi_noslip = f.zhi_bc == ERF_BC_NO_SLIP_WALL;
#ifdef ERF_B200_BOUNDS
    g.oob = c->status;
#endif
    Params& P = c->P;
    P.g = g;
    P.ncomp = f.ncomp; P.nprim = f.ncomp - 1;
    P.moist = f.moisture != ERF_MOIST_NONE;
    P.kessler_rain = f.moisture == ERF_MOIST_KESSLER;
    P.use_turb = f.les_type != ERF_LES_NONE;
    P.use_diff = (f.molec_diff_type != ERF_MOLEC_NONE) || P.use_turb;
    P.use_consA = f.molec_diff_type == ERF_MOLEC_CONSTANT_ALPHA;
    P.les = f.les_type;
    // Smagorinsky length scale in the reference's order
    // (ERF_ComputeTurbulentViscosity.cpp:95-97), with map factors 1
    double cellVolMsf = 1.0 / (g.dxi * 1.0 * g.dyi * 1.0 * g.dzi);
    double DeltaMsf = std::pow(cellVolMsf, 1.0 / 3.0);
    P.CsDeltaSqr = f.Cs * f.Cs * DeltaMsf * DeltaMsf;
    P.Cs = f.Cs;
    P.ter = f.use_terrain;
    P.znd = c->znd;
    P.detJ = c->detJ;
    P.met = c->met;
    P.mt_zt = nullptr;
    P.mt_znew = nullptr;
    P.mt_fac = c->mt.fac;
    {
        const double PI = 3.14159265358979323846264338327950288;
        P.mt_ampl = f.mt_ampl;
        P.mt_kp = f.mt_wavelength > 0.0 ? 2.0 * PI / f.mt_wavelength : 0.0;
        P.mt_om = std::sqrt(9.81 * P.mt_kp);   // deep-water gravity wave, CONST_GRAV
        P.mt_dx = f.dx;
        P.mt_dz = f.dz;
    }
    // Deardorff constants (ERF_ComputeTurbulentViscosity.cpp:129-142) and the
    // buoyancy factor of the TKE source (ERF_DiffusionSrcForState_N.cpp:681-697)
    P.Delta = DeltaMsf;
    P.Ck = f.Ck;
    P.Ce_wall = f.Ce_wall;
    P.Ce_lcoeff = std::max(0.0, f.Ce - 1.9 * f.Ck);
    P.g_over_theta0 = std::fabs(f.gravity) * (1.0 / f.theta_ref);
    P.invSigmaK = 1.0 / f.sigma_k;
    P.invPr = 1.0 / f.Pr_t;
    P.invSc = 1.0 / f.Sc_t;
    P.alphaT_eff = P.use_consA ? f.alpha_T : f.rho0_trans * f.alpha_T;
    P.alphaC_eff = P.use_consA ? f.alpha_C : f.rho0_trans * f.alpha_C;
    P.mu_eff = P.use_consA ? 2.0 * f.dynamic_viscosity / f.rho0_trans : 2.0 * f.dynamic_viscosity;
    P.gravity = f.gravity;
    P.rdOcp = R_d / f.c_p;
    P.c_p = f.c_p;
    P.c_v = f.c_p - R_d;
    P.halfg = std::abs(0.5 * -f.gravity);
    P.buoy_type = f.buoyancy_type;
    P.coriolis = f.use_coriolis;
    P.cf = f.coriolis_factor; P.sinphi = f.sinphi; P.cosphi = f.cosphi;
    P.geo0 = f.abl_geo_forcing[0]; P.geo1 = f.abl_geo_forcing[1]; P.geo2 = f.abl_geo_forcing[2];
    P.dyc_h = f.dycore_horiz_adv; P.dyc_v = f.dycore_vert_adv;
    P.dry_h = f.dryscal_horiz_adv; P.dry_v = f.dryscal_vert_adv;
    P.moi_h = f.moistscal_horiz_adv; P.moi_v = f.moistscal_vert_adv;
    P.f_dyc_h = f.dycore_horiz_upw_frac; P.f_dyc_v = f.dycore_vert_upw_frac;
    P.f_dry_h = f.dryscal_horiz_upw_frac; P.f_dry_v = f.dryscal_vert_upw_frac;
    P.f_moi_h = f.moistscal_horiz_upw_frac; P.f_moi_v = f.moistscal_vert_upw_frac;
    P.r0 = c->r0; P.p0 = c->p0; P.pi0 = c->pi0;
    P.status = c->status;
    P.most = f.zlo_bc == ERF_BC_MOST;
    most_reference_level(f, P.most_k, P.most_zref);
    P.most_z0 = f.most_z0;
    P.most_dz = f.dz;
    P.most_avg = c->most_avg;
    P.most_mut_f32 = c->mixed ? 1 : 0;
    P.most_mut = c->mixed ? (const void*)c->bf.mut : (const void*)c->bd.mut;
}

dim3 cell_block() { return dim3(32, 4, 1); }
dim3 cell_grid(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz); }
dim3 col_block() { return dim3(32, 4, 1); }
dim3 col_grid(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, 1); }

// Substep schedule of MRISplitIntegrator::advance (ERF_MRI.H:255-282).
// Without substepping every stage takes one update of its whole length.
bool no_substepping(const erf_b200_config& f) { return f.substepping_type == ERF_SUBSTEP_NONE; }
void stage_schedule(const erf_b200_config& f, int nrk, int& nsub, double& dtau, double& slow_dt) {
    double dt = f.dt;
    const bool nosub = no_substepping(f);
    double sub_dt = nosub ? 0.0 : dt / f.mri_ratio;
    if (nrk == 0) {
        if (f.force_stage1_single_substep || nosub) { nsub = 1; dtau = dt / 3.0; }
        else { nsub = f.mri_ratio / 3; dtau = sub_dt; }
        slow_dt = dt / 3.0;
    } else if (nrk == 1) {
        if (nosub) { nsub = 1; dtau = 0.5 * dt; }
        else { nsub = f.mri_ratio / 2; dtau = sub_dt; }
        slow_dt = dt / 2.0;
    } else {
        if (nosub) { nsub = 1; dtau = dt; }
        else { nsub = f.mri_ratio; dtau = sub_dt; }
        slow_dt = dt;
    }
}

int substeps_per_step(const erf_b200_config& f) {
    if (no_substepping(f)) return 0;   // no acoustic substeps, no lagged d(rho theta)
    int tot = 0;
    for (int nrk = 0; nrk < 3; ++nrk) { int n; double a, b; stage_schedule(f, nrk, n, a, b); tot += n; }
    return tot;
}

// Optional per-launch event timing (profiling entry point only).
struct LaunchTimer {
    cudaStream_t st;
    std::vector<cudaEvent_t> ev;
    std::vector<int> slot;
    size_t used = 0;
    void mark(int s) {
        if (used + 2 > ev.size()) {
            for (int q = 0; q < 64; ++q) { cudaEvent_t e; cudaEventCreate(&e); ev.push_back(e); }
        }
        cudaEventRecord(ev[used], st);
        slot.push_back(s);
        used += 2;
    }
    void done() { cudaEventRecord(ev[used - 1], st); }
};
// NVTX range names of the pass slots (the tracing tools' timeline; the
// calls cost a pointer test when no tool is attached)
static const char* const kPassName[] = {"step_begin", "stress", "slow_cell", "plane_avg", "slow_mom",
                                        "fast_horizontal", "fast_column", "slow_post", "kessler", "fast_coeffs",
                                        "no_substep"};
#define TIMED(slotid, launch)                 \
    do {                                      \
        nvtxRangePushA(kPassName[slotid]);    \
        if (T) T->mark(slotid);               \
        launch;                               \
        if (T) T->done();                     \
        nvtxRangePop();                       \
    } while (0)

// One full step over static terrain: the same stage / substep schedule with
// the terrain passes (dry states only).
template <class R>
void enqueue_step_ter(erf_b200_ctx* c, Bulk<R>& B, int p, LaunchTimer* T) {
    const Params& P = c->P;
    const Geo& g = c->g;
    cudaStream_t st = c->stream;
    StateBuf OLD = c->S[p], N0 = c->S[1 - p], N1 = c->S[2], SUM = c->S[3];
    double** Vold = c->vel[p];
    double** Vnew = c->vel[1 - p];
    TIMED(0, launch_ter_step_begin<R>(P, st, OLD.cons, Vold[0], Vold[1], Vold[2], OLD, Vnew[0], Vnew[1], Vnew[2],
                                      B.aux[0], B.mut, B.tke));
    // stage outputs alternate between the two scratch states so that the last
    // one lands in slot 1-p (or in N1 when Kessler moves it to slot 1-p)
    StateBuf outs[3] = {N0, N1, N0};
    if (P.moist) { outs[0] = N1; outs[1] = N0; outs[2] = N1; }
    StateBuf stage[3] = {OLD, outs[0], outs[1]};
    dim3 tg((g.nx + c->tile_tx - 1) / c->tile_tx, g.ny, 1), tcb(c->tile_tx, c->coef_warps, 1);
    const bool fork = T == nullptr && c->side;
    int a = 0;
    int lp = (p * c->lag_parity_per_step) & 1;
    const double beta_s = 0.1;
    const double beta_1 = 0.5 * (1.0 - beta_s), beta_2 = 0.5 * (1.0 + beta_s);
    const bool nosub = no_substepping(c->cfg);
    for (int nrk = 0; nrk < 3; ++nrk) {
        StateBuf Sst = stage[nrk], Snew = outs[nrk];
        StageAux<R> Acur = B.aux[a], Anext = B.aux[1 - a];
        int nsub; double dtau, slow_dt;
        stage_schedule(c->cfg, nrk, nsub, dtau, slow_dt);
        double facinv = 1.0 / (double)nsub;
        double D = dtau * dtau * beta_2 * beta_2 * g.dzi;
        if (fork && !nosub) {
            cudaEventRecord(c->ev_fork, st);
            cudaStreamWaitEvent(c->side, c->ev_fork, 0);
            launch_fast_coef<R>(P, c->side, tg, tcb, c->coef_smem, D, Sst, Acur, B.cA, B.cInvB, B.cCB, B.cP, B.cQ);
            cudaEventRecord(c->ev_coef, c->side);
        }
        if (P.use_diff)
            TIMED(1, launch_ter_tau<R>(P, st, nrk, Sst.cons, Vnew[0], Vnew[1], Vnew[2], B.mut, B.ter, B.tke, B.t11,
                                       B.t22, B.t33, B.t12, B.t13, B.t23));
        TIMED(2, launch_ter_slow_cell<R>(P, st, Sst, Acur, Vnew[0], Vnew[1], B.mut, B.tke, B.ter, B.Fcons, B.avx,
                                         B.avy, B.avz));
        TIMED(4, launch_ter_slow_mom<R>(P, st, Sst, Acur, Vnew[0], Vnew[1], Vnew[2], B.t11, B.t22, B.t33, B.t12, B.t13,
                                        B.t23, B.ter, B.avz, B.Fmx, B.Fmy, B.Fmz));
        if (nosub)
            TIMED(10, launch_no_substep<R>(P, st, slow_dt, OLD, B.Fcons, B.Fmx, B.Fmy, B.Fmz, SUM));
        else if (!fork)
            TIMED(9, launch_fast_coef<R>(P, st, tg, tcb, c->coef_smem, D, Sst, Acur, B.cA, B.cInvB, B.cCB, B.cP, B.cQ));
        else
            cudaStreamWaitEvent(st, c->ev_coef, 0);
        for (int ks = 0; ks < (nosub ? 0 : nsub); ++ks) {
            StateBuf Sprev = (ks == 0) ? OLD : SUM;
            int prt = ks > 0;
            TIMED(5, launch_ter_fast_h<R>(P, st, ks, dtau, facinv, Sprev, prt, Sst, Acur, B.Fmx, B.Fmy, B.lag[lp],
                                          B.lag[1 - lp], B.ter, B.avx, B.avy, SUM.mx, SUM.my));
            lp ^= 1;
            TIMED(6, launch_ter_fast_vert<R>(P, st, c->ter_tx, c->ter_smem, dtau, facinv, beta_1, beta_2, Sprev, prt,
                                             Sst, Acur, B.Fcons, B.Fmz, B.ter, B.cA, B.cInvB, B.cCB, B.cP, B.cQ,
                                             B.avz, SUM.cons, SUM.mz));
        }
        TIMED(7, launch_ter_post<R>(P, st, c->tkz.ter_post, slow_dt, OLD, Sst, SUM, Snew, Acur, Anext, nrk < 2 ? 1 : 0, B.mut, B.tke,
                                    B.ter, B.avx, B.avy, B.avz, Vnew[0], Vnew[1], Vnew[2]));
        a = 1 - a;
    }
    if (P.moist) {   // Kessler with the sedimentation over detJ
        dim3 kb(32, 1, KESS_KB), kg((g.nx + 31) / 32, g.ny, (g.nz + KESS_KB - 1) / KESS_KB);
        TIMED(8, (k_kessler_cells<<<kg, kb, 0, st>>>(P, N1.cons, N0.cons, c->cfg.dt, c->cfg.dz)));
    }
}

// One step over moving terrain without acoustic substepping
// (MRISplitIntegrator::advance with the moving-terrain branches of
// slow_rhs_fun_pre, no_substep_fun and slow_rhs_fun_post, then
// post_timestep).  The grid at the step's old time and its tables serve the
// step prologue and the slow-variable pass; each stage regenerates the grid
// at its source time (tables for the slow right-hand side) and at its new
// time, forms z_t, updates the base state after the slow right-hand side
// and applies the detJ-weighted stage update.  Every launch reads the
// device clock, so the captured graph replays for any step.
template <class R>
void enqueue_step_mt(erf_b200_ctx* c, Bulk<R>& B, int p, LaunchTimer* T) {
    Params Po = c->P;
    Po.mt_zt = c->mt.zt;
    Po.mt_znew = c->mt.z[2];
    const bool nosub = no_substepping(c->cfg);
    Params Ps = Po;
    Ps.znd = c->mt.z[1];
    Ps.met = c->mt.met1;
    Ps.detJ = c->mt.detJ1;
    const double dt = c->cfg.dt;
    cudaStream_t st = c->stream;
    const size_t nb = (size_t)(c->cfg.nz + 2) * c->cfg.nx * c->cfg.ny * sizeof(double);
    StateBuf OLD = c->S[p], N0 = c->S[1 - p], N1 = c->S[2], SUM = c->S[3];
    double** Vold = c->vel[p];
    double** Vnew = c->vel[1 - p];
    launch_mt_grid(Po, st, c->mt.time, dt, 0, c->mt.z[0]);
    launch_ter_metrics(Po, st, c->detJ, c->zcc);
    cudaMemcpyAsync(c->mt.r0o, c->r0, nb, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(c->mt.p0o, c->p0, nb, cudaMemcpyDeviceToDevice, st);
    TIMED(0, launch_ter_step_begin<R>(Po, st, OLD.cons, Vold[0], Vold[1], Vold[2], OLD, Vnew[0], Vnew[1], Vnew[2],
                                      B.aux[0], B.mut, B.tke));
    StateBuf outs[3] = {N0, N1, N0};
    StateBuf stage[3] = {OLD, outs[0], outs[1]};
    int a = 0;
    for (int nrk = 0; nrk < 3; ++nrk) {
        StateBuf Sst = stage[nrk], Snew = outs[nrk];
        StageAux<R> Acur = B.aux[a], Anext = B.aux[1 - a];
        int nsub; double dtau, slow_dt;
        stage_schedule(c->cfg, nrk, nsub, dtau, slow_dt);
        const int ts_src = nrk, ts_new = nrk + 1;   // T, T + dt/3, T + dt/2, T + dt
        launch_mt_grid(Po, st, c->mt.time, dt, ts_src, c->mt.z[1]);
        launch_mt_grid(Po, st, c->mt.time, dt, ts_new, c->mt.z[2]);
        launch_ter_metrics(Ps, st, c->mt.detJ1, c->mt.zcc1);
        launch_mt_zt(Po, st, c->mt.z[0], c->mt.z[2], c->mt.time, dt, ts_new, c->mt.zt);
        TIMED(2, launch_ter_slow_cell<R>(Ps, st, Sst, Acur, Vnew[0], Vnew[1], B.mut, B.tke, B.ter, B.Fcons, B.avx,
                                         B.avy, B.avz));
        TIMED(4, launch_ter_slow_mom<R>(Ps, st, Sst, Acur, Vnew[0], Vnew[1], Vnew[2], B.t11, B.t22, B.t33, B.t12,
                                        B.t13, B.t23, B.ter, B.avz, B.Fmx, B.Fmy, B.Fmz));
        launch_mt_base_state(Po, st, c->mt.r0o, c->mt.p0o, c->mt.z[0], c->mt.z[1], c->mt.z[2], c->mt.time, dt,
                             ts_new, c->r0, c->p0);
        Params Pp = Po;   // the slow-variable pass: the level's grid when it runs
        if (nosub) {
            TIMED(10, launch_mt_no_substep<R>(Po, st, nsub * dtau, OLD, B.Fcons, B.Fmx, B.Fmy, B.Fmz, c->mt.z[0],
                                              c->mt.z[2], SUM));
        } else {
            // fast_rhs_fun, moving terrain (ERF_TI_fast_rhs_fun.H:47-118): per
            // substep the grids at its old and new times, z_t'', the fast
            // coefficients on the old grid with the step's old base state;
            // the level keeps the last substep's old grid and its new one
            // serves the slow-variable update
            const double beta_s = 0.1;
            const double D = dtau * dtau * (0.5 * (1.0 + beta_s)) * (0.5 * (1.0 + beta_s)) * c->g.dzi;
            dim3 tg((c->g.nx + c->tile_tx - 1) / c->tile_tx, c->g.ny, 1), tcb(c->tile_tx, c->coef_warps, 1);
            Params Pf = Po;
            Pf.detJ = c->mt.detJso;
            Pf.r0 = c->mt.r0o;
            int lp = 0;
            // the substep grids alternate: a substep's new grid is the next one's old grid
            double *zso = c->mt.z[3], *zsn = c->mt.z[4];
            launch_mt_grid_sub(Po, st, c->mt.time, dtau, 0, zso);
            for (int ks = 0; ks < nsub; ++ks) {
                if (ks > 0) std::swap(zso, zsn);
                launch_mt_grid_sub(Po, st, c->mt.time, dtau, ks + 1, zsn);
                launch_mt_zpt(Po, st, zso, zsn, dtau, c->mt.zpt);
                launch_mt_detj(Po, st, zso, c->mt.detJso);
                TIMED(9, launch_fast_coef<R>(Pf, st, tg, tcb, c->coef_smem, D, Sst, Acur, B.cA, B.cInvB, B.cCB, B.cP,
                                             B.cQ));
                TIMED(6, launch_mt_fast<R>(Po, st, ks, c->cfg.no_lagged_delta_rt ? 0 : 1, dtau, beta_s,
                                           1.0 / (double)nsub, ks == 0 ? OLD : SUM, Sst, Acur, B.Fcons, B.Fmx, B.Fmy,
                                           B.Fmz, B.lag[lp], B.lag[1 - lp], B.cA, B.cInvB, B.cCB, B.cP, B.cQ,
                                           zso, zsn, c->mt.z[1], c->mt.zpt, c->mt.trhs, c->mt.om,
                                           c->mt.soln, B.avx, B.avy, B.avz, SUM, ks == nsub - 1 ? 1 : 0));
                lp ^= 1;
            }
            Pp.znd = zso;
            Pp.detJ = c->mt.detJso;
            Pp.mt_znew = zsn;
        }
        TIMED(7, launch_ter_post<R>(Pp, st, c->tkz.ter_post, slow_dt, OLD, Sst, SUM, Snew, Acur, Anext,
                                    nrk < 2 ? 1 : 0, B.mut, B.tke, B.ter, B.avx, B.avy, B.avz, Vnew[0], Vnew[1],
                                    Vnew[2]));
        a = 1 - a;
    }
    launch_mt_advance_time(st, c->mt.time, dt);
}

// Enqueue one full step with parity p (state slot p is the old state).
template <class R>
void enqueue_step_t(erf_b200_ctx* c, Bulk<R>& B, int p, LaunchTimer* T) {
    if (c->P.ter) {
        if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) enqueue_step_mt<R>(c, B, p, T);
        else enqueue_step_ter<R>(c, B, p, T);
        return;
    }
    const Params& P = c->P;
    const Geo& g = c->g;
    cudaStream_t st = c->stream;
    StateBuf OLD = c->S[p], N0 = c->S[1 - p], N1 = c->S[2], SUM = c->S[3];
    double** Vold = c->vel[p];
    double** Vnew = c->vel[1 - p];

    TIMED(0, launch_step_begin<R>(P, st, OLD.cons, Vold[0], Vold[1], Vold[2], OLD, Vnew[0], Vnew[1], Vnew[2],
                                  B.aux[0], B.mut, B.tke));
    // the MOST plane means and u* of the step (ERF_Advance.cpp:62-86)
    if (P.most) TIMED(0, launch_most_avg(P, st, Vold[0], Vold[1]));
    // stage outputs alternate between the two scratch states so that the last
    // one lands in slot 1-p (or in N1 when Kessler moves it to slot 1-p)
    StateBuf outs[3] = {N0, N1, N0};
    if (P.moist) { outs[0] = N1; outs[1] = N0; outs[2] = N1; }
    StateBuf stage[3] = {OLD, outs[0], outs[1]};
    dim3 tb(c->tile_tx, c->vert_warps, 1), tg((g.nx + c->tile_tx - 1) / c->tile_tx, g.ny, 1);
    dim3 tcb(c->tile_tx, c->coef_warps, 1);
    const bool fork = T == nullptr && c->side;   // per-kernel timing keeps one stream
    int a = 0;
    int lp = (p * c->lag_parity_per_step) & 1;
    const double beta_s = 0.1;
    const double beta_1 = 0.5 * (1.0 - beta_s), beta_2 = 0.5 * (1.0 + beta_s);
    const bool nosub = no_substepping(c->cfg);
    for (int nrk = 0; nrk < 3; ++nrk) {
        StateBuf Sst = stage[nrk], Snew = outs[nrk];
        StageAux<R> Acur = B.aux[a], Anext = B.aux[1 - a];
        int nsub; double dtau, slow_dt;
        stage_schedule(c->cfg, nrk, nsub, dtau, slow_dt);
        const bool plane = P.moist && P.buoy_type == 2;
        double facinv = 1.0 / (double)nsub;
        double D = dtau * dtau * beta_2 * beta_2 * g.dzi;
        if (fork) {
            cudaEventRecord(c->ev_fork, st);
            cudaStreamWaitEvent(c->side, c->ev_fork, 0);
            if (plane) {
                launch_plane_avg<R>(P, c->side, Sst.cons, Acur.prim, c->pavg);
                cudaEventRecord(c->ev_pavg, c->side);
            }
            if (!nosub)
                launch_fast_coef<R>(P, c->side, tg, tcb, c->coef_smem, D, Sst, Acur, B.cA, B.cInvB, B.cCB, B.cP, B.cQ);
            cudaEventRecord(c->ev_coef, c->side);
        }
        if (P.les == ERF_LES_MLP) {
            ClosureNet net{c->net->wpack, c->net->bias, c->net->norm, c->net->env, c->fallback};
            TIMED(1, launch_closure<R>(P, net, c->closure_grid, st, Sst.cons, Vnew[0], Vnew[1], Vnew[2], Acur.prim,
                                       B.t11, B.t22, B.t33, B.c12, B.c13, B.c23, B.t12, B.t13, B.t23, B.hx, B.hy,
                                       B.hz));
        } else if (P.use_diff) {
            TIMED(1, launch_tau<R>(P, st, Sst.cons, Vnew[0], Vnew[1], Vnew[2], B.mut, B.t11, B.t22, B.t33, B.t12,
                                   B.t13, B.t23));
        }
        TIMED(2, launch_slow_cell<R>(P, c->tkz, st, Sst, Acur, B.mut, B.hx, B.hy, B.hz, B.tke, B.Fcons, B.avx,
                                     B.avy, B.avz));
        if (plane && !fork) TIMED(3, launch_plane_avg<R>(P, st, Sst.cons, Acur.prim, c->pavg));
        if (plane && fork) cudaStreamWaitEvent(st, c->ev_pavg, 0);
        TIMED(4, launch_slow_mom<R>(P, c->tkz, st, Sst, Acur, Vnew[0], Vnew[1], Vnew[2], B.t11, B.t22, B.t33, B.t12,
                                    B.t13, B.t23, c->pavg, B.Fmx, B.Fmy, B.Fmz));
        if (fork)
            cudaStreamWaitEvent(st, c->ev_coef, 0);
        if (nosub)
            TIMED(10, launch_no_substep<R>(P, st, slow_dt, OLD, B.Fcons, B.Fmx, B.Fmy, B.Fmz, SUM));
        else if (!fork)
            TIMED(9, launch_fast_coef<R>(P, st, tg, tcb, c->coef_smem, D, Sst, Acur, B.cA, B.cInvB, B.cCB, B.cP, B.cQ));
        for (int ks = 0; ks < (nosub ? 0 : nsub); ++ks) {
            StateBuf Sprev = (ks == 0) ? OLD : SUM;
            int prt = ks > 0;
            TIMED(5, launch_fast_h<R>(P, st, ks, nrk, dtau, facinv, Sprev, prt, Sst, Acur, B.Fmx, B.Fmy, B.lag[lp],
                                      B.lag[1 - lp], B.avx, B.avy, SUM.mx, SUM.my));
            lp ^= 1;
            TIMED(6, launch_fast_vert<R>(P, st, tg, tb, c->vert_smem, dtau, facinv, beta_1, beta_2, Sprev, prt, Sst,
                                         Acur, B.Fcons, B.Fmz, SUM.mx, SUM.my, B.cA, B.cInvB, B.cCB, B.cP, B.cQ,
                                         B.avz, SUM.cons, SUM.mz));
        }
        TIMED(7, launch_post<R>(P, c->tkz, st, slow_dt, OLD, Sst, SUM, Snew, Acur, Anext, nrk < 2 ? 1 : 0, B.mut,
                                B.tke, B.avx, B.avy, B.avz, Vnew[0], Vnew[1], Vnew[2]));
        a = 1 - a;
    }
    if (P.moist) {
        dim3 kb(32, 1, KESS_KB), kg((g.nx + 31) / 32, g.ny, (g.nz + KESS_KB - 1) / KESS_KB);
        TIMED(8, (k_kessler_cells<<<kg, kb, 0, st>>>(P, N1.cons, N0.cons, c->cfg.dt, c->cfg.dz)));
    }
}

void enqueue_step(erf_b200_ctx* c, int p, LaunchTimer* T = nullptr) {
    if (c->mixed) enqueue_step_t<float>(c, c->bf, p, T);
    else enqueue_step_t<double>(c, c->bd, p, T);
}

template <class R>
int alloc_bulk(erf_b200_ctx* c, Bulk<R>& B) {
    const erf_b200_config* cfg = &c->cfg;
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    const int64_t NZF = (int64_t)cfg->nx * cfg->ny * (cfg->nz + 1);
    const int nc = cfg->ncomp;
    int rc = ERF_B200_OK;
    auto A = [&](R** p, size_t n) { if (rc == ERF_B200_OK) rc = dalloc(c, p, n); };
    A(&B.Fcons, 2 * N); A(&B.Fmx, N); A(&B.Fmy, N); A(&B.Fmz, NZF);
    A(&B.avx, N); A(&B.avy, N); A(&B.avz, NZF);
    A(&B.lag[0], N); A(&B.lag[1], N);
    for (int p = 0; p < 2; ++p) { A(&B.aux[p].prim, (nc - 1) * N); A(&B.aux[p].pi, N); A(&B.aux[p].pp, N); }
    A(&B.mut, N);
    A(&B.t11, N); A(&B.t22, N); A(&B.t33, N); A(&B.t12, N); A(&B.t13, NZF); A(&B.t23, NZF);
    A(&B.cA, NZF); A(&B.cInvB, NZF); A(&B.cCB, NZF); A(&B.cP, NZF); A(&B.cQ, NZF);
    if (cfg->les_type == ERF_LES_MLP) {
        A(&B.c12, N); A(&B.c13, N); A(&B.c23, N); A(&B.hx, N); A(&B.hy, N); A(&B.hz, N);
    }
    if (cfg->les_type == ERF_LES_DEARDORFF) {
        A(&B.tke.kthv, N); A(&B.tke.diss, N); A(&B.tke.smn, N); A(&B.tke.hfz, NZF);
    }
    if (cfg->use_terrain) {
        A(&B.ter.s11, N); A(&B.ter.s22, N); A(&B.ter.s33, N); A(&B.ter.s12, N); A(&B.ter.s13, NZF);
        A(&B.ter.s23, NZF); A(&B.ter.t31, NZF); A(&B.ter.t32, NZF);
        A(&B.ter.ndu, N); A(&B.ter.ndv, N); A(&B.ter.odu, N); A(&B.ter.odv, N);
        A(&B.ter.fx[0], N); A(&B.ter.fy[0], N); A(&B.ter.fx[1], N); A(&B.ter.fy[1], N);
        auto D = [&](double** q, size_t n) { if (rc == ERF_B200_OK) rc = dalloc(c, q, n); };
        D(&B.ter.bnd, 2 * (int64_t)cfg->nx * cfg->ny);
    }
    return rc;
}

int build_graphs(erf_b200_ctx* c) {
    for (int p = 0; p < 2; ++p) {
        if (c->graph[p]) continue;
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(c, p);
        CK(cudaStreamEndCapture(c->stream, &gr));
        cudaError_t e = cudaGraphInstantiate(&c->graph[p], gr, 0);
        if (c->graph_raw[p]) cudaGraphDestroy(c->graph_raw[p]);
        c->graph_raw[p] = gr;
        CK(e);
    }
    return ERF_B200_OK;
}

void drop_graphs(erf_b200_ctx* c) {
    for (int p = 0; p < 2; ++p) {
        if (c->graph[p]) cudaGraphExecDestroy(c->graph[p]);
        if (c->graph_raw[p]) cudaGraphDestroy(c->graph_raw[p]);
        c->graph[p] = nullptr;
        c->graph_raw[p] = nullptr;
    }
}

bool fab_ok(const erf_b200_fab* f, int kind, const Geo& g, int ncomp) {
    if (!f || !f->p) return false;
    int hx = g.nx - 1 + (kind == 1), hy = g.ny - 1 + (kind == 2), hz = g.nz - 1 + (kind == 3);
    if (f->lo[0] > 0 || f->lo[1] > 0 || f->lo[2] > 0) return false;
    if (f->hi[0] < hx || f->hi[1] < hy || f->hi[2] < hz) return false;
    if (f->ncomp < ncomp) return false;
    return true;
}

int pack(erf_b200_ctx* c, const erf_b200_fab* f, int kind, int ncomp, double* dst) {
    const Geo& g = c->g;
    dim3 b(32, 4, 1), gr((g.nx + 31) / 32, (g.ny + 3) / 4, kind == 3 ? g.nz + 1 : g.nz);
    k_pack<<<gr, b, 0, c->stream>>>(g, *f, kind, ncomp, dst);
    return cuda_fail(cudaGetLastError());
}
int unpack(erf_b200_ctx* c, const erf_b200_fab* f, int kind, int ncomp, const double* src) {
    const Geo& g = c->g;
    int nxb = f->hi[0] - f->lo[0] + 1, nyb = f->hi[1] - f->lo[1] + 1, nzb = f->hi[2] - f->lo[2] + 1;
    dim3 b(32, 4, 1), gr((nxb + 31) / 32, (nyb + 3) / 4, nzb);
    k_unpack<<<gr, b, 0, c->stream>>>(g, *f, kind, ncomp, src, g.zlo_noslip, g.zhi_noslip, c->P.ter);
    return cuda_fail(cudaGetLastError());
}

}  // namespace

// The configuration checks of erf_b200_create, shared with the entry points
// that take a configuration without a context.
int erfb::validate_config(const erf_b200_config* c) { return validate(c); }

extern "C" {

int erf_b200_config_defaults(erf_b200_config* cfg) {
    if (!cfg) return ERF_B200_EINVAL;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->nx = cfg->ny = cfg->nz = 16;
    cfg->dx = cfg->dy = cfg->dz = 1.0;
    cfg->zlo_bc = cfg->zhi_bc = ERF_BC_SLIP_WALL;
    cfg->dt = 1.0;
    cfg->mri_ratio = 6;
    cfg->force_stage1_single_substep = 1;
    cfg->most_z0 = 0.1;
    cfg->most_zref = 0.0;
    cfg->terrain_type = ERF_TERRAIN_STATIC;
    cfg->mt_ampl = 0.0;
    cfg->mt_wavelength = 100.0;
    cfg->ncomp = 5;
    cfg->dycore_horiz_adv = cfg->dycore_vert_adv = ERF_ADV_UPWIND_3RD;
    cfg->dryscal_horiz_adv = cfg->dryscal_vert_adv = ERF_ADV_UPWIND_3RD;
    cfg->moistscal_horiz_adv = cfg->moistscal_vert_adv = ERF_ADV_WENO_3;
    cfg->dycore_horiz_upw_frac = cfg->dycore_vert_upw_frac = 1.0;
    cfg->dryscal_horiz_upw_frac = cfg->dryscal_vert_upw_frac = 1.0;
    cfg->moistscal_horiz_upw_frac = cfg->moistscal_vert_upw_frac = 1.0;
    cfg->molec_diff_type = ERF_MOLEC_CONSTANT;
    cfg->rho0_trans = 1.0;
    cfg->Pr_t = 1.0 / 3.0;
    cfg->Sc_t = 1.0;
    cfg->Ck = 0.1;
    cfg->Ce = 0.93;
    cfg->sigma_k = 0.5;
    cfg->theta_ref = 300.0;
    cfg->c_p = Cp_d;
    cfg->buoyancy_type = 1;
    return ERF_B200_OK;
}

int erf_b200_create(erf_b200_ctx** out, const erf_b200_config* cfg, void* stream) {
    if (!out) return ERF_B200_EINVAL;
    *out = nullptr;
    int v = validate(cfg);
    if (v != ERF_B200_OK) return v;
    erf_b200_ctx* c = new (std::nothrow) erf_b200_ctx();
    if (!c) return ERF_B200_ENOMEM;
    c->cfg = *cfg;
    cudaGetDevice(&c->device);
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return ERF_B200_ECUDA; }
        c->own_stream = true;
    }
    if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_pavg, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_coef, cudaEventDisableTiming) != cudaSuccess) {
        erf_b200_destroy(c);
        return ERF_B200_ECUDA;
    }
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    const int64_t NZF = (int64_t)cfg->nx * cfg->ny * (cfg->nz + 1);
    const int nc = cfg->ncomp;
    int rc = ERF_B200_OK;
    auto A = [&](double** p, size_t n) { if (rc == ERF_B200_OK) rc = dalloc(c, p, n); };
    for (int s = 0; s < 4; ++s) {
        A(&c->S[s].cons, nc * N); A(&c->S[s].mx, N); A(&c->S[s].my, N); A(&c->S[s].mz, NZF);
    }
    for (int p = 0; p < 2; ++p) { A(&c->vel[p][0], N); A(&c->vel[p][1], N); A(&c->vel[p][2], NZF); }
    A(&c->pavg, plane_avg_doubles(cfg->nz));
    A(&c->most_avg, 4);
    c->mixed = cfg->precision == ERF_PREC_MIXED;
    if (rc == ERF_B200_OK) rc = c->mixed ? alloc_bulk(c, c->bf) : alloc_bulk(c, c->bd);
    {
        const size_t nb = cfg->use_terrain ? (size_t)(cfg->nz + 2) * cfg->nx * cfg->ny : (size_t)(cfg->nz + 2);
        A(&c->r0, nb); A(&c->p0, nb); A(&c->pi0, nb); A(&c->th0, nb);
    }
    if (cfg->use_terrain) {
        const size_t sk = (size_t)cfg->nx * cfg->ny;
        A(&c->znd, (size_t)(cfg->nz + 3) * sk); A(&c->detJ, N); A(&c->zcc, (size_t)(cfg->nz + 1) * sk);
        A(&c->met, (size_t)TER_NMET * NZF);
        if (cfg->terrain_type == ERF_TERRAIN_MOVING) {
            c->mt.z[0] = c->znd;
            A(&c->mt.z[1], (size_t)(cfg->nz + 3) * sk); A(&c->mt.z[2], (size_t)(cfg->nz + 3) * sk);
            A(&c->mt.met1, (size_t)TER_NMET * NZF); A(&c->mt.detJ1, N); A(&c->mt.zcc1, (size_t)(cfg->nz + 1) * sk);
            A(&c->mt.zt, NZF);
            A(&c->mt.r0o, (size_t)(cfg->nz + 2) * sk); A(&c->mt.p0o, (size_t)(cfg->nz + 2) * sk);
            A(&c->mt.time, 1);
            A(&c->mt.fac, (size_t)cfg->nz + 1);
            if (rc == ERF_B200_OK) cudaMemsetAsync(c->mt.time, 0, sizeof(double), c->stream);
            if (cfg->substepping_type == ERF_SUBSTEP_IMPLICIT) {
                A(&c->mt.z[3], (size_t)(cfg->nz + 3) * sk); A(&c->mt.z[4], (size_t)(cfg->nz + 3) * sk);
                A(&c->mt.detJso, N); A(&c->mt.zpt, NZF); A(&c->mt.trhs, 2 * N); A(&c->mt.om, NZF);
                A(&c->mt.soln, NZF);
            }
        }
    }
    if (rc == ERF_B200_OK) {
        void* q = nullptr;
        if (cudaMalloc(&q, sizeof(int)) != cudaSuccess) rc = ERF_B200_ENOMEM;
        else { c->allocs.push_back(q); c->status = (int*)q; cudaMemsetAsync(q, 0, sizeof(int), c->stream); }
    }
    if (rc != ERF_B200_OK) { erf_b200_destroy(c); return rc; }
    make_params(c);
    // a moving grid is generated by the step itself
    if (cfg->use_terrain && cfg->terrain_type == ERF_TERRAIN_MOVING) {
        c->ter_set = true;
        // Sullivan's factor (1 - z_k / z_top)^3 of each level, formed on the
        // host with the C library's pow as init_which_terrain_grid's is
        std::vector<double> fac((size_t)cfg->nz + 1);
        const double ztop = cfg->nz * cfg->dz;
        for (int k = 0; k <= cfg->nz; ++k) {
            const double zl = k * cfg->dz;
            fac[k] = std::pow(1. - zl / ztop, 3.0);
        }
        if (cudaMemcpy(c->mt.fac, fac.data(), fac.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = ERF_B200_ECUDA;
        if (rc != ERF_B200_OK) { erf_b200_destroy(c); return rc; }
    }
    if (c->mixed) tiled_setup<float>(c->P, &c->tkz);
    else tiled_setup<double>(c->P, &c->tkz);
    c->tkz.ter_post = !cfg->use_terrain ? 0 : (c->mixed ? ter_post_kz<float>(c->P) : ter_post_kz<double>(c->P));
    c->lag_parity_per_step = substeps_per_step(c->cfg) & 1;
    // shared-memory tiles of the vertical kernels: TX columns x all levels
    {
        const size_t max_smem = 227 * 1024;
        int nz = cfg->nz;
        // the widest tile that fits: wide tiles read long contiguous rows
        // (64 columns: 18 % faster than 32 in the mixed form, where it fits)
        c->tile_tx = 64;
        const size_t rs = c->mixed ? sizeof(float) : sizeof(double);
        while (c->tile_tx > 4 && (size_t)(7 * nz + 5) * c->tile_tx * rs > max_smem) c->tile_tx /= 2;
        c->vert_smem = (size_t)(7 * nz + 5) * c->tile_tx * rs;
        c->coef_smem = (size_t)3 * (nz + 1) * c->tile_tx * rs;
        if (c->vert_smem > max_smem) rc = ERF_B200_ECONFIG;
        c->vert_warps = ERFB_VERT_THREADS / c->tile_tx;
        c->coef_warps = c->tile_tx >= 32 ? 8 : 16;
        if (rc == ERF_B200_OK) {
            if ((c->mixed ? vert_setup<float>(c->vert_smem, c->coef_smem) : vert_setup<double>(c->vert_smem, c->coef_smem)) != 0)
                rc = ERF_B200_ECUDA;
        }
        if (rc == ERF_B200_OK && cfg->use_terrain) {
            ter_vert_shape(nz, &c->ter_tx, &c->ter_smem);
            if (c->ter_tx < 1) rc = ERF_B200_ECONFIG;
        }
        if (rc != ERF_B200_OK) { erf_b200_destroy(c); return rc; }
    }
    if (cfg->les_type == ERF_LES_MLP) {
        // the step graphs are built when the network is attached
        void* q = nullptr;
        if (cudaMalloc(&q, sizeof(unsigned int)) != cudaSuccess) rc = ERF_B200_ENOMEM;
        else { c->allocs.push_back(q); c->fallback = (unsigned int*)q; cudaMemsetAsync(q, 0, sizeof(unsigned int), c->stream); }
        if (rc == ERF_B200_OK) c->closure_grid = c->mixed ? closure_grid<float>(c->P) : closure_grid<double>(c->P);
    } else {
        rc = build_graphs(c);
    }
    if (rc == ERF_B200_OK) rc = cuda_fail(cudaStreamSynchronize(c->stream));
    if (rc != ERF_B200_OK) { erf_b200_destroy(c); return rc; }
    *out = c;
    return ERF_B200_OK;
}

int erf_b200_destroy(erf_b200_ctx* c) {
    if (!c) return ERF_B200_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->side) cudaStreamSynchronize(c->side);
    drop_graphs(c);
    for (void* q : c->allocs) cudaFree(q);
    if (c->side) cudaStreamDestroy(c->side);
    for (cudaEvent_t e : {c->ev_fork, c->ev_pavg, c->ev_coef})
        if (e) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return ERF_B200_OK;
}

int erf_b200_set_stream(erf_b200_ctx* c, void* stream) {
    if (!c) return ERF_B200_EINVAL;
    if (!stream) return ERF_B200_EINVAL;
    cudaStreamSynchronize(c->stream);
    if (c->own_stream) { cudaStreamDestroy(c->stream); c->own_stream = false; }
    c->stream = (cudaStream_t)stream;
    return ERF_B200_OK;
}

int erf_b200_get_status(erf_b200_ctx* c) {
    if (!c) return ERF_B200_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    int h = 0;
    CK(cudaMemcpy(&h, c->status, sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemset(c->status, 0, sizeof(int)));
    if (h & ST_BOUNDS) return ERF_B200_EBOUNDS;
    if (h & ST_TIMEOUT) return ERF_B200_ETIMEOUT;
    if (h & ST_NAN) return ERF_B200_ENAN;
    if (h & ST_BADSTATE) return ERF_B200_EBADSTATE;
    return ERF_B200_OK;
}

int erf_b200_scratch_bytes(const erf_b200_ctx* c, size_t* bytes) {
    if (!c || !bytes) return ERF_B200_EINVAL;
    *bytes = c->bytes;
    return ERF_B200_OK;
}

int erf_b200_make_base_state(erf_b200_ctx* c, const double* theta_cc, const double* qv_cc, double theta_sfc,
                             double qv_sfc, double p_sfc, double* rho0, double* p0, double* pi0, double* th0) {
    if (!c || !theta_cc || !qv_cc || !rho0 || !p0 || !pi0 || !th0) return ERF_B200_EINVAL;
    k_base_state<<<1, 1, 0, c->stream>>>(c->cfg.nz, c->cfg.dz, c->cfg.gravity, R_d / c->cfg.c_p, theta_cc, qv_cc,
                                         theta_sfc, qv_sfc, p_sfc, rho0, p0, pi0, th0);
    return cuda_fail(cudaGetLastError());
}

int erf_b200_set_base_state(erf_b200_ctx* c, const double* rho0, const double* p0, const double* pi0,
                            const double* th0) {
    if (!c || !rho0 || !p0 || !pi0 || !th0) return ERF_B200_EINVAL;
    size_t b = (c->cfg.nz + 2) * sizeof(double);
    if (c->cfg.use_terrain) b *= (size_t)c->cfg.nx * c->cfg.ny;
    CK(cudaMemcpyAsync(c->r0, rho0, b, cudaMemcpyDefault, c->stream));
    CK(cudaMemcpyAsync(c->p0, p0, b, cudaMemcpyDefault, c->stream));
    CK(cudaMemcpyAsync(c->pi0, pi0, b, cudaMemcpyDefault, c->stream));
    CK(cudaMemcpyAsync(c->th0, th0, b, cudaMemcpyDefault, c->stream));
    c->base_set = true;
    return ERF_B200_OK;
}

// Install z_phys_nd for a context created with use_terrain: (nz+1)(ny+1)(nx+1)
// node heights, i fastest (host or device memory).  The terrain must be
// periodic (node nx equal to node 0, node ny to node 0).  The ghost levels
// are extrapolated as init_terrain_grid does (ERF_TerrainMetrics.cpp:320-333)
// and detJ / z_cc formed on the GPU (make_J, make_zcc).
int erf_b200_set_terrain(erf_b200_ctx* c, const double* z_nd) {
    if (!c || !z_nd || !c->cfg.use_terrain) return ERF_B200_EINVAL;
    if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) return ERF_B200_EINVAL;   // the grid is generated
    const int nx = c->cfg.nx, ny = c->cfg.ny, nz = c->cfg.nz;
    const size_t nn = (size_t)(nx + 1) * (ny + 1) * (nz + 1), sk = (size_t)nx * ny;
    std::vector<double> h(nn), z((size_t)(nz + 3) * sk);
    CK(cudaMemcpy(h.data(), z_nd, nn * sizeof(double), cudaMemcpyDefault));
    auto at = [&](int i, int j, int k) { return h[((size_t)k * (ny + 1) + j) * (nx + 1) + i]; };
    for (int k = 0; k <= nz; ++k)
        for (int j = 0; j <= ny; ++j)
            if (at(nx, j, k) != at(0, j, k)) return ERF_B200_EINVAL;
    for (int k = 0; k <= nz; ++k)
        for (int i = 0; i <= nx; ++i)
            if (at(i, ny, k) != at(i, 0, k)) return ERF_B200_EINVAL;
    for (int k = -1; k <= nz + 1; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double v;
                if (k == -1) v = 2.0 * at(i, j, 0) - at(i, j, 1);
                else if (k == nz + 1) v = 2.0 * at(i, j, nz) - at(i, j, nz - 1);
                else v = at(i, j, k);
                if (std::isnan(v)) return ERF_B200_EINVAL;
                z[(size_t)(k + 1) * sk + (size_t)j * nx + i] = v;
            }
    CK(cudaMemcpyAsync(c->znd, z.data(), z.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_ter_metrics(c->P, c->stream, c->detJ, c->zcc);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    std::vector<double> J(sk * nz);
    CK(cudaMemcpy(J.data(), c->detJ, J.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (double v : J)
        if (!(v > 0.0)) return ERF_B200_EINVAL;   // folded or inverted cells
    c->ter_set = true;
    return ERF_B200_OK;
}

// Diagnostics of the latest state (the resident one, or the one the last
// erf_b200_advance left): out[0] the mass (integral of rho over the
// physical volume, dx dy dz detJ per cell), out[1] the integral of rho
// theta, out[2] max |w|.  Synchronises the stream.
int erf_b200_diagnostics(erf_b200_ctx* c, double* out) {
    if (!c || !out) return ERF_B200_EINVAL;
    const int p = c->cur >= 0 ? c->cur : c->last;
    if (p < 0) return ERF_B200_EBADSTATE;
    if (c->cfg.use_terrain && !c->ter_set) return ERF_B200_EBADSTATE;
    if (!c->diag) {
        int rc = dalloc(c, &c->diag, (size_t)diagnostics_scratch_doubles());
        if (rc) return rc;
    }
    const double* zg = nullptr;
    if (c->cfg.use_terrain && c->cfg.terrain_type == ERF_TERRAIN_MOVING) {   // the grid at the clock's time
        launch_mt_grid(c->P, c->stream, c->mt.time, c->cfg.dt, 0, c->mt.z[1]);
        zg = c->mt.z[1];
    }
    double* res = c->diag + diagnostics_scratch_doubles() - 3;
    launch_diagnostics(c->P, c->stream, c->S[p].cons, c->vel[p][2], zg, c->diag, res);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ERF_B200_OK;
}

// Moving terrain: set the device clock (the old time of the next step).
int erf_b200_set_time(erf_b200_ctx* c, double time) {
    if (!c || c->cfg.terrain_type != ERF_TERRAIN_MOVING || !c->cfg.use_terrain) return ERF_B200_EINVAL;
    CK(cudaMemcpyAsync(c->mt.time, &time, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ERF_B200_OK;
}

// Moving terrain: the clock, the grid at that time ((nz+1)(ny+1)(nx+1)
// nodes, i fastest; node nx / ny repeat node 0) and the evolved base state
// (rho0, p0: (nz+2) planes of nx*ny) into host memory; NULL skips an output.
int erf_b200_moving_terrain_state(erf_b200_ctx* c, double* time, double* z_nd, double* rho0, double* p0) {
    if (!c || c->cfg.terrain_type != ERF_TERRAIN_MOVING || !c->cfg.use_terrain) return ERF_B200_EINVAL;
    const int nx = c->cfg.nx, ny = c->cfg.ny, nz = c->cfg.nz;
    const size_t sk = (size_t)nx * ny;
    if (z_nd) {
        Params Po = c->P;
        launch_mt_grid(Po, c->stream, c->mt.time, c->cfg.dt, 0, c->mt.z[1]);
        CK(cudaGetLastError());
        std::vector<double> z((size_t)(nz + 3) * sk);
        CK(cudaMemcpyAsync(z.data(), c->mt.z[1], z.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx; ++i)
                    z_nd[((size_t)k * (ny + 1) + j) * (nx + 1) + i] = z[(size_t)(k + 1) * sk + (size_t)(j % ny) * nx + (i % nx)];
    }
    if (time) CK(cudaMemcpyAsync(time, c->mt.time, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (rho0) CK(cudaMemcpyAsync(rho0, c->r0, (size_t)(nz + 2) * sk * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (p0) CK(cudaMemcpyAsync(p0, c->p0, (size_t)(nz + 2) * sk * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ERF_B200_OK;
}

// Base state over the terrain (device pointers): theta3 / qv3 at the cell
// centres (nz planes of nx*ny); rho0 / p0 / pi0 / th0 receive (nz+2) planes,
// plane k+1 for level k.  calc_rho_p + erf_enforce_hse per column.
int erf_b200_make_base_state_terrain(erf_b200_ctx* c, const double* theta3, const double* qv3, double theta_sfc,
                                     double qv_sfc, double p_sfc, double* rho0, double* p0, double* pi0,
                                     double* th0) {
    if (!c || !c->ter_set || !theta3 || !qv3 || !rho0 || !p0 || !pi0 || !th0) return ERF_B200_EINVAL;
    launch_ter_base_state(c->P, c->stream, c->zcc, theta3, qv3, theta_sfc, qv_sfc, p_sfc, rho0, p0, pi0, th0);
    return cuda_fail(cudaGetLastError());
}

int erf_b200_advance(erf_b200_ctx* c, const erf_b200_fab* cons, const erf_b200_fab* xvel,
                     const erf_b200_fab* yvel, const erf_b200_fab* zvel, int nsteps) {
    if (!c || nsteps < 0) return ERF_B200_EINVAL;
    if (!c->base_set) return ERF_B200_EINVAL;
    if (c->cfg.use_terrain && !c->ter_set) return ERF_B200_EBADSTATE;
    const Geo& g = c->g;
    if (!fab_ok(cons, 0, g, c->cfg.ncomp) || !fab_ok(xvel, 1, g, 1) || !fab_ok(yvel, 2, g, 1) || !fab_ok(zvel, 3, g, 1))
        return ERF_B200_EINVAL;
    int rc;
    if ((rc = pack(c, cons, 0, c->cfg.ncomp, c->S[0].cons))) return rc;
    if ((rc = pack(c, xvel, 1, 1, c->vel[0][0]))) return rc;
    if ((rc = pack(c, yvel, 2, 1, c->vel[0][1]))) return rc;
    if ((rc = pack(c, zvel, 3, 1, c->vel[0][2]))) return rc;
    if (!c->graph[0] || !c->graph[1]) return ERF_B200_EBADSTATE;   // learned closure not attached
    c->cur = -1;
    {
        NvtxRange r("erf_b200_advance");
        for (int s = 0; s < nsteps; ++s) {
            NvtxRange rs("step");
            CK(cudaGraphLaunch(c->graph[s & 1], c->stream));
        }
    }
    int p = nsteps & 1;
    c->last = p;
    if ((rc = unpack(c, cons, 0, c->cfg.ncomp, c->S[p].cons))) return rc;
    if ((rc = unpack(c, xvel, 1, 1, c->vel[p][0]))) return rc;
    if ((rc = unpack(c, yvel, 2, 1, c->vel[p][1]))) return rc;
    if ((rc = unpack(c, zvel, 3, 1, c->vel[p][2]))) return rc;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_advance_host(erf_b200_ctx* c, double* cons, double* u, double* v, double* w, int nsteps) {
    if (!c || !cons || !u || !v || !w) return ERF_B200_EINVAL;
    const erf_b200_config& f = c->cfg;
    const int64_t nc = f.ncomp, nx = f.nx, ny = f.ny, nz = f.nz;
    const int64_t ncons = nc * nx * ny * nz, nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
    if (!c->h_stage) {
        int rc = dalloc(c, &c->h_stage, ncons + nu + nv + nw);
        if (rc) return rc;
    }
    double* dc = c->h_stage;
    double* du = dc + ncons;
    double* dv = du + nu;
    double* dw = dv + nv;
    // Components the configuration neither reads nor changes (rho*KE without
    // Deardorff, rho*QKE always: no PBL scheme on this path) keep their host
    // values and are not copied; the others move as contiguous runs.
    const int64_t ncell = nx * ny * nz;
    auto live = [&](int n) { return !(n == ERF_RHOQKE_COMP || (n == ERF_RHOKE_COMP && f.les_type != ERF_LES_DEARDORFF)); };
    auto copy_cons = [&](bool to_device) -> int {
        for (int n0 = 0; n0 < nc;) {
            if (!live(n0)) { ++n0; continue; }
            int n1 = n0;
            while (n1 < nc && live(n1)) ++n1;
            size_t off = (size_t)n0 * ncell, cnt = (size_t)(n1 - n0) * ncell;
            cudaError_t e = to_device ? cudaMemcpyAsync(dc + off, cons + off, cnt * sizeof(double), cudaMemcpyHostToDevice, c->stream)
                                      : cudaMemcpyAsync(cons + off, dc + off, cnt * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
            if (e != cudaSuccess) return cuda_fail(e);
            n0 = n1;
        }
        return ERF_B200_OK;
    };
    int crc = copy_cons(true);
    if (crc) return crc;
    CK(cudaMemcpyAsync(du, u, nu * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dv, v, nv * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dw, w, nw * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    auto mk = [&](double* p, int hx, int hy, int hz, int ncomp) {
        erf_b200_fab fb;
        fb.p = p; fb.lo[0] = fb.lo[1] = fb.lo[2] = 0; fb.hi[0] = hx; fb.hi[1] = hy; fb.hi[2] = hz;
        fb.jstride = hx + 1; fb.kstride = (int64_t)(hx + 1) * (hy + 1); fb.nstride = fb.kstride * (hz + 1);
        fb.ncomp = ncomp;
        return fb;
    };
    erf_b200_fab fc = mk(dc, nx - 1, ny - 1, nz - 1, nc), fu = mk(du, nx, ny - 1, nz - 1, 1),
                 fv = mk(dv, nx - 1, ny, nz - 1, 1), fw = mk(dw, nx - 1, ny - 1, nz, 1);
    int rc = erf_b200_advance(c, &fc, &fu, &fv, &fw, nsteps);
    if (rc) return rc;
    crc = copy_cons(false);
    if (crc) return crc;
    CK(cudaMemcpyAsync(u, du, nu * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(v, dv, nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(w, dw, nw * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ERF_B200_OK;
}

int erf_b200_advance_profiled(erf_b200_ctx* c, const erf_b200_fab* cons, const erf_b200_fab* xvel,
                              const erf_b200_fab* yvel, const erf_b200_fab* zvel, int nsteps, double* kernel_ms,
                              int* kernel_launches, int nslots) {
    if (!c || nsteps < 0 || !kernel_ms || !kernel_launches || nslots < ERF_B200_NUM_KERNEL_SLOTS) return ERF_B200_EINVAL;
    if (!c->base_set) return ERF_B200_EINVAL;
    if (c->P.les == ERF_LES_MLP && !c->net) return ERF_B200_EBADSTATE;
    const Geo& g = c->g;
    if (!fab_ok(cons, 0, g, c->cfg.ncomp) || !fab_ok(xvel, 1, g, 1) || !fab_ok(yvel, 2, g, 1) || !fab_ok(zvel, 3, g, 1))
        return ERF_B200_EINVAL;
    for (int q = 0; q < nslots; ++q) { kernel_ms[q] = 0.0; kernel_launches[q] = 0; }
    int rc;
    if ((rc = pack(c, cons, 0, c->cfg.ncomp, c->S[0].cons))) return rc;
    if ((rc = pack(c, xvel, 1, 1, c->vel[0][0]))) return rc;
    if ((rc = pack(c, yvel, 2, 1, c->vel[0][1]))) return rc;
    if ((rc = pack(c, zvel, 3, 1, c->vel[0][2]))) return rc;
    LaunchTimer T;
    T.st = c->stream;
    for (int s = 0; s < nsteps; ++s) {
        T.used = 0;
        T.slot.clear();
        enqueue_step(c, s & 1, &T);
        CK(cudaStreamSynchronize(c->stream));
        for (size_t q = 0; q < T.slot.size(); ++q) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, T.ev[2 * q], T.ev[2 * q + 1]);
            kernel_ms[T.slot[q]] += ms;
            kernel_launches[T.slot[q]] += 1;
        }
    }
    for (cudaEvent_t e : T.ev) cudaEventDestroy(e);
    int p = nsteps & 1;
    if ((rc = unpack(c, cons, 0, c->cfg.ncomp, c->S[p].cons))) return rc;
    if ((rc = unpack(c, xvel, 1, 1, c->vel[p][0]))) return rc;
    if ((rc = unpack(c, yvel, 2, 1, c->vel[p][1]))) return rc;
    if ((rc = unpack(c, zvel, 3, 1, c->vel[p][2]))) return rc;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_kernels_per_step(const erf_b200_ctx* c, int* launches) {
    if (!c || !launches) return ERF_B200_EINVAL;
    int n = 1 + (c->P.moist ? 1 : 0) + (c->P.most ? 1 : 0);
    for (int nrk = 0; nrk < 3; ++nrk) {
        int nsub; double a, b;
        stage_schedule(c->cfg, nrk, nsub, a, b);
        int stress = c->P.les == ERF_LES_MLP ? 2 : (c->P.use_diff ? (c->P.most ? 2 : 1) : 0);
        // slow_cell, slow_mom, post + (fast_coeffs and 2 per substep, or the no-substep update)
        int fast = no_substepping(c->cfg) ? 1 : 1 + 2 * nsub;
        n += 3 + fast + stress + ((c->P.moist && c->P.buoy_type == 2) ? 1 : 0);
    }
    *launches = n;
    return ERF_B200_OK;
}

// ---------------------------------------------------------------------------
// Per-pass entry points (plain form).  Each packs the caller's fabs into the
// context's valid-region arrays, runs the kernels of that pass and unpacks
// the outputs.  State carried between passes lives in the context, as in
// MRISplitIntegrator: the eddy viscosity (erf_b200_turbulent_viscosity), the
// stage primitives of the last slow_rhs_pre (used by slow_rhs_post), and the
// fast coefficients of the stage (made at substep 0).  A vector of fabs
// S[4] is {cons, x-momentum, y-momentum, z-momentum}.
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

// The fab of one component of a multi-component fab.
erf_b200_fab comp_fab(const erf_b200_fab* f, int n, int ncomp) {
    erf_b200_fab r = *f;
    r.p = f->p + (int64_t)n * f->nstride;
    r.ncomp = ncomp;
    return r;
}

bool fab4_ok(const erf_b200_fab* S, const Geo& g, int ncons) {
    return S && fab_ok(&S[0], 0, g, ncons) && fab_ok(&S[1], 1, g, 1) && fab_ok(&S[2], 2, g, 1) &&
           fab_ok(&S[3], 3, g, 1);
}

int pack4(erf_b200_ctx* c, const erf_b200_fab* S, int ncons, double* cons, double* mx, double* my, double* mz) {
    int rc;
    if (cons && (rc = pack(c, &S[0], 0, ncons, cons))) return rc;
    if ((rc = pack(c, &S[1], 1, 1, mx))) return rc;
    if ((rc = pack(c, &S[2], 2, 1, my))) return rc;
    return pack(c, &S[3], 3, 1, mz);
}

int unpack4(erf_b200_ctx* c, const erf_b200_fab* S, int ncons, const double* cons, const double* mx,
            const double* my, const double* mz) {
    int rc;
    if (cons && (rc = unpack(c, &S[0], 0, ncons, cons))) return rc;
    if ((rc = unpack(c, &S[1], 1, 1, mx))) return rc;
    if ((rc = unpack(c, &S[2], 2, 1, my))) return rc;
    return unpack(c, &S[3], 3, 1, mz);
}

// A, 1/B', C, P, Q on the valid z-faces of a 5-component z-face fab; C is
// recovered from the stored C/B'.
__global__ void k_coef_export(Geo g, erf_b200_fab f, const double* cA, const double* cInvB, const double* cCB,
                              const double* cP, const double* cQ) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    int64_t s = cidx(g, i, j, k);
    int64_t d = (int64_t)(i - f.lo[0]) + (int64_t)(j - f.lo[1]) * f.jstride + (int64_t)(k - f.lo[2]) * f.kstride;
    double invb = cInvB[s];
    double cc = cCB[s] / invb;   // C/B' * B' (wall rows hold B' itself)
    f.p[d] = cA[s];
    f.p[d + f.nstride] = invb;
    f.p[d + 2 * f.nstride] = cc;
    f.p[d + 3 * f.nstride] = cP[s];
    f.p[d + 4 * f.nstride] = cQ[s];
}

const double kBeta1 = 0.5 * (1.0 - 0.1), kBeta2 = 0.5 * (1.0 + 0.1);

}  // namespace

extern "C" {

int erf_b200_turbulent_viscosity(erf_b200_ctx* c, const erf_b200_fab* xvel, const erf_b200_fab* yvel,
                                 const erf_b200_fab* zvel, const erf_b200_fab* cons) {
    if (!c || c->mixed || !c->base_set) return ERF_B200_EINVAL;
    if (c->P.ter && !c->ter_set) return ERF_B200_EBADSTATE;
    if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) return ERF_B200_EINVAL;   // fused step only
    const Geo& g = c->g;
    if (!fab_ok(cons, 0, g, c->cfg.ncomp) || !fab_ok(xvel, 1, g, 1) || !fab_ok(yvel, 2, g, 1) || !fab_ok(zvel, 3, g, 1))
        return ERF_B200_EINVAL;
    int rc;
    if ((rc = pack(c, cons, 0, c->cfg.ncomp, c->S[0].cons))) return rc;
    if ((rc = pack(c, xvel, 1, 1, c->vel[0][0])) || (rc = pack(c, yvel, 2, 1, c->vel[0][1])) ||
        (rc = pack(c, zvel, 3, 1, c->vel[0][2])))
        return rc;
    // the step prologue forms the eddy viscosity from these velocities (its
    // other outputs go to scratch slots of the context)
    if (c->P.ter) {   // ComputeStrain_T + the terrain filter width
        launch_ter_step_begin<double>(c->P, c->stream, c->S[0].cons, c->vel[0][0], c->vel[0][1], c->vel[0][2],
                                      c->S[1], c->vel[1][0], c->vel[1][1], c->vel[1][2], c->bd.aux[1], c->bd.mut,
                                      c->bd.tke);
        return cuda_fail(cudaGetLastError());
    }
    launch_step_begin<double>(c->P, c->stream, c->S[0].cons, c->vel[0][0], c->vel[0][1], c->vel[0][2], c->S[1],
                              c->vel[1][0], c->vel[1][1], c->vel[1][2], c->bd.aux[1], c->bd.mut, c->bd.tke);
    return cuda_fail(cudaGetLastError());
}

int erf_b200_most_update_fluxes(erf_b200_ctx* c, const erf_b200_fab* xvel, const erf_b200_fab* yvel) {
    if (!c || c->mixed) return ERF_B200_EINVAL;
    if (!c->P.most) return ERF_B200_ECONFIG;
    const Geo& g = c->g;
    if (!fab_ok(xvel, 1, g, 1) || !fab_ok(yvel, 2, g, 1)) return ERF_B200_EINVAL;
    int rc;
    if ((rc = pack(c, xvel, 1, 1, c->vel[0][0])) || (rc = pack(c, yvel, 2, 1, c->vel[0][1]))) return rc;
    launch_most_avg(c->P, c->stream, c->vel[0][0], c->vel[0][1]);
    rc = cuda_fail(cudaGetLastError());
    if (rc == ERF_B200_OK) c->most_set = true;
    return rc;
}

int erf_b200_slow_rhs_pre(erf_b200_ctx* c, int nrk, double slow_dt, const erf_b200_fab* S_rhs,
                          const erf_b200_fab* S_data, const erf_b200_fab* S_scratch, const erf_b200_fab* xvel,
                          const erf_b200_fab* yvel, const erf_b200_fab* zvel) {
    (void)slow_dt;
    if (!c || c->mixed || !c->base_set || nrk < 0 || nrk > 2) return ERF_B200_EINVAL;
    if (c->P.ter && !c->ter_set) return ERF_B200_EBADSTATE;
    if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) return ERF_B200_EINVAL;   // fused step only
    if (c->P.most && !c->most_set) return ERF_B200_EBADSTATE;
    if (c->P.les == ERF_LES_MLP && !c->net) return ERF_B200_EBADSTATE;
    const Geo& g = c->g;
    const int nc = c->cfg.ncomp;
    if (!fab4_ok(S_data, g, nc) || !fab4_ok(S_rhs, g, 2) || !fab4_ok(S_scratch, g, 1) || !fab_ok(xvel, 1, g, 1) ||
        !fab_ok(yvel, 2, g, 1) || !fab_ok(zvel, 3, g, 1))
        return ERF_B200_EINVAL;
    const Params& P = c->P;
    Bulk<double>& B = c->bd;
    StateBuf Sst = c->S[2];
    double** V = c->vel[1];
    int rc;
    if ((rc = pack4(c, S_data, nc, Sst.cons, Sst.mx, Sst.my, Sst.mz))) return rc;
    if ((rc = pack(c, xvel, 1, 1, V[0])) || (rc = pack(c, yvel, 2, 1, V[1])) || (rc = pack(c, zvel, 3, 1, V[2])))
        return rc;
    cudaStream_t st = c->stream;
    launch_stage_aux<double>(P, st, Sst.cons, B.aux[0]);
    if (P.ter) {   // terrain passes; S_scratch's z-momentum receives Omega (avg_zmom)
        if (P.use_diff)
            launch_ter_tau<double>(P, st, nrk, Sst.cons, V[0], V[1], V[2], B.mut, B.ter, B.tke, B.t11, B.t22, B.t33,
                                   B.t12, B.t13, B.t23);
        launch_ter_slow_cell<double>(P, st, Sst, B.aux[0], V[0], V[1], B.mut, B.tke, B.ter, B.Fcons, B.avx, B.avy,
                                     B.avz);
        launch_ter_slow_mom<double>(P, st, Sst, B.aux[0], V[0], V[1], V[2], B.t11, B.t22, B.t33, B.t12, B.t13, B.t23,
                                    B.ter, B.avz, B.Fmx, B.Fmy, B.Fmz);
        if ((rc = unpack4(c, S_rhs, 2, B.Fcons, B.Fmx, B.Fmy, B.Fmz))) return rc;
        if ((rc = unpack4(c, S_scratch, 0, nullptr, B.avx, B.avy, B.avz))) return rc;
        return cuda_fail(cudaGetLastError());
    }
    if (P.les == ERF_LES_MLP) {
        ClosureNet net{c->net->wpack, c->net->bias, c->net->norm, c->net->env, c->fallback};
        launch_closure<double>(P, net, c->closure_grid, st, Sst.cons, V[0], V[1], V[2], B.aux[0].prim, B.t11, B.t22,
                               B.t33, B.c12, B.c13, B.c23, B.t12, B.t13, B.t23, B.hx, B.hy, B.hz);
    } else if (P.use_diff) {
        launch_tau<double>(P, st, Sst.cons, V[0], V[1], V[2], B.mut, B.t11, B.t22, B.t33, B.t12, B.t13, B.t23);
    }
    launch_slow_cell<double>(P, c->tkz, st, Sst, B.aux[0], B.mut, B.hx, B.hy, B.hz, B.tke, B.Fcons, B.avx, B.avy,
                             B.avz);
    if (P.moist && P.buoy_type == 2) launch_plane_avg<double>(P, st, Sst.cons, B.aux[0].prim, c->pavg);
    launch_slow_mom<double>(P, c->tkz, st, Sst, B.aux[0], V[0], V[1], V[2], B.t11, B.t22, B.t33, B.t12, B.t13, B.t23,
                            c->pavg, B.Fmx, B.Fmy, B.Fmz);
    if ((rc = unpack4(c, S_rhs, 2, B.Fcons, B.Fmx, B.Fmy, B.Fmz))) return rc;
    if ((rc = unpack4(c, S_scratch, 0, nullptr, B.avx, B.avy, B.avz))) return rc;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_make_fast_coeffs(erf_b200_ctx* c, const erf_b200_fab* fast_coeffs, const erf_b200_fab* S_stage,
                              double dtau) {
    if (!c || c->mixed || !c->base_set || !fast_coeffs) return ERF_B200_EINVAL;
    if (c->P.ter && !c->ter_set) return ERF_B200_EBADSTATE;
    if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) return ERF_B200_EINVAL;   // fused step only
    const Geo& g = c->g;
    if (!fab4_ok(S_stage, g, c->cfg.ncomp) || !fab_ok(fast_coeffs, 3, g, 5)) return ERF_B200_EINVAL;
    StateBuf Sst = c->S[2];
    Bulk<double>& B = c->bd;
    int rc;
    if ((rc = pack4(c, S_stage, c->cfg.ncomp, Sst.cons, Sst.mx, Sst.my, Sst.mz))) return rc;
    launch_stage_aux<double>(c->P, c->stream, Sst.cons, B.aux[0]);
    dim3 tg((g.nx + c->tile_tx - 1) / c->tile_tx, g.ny, 1), tcb(c->tile_tx, c->coef_warps, 1);
    double D = dtau * dtau * kBeta2 * kBeta2 * g.dzi;
    launch_fast_coef<double>(c->P, c->stream, tg, tcb, c->coef_smem, D, Sst, B.aux[0], B.cA, B.cInvB, B.cCB, B.cP, B.cQ);
    k_coef_export<<<dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz + 1), dim3(32, 4, 1), 0, c->stream>>>(
        g, *fast_coeffs, B.cA, B.cInvB, B.cCB, B.cP, B.cQ);
    return cuda_fail(cudaGetLastError());
}

}  // extern "C"

namespace {
// erf_fast_rhs_N / erf_fast_rhs_T per-pass body (terrain selects the _T kernels)
int fast_rhs_pass(erf_b200_ctx* c, bool terrain, int step, int nrk, const erf_b200_fab* S_slow_rhs,
                  const erf_b200_fab* S_prev, const erf_b200_fab* S_stage, const erf_b200_fab* S_data,
                  const erf_b200_fab* S_scratch, double dtau, double facinv) {
    if (!c || c->mixed || !c->base_set || step < 0 || nrk < 0 || nrk > 2) return ERF_B200_EINVAL;
    if (terrain != (c->P.ter != 0)) return ERF_B200_ECONFIG;   // _N without terrain, _T with it
    if (terrain && !c->ter_set) return ERF_B200_EBADSTATE;
    if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) return ERF_B200_EINVAL;   // fused step only
    const Geo& g = c->g;
    const int nc = c->cfg.ncomp;
    if (!fab4_ok(S_slow_rhs, g, 2) || !fab4_ok(S_prev, g, 2) || !fab4_ok(S_stage, g, nc) || !fab4_ok(S_data, g, 2) ||
        !fab4_ok(S_scratch, g, 2))
        return ERF_B200_EINVAL;
    const Params& P = c->P;
    Bulk<double>& B = c->bd;
    StateBuf Sprev = c->S[0], Sst = c->S[2], OUT = c->S[3];
    cudaStream_t st = c->stream;
    int rc;
    if ((rc = pack4(c, S_slow_rhs, 2, B.Fcons, B.Fmx, B.Fmy, B.Fmz))) return rc;
    if ((rc = pack4(c, S_prev, 2, Sprev.cons, Sprev.mx, Sprev.my, Sprev.mz))) return rc;
    if ((rc = pack4(c, S_stage, nc, Sst.cons, Sst.mx, Sst.my, Sst.mz))) return rc;
    if ((rc = pack4(c, S_scratch, 0, nullptr, B.avx, B.avy, B.avz))) return rc;
    erf_b200_fab lagf = comp_fab(&S_scratch[0], 1, 1);   // lagged d(rho theta) in the rho-theta slot
    if ((rc = pack(c, &lagf, 0, 1, B.lag[0]))) return rc;
    if (step == 0) {
        // make_fast_coeffs at the stage's first substep (ERF_fast_rhs_N.cpp:60-70)
        launch_stage_aux<double>(P, st, Sst.cons, B.aux[0]);
        dim3 tg((g.nx + c->tile_tx - 1) / c->tile_tx, g.ny, 1), tcb(c->tile_tx, c->coef_warps, 1);
        double D = dtau * dtau * kBeta2 * kBeta2 * g.dzi;
        launch_fast_coef<double>(P, st, tg, tcb, c->coef_smem, D, Sst, B.aux[0], B.cA, B.cInvB, B.cCB, B.cP, B.cQ);
    }
    if (terrain) {
        launch_ter_fast_h<double>(P, st, step, dtau, facinv, Sprev, 0, Sst, B.aux[0], B.Fmx, B.Fmy, B.lag[0],
                                  B.lag[1], B.ter, B.avx, B.avy, OUT.mx, OUT.my);
        launch_ter_fast_vert<double>(P, st, c->ter_tx, c->ter_smem, dtau, facinv, kBeta1, kBeta2, Sprev, 0, Sst,
                                     B.aux[0], B.Fcons, B.Fmz, B.ter, B.cA, B.cInvB, B.cCB, B.cP, B.cQ, B.avz,
                                     OUT.cons, OUT.mz);
    } else {
        launch_fast_h<double>(P, st, step, nrk, dtau, facinv, Sprev, 0, Sst, B.aux[0], B.Fmx, B.Fmy, B.lag[0],
                              B.lag[1], B.avx, B.avy, OUT.mx, OUT.my);
        dim3 tb(c->tile_tx, c->vert_warps, 1), tg((g.nx + c->tile_tx - 1) / c->tile_tx, g.ny, 1);
        launch_fast_vert<double>(P, st, tg, tb, c->vert_smem, dtau, facinv, kBeta1, kBeta2, Sprev, 0, Sst, B.aux[0],
                                 B.Fcons, B.Fmz, OUT.mx, OUT.my, B.cA, B.cInvB, B.cCB, B.cP, B.cQ, B.avz, OUT.cons,
                                 OUT.mz);
    }
    if ((rc = unpack4(c, S_data, 2, OUT.cons, OUT.mx, OUT.my, OUT.mz))) return rc;
    if ((rc = unpack4(c, S_scratch, 0, nullptr, B.avx, B.avy, B.avz))) return rc;
    if ((rc = unpack(c, &lagf, 0, 1, B.lag[1]))) return rc;
    return cuda_fail(cudaGetLastError());
}

}  // namespace

extern "C" {

int erf_b200_fast_rhs_N(erf_b200_ctx* c, int step, int nrk, const erf_b200_fab* S_slow_rhs,
                        const erf_b200_fab* S_prev, const erf_b200_fab* S_stage, const erf_b200_fab* S_data,
                        const erf_b200_fab* S_scratch, double dtau, double facinv) {
    return fast_rhs_pass(c, false, step, nrk, S_slow_rhs, S_prev, S_stage, S_data, S_scratch, dtau, facinv);
}

int erf_b200_fast_rhs_T(erf_b200_ctx* c, int step, int nrk, const erf_b200_fab* S_slow_rhs,
                        const erf_b200_fab* S_prev, const erf_b200_fab* S_stage, const erf_b200_fab* S_data,
                        const erf_b200_fab* S_scratch, double dtau, double facinv) {
    return fast_rhs_pass(c, true, step, nrk, S_slow_rhs, S_prev, S_stage, S_data, S_scratch, dtau, facinv);
}

// The no_substep hook (ERF_TI_no_substep_fun.H:6-150): S_sum's fast
// variables (rho, rho*theta, momenta) = S_old + slow_dt * F_slow, then the
// boundary fill of S_sum's ghost cells.
int erf_b200_no_substep(erf_b200_ctx* c, const erf_b200_fab* S_sum, const erf_b200_fab* S_old,
                        const erf_b200_fab* F_slow, double slow_dt, int nrk) {
    if (!c || c->mixed || nrk < 0 || nrk > 2) return ERF_B200_EINVAL;
    const Geo& g = c->g;
    if (!fab4_ok(S_sum, g, 2) || !fab4_ok(S_old, g, 2) || !fab4_ok(F_slow, g, 2)) return ERF_B200_EINVAL;
    Bulk<double>& B = c->bd;
    StateBuf OLD = c->S[0], SUM = c->S[3];
    int rc;
    if ((rc = pack4(c, F_slow, 2, B.Fcons, B.Fmx, B.Fmy, B.Fmz))) return rc;
    if ((rc = pack4(c, S_old, 2, OLD.cons, OLD.mx, OLD.my, OLD.mz))) return rc;
    launch_no_substep<double>(c->P, c->stream, slow_dt, OLD, B.Fcons, B.Fmx, B.Fmy, B.Fmz, SUM);
    if ((rc = unpack4(c, S_sum, 2, SUM.cons, SUM.mx, SUM.my, SUM.mz))) return rc;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_slow_rhs_post(erf_b200_ctx* c, int nrk, double slow_dt, const erf_b200_fab* S_rhs,
                           const erf_b200_fab* S_old, const erf_b200_fab* S_new, const erf_b200_fab* S_data,
                           const erf_b200_fab* S_scratch) {
    (void)S_rhs;
    if (!c || c->mixed || !c->base_set || nrk < 0 || nrk > 2) return ERF_B200_EINVAL;
    if (c->P.ter && !c->ter_set) return ERF_B200_EBADSTATE;
    if (c->cfg.terrain_type == ERF_TERRAIN_MOVING) return ERF_B200_EINVAL;   // fused step only
    const Geo& g = c->g;
    const int nc = c->cfg.ncomp;
    if (!fab4_ok(S_old, g, nc) || !fab4_ok(S_new, g, nc) || !fab4_ok(S_data, g, nc) || !fab4_ok(S_scratch, g, 1))
        return ERF_B200_EINVAL;
    Bulk<double>& B = c->bd;
    StateBuf OLD = c->S[0], NEW = c->S[1], SUM = c->S[3];
    int rc;
    if ((rc = pack4(c, S_old, nc, OLD.cons, OLD.mx, OLD.my, OLD.mz))) return rc;
    if ((rc = pack4(c, S_data, nc, SUM.cons, SUM.mx, SUM.my, SUM.mz))) return rc;
    if ((rc = pack4(c, S_scratch, 0, nullptr, B.avx, B.avy, B.avz))) return rc;
    // stage state and primitives: those of the preceding slow_rhs_pre
    if (c->P.ter)
        launch_ter_post<double>(c->P, c->stream, c->tkz.ter_post, slow_dt, OLD, c->S[2], SUM, NEW, B.aux[0], B.aux[1], 0, B.mut, B.tke,
                                B.ter, B.avx, B.avy, B.avz, c->vel[1][0], c->vel[1][1], c->vel[1][2]);
    else
    launch_post<double>(c->P, c->tkz, c->stream, slow_dt, OLD, c->S[2], SUM, NEW, B.aux[0], B.aux[1], 0, B.mut, B.tke,
                        B.avx, B.avy, B.avz, c->vel[1][0], c->vel[1][1], c->vel[1][2]);
    if ((rc = unpack4(c, S_new, nc, NEW.cons, NEW.mx, NEW.my, NEW.mz))) return rc;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_kessler_advance(erf_b200_ctx* c, const erf_b200_fab* cons, double dt) {
    if (!c || !c->P.moist) return ERF_B200_EINVAL;
    if (c->P.ter && !c->ter_set) return ERF_B200_EBADSTATE;   // the sedimentation reads detJ
    const Geo& g = c->g;
    if (!fab_ok(cons, 0, g, c->cfg.ncomp)) return ERF_B200_EINVAL;
    int rc;
    if ((rc = pack(c, cons, 0, c->cfg.ncomp, c->S[2].cons))) return rc;
    k_kessler<<<col_grid(g), col_block(), 0, c->stream>>>(c->P, c->S[2].cons, dt, c->cfg.dz);
    if ((rc = unpack(c, cons, 0, c->cfg.ncomp, c->S[2].cons))) return rc;
    return cuda_fail(cudaGetLastError());
}

// Attach a trained network to a context created with les_type
// ERF_LES_MLP; the step graphs are (re)built with its arrays.
int erf_b200_set_closure(erf_b200_ctx* c, const erf_b200_mlp* m) {
    if (!c || !m || c->P.les != ERF_LES_MLP) return ERF_B200_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->net = m;
    int rc = build_graphs(c);
    if (rc) return rc;
    return cuda_fail(cudaStreamSynchronize(c->stream));
}

// Cells that fell back to Smagorinsky since the last call (reset on read).
int erf_b200_closure_fallbacks(erf_b200_ctx* c, unsigned long long* count) {
    if (!c || !count || !c->fallback) return ERF_B200_EINVAL;
    CK(cudaStreamSynchronize(c->stream));
    unsigned int h = 0;
    CK(cudaMemcpy(&h, c->fallback, sizeof(h), cudaMemcpyDeviceToHost));
    CK(cudaMemset(c->fallback, 0, sizeof(h)));
    *count = h;
    return ERF_B200_OK;
}

// Closure features (13 per cell, cell order i fastest) of a state given as
// dense host arrays in the layout of erf_b200_advance_host.
int erf_b200_closure_features_host(erf_b200_ctx* c, const double* cons, const double* u, const double* v,
                                   const double* w, float* features) {
    if (!c || !cons || !u || !v || !w || !features) return ERF_B200_EINVAL;
    const erf_b200_config& f = c->cfg;
    const int64_t nc = f.ncomp, nx = f.nx, ny = f.ny, nz = f.nz, N = nx * ny * nz;
    const int64_t ncons = nc * N, nu = (nx + 1) * ny * nz, nv = nx * (ny + 1) * nz, nw = nx * ny * (nz + 1);
    int rc;
    if (!c->h_stage && (rc = dalloc(c, &c->h_stage, ncons + nu + nv + nw))) return rc;
    if (!c->feat_theta && (rc = dalloc(c, &c->feat_theta, N))) return rc;
    if (!c->feat_out && (rc = dalloc(c, &c->feat_out, N * 13))) return rc;
    double* dc = c->h_stage;
    double* du = dc + ncons;
    double* dv = du + nu;
    double* dw = dv + nv;
    CK(cudaMemcpyAsync(dc, cons, ncons * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(du, u, nu * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dv, v, nv * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dw, w, nw * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    auto mk = [&](double* p, int hx, int hy, int hz, int ncomp) {
        erf_b200_fab fb;
        fb.p = p; fb.lo[0] = fb.lo[1] = fb.lo[2] = 0; fb.hi[0] = hx; fb.hi[1] = hy; fb.hi[2] = hz;
        fb.jstride = hx + 1; fb.kstride = (int64_t)(hx + 1) * (hy + 1); fb.nstride = fb.kstride * (hz + 1);
        fb.ncomp = ncomp;
        return fb;
    };
    erf_b200_fab fc = mk(dc, nx - 1, ny - 1, nz - 1, nc), fu = mk(du, nx, ny - 1, nz - 1, 1),
                 fv = mk(dv, nx - 1, ny, nz - 1, 1), fw = mk(dw, nx - 1, ny - 1, nz, 1);
    if ((rc = pack(c, &fc, 0, f.ncomp, c->S[0].cons))) return rc;
    if ((rc = pack(c, &fu, 1, 1, c->vel[0][0]))) return rc;
    if ((rc = pack(c, &fv, 2, 1, c->vel[0][1]))) return rc;
    if ((rc = pack(c, &fw, 3, 1, c->vel[0][2]))) return rc;
    launch_features(c->P, c->stream, c->S[0].cons, c->vel[0][0], c->vel[0][1], c->vel[0][2], c->feat_theta,
                    c->feat_out);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(features, c->feat_out, N * 13 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ERF_B200_OK;
}

// ---------------------------------------------------------------------------
// Resident state, ensembles and autotuning (no reference counterpart: the
// reference advances one level of one domain per call).
// ---------------------------------------------------------------------------
int erf_b200_load_state(erf_b200_ctx* c, const erf_b200_fab* cons, const erf_b200_fab* xvel,
                        const erf_b200_fab* yvel, const erf_b200_fab* zvel) {
    if (!c || !c->base_set) return ERF_B200_EINVAL;
    const Geo& g = c->g;
    if (!fab_ok(cons, 0, g, c->cfg.ncomp) || !fab_ok(xvel, 1, g, 1) || !fab_ok(yvel, 2, g, 1) || !fab_ok(zvel, 3, g, 1))
        return ERF_B200_EINVAL;
    int rc;
    if ((rc = pack(c, cons, 0, c->cfg.ncomp, c->S[0].cons))) return rc;
    if ((rc = pack(c, xvel, 1, 1, c->vel[0][0])) || (rc = pack(c, yvel, 2, 1, c->vel[0][1])) ||
        (rc = pack(c, zvel, 3, 1, c->vel[0][2])))
        return rc;
    c->cur = 0;
    c->last = 0;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_store_state(erf_b200_ctx* c, const erf_b200_fab* cons, const erf_b200_fab* xvel,
                         const erf_b200_fab* yvel, const erf_b200_fab* zvel) {
    if (!c) return ERF_B200_EINVAL;
    if (c->cur < 0) return ERF_B200_EBADSTATE;
    const Geo& g = c->g;
    if (!fab_ok(cons, 0, g, c->cfg.ncomp) || !fab_ok(xvel, 1, g, 1) || !fab_ok(yvel, 2, g, 1) || !fab_ok(zvel, 3, g, 1))
        return ERF_B200_EINVAL;
    int p = c->cur, rc;
    if ((rc = unpack(c, cons, 0, c->cfg.ncomp, c->S[p].cons))) return rc;
    if ((rc = unpack(c, xvel, 1, 1, c->vel[p][0])) || (rc = unpack(c, yvel, 2, 1, c->vel[p][1])) ||
        (rc = unpack(c, zvel, 3, 1, c->vel[p][2])))
        return rc;
    return cuda_fail(cudaGetLastError());
}

int erf_b200_advance_resident(erf_b200_ctx* c, int nsteps) {
    if (!c || nsteps < 0) return ERF_B200_EINVAL;
    if (c->cur < 0 || !c->graph[0] || !c->graph[1]) return ERF_B200_EBADSTATE;
    NvtxRange r("erf_b200_advance_resident");
    for (int s = 0; s < nsteps; ++s) {
        NvtxRange rs("step");
        CK(cudaGraphLaunch(c->graph[c->cur], c->stream));
        c->cur ^= 1;
    }
    c->last = c->cur;
    return ERF_B200_OK;
}

// Runtime launch shapes of one context, chosen by timing candidate shapes on
// the resident state.  Every trial recomputes the step from the resident slot
// (a step reads only that slot's state and velocities and writes the other
// slots), so the resident state is left unchanged.  Coordinate search over
// the vertical solver's threads per block, the coefficient kernel's warps and
// the levels per block of the three tiled transport kernels.
int erf_b200_autotune(erf_b200_ctx* c, int reps, double* best_ms) {
    if (!c || reps < 1) return ERF_B200_EINVAL;
    if (c->cur < 0 || (c->P.les == ERF_LES_MLP && !c->net)) return ERF_B200_EBADSTATE;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int p = c->cur;
    auto trial = [&](float& ms) -> int {
        drop_graphs(c);
        int rc = build_graphs(c);
        if (rc) return rc;
        CK(cudaGraphLaunch(c->graph[p], c->stream));
        CK(cudaEventRecord(e0, c->stream));
        for (int r = 0; r < reps; ++r) CK(cudaGraphLaunch(c->graph[p], c->stream));
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        CK(cudaEventElapsedTime(&ms, e0, e1));
        ms /= reps;
        return ERF_B200_OK;
    };
    float best = 0.f;
    int rc = trial(best);
    const int nz = c->cfg.nz;
    // vertical kernels: columns per block (smaller tiles let two blocks share
    // an SM, overlapping one block's serial sweep with the other's loads) and
    // threads per block
    const size_t rs = c->mixed ? sizeof(float) : sizeof(double);
    for (int tx : {c->tile_tx, c->tile_tx / 2}) {
        for (int threads : {256, 512, 1024}) {
            int vw = threads / tx;
            if (rc || tx < 4 || vw < 1 || (tx == c->tile_tx && vw == c->vert_warps)) continue;
            int keep_tx = c->tile_tx, keep_vw = c->vert_warps, keep_cw = c->coef_warps;
            size_t keep_vs = c->vert_smem, keep_cs = c->coef_smem;
            c->tile_tx = tx;
            c->vert_warps = vw;
            c->vert_smem = (size_t)(7 * nz + 5) * tx * rs;
            c->coef_smem = (size_t)3 * (nz + 1) * tx * rs;
            if (c->coef_warps * tx > 1024) c->coef_warps = 1024 / tx;
            float ms;
            if (trial(ms) == ERF_B200_OK && ms < best) {
                best = ms;
            } else {   // slower, or not launchable: keep the previous shape
                cudaGetLastError();
                c->tile_tx = keep_tx; c->vert_warps = keep_vw; c->coef_warps = keep_cw;
                c->vert_smem = keep_vs; c->coef_smem = keep_cs;
            }
        }
    }
    for (int cw : {4, 8, 16}) {
        if (rc || cw == c->coef_warps || cw * c->tile_tx > 1024) continue;
        int keep = c->coef_warps;
        c->coef_warps = cw;
        float ms;
        if (trial(ms) == ERF_B200_OK && ms < best) best = ms;
        else { cudaGetLastError(); c->coef_warps = keep; }
    }
    int* kz[3] = {&c->tkz.cell, &c->tkz.mom, &c->tkz.post};
    for (int q = 0; q < 3 && !rc; ++q) {
        const int k0 = *kz[q];
        for (int cand : {k0 / 2, k0 * 2, k0 * 3 / 2}) {
            if (cand < 1 || cand > nz || cand == *kz[q]) continue;
            int keep = *kz[q];
            *kz[q] = cand;
            float ms;
            if (trial(ms) == ERF_B200_OK && ms < best) best = ms;
            else { cudaGetLastError(); *kz[q] = keep; }
        }
    }
    drop_graphs(c);
    int rc2 = build_graphs(c);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_ms) *best_ms = best;
    return rc ? rc : rc2;
}

}  // extern "C"

// An ensemble of contexts advanced inside one graph launch: a conditional
// WHILE node whose body runs two steps of every member (the members' step
// graphs as child graphs, members concurrently) and then a one-thread
// kernel that counts the steps, polls the host's abort word (mapped pinned
// memory) and sets the loop condition.  An odd remaining step runs in a
// second graph whose IF node is gated by the same word.  An abort is seen
// between two steps, so every member's state is a whole number of steps old;
// the device counts the steps that ran and the host reads the count at the
// next sync to put the members' state slots right.
struct EnsCtl {
    int aborted;      // sticky: set when the abort word was seen
    int steps_done;   // steps run since the ensemble was made
    int pairs_left;   // pairs still to run in this launch
    int pairs_req;    // pairs asked for by the launch (written before it)
};

__global__ void k_ens_loop_begin(const volatile int* abort_word, EnsCtl* ctl, cudaGraphConditionalHandle h) {
    const int ab = ctl->aborted | (*abort_word != 0);
    ctl->aborted = ab;
    ctl->pairs_left = ctl->pairs_req;
    cudaGraphSetConditional(h, (!ab && ctl->pairs_left > 0) ? 1u : 0u);
}
__global__ void k_ens_loop_end(const volatile int* abort_word, EnsCtl* ctl, cudaGraphConditionalHandle h) {
    ctl->steps_done += 2;
    const int left = --ctl->pairs_left;
    const int ab = ctl->aborted | (*abort_word != 0);
    ctl->aborted = ab;
    cudaGraphSetConditional(h, (!ab && left > 0) ? 1u : 0u);
}
__global__ void k_ens_gate(const volatile int* abort_word, EnsCtl* ctl, cudaGraphConditionalHandle h) {
    const int ab = ctl->aborted | (*abort_word != 0);
    ctl->aborted = ab;
    if (!ab) ctl->steps_done += 1;
    cudaGraphSetConditional(h, ab ? 0u : 1u);
}

struct erf_b200_ensemble {
    std::vector<erf_b200_ctx*> m;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraphExec_t loop[2] = {nullptr, nullptr};   // pairs of steps from slot parity p
    cudaGraphExec_t one[2] = {nullptr, nullptr};    // one gated step from parity p
    int* abort_word = nullptr;                      // pinned, mapped
    EnsCtl* ctl = nullptr;                          // device
    int parity = 0;                                 // slot parity when all launched steps have run
    int parity_synced = 0;                          // parity at the last sync
    int steps_synced = 0;                           // ctl->steps_done at the last sync
};

namespace {
cudaError_t add_kernel(cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps, size_t ndeps, void* fn,
                       void** args) {
    cudaKernelNodeParams kp{};
    kp.func = fn;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    return cudaGraphAddKernelNode(node, g, deps, ndeps, &kp);
}
cudaError_t add_conditional(cudaGraph_t g, cudaGraphNode_t* node, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                            cudaGraphConditionalNodeType type, cudaGraph_t* body) {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(node, g, &dep, 1, &cp);
    if (e == cudaSuccess) *body = cp.conditional.phGraph_out[0];
    return e;
}
// The loop graph from parity p: begin kernel, then WHILE { steps p and 1-p
// of every member, end kernel }.
cudaError_t build_loop_graph(erf_b200_ensemble* e, int p, cudaGraphExec_t* out) {
    cudaGraph_t g;
    cudaError_t err = cudaGraphCreate(&g, 0);
    if (err != cudaSuccess) return err;
    cudaGraphConditionalHandle h;
    err = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
    const volatile int* aw = e->abort_word;
    EnsCtl* ctl = e->ctl;
    void* args[3] = {(void*)&aw, (void*)&ctl, (void*)&h};
    cudaGraphNode_t begin, wnode, endk;
    cudaGraph_t body = nullptr;
    if (err == cudaSuccess) err = add_kernel(g, &begin, nullptr, 0, (void*)k_ens_loop_begin, args);
    if (err == cudaSuccess) err = add_conditional(g, &wnode, begin, h, cudaGraphCondTypeWhile, &body);
    std::vector<cudaGraphNode_t> second;
    for (size_t q = 0; q < e->m.size() && err == cudaSuccess; ++q) {
        cudaGraphNode_t a, b;
        err = cudaGraphAddChildGraphNode(&a, body, nullptr, 0, e->m[q]->graph_raw[p]);
        if (err == cudaSuccess) err = cudaGraphAddChildGraphNode(&b, body, &a, 1, e->m[q]->graph_raw[1 - p]);
        if (err == cudaSuccess) second.push_back(b);
    }
    if (err == cudaSuccess) err = add_kernel(body, &endk, second.data(), second.size(), (void*)k_ens_loop_end, args);
    if (err == cudaSuccess) err = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return err;
}
// One gated step from parity p: gate kernel, then IF { step p of every member }.
cudaError_t build_one_graph(erf_b200_ensemble* e, int p, cudaGraphExec_t* out) {
    cudaGraph_t g;
    cudaError_t err = cudaGraphCreate(&g, 0);
    if (err != cudaSuccess) return err;
    cudaGraphConditionalHandle h;
    err = cudaGraphConditionalHandleCreate(&h, g, 0, 0);
    const volatile int* aw = e->abort_word;
    EnsCtl* ctl = e->ctl;
    void* args[3] = {(void*)&aw, (void*)&ctl, (void*)&h};
    cudaGraphNode_t gate, inode;
    cudaGraph_t body = nullptr;
    if (err == cudaSuccess) err = add_kernel(g, &gate, nullptr, 0, (void*)k_ens_gate, args);
    if (err == cudaSuccess) err = add_conditional(g, &inode, gate, h, cudaGraphCondTypeIf, &body);
    for (size_t q = 0; q < e->m.size() && err == cudaSuccess; ++q) {
        cudaGraphNode_t a;
        err = cudaGraphAddChildGraphNode(&a, body, nullptr, 0, e->m[q]->graph_raw[p]);
    }
    if (err == cudaSuccess) err = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return err;
}
}  // namespace

extern "C" {

int erf_b200_ensemble_destroy(erf_b200_ensemble* e) {
    if (!e) return ERF_B200_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (int p = 0; p < 2; ++p) {
        if (e->loop[p]) cudaGraphExecDestroy(e->loop[p]);
        if (e->one[p]) cudaGraphExecDestroy(e->one[p]);
    }
    if (e->ctl) cudaFree(e->ctl);
    if (e->abort_word) cudaFreeHost(e->abort_word);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    delete e;
    return ERF_B200_OK;
}

int erf_b200_ensemble_create(erf_b200_ensemble** out, erf_b200_ctx* const* members, int n, void* stream) {
    if (!out || !members || n < 1) return ERF_B200_EINVAL;
    *out = nullptr;
    int parity = members[0] ? members[0]->cur : -1;
    for (int q = 0; q < n; ++q) {
        erf_b200_ctx* c = members[q];
        if (!c || c->cur < 0 || c->cur != parity || !c->graph_raw[0] || !c->graph_raw[1]) return ERF_B200_EBADSTATE;
        CK(cudaStreamSynchronize(c->stream));
    }
    erf_b200_ensemble* e = new (std::nothrow) erf_b200_ensemble();
    if (!e) return ERF_B200_ENOMEM;
    e->m.assign(members, members + n);
    e->parity = e->parity_synced = parity;
    auto fail = [&](cudaError_t err) { erf_b200_ensemble_destroy(e); return cuda_fail(err); };
    if (stream) {
        e->stream = (cudaStream_t)stream;
    } else {
        cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
        if (err != cudaSuccess) { e->stream = nullptr; return fail(err); }
        e->own_stream = true;
    }
    cudaError_t err = cudaHostAlloc((void**)&e->abort_word, sizeof(int), cudaHostAllocMapped);
    if (err != cudaSuccess) { e->abort_word = nullptr; return fail(err); }
    *(volatile int*)e->abort_word = 0;
    err = cudaMalloc((void**)&e->ctl, sizeof(EnsCtl));
    if (err != cudaSuccess) { e->ctl = nullptr; return fail(err); }
    if ((err = cudaMemsetAsync(e->ctl, 0, sizeof(EnsCtl), e->stream)) != cudaSuccess) return fail(err);
    for (int p = 0; p < 2; ++p) {
        if ((err = build_loop_graph(e, p, &e->loop[p])) != cudaSuccess) return fail(err);
        if ((err = build_one_graph(e, p, &e->one[p])) != cudaSuccess) return fail(err);
    }
    if ((err = cudaStreamSynchronize(e->stream)) != cudaSuccess) return fail(err);
    *out = e;
    return ERF_B200_OK;
}

// nsteps steps of every member: the pairs in one launch of the loop graph,
// an odd last step in one launch of the gated single-step graph.  The
// members' resident states advance; the slot parity is settled at the next
// erf_b200_ensemble_sync.
int erf_b200_ensemble_advance(erf_b200_ensemble* e, int nsteps) {
    if (!e || nsteps < 0) return ERF_B200_EINVAL;
    const int pairs = nsteps / 2;
    if (pairs > 0) {
        CK(cudaMemcpyAsync(&e->ctl->pairs_req, &pairs, sizeof(int), cudaMemcpyHostToDevice, e->stream));
        CK(cudaGraphLaunch(e->loop[e->parity], e->stream));
    }
    if (nsteps & 1) {
        CK(cudaGraphLaunch(e->one[e->parity], e->stream));
        e->parity ^= 1;
    }
    for (erf_b200_ctx* c : e->m) c->cur = -1;   // unknown until the next sync
    return ERF_B200_OK;
}

// Ask the ensemble's device loop to stop (flag != 0) or clear a stop (0).
// The loop reads the word between steps; the members then keep the state of
// the last whole step and erf_b200_ensemble_sync returns ERF_B200_EABORTED.
// Clearing waits for the ensemble's stream and resets the device's sticky
// flag, so that later advances run again.
int erf_b200_ensemble_abort(erf_b200_ensemble* e, int flag) {
    if (!e) return ERF_B200_EINVAL;
    *(volatile int*)e->abort_word = flag ? 1 : 0;
    if (!flag) {
        CK(cudaStreamSynchronize(e->stream));
        CK(cudaMemsetAsync(&e->ctl->aborted, 0, sizeof(int), e->stream));
        CK(cudaStreamSynchronize(e->stream));
    }
    return ERF_B200_OK;
}

// Wait for the ensemble's work, then settle the members' state slots from
// the steps that ran (before store_state or status reads on the members'
// own streams).  ERF_B200_EABORTED when an abort stopped the loop.
int erf_b200_ensemble_sync(erf_b200_ensemble* e) {
    if (!e) return ERF_B200_EINVAL;
    CK(cudaStreamSynchronize(e->stream));
    EnsCtl h;
    CK(cudaMemcpy(&h, e->ctl, sizeof(EnsCtl), cudaMemcpyDeviceToHost));
    const int ran = h.steps_done - e->steps_synced;
    e->steps_synced = h.steps_done;
    e->parity_synced ^= (ran & 1);
    e->parity = e->parity_synced;
    for (erf_b200_ctx* c : e->m) c->cur = e->parity;
    return h.aborted ? ERF_B200_EABORTED : ERF_B200_OK;
}

// Steps every member ran since the ensemble was made (after a sync).
int erf_b200_ensemble_steps(const erf_b200_ensemble* e, int* steps) {
    if (!e || !steps) return ERF_B200_EINVAL;
    *steps = e->steps_synced;
    return ERF_B200_OK;
}

// Name of the last CUDA error behind an ERF_B200_ECUDA / ENOMEM return on
// this host thread ("no error" if none).
const char* erf_b200_last_cuda_error(void) { return cudaGetErrorString(g_last_cuda_error); }

}  // extern "C"
