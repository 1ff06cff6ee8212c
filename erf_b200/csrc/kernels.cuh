// kernels.cuh -- parameter block and device-array bundle shared by the
// dycore kernels (kernels.cu) and the host driver (api.cu).
#pragma once
#include "common.cuh"

namespace erfb {

// Scalar parameters of one context, passed by value to every kernel.
struct Params {
    Geo g;
    int ncomp, nprim;
    int moist, kessler_rain;
    int use_diff, use_turb, use_consA, les;
    double CsDeltaSqr;          // Cs^2 Delta^2 (host-computed, reference order)
    double Cs;
    double Delta;               // (dx dy dz)^(1/3)
    double Ck, Ce_wall, Ce_lcoeff, g_over_theta0, invSigmaK;   // Deardorff constants
    double invPr, invSc;
    double alphaT_eff, alphaC_eff; // rhoAlpha (Constant) or alpha (ConstantAlpha)
    double mu_eff;              // 2*dynamicViscosity (/rho0_trans for ConstantAlpha)
    double gravity, rdOcp, c_p, c_v, halfg;
    int buoy_type;
    int coriolis;
    double cf, sinphi, cosphi, geo0, geo1, geo2;
    int dyc_h, dyc_v, dry_h, dry_v, moi_h, moi_v;
    double f_dyc_h, f_dyc_v, f_dry_h, f_dry_v, f_moi_h, f_moi_v;
    const double* r0;           // base state, index k+1 for cell k (nz+2); with
    const double* p0;           // terrain (nz+2) planes of nx*ny, plane k+1
    const double* pi0;          // for level k
    int* status;
    // static terrain: z_phys_nd as (nz+3) planes of nx*ny nodes (plane k+1
    // for node level k, lateral node index periodic) and detJ per cell
    int ter;
    const double* znd;
    const double* detJ;
    const double* met;          // metric tables (terrain.cu), TER_NMET planes of nzf
    // moving terrain (terrain_type Moving; null pointers otherwise): z_t on
    // the z faces ((nz+1) planes of nx*ny), the nodes at the stage's new time
    // (detJ_new of the slow-variable update), and the surface wave
    // h = mt_ampl sin(mt_kp x - mt_om t) on x = i mt_dx, levels k mt_dz
    const double* mt_zt;
    const double* mt_znew;
    const double* mt_fac;       // Sullivan's factor of each level (nz+1)
    double mt_ampl, mt_kp, mt_om, mt_dx, mt_dz;
    // MOST ground (Moeng stress, adiabatic): the level of the reference
    // height, the step's plane means {u, v, |U|, u*} (most_avg, device), the
    // eddy viscosity (R = double or float by most_mut_f32) for eta
    int most, most_k, most_mut_f32;
    double most_zref, most_z0, most_dz;
    double* most_avg;
    const void* most_mut;
};

// Number of static-terrain metric tables (planes of nzf values each).
constexpr int TER_NMET = 21;

// One copy of the prognostic state: cons (ncomp*ncell), face momenta.
struct StateBuf {
    double* cons;
    double* mx;   // ncell (periodic x faces)
    double* my;   // ncell
    double* mz;   // nzf
};

// Quantities derived from a stage state, stored in the bulk type R.
template <class R>
struct StageAux {
    R* prim;   // nprim*ncell
    R* pi;     // ncell
    R* pp;     // ncell (p - p0)
};

// Deardorff TKE closure arrays (R): vertical heat diffusivity Theta_v,
// dissipation and SmnSmn per cell, theta's vertical diffusive flux per z-face
// (hfx_z).  All null for the other closures.
template <class R>
struct TkeBuf {
    R* kthv;
    R* diss;
    R* smn;
    R* hfz;
};

// Terrain scratch (R): strain components of the stage (tau_ii with the
// expansion-rate third removed, S12, S13, S23 on edges), the non-symmetric
// stresses tau31 / tau32, the substep's horizontal momentum increments, and
// the boundary-face momenta of the previous substep (FP64).
template <class R>
struct TerBuf {
    R *s11, *s22, *s33, *s12, *s13, *s23;
    R *t31, *t32;
    R *ndu, *ndv, *odu, *odv;
    R *fx[2], *fy[2];            // raw diffusive face fluxes (two fields)
    double* bnd;                 // substep: the previous momentum on the ground
                                 // and lid faces (two planes)
};

// x-y tile of the transport kernels (slow_cell, slow_mom, post) and the
// levels each of their blocks marches through (chosen per context).
constexpr int TTX = 32, TTY = 8;
struct TiledKz {
    int cell, mom, post;
    int ter_post;   // the terrain post pass (terrain contexts)
};

// erf_b200_create's configuration checks (api.cu): ERF_B200_OK or an error code.
int validate_config(const erf_b200_config* c);

// Host launchers of the dycore kernels (kernels.cu), instantiated for
// R = double (plain form) and R = float (mixed form).
// Levels per block of k_kessler_cells (blocks of 32 columns x KESS_KB levels)
constexpr int KESS_KB = 8;
template <class R>
void tiled_setup(const Params& P, TiledKz* t);
template <class R>
int vert_setup(size_t vert_smem, size_t coef_smem);
template <class R>
void launch_step_begin(const Params& P, cudaStream_t st, const double* cons, const double* uo, const double* vo,
                       const double* wo, StateBuf S, double* un, double* vn, double* wn, StageAux<R> A, R* mut,
                       TkeBuf<R> tke);
template <class R>
void launch_tau(const Params& P, cudaStream_t st, const double* cons, const double* u, const double* v,
                const double* w, const R* mut, R* t11, R* t22, R* t33, R* t12, R* t13, R* t23);
template <class R>
void launch_stage_aux(const Params& P, cudaStream_t st, const double* cons, StageAux<R> A);
// Blocks per level of the plane averages; the avg buffer holds 6 nz results,
// 5 nz PAVG_PARTS partial sums and nz tickets (plane_avg_doubles(nz) doubles,
// zero-initialised).
constexpr int PAVG_PARTS = 16;
inline size_t plane_avg_doubles(int nz) { return (size_t)6 * nz + (size_t)5 * nz * PAVG_PARTS + nz; }
template <class R>
void launch_plane_avg(const Params& P, cudaStream_t st, const double* cons, const R* prim, double* avg);
template <class R>
void launch_fast_h(const Params& P, cudaStream_t st, int step, int nrk, double dtau, double facinv, StateBuf Sprev,
                   int prev_rt, StateBuf Sst, StageAux<R> A, const R* Fmx, const R* Fmy, const R* lag_in, R* lag_out,
                   R* avx, R* avy, double* outx, double* outy);
// MOST plane means and friction velocity of a step from its old velocities
void launch_most_avg(const Params& P, cudaStream_t st, const double* u, const double* v);
template <class R>
void launch_no_substep(const Params& P, cudaStream_t st, double slow_dt, StateBuf Sold, const R* Fcons, const R* Fmx,
                       const R* Fmy, const R* Fmz, StateBuf Ssum);
template <class R>
void launch_fast_coef(const Params& P, cudaStream_t st, dim3 grid, dim3 block, size_t smem, double D, StateBuf Sst,
                      StageAux<R> A, R* cA, R* cInvB, R* cCB, R* cP, R* cQ);
template <class R>
void launch_fast_vert(const Params& P, cudaStream_t st, dim3 grid, dim3 block, size_t smem, double dtau,
                      double facinv, double beta_1, double beta_2, StateBuf Sprev, int prev_rt, StateBuf Sst,
                      StageAux<R> A, const R* Fcons, const R* Fmz, const double* newx, const double* newy,
                      const R* cA, const R* cInvB, const R* cCB, const R* cP, const R* cQ, R* avz, double* out_cons,
                      double* out_mz);
template <class R>
void launch_slow_cell(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux<R> A, const R* mut,
                      const R* hx, const R* hy, const R* hz, TkeBuf<R> tke, R* Fcons, R* avx, R* avy, R* avz);

// Learned closure (closure.cu): network arrays on the device, the fused
// stress / heat-flux kernel with its edge averaging, and feature extraction.
struct ClosureNet {
    const unsigned char* wpack;
    const float* bias;
    const float* norm;   // in mean[13], in std[13], out mean[9], out std[9]
    const float* env;    // lo[13], hi[13]
    unsigned int* fallback;
};
template <class R>
void launch_closure(const Params& P, const ClosureNet& net, int grid, cudaStream_t st, const double* cons,
                    const double* u, const double* v, const double* w, const R* theta, R* t11, R* t22, R* t33, R* c12,
                    R* c13, R* c23, R* t12, R* t13, R* t23, R* hx, R* hy, R* hz);
template <class R>
int closure_grid(const Params& P);
void launch_features(const Params& P, cudaStream_t st, const double* cons, const double* u, const double* v,
                     const double* w, double* theta_scratch, float* out);
template <class R>
void launch_slow_mom(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux<R> A, const double* u,
                     const double* v, const double* w, const R* t11, const R* t22, const R* t33, const R* t12,
                     const R* t13, const R* t23, const double* pavg, R* Fmx, R* Fmy, R* Fmz);
template <class R>
void launch_post(const Params& P, const TiledKz& t, cudaStream_t st, double slow_dt, StateBuf Sold, StateBuf Sst,
                 StateBuf Ssum, StateBuf Snew, StageAux<R> Acur, StageAux<R> Anext, int make_next, const R* mut,
                 TkeBuf<R> tke, const R* avx, const R* avy, const R* avz, double* un, double* vn, double* wn);

// Static terrain (terrain.cu): metrics, base state and the _T passes.
void launch_ter_metrics(const Params& P, cudaStream_t st, double* detJ, double* zcc);
// Moving terrain (terrain.cu).  tdev: the step's old time on the device;
// tsel 0..3 picks T, T + dt/3, T + dt/2, T + dt.
void launch_mt_grid(const Params& P, cudaStream_t st, const double* tdev, double dt, int tsel, double* z);
void launch_mt_zt(const Params& P, cudaStream_t st, const double* zo, const double* zn, const double* tdev,
                  double dt, int tsel_new, double* zt);
void launch_mt_base_state(const Params& P, cudaStream_t st, const double* r0o, const double* p0o, const double* zo,
                          const double* zs, const double* zn, const double* tdev, double dt, int tsel_new,
                          double* r0n, double* p0n);
template <class R>
void launch_mt_no_substep(const Params& P, cudaStream_t st, double slow_dt, StateBuf Sold, const R* Fcons,
                          const R* Fmx, const R* Fmy, const R* Fmz, const double* zo, const double* zn, StateBuf Ssum);
void launch_mt_advance_time(cudaStream_t st, double* tdev, double dt);
// step diagnostics (terrain.cu): out = {mass, integral of rho theta, max |w|};
// zgrid: moving terrain's nodes (NULL: P.detJ with terrain, 1 without);
// part: diagnostics_scratch_doubles() - 3 values
void launch_diagnostics(const Params& P, cudaStream_t st, const double* cons, const double* w, const double* zgrid,
                        double* part, double* out);
int diagnostics_scratch_doubles();
// acoustic substeps over moving terrain: the grid at T + ks dtau, z_t'' of
// the substep, detJ of a grid, and one substep (last: no boundary fill after
// it, the slow-variable pass does that)
void launch_mt_grid_sub(const Params& P, cudaStream_t st, const double* tdev, double dtau, int ks, double* z);
void launch_mt_zpt(const Params& P, cudaStream_t st, const double* zo, const double* zn, double dtau, double* zpt);
void launch_mt_detj(const Params& P, cudaStream_t st, const double* z, double* detJ);
template <class R>
void launch_mt_fast(const Params& P, cudaStream_t st, int step, int lagged, double dtau, double beta_s, double facinv,
                    StateBuf Sprev, StateBuf Sst, StageAux<R> A, const R* Fcons, const R* Fmx, const R* Fmy,
                    const R* Fmz, const R* lag_in, R* lag_out, const R* cA, const R* cInvB, const R* cCB, const R* cP,
                    const R* cQ, const double* zo, const double* zn, const double* zs, const double* zpt,
                    double* trhs, double* om, double* soln, R* avx, R* avy, R* avz, StateBuf Ssum, int last);
void launch_ter_base_state(const Params& P, cudaStream_t st, const double* zcc, const double* th3, const double* qv3,
                           double th_s, double qv_s, double p_s, double* rho0, double* p0, double* pi0, double* th0);
template <class R>
void launch_ter_step_begin(const Params& P, cudaStream_t st, const double* cons, const double* uo, const double* vo,
                           const double* wo, StateBuf S, double* un, double* vn, double* wn, StageAux<R> A, R* mut,
                           TkeBuf<R> tke);
template <class R>
void launch_ter_tau(const Params& P, cudaStream_t st, int nrk, const double* cons, const double* u, const double* v,
                    const double* w, const R* mut, TerBuf<R> T, TkeBuf<R> tke, R* t11, R* t22, R* t33, R* t12, R* t13,
                    R* t23);
template <class R>
void launch_ter_slow_cell(const Params& P, cudaStream_t st, StateBuf S, StageAux<R> A, const double* u,
                          const double* v, const R* mut, TkeBuf<R> tke, TerBuf<R> T, R* Fcons, R* avx, R* avy,
                          R* avz);
template <class R>
void launch_ter_slow_mom(const Params& P, cudaStream_t st, StateBuf S, StageAux<R> A, const double* u,
                         const double* v, const double* w, const R* t11, const R* t22, const R* t33, const R* t12,
                         const R* t13, const R* t23, TerBuf<R> T, const R* Om, R* Fmx, R* Fmy, R* Fmz);
template <class R>
void launch_ter_fast_h(const Params& P, cudaStream_t st, int step, double dtau, double facinv, StateBuf Sprev,
                       int prev_rt, StateBuf Sst, StageAux<R> A, const R* Fmx, const R* Fmy, const R* lag_in,
                       R* lag_out, TerBuf<R> T, R* avx, R* avy, double* outx, double* outy);
template <class R>
void launch_ter_fast_vert(const Params& P, cudaStream_t st, int tx, size_t smem, double dtau, double facinv,
                          double beta_1, double beta_2, StateBuf Sprev, int prev_rt, StateBuf Sst, StageAux<R> A,
                          const R* Fcons, const R* Fmz, TerBuf<R> T, const R* cA, const R* cInvB, const R* cCB,
                          const R* cP, const R* cQ, R* avz, double* out_cons, double* out_mz);
void ter_vert_shape(int nz, int* tx, size_t* smem);
template <class R>
void launch_ter_post(const Params& P, cudaStream_t st, int kz, double slow_dt, StateBuf Sold, StateBuf Sst,
                     StateBuf Ssum, StateBuf Snew, StageAux<R> Acur, StageAux<R> Anext, int make_next, const R* mut,
                     TkeBuf<R> tke, TerBuf<R> T, const R* avx, const R* avy, const R* avz, double* un, double* vn,
                     double* wn);
// Levels per block of the tiled terrain post pass (from the occupancy API).
template <class R>
int ter_post_kz(const Params& P);

}  // namespace erfb
