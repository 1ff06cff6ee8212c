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
    double invPr, invSc;
    double alphaT_eff, alphaC_eff; // rhoAlpha (Constant) or alpha (ConstantAlpha)
    double mu_eff;              // 2*dynamicViscosity (/rho0_trans for ConstantAlpha)
    double gravity, rdOcp, c_p, c_v, halfg;
    int buoy_type;
    int coriolis;
    double cf, sinphi, cosphi, geo0, geo1, geo2;
    int dyc_h, dyc_v, dry_h, dry_v, moi_h, moi_v;
    double f_dyc_h, f_dyc_v, f_dry_h, f_dry_v, f_moi_h, f_moi_v;
    const double* r0;           // base state, index k+1 for cell k (nz+2)
    const double* p0;
    const double* pi0;
    int* status;
};

// One copy of the prognostic state: cons (ncomp*ncell), face momenta.
struct StateBuf {
    double* cons;
    double* mx;   // ncell (periodic x faces)
    double* my;   // ncell
    double* mz;   // nzf
};

// Quantities derived from a stage state.
struct StageAux {
    double* prim;   // nprim*ncell
    double* pi;     // ncell
    double* pp;     // ncell (p - p0)
};

// x-y tile of the transport kernels (slow_cell, slow_mom, post) and the
// levels each of their blocks marches through (chosen per context).
constexpr int TTX = 32, TTY = 8;
struct TiledKz {
    int cell, mom, post;
};
void tiled_setup(const Params& P, TiledKz* t);
void launch_slow_cell(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux A, const double* mut,
                      double* Fcons, double* avx, double* avy, double* avz);
void launch_slow_mom(const Params& P, const TiledKz& t, cudaStream_t st, StateBuf S, StageAux A, const double* u,
                     const double* v, const double* w, const double* t11, const double* t22, const double* t33,
                     const double* t12, const double* t13, const double* t23, const double* pavg, double* Fmx,
                     double* Fmy, double* Fmz);
void launch_post(const Params& P, const TiledKz& t, cudaStream_t st, double slow_dt, StateBuf Sold, StateBuf Sst,
                 StateBuf Ssum, StateBuf Snew, StageAux Acur, StageAux Anext, int make_next, const double* mut,
                 const double* avx, const double* avy, const double* avz, double* un, double* vn, double* wn);

}  // namespace erfb
