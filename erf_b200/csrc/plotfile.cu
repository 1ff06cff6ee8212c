// plotfile.cu -- AMReX single-level plotfile writer (host code).
//
// Writes the state in the layout of ERF::WritePlotFile (Source/IO/
// ERF_Plotfile.cpp:186-1400 with the derived fields of Source/ERF_Derive.cpp)
// so that AMReX tooling (fcompare, yt, ParaView, Amrvis) reads it:
//   <dir>/Header                  "HyperCLaw-V1.1" header: variable names,
//                                 time, domain, cell sizes, one grid;
//   <dir>/Level_0/Cell_H          FabArray header: box list, FabOnDisk,
//                                 per-component min / max;
//   <dir>/Level_0/Cell_D_00000    one FAB: text header, then little-endian
//                                 FP64, component-major, i fastest.
// Variables, in the reference's order: density, x/y/z_velocity (face
// averages to cell centres), temp, theta, KE (Deardorff), scalar, pres_hse and
// dens_hse (when a base state is given), pressure, and qv / qc / qrain with
// moisture, and z_phys (cell-centre heights) and detJ when terrain node
// heights are given; the terrain plotfile also carries the nodal MultiFab
// Level_0/Nu_nd (node displacements 0, 0, z - k dz) listed at the end of the
// Header, as WriteMultiLevelPlotfileWithTerrain (ERF_Plotfile.cpp:1505-1680)
// writes it.  The MultiFab files themselves are written by amrex_io.h.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/erf_b200.h"
#include "amrex_io.h"

namespace {

constexpr double kRd = 287.0, kRv = 461.505, kP0 = 1.0e5, kIP0 = 1. / kP0, kGamma = 1.4;

// getPgivenRTh / getTgivenRandRTh (Source/Utils/ERF_EOS.H:42-79), same
// operation order so the derived fields match the reference's to the bit
double eos_p(double rt, double qv) { return kP0 * std::pow(kRd * rt * (1.0 + (kRv / kRd) * qv) * kIP0, kGamma); }
double eos_T(double rho, double rt, double qv) {
    double p = kP0 * std::pow(kRd * rt * (1.0 + kRv / kRd * qv) * kIP0, kGamma);
    return p / (kRd * rho * (1.0 + kRv / kRd * qv));
}

}  // namespace

extern "C" {

int erf_b200_write_plotfile(const erf_b200_config* cfg, const char* dir, const double* cons, const double* u,
                            const double* v, const double* w, const double* rho0, const double* p0,
                            const double* z_nd, double time, int step) {
    if (!cfg || !dir || !cons || !u || !v || !w) return ERF_B200_EINVAL;
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, nc = cfg->ncomp;
    if (nx < 1 || ny < 1 || nz < 1) return ERF_B200_EINVAL;
    const size_t N = (size_t)nx * ny * nz;
    const bool moist = cfg->moisture != ERF_MOIST_NONE;
    const bool dd = cfg->les_type == ERF_LES_DEARDORFF;
    const bool terrain = cfg->use_terrain && z_nd;
    // base state: nz+2 values (or planes of nx*ny with terrain), plane k+1 for level k
    auto base_at = [&](const double* b, int i, int j, int k) {
        return cfg->use_terrain ? b[(size_t)(k + 1) * nx * ny + (size_t)j * nx + i] : b[k + 1];
    };
    std::vector<std::string> names = {"density", "x_velocity", "y_velocity", "z_velocity", "temp", "theta"};
    if (dd) names.push_back("KE");
    names.push_back("scalar");
    if (rho0 && p0) { names.push_back("pres_hse"); names.push_back("dens_hse"); }
    names.push_back("pressure");
    if (moist) {
        names.push_back("qv");
        if (nc > ERF_RHOQ1_COMP + 1) names.push_back("qc");
        if (nc > ERF_RHOQ1_COMP + 2) names.push_back("qrain");
    }
    if (terrain) { names.push_back("z_phys"); names.push_back("detJ"); }
    const int nvar = (int)names.size();
    std::vector<double> data((size_t)nvar * N);
    auto C = [&](int n, size_t c) { return cons[(size_t)n * N + c]; };
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                size_t c = ((size_t)k * ny + j) * nx + i;
                double rho = C(0, c), rt = C(1, c);
                double qv = moist ? C(ERF_RHOQ1_COMP, c) / rho : 0.0;
                int q = 0;
                auto put = [&](double val) { data[(size_t)(q++) * N + c] = val; };
                put(rho);
                put(0.5 * (u[((size_t)k * ny + j) * (nx + 1) + i] + u[((size_t)k * ny + j) * (nx + 1) + i + 1]));
                put(0.5 * (v[((size_t)k * (ny + 1) + j) * nx + i] + v[((size_t)k * (ny + 1) + j + 1) * nx + i]));
                put(0.5 * (w[((size_t)k * ny + j) * nx + i] + w[((size_t)(k + 1) * ny + j) * nx + i]));
                put(eos_T(rho, rt, qv));
                put(rt / rho);
                if (dd) put(C(ERF_RHOKE_COMP, c) / rho);
                put(C(ERF_RHOSCALAR_COMP, c) / rho);
                if (rho0 && p0) { put(base_at(p0, i, j, k)); put(base_at(rho0, i, j, k)); }
                put(eos_p(rt, qv));
                if (moist) {
                    put(qv);
                    if (nc > ERF_RHOQ1_COMP + 1) put(C(ERF_RHOQ1_COMP + 1, c) / rho);
                    if (nc > ERF_RHOQ1_COMP + 2) put(C(ERF_RHOQ1_COMP + 2, c) / rho);
                }
                if (terrain) {
                    auto Z = [&](int a, int b, int kk) { return z_nd[((size_t)kk * (ny + 1) + b) * (nx + 1) + a]; };
                    put(.125 * (Z(i, j, k) + Z(i + 1, j, k) + Z(i, j + 1, k) + Z(i + 1, j + 1, k) + Z(i, j, k + 1) +
                                Z(i + 1, j, k + 1) + Z(i, j + 1, k + 1) + Z(i + 1, j + 1, k + 1)));
                    put(.25 * (Z(i, j, k + 1) - Z(i, j, k) + Z(i + 1, j, k + 1) - Z(i + 1, j, k) + Z(i, j + 1, k + 1) -
                               Z(i, j + 1, k) + Z(i + 1, j + 1, k + 1) - Z(i + 1, j + 1, k)) /
                        cfg->dz);
                }
            }

    const std::string root(dir);
    if (erfio::make_dir(root) || erfio::make_dir(root + "/Level_0")) return ERF_B200_EINVAL;
    const double prob_hi[3] = {nx * cfg->dx, ny * cfg->dy, nz * cfg->dz};
    const double dxs[3] = {cfg->dx, cfg->dy, cfg->dz};
    // ---- Header
    {
        FILE* f = std::fopen((root + "/Header").c_str(), "w");
        if (!f) return ERF_B200_EINVAL;
        std::fprintf(f, "HyperCLaw-V1.1\n%d\n", nvar);
        for (auto& s : names) std::fprintf(f, "%s\n", s.c_str());
        std::fprintf(f, "3\n%.17g\n0\n", time);
        std::fprintf(f, "%.17g %.17g %.17g \n", 0.0, 0.0, 0.0);
        std::fprintf(f, "%.17g %.17g %.17g \n", prob_hi[0], prob_hi[1], prob_hi[2]);
        std::fprintf(f, "\n((0,0,0) (%d,%d,%d) (0,0,0)) \n", nx - 1, ny - 1, nz - 1);
        std::fprintf(f, "%d \n%.17g %.17g %.17g \n0\n0\n", step, dxs[0], dxs[1], dxs[2]);
        std::fprintf(f, "0 1 %.17g\n%d\n", time, step);
        for (int d = 0; d < 3; ++d) std::fprintf(f, "%.17g %.17g\n", 0.0, prob_hi[d]);
        std::fprintf(f, "Level_0/Cell\n");
        if (terrain) std::fprintf(f, "1\n3\namrexvec_nu_x\namrexvec_nu_y\namrexvec_nu_z\nLevel_0/Nu_nd\n");
        std::fclose(f);
    }
    if (erfio::write_multifab(root + "/Level_0/Cell", erfio::box(nx - 1, ny - 1, nz - 1), 0, nvar, data))
        return ERF_B200_EINVAL;
    if (terrain) {
        // node displacements (0, 0, z - k dz) over the nodal box, as the reference's Nu_nd
        const size_t M = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
        std::vector<double> nd(3 * M, 0.0);
        for (int k = 0; k <= nz; ++k)
            for (size_t p = 0; p < (size_t)(nx + 1) * (ny + 1); ++p) {
                size_t c = (size_t)k * (nx + 1) * (ny + 1) + p;
                nd[2 * M + c] = z_nd[c] - k * cfg->dz;
            }
        if (erfio::write_multifab(root + "/Level_0/Nu_nd", erfio::box(nx, ny, nz, 1, 1, 1), 0, 3, nd))
            return ERF_B200_EINVAL;
    }
    return ERF_B200_OK;
}

}  // extern "C"
