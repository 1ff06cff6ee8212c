// checkpoint.cu -- ERF native checkpoints of a host state (host code).
//
// Layout of ERF::WriteCheckpointFile / ReadCheckpointFile
// (Source/IO/ERF_Checkpoint.cpp:25-265 and :264-470), single level:
//   <dir>/Header                 "Checkpoint file for ERF", finest_level 0,
//                                ncomp of cons, 1 / 1 / 1 (face velocities),
//                                istep, dt, t_new, the level's BoxArray;
//   <dir>/Level_0/Cell           cons, no ghost cells;
//   <dir>/Level_0/XFace, YFace, ZFace   face velocities, no ghost cells;
//   <dir>/Level_0/BaseState      r0, p0, pi0, th0 with 3 ghost cells;
//   <dir>/Level_0/Z_Phys_nd      terrain node heights with the reference's
//                                ghost width (ComputeGhostCells + 2);
//   <dir>/Level_0/MapFactor_m, _u, _v   2-D map factors (1: no map projection
//                                on this path) with 3 ghost cells.
// Ghost values the state does not carry are filled the way the reference's
// FillBoundary / extrapolation leaves them: periodic images laterally, base
// state levels beyond k = -1 .. nz held at the nearest level, node heights
// below / above the grid linearly extrapolated from the nearest two levels.
// The reader takes any number of FABs and any ghost width, so checkpoints
// written by the reference itself restart here too.
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/erf_b200.h"
#include "amrex_io.h"

namespace {

// ERF::ComputeGhostCells (Source/ERF.H:1081-1125) with use_NumDiff false:
// the ghost width the reference sizes its MultiFabs with for an advection choice
int ghost_cells(const erf_b200_config& c) {
    auto any = [&](int a) {
        return c.dycore_horiz_adv == a || c.dycore_vert_adv == a || c.moistscal_horiz_adv == a ||
               c.dryscal_horiz_adv == a || c.dryscal_vert_adv == a;
    };
    auto any_scal = [&](int a) {
        return c.dryscal_horiz_adv == a || c.dryscal_vert_adv == a || c.moistscal_horiz_adv == a ||
               c.moistscal_vert_adv == a;
    };
    if (any(ERF_ADV_CENTERED_6TH) || any(ERF_ADV_UPWIND_5TH)) return 3;
    if (any_scal(ERF_ADV_WENO_5) || any_scal(ERF_ADV_WENO_5Z)) return 3;
    if (any_scal(ERF_ADV_WENO_7) || any_scal(ERF_ADV_WENO_7Z)) return 4;
    return 2;
}

int wrap(int i, int n) { return ((i % n) + n) % n; }

}  // namespace

extern "C" {

int erf_b200_write_checkpoint(const erf_b200_config* cfg, const char* dir, const double* cons, const double* u,
                              const double* v, const double* w, const double* r0, const double* p0,
                              const double* pi0, const double* th0, const double* z_nd, int step, double dt,
                              double time) {
    if (!cfg || !dir || !cons || !u || !v || !w || !r0 || !p0 || !pi0 || !th0) return ERF_B200_EINVAL;
    if (cfg->use_terrain && !z_nd) return ERF_B200_EINVAL;
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, nc = cfg->ncomp;
    if (nx < 1 || ny < 1 || nz < 2 || nc < 1) return ERF_B200_EINVAL;
    const size_t N = (size_t)nx * ny * nz;
    const std::string root(dir), lev = root + "/Level_0/";
    if (erfio::make_dir(root) || erfio::make_dir(root + "/Level_0")) return ERF_B200_EINVAL;
    {
        FILE* f = std::fopen((root + "/Header").c_str(), "w");
        if (!f) return ERF_B200_EINVAL;
        std::fprintf(f, "Checkpoint file for ERF\n0\n%d\n1\n1\n1\n%d \n%.17g \n%.17g \n(1 0\n%s\n)\n", nc, step, dt, time,
                     erfio::box_str(erfio::box(nx - 1, ny - 1, nz - 1)).c_str());
        std::fclose(f);
    }
    const erfio::Box cell = erfio::box(nx - 1, ny - 1, nz - 1);
    int rc = 0;
    rc |= erfio::write_multifab(lev + "Cell", cell, 0, nc, std::vector<double>(cons, cons + nc * N));
    rc |= erfio::write_multifab(lev + "XFace", erfio::box(nx, ny - 1, nz - 1, 1, 0, 0), 0, 1,
                                std::vector<double>(u, u + (size_t)(nx + 1) * ny * nz));
    rc |= erfio::write_multifab(lev + "YFace", erfio::box(nx - 1, ny, nz - 1, 0, 1, 0), 0, 1,
                                std::vector<double>(v, v + (size_t)nx * (ny + 1) * nz));
    rc |= erfio::write_multifab(lev + "ZFace", erfio::box(nx - 1, ny - 1, nz, 0, 0, 1), 0, 1,
                                std::vector<double>(w, w + N + (size_t)nx * ny));
    if (rc) return ERF_B200_EINVAL;
    {   // base state: levels k = -1 .. nz per column (one column when flat)
        const int g = 3;
        const erfio::Box gb = erfio::grow(cell, g);
        std::vector<double> bs(4 * gb.size());
        const double* B[4] = {r0, p0, pi0, th0};
        size_t c = 0;
        for (int q = 0; q < 4; ++q)
            for (int k = gb.lo[2]; k <= gb.hi[2]; ++k)
                for (int j = gb.lo[1]; j <= gb.hi[1]; ++j)
                    for (int i = gb.lo[0]; i <= gb.hi[0]; ++i) {
                        int kk = k < -1 ? -1 : (k > nz ? nz : k);
                        size_t col = cfg->use_terrain ? (size_t)wrap(j, ny) * nx + wrap(i, nx) : 0;
                        bs[c++] = B[q][(size_t)(kk + 1) * (cfg->use_terrain ? (size_t)nx * ny : 1) + col];
                    }
        if (erfio::write_multifab(lev + "BaseState", cell, g, 4, bs)) return ERF_B200_EINVAL;
    }
    if (cfg->use_terrain) {
        const int g = ghost_cells(*cfg) + 2;
        const erfio::Box nb = erfio::box(nx, ny, nz, 1, 1, 1), gb = erfio::grow(nb, g);
        std::vector<double> zn(gb.size());
        auto Z = [&](int i, int j, int k) { return z_nd[((size_t)k * (ny + 1) + j) * (nx + 1) + i]; };
        size_t c = 0;
        for (int k = gb.lo[2]; k <= gb.hi[2]; ++k)
            for (int j = gb.lo[1]; j <= gb.hi[1]; ++j)
                for (int i = gb.lo[0]; i <= gb.hi[0]; ++i) {
                    int ii = wrap(i, nx), jj = wrap(j, ny);  // node n == node 0 on a periodic grid
                    double z;
                    if (k < 0) z = Z(ii, jj, 0) + k * (Z(ii, jj, 1) - Z(ii, jj, 0));
                    else if (k > nz) z = Z(ii, jj, nz) + (k - nz) * (Z(ii, jj, nz) - Z(ii, jj, nz - 1));
                    else z = Z(ii, jj, k);
                    zn[c++] = z;
                }
        if (erfio::write_multifab(lev + "Z_Phys_nd", nb, g, 1, zn)) return ERF_B200_EINVAL;
    }
    {
        const int g = 3;
        const erfio::Box m = erfio::box(nx - 1, ny - 1, 0), mu = erfio::box(nx, ny - 1, 0, 1, 0, 0),
                         mv = erfio::box(nx - 1, ny, 0, 0, 1, 0);
        rc |= erfio::write_multifab(lev + "MapFactor_m", m, g, 1, std::vector<double>(erfio::grow(m, g).size(), 1.0));
        rc |= erfio::write_multifab(lev + "MapFactor_u", mu, g, 1, std::vector<double>(erfio::grow(mu, g).size(), 1.0));
        rc |= erfio::write_multifab(lev + "MapFactor_v", mv, g, 1, std::vector<double>(erfio::grow(mv, g).size(), 1.0));
        if (rc) return ERF_B200_EINVAL;
    }
    return ERF_B200_OK;
}

int erf_b200_read_checkpoint(const erf_b200_config* cfg, const char* dir, double* cons, double* u, double* v,
                             double* w, double* r0, double* p0, double* pi0, double* th0, double* z_nd, int* step,
                             double* dt, double* time) {
    if (!cfg || !dir || !cons || !u || !v || !w) return ERF_B200_EINVAL;
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, nc = cfg->ncomp;
    if (nx < 1 || ny < 1 || nz < 1 || nc < 1) return ERF_B200_EINVAL;
    const std::string root(dir), lev = root + "/Level_0/";
    {
        FILE* f = std::fopen((root + "/Header").c_str(), "r");
        if (!f) return ERF_B200_EINVAL;
        char title[256];
        int finest = -1, ncons = 0, n1 = 0, n2 = 0, n3 = 0, st = 0;
        double d = 0, t = 0;
        bool ok = std::fgets(title, sizeof title, f) && std::string(title) == "Checkpoint file for ERF\n" &&
                  std::fscanf(f, "%d %d %d %d %d %d %lf %lf", &finest, &ncons, &n1, &n2, &n3, &st, &d, &t) == 8;
        std::fclose(f);
        // single level, the same conserved components, one component per face velocity
        if (!ok || finest != 0 || ncons != nc || n1 != 1 || n2 != 1 || n3 != 1) return ERF_B200_EINVAL;
        if (step) *step = st;
        if (dt) *dt = d;
        if (time) *time = t;
    }
    std::vector<double> buf;
    auto take = [&](const std::string& name, const erfio::Box& b, int ncomp, double* dst) {
        if (erfio::read_multifab(lev + name, b, ncomp, buf)) return false;
        std::copy(buf.begin(), buf.end(), dst);
        return true;
    };
    if (!take("Cell", erfio::box(nx - 1, ny - 1, nz - 1), nc, cons) ||
        !take("XFace", erfio::box(nx, ny - 1, nz - 1, 1, 0, 0), 1, u) ||
        !take("YFace", erfio::box(nx - 1, ny, nz - 1, 0, 1, 0), 1, v) ||
        !take("ZFace", erfio::box(nx - 1, ny - 1, nz, 0, 0, 1), 1, w))
        return ERF_B200_EINVAL;
    if (r0 || p0 || pi0 || th0) {
        if (!(r0 && p0 && pi0 && th0)) return ERF_B200_EINVAL;
        // levels k = -1 .. nz; every column over terrain, column (0,0) on a flat grid
        erfio::Box b = cfg->use_terrain ? erfio::box(nx - 1, ny - 1, nz) : erfio::box(0, 0, nz);
        b.lo[2] = -1;
        if (erfio::read_multifab(lev + "BaseState", b, 4, buf)) return ERF_B200_EINVAL;
        double* B[4] = {r0, p0, pi0, th0};
        for (int q = 0; q < 4; ++q) std::copy(buf.begin() + q * b.size(), buf.begin() + (q + 1) * b.size(), B[q]);
    }
    if (z_nd && !take("Z_Phys_nd", erfio::box(nx, ny, nz, 1, 1, 1), 1, z_nd)) return ERF_B200_EINVAL;
    return ERF_B200_OK;
}

}  // extern "C"
