// amrex_io.h -- host-side AMReX VisMF MultiFab files (single grid on write,
// any number of grids on read), shared by the plotfile and checkpoint
// writers.
//
// A MultiFab named <prefix> is two kinds of file:
//   <prefix>_H         VisMF header: version 1, "how" 1, ncomp, ngrow, the
//                      BoxArray of valid boxes, the FabOnDisk list, and the
//                      per-FAB min / max of each component over its valid box;
//   <prefix>_D_00000   the FABs: a text line
//                      "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))(box) ncomp"
//                      (IEEE FP64, little endian) followed by the grown box's
//                      values, component-major, i fastest.
// Boxes are written "((lo) (hi) (type))" with type 1 in a nodal direction.
#pragma once

#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace erfio {

struct Box {
    int lo[3], hi[3], t[3];
    long long n(int d) const { return (long long)hi[d] - lo[d] + 1; }
    size_t size() const { return (size_t)(n(0) * n(1) * n(2)); }
};

inline Box box(int hx, int hy, int hz, int tx = 0, int ty = 0, int tz = 0) {
    return Box{{0, 0, 0}, {hx, hy, hz}, {tx, ty, tz}};
}

inline Box grow(const Box& b, int g) {
    Box r = b;
    for (int d = 0; d < 3; ++d) { r.lo[d] -= g; r.hi[d] += g; }
    return r;
}

inline std::string box_str(const Box& b) {
    char s[160];
    std::snprintf(s, sizeof s, "((%d,%d,%d) (%d,%d,%d) (%d,%d,%d))", b.lo[0], b.lo[1], b.lo[2], b.hi[0], b.hi[1],
                  b.hi[2], b.t[0], b.t[1], b.t[2]);
    return s;
}

inline int make_dir(const std::string& d) {
    if (mkdir(d.c_str(), 0755) != 0 && errno != EEXIST) return -1;
    return 0;
}

// Write MultiFab <prefix> of one FAB: valid box `vb`, `ng` ghost cells, data
// over the grown box (ncomp * grow(vb, ng).size() values).
inline int write_multifab(const std::string& prefix, const Box& vb, int ng, int ncomp, const std::vector<double>& data) {
    const Box gb = grow(vb, ng);
    const size_t n = gb.size();
    if (data.size() != n * ncomp) return -1;
    const std::string dname = prefix.substr(prefix.rfind('/') + 1) + "_D_00000";
    FILE* f = std::fopen((prefix + "_D_00000").c_str(), "wb");
    if (!f) return -1;
    std::fprintf(f, "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))%s %d\n", box_str(gb).c_str(), ncomp);
    size_t wrote = std::fwrite(data.data(), sizeof(double), data.size(), f);
    std::fclose(f);
    if (wrote != data.size()) return -1;
    f = std::fopen((prefix + "_H").c_str(), "w");
    if (!f) return -1;
    std::fprintf(f, "1\n1\n%d\n%d\n(1 0\n%s\n)\n1\nFabOnDisk: %s 0\n\n", ncomp, ng, box_str(vb).c_str(), dname.c_str());
    for (int pass = 0; pass < 2; ++pass) {
        std::fprintf(f, "1,%d\n", ncomp);
        for (int q = 0; q < ncomp; ++q) {
            double m = 0.0;
            bool first = true;
            for (int k = vb.lo[2]; k <= vb.hi[2]; ++k)
                for (int j = vb.lo[1]; j <= vb.hi[1]; ++j)
                    for (int i = vb.lo[0]; i <= vb.hi[0]; ++i) {
                        size_t c = (size_t)q * n + ((size_t)(k - gb.lo[2]) * gb.n(1) + (j - gb.lo[1])) * gb.n(0) +
                                   (i - gb.lo[0]);
                        double x = data[c];
                        m = first ? x : (pass == 0 ? std::fmin(m, x) : std::fmax(m, x));
                        first = false;
                    }
            std::fprintf(f, "%.16e,", m);
        }
        std::fprintf(f, "\n\n");
    }
    std::fclose(f);
    return 0;
}

inline bool parse_box(const char* s, Box& b) {
    return std::sscanf(s, " ((%d,%d,%d) (%d,%d,%d) (%d,%d,%d))", &b.lo[0], &b.lo[1], &b.lo[2], &b.hi[0], &b.hi[1],
                       &b.hi[2], &b.t[0], &b.t[1], &b.t[2]) == 9;
}

// Read MultiFab <prefix> (any number of FABs, any ghost width) into `out`,
// ncomp values over box `want` (component-major, i fastest).  Every point of
// `want` must be covered by some FAB's stored (grown) box; the valid boxes
// are preferred, so values in ghost cells never overwrite valid ones.
// Returns 0, or -1 on a missing file, a malformed header, a component-count
// or index-type mismatch, a non-FP64 / big-endian FAB or an uncovered point.
inline int read_multifab(const std::string& prefix, const Box& want, int ncomp, std::vector<double>& out) {
    FILE* f = std::fopen((prefix + "_H").c_str(), "r");
    if (!f) return -1;
    char line[4096];
    int vers = 0, how = 0, nc = 0, nboxes = 0;
    auto next = [&]() { return std::fgets(line, sizeof line, f) != nullptr; };
    bool ok = next() && std::sscanf(line, "%d", &vers) == 1 && next() && std::sscanf(line, "%d", &how) == 1 &&
              next() && std::sscanf(line, "%d", &nc) == 1 && next() && next() &&
              std::sscanf(line, " (%d", &nboxes) == 1;
    std::vector<Box> valid;
    for (int b = 0; ok && b < nboxes; ++b) {
        Box bx;
        ok = next() && parse_box(line, bx);
        valid.push_back(bx);
    }
    ok = ok && next() && next();  // ")" and the FAB count
    std::vector<std::pair<std::string, long>> fabs;
    for (int b = 0; ok && b < nboxes; ++b) {
        char name[1024];
        long off = 0;
        ok = next() && std::sscanf(line, "FabOnDisk: %1023s %ld", name, &off) == 2;
        fabs.emplace_back(name, off);
    }
    std::fclose(f);
    if (!ok || nc != ncomp) return -1;
    const std::string dir = prefix.substr(0, prefix.rfind('/') + 1);
    out.assign((size_t)ncomp * want.size(), 0.0);
    std::vector<char> have(want.size(), 0);
    for (int pass = 0; pass < 2; ++pass)  // pass 0: ghost regions, pass 1: valid boxes (win)
        for (int b = 0; b < nboxes; ++b) {
            FILE* d = std::fopen((dir + fabs[b].first).c_str(), "rb");
            if (!d) return -1;
            std::fseek(d, fabs[b].second, SEEK_SET);
            if (!std::fgets(line, sizeof line, d)) { std::fclose(d); return -1; }
            const char* desc = "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))";
            Box gb;
            int fnc = 0;
            const char* rest = line + std::strlen(desc);
            if (std::strncmp(line, desc, std::strlen(desc)) != 0 || !parse_box(rest, gb) ||
                std::sscanf(std::strrchr(rest, ')') + 1, "%d", &fnc) != 1 || fnc != ncomp) {
                std::fclose(d);
                return -1;
            }
            for (int q = 0; q < 3; ++q)
                if (gb.t[q] != want.t[q]) { std::fclose(d); return -1; }
            std::vector<double> fab((size_t)ncomp * gb.size());
            size_t got = std::fread(fab.data(), sizeof(double), fab.size(), d);
            std::fclose(d);
            if (got != fab.size()) return -1;
            Box src = pass == 0 ? gb : valid[b];
            for (int q = 0; q < 3; ++q) {  // never read outside the stored box
                src.lo[q] = std::max(src.lo[q], gb.lo[q]);
                src.hi[q] = std::min(src.hi[q], gb.hi[q]);
            }
            for (int k = std::max(src.lo[2], want.lo[2]); k <= std::min(src.hi[2], want.hi[2]); ++k)
                for (int j = std::max(src.lo[1], want.lo[1]); j <= std::min(src.hi[1], want.hi[1]); ++j)
                    for (int i = std::max(src.lo[0], want.lo[0]); i <= std::min(src.hi[0], want.hi[0]); ++i) {
                        size_t w = ((size_t)(k - want.lo[2]) * want.n(1) + (j - want.lo[1])) * want.n(0) +
                                   (i - want.lo[0]);
                        size_t s = ((size_t)(k - gb.lo[2]) * gb.n(1) + (j - gb.lo[1])) * gb.n(0) + (i - gb.lo[0]);
                        for (int q = 0; q < ncomp; ++q)
                            out[(size_t)q * want.size() + w] = fab[(size_t)q * gb.size() + s];
                        have[w] = 1;
                    }
        }
    for (char h : have)
        if (!h) return -1;
    return 0;
}

}  // namespace erfio
