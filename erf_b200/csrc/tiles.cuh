// tiles.cuh -- x-y tiles marching in k, shared by the flat transport
// kernels (kernels.cu) and the terrain post pass (terrain.cu): the staged
// level of a scalar with its halo, the face-flux tile, the tile-edge faces
// and the divergence.  A block of TTX x TTY columns stages each level's
// plane in shared memory, evaluates the advective flux through every cell's
// low x and y faces (two designated warps also the tile's high-side faces)
// and carries the flux through each cell's top face to the next level, so
// every face flux is evaluated once per block.
#pragma once
#include "kernels.cuh"

namespace erfb {

// Cell-centred scalar with foextrap in z.
template <class V>
__device__ __forceinline__ V ccz(const V* __restrict__ f, const Geo& g, int i, int j, int k) {
    return __ldg(f + cidx(g, i, j, clampk(k, g.nz)));
}

// Advective flux of a primitive scalar phi (type R) through the low z face
// of cell (i,j,k): mom * interp(phi) (Advection/ERF_AdvectionSrcForScalars.H:
// 7-58).  The advecting momentum M is the FP64 stage momentum (rho, theta)
// or the R average momentum (slow scalars).
template <int T, class R, class M>
__device__ __forceinline__ R adv_flux_z(const Geo& g, const R* __restrict__ phi, const M* __restrict__ mom, int type,
                                        R frac, int i, int j, int k) {
    R s[6];
    const int w = width_of<T>(type);
    for (int m = 0; m < 6; ++m) {
        int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? ccz(phi, g, i, j, k + off) : R(0);
    }
    R a = R(__ldg(mom + cidx(g, i, j, k)));
    return a * interp_of<T, R>(type, s, a, frac);
}

template <class R>
struct FluxTile {
    R fx[TTY][TTX + 1];
    R fy[TTY + 1][TTX];
};

// One level of a scalar over the block's tile plus a 3-cell halo on every
// side (periodic in x and y), staged in shared memory so that the x and y
// stencils read it at fixed offsets.
constexpr int PH = 3;   // halo width (Upwind_5th / WENO5 stencils)
template <class R>
struct Plane {
    R v[TTY + 2 * PH][TTX + 2 * PH];
};
// Asynchronous copy of the plane (cp.async): the copies land in shared
// memory while the block works on the previous level; plane_wait() makes
// this thread's copies complete (a barrier then publishes them).
template <class R>
__device__ __forceinline__ void load_plane(const Geo& g, Plane<R>& p, const R* __restrict__ phi, int k) {
    const int t = threadIdx.y * TTX + threadIdx.x;
    const int i0 = blockIdx.x * TTX - PH, j0 = blockIdx.y * TTY - PH;
    const R* __restrict__ lev = phi + g.sk * k;
    constexpr int W = TTX + 2 * PH, NE = W * (TTY + 2 * PH);
    for (int e = t; e < NE; e += TTX * TTY) {
        const int b = e / W, a = e - b * W;
        const int gi = wrap_far(i0 + a, g.nx), gj = wrap_far(j0 + b, g.ny);
        const unsigned dst = (unsigned)__cvta_generic_to_shared(&p.v[b][a]);
        const R* src = lev + gi + (int64_t)g.nx * gj;
        if constexpr (sizeof(R) == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void plane_wait() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Flux through a face from the plane: x faces read row ty+PH from column
// c0 (c0 = tx for the low face, tx+1 for the high face); y faces read column
// tx+PH from row r0.
template <int T, class R>
__device__ __forceinline__ R plane_flux_x(const Plane<R>& p, int ty, int c0, R a, int type, R frac) {
    R s[6];
    const int w = width_of<T>(type);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? p.v[ty + PH][c0 + m] : R(0);
    }
    return a * interp_of<T, R>(type, s, a, frac);
}
template <int T, class R>
__device__ __forceinline__ R plane_flux_y(const Plane<R>& p, int r0, int tx, R a, int type, R frac) {
    R s[6];
    const int w = width_of<T>(type);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const int off = m - 3;
        s[m] = (off >= -w && off <= w - 1) ? p.v[r0 + m][tx + PH] : R(0);
    }
    return a * interp_of<T, R>(type, s, a, frac);
}

// The tile's high-side halo faces: the x-face after the last valid column
// of each valid row (nvy of them) and the y-face above the last valid row
// of each valid column (nvx).  Warp 0 evaluates the y-faces (lane = column)
// and warp 1 the x-faces (lane = row), so the other warps run no extra
// interpolant pass; with the faces assigned to the cells' own threads
// instead, every warp would repeat the whole interpolant for its last lane.
struct TileEdge {
    int nvx, nvy;   // valid columns / rows of the tile
    int col;        // >= 0: this thread evaluates the high y-face of column col
    int row;        // >= 0: this thread evaluates the high x-face of row row
    int i0, j0;
};
__device__ __forceinline__ TileEdge tile_edge(const Geo& g) {
    TileEdge e;
    e.i0 = blockIdx.x * TTX;
    e.j0 = blockIdx.y * TTY;
    e.nvx = min(TTX, g.nx - e.i0);
    e.nvy = min(TTY, g.ny - e.j0);
    const int t = threadIdx.y * TTX + threadIdx.x;
    e.col = t < e.nvx ? t : -1;
    e.row = (t >= TTX && t < TTX + e.nvy) ? t - TTX : -1;
    return e;
}

// Fluxes of one scalar for cell (i,j,k): the low x / y faces into the tile
// from the staged plane, z through zl/zh (zl is computed only on the block's
// first level; otherwise it is the carried top flux of the level below).
template <int TH, int TV, class R, class M>
__device__ __forceinline__ void tile_put(const Geo& g, FluxTile<R>& t, const Plane<R>& pl, const R* __restrict__ phi,
                                         const M* __restrict__ ax, const M* __restrict__ ay,
                                         const M* __restrict__ az, int th, int tv, R fh, R fv, int i, int j, int k,
                                         bool first, R& zl, R& zh) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t c = cidx(g, i, j, k);
    t.fx[ty][tx] = plane_flux_x<TH>(pl, ty, tx, R(__ldg(ax + c)), th, fh);
    t.fy[ty][tx] = plane_flux_y<TH>(pl, ty, tx, R(__ldg(ay + c)), th, fh);
    if (first) zl = adv_flux_z<TV>(g, phi, az, tv, fv, i, j, k);
    zh = adv_flux_z<TV>(g, phi, az, tv, fv, i, j, k + 1);
}
// The tile's high-side halo faces of one scalar at level k (see TileEdge).
template <int TH, class R, class M>
__device__ __forceinline__ void tile_put_edge(const Geo& g, const TileEdge& e, FluxTile<R>& t, const Plane<R>& pl,
                                              const M* __restrict__ ax, const M* __restrict__ ay, int th, R fh,
                                              int k) {
    if (e.row >= 0) {
        const int ih = wrap(e.i0 + e.nvx, g.nx);
        t.fx[e.row][e.nvx] = plane_flux_x<TH>(pl, e.row, e.nvx, R(__ldg(ax + cidx(g, ih, e.j0 + e.row, k))), th, fh);
    }
    if (e.col >= 0) {
        const int jh = wrap(e.j0 + e.nvy, g.ny);
        t.fy[e.nvy][e.col] = plane_flux_y<TH>(pl, e.nvy, e.col, R(__ldg(ay + cidx(g, e.i0 + e.col, jh, k))), th, fh);
    }
}
template <class R>
__device__ __forceinline__ R tile_div(const Geo& g, const FluxTile<R>& t, R zl, R zh) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    return R(-1.0 * 1.0) * ((t.fx[ty][tx + 1] - t.fx[ty][tx]) * R(g.dxi) + (t.fy[ty + 1][tx] - t.fy[ty][tx]) * R(g.dyi) +
                            (zh - zl) * R(g.dzi));
}

// Host side of the tiles.
// Levels per block: minimise waves x (levels + 1), the cost of a block being
// its levels plus the extra bottom-face flux evaluation.
template <typename K>
inline int pick_kz(K kern, const Geo& g) {
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, TTX * TTY, 0) != cudaSuccess || per < 1) per = 1;
    const long cap = (long)per * nsm;
    const long nxy = (long)((g.nx + TTX - 1) / TTX) * ((g.ny + TTY - 1) / TTY);
    int best = g.nz;
    double best_cost = 1e30;
    for (int zb = 1; zb <= g.nz; ++zb) {
        int kz = (g.nz + zb - 1) / zb;
        int zb2 = (g.nz + kz - 1) / kz;
        long waves = (nxy * zb2 + cap - 1) / cap;
        double cost = (double)waves * (kz + 1);
        if (cost < best_cost) { best_cost = cost; best = kz; }
    }
    return best;
}

inline dim3 tile_grid(const Geo& g, int kz) { return dim3((g.nx + TTX - 1) / TTX, (g.ny + TTY - 1) / TTY, (g.nz + kz - 1) / kz); }

}  // namespace erfb
