// noalloc.cu -- Kessler microphysics for callers that cannot allocate device
// memory.
//
// erf_b200_kessler_advance stages the caller's state (an Array4 view with
// arbitrary ghost widths and strides) in a dense scratch copy owned by the
// context, runs the column kernel on it and writes the result back.  Creating
// a context allocates.  Some callers cannot do that: a host code whose device
// memory is entirely reserved up front by its own pool (AMReX's arenas, for
// example) and which must not see a second allocator, or code running while
// a CUDA graph is being captured on its stream, where cudaMalloc is not
// permitted.  erf_b200_kessler_advance_noalloc does the same work with no
// context and no allocation: its scratch is the file-scope device array
// below, loaded with the library.
#include <mutex>

#include "kernels.cuh"

namespace erfb {
__global__ void k_kessler(Params P, double* cons, double dtn, double dz);
__global__ void k_pack(Geo g, erf_b200_fab f, int kind, int ncomp, double* dst);
__global__ void k_unpack(Geo g, erf_b200_fab f, int kind, int ncomp, const double* src, int tang_lo_zero,
                         int tang_hi_zero, int wall_w);
}  // namespace erfb

using namespace erfb;

// Shared scratch: ERF_B200_NOALLOC_MAX_DOUBLES doubles (16 MiB) on every GPU
// that loads the library, held until the process exits.  Host code must not
// pass this symbol to a kernel (on the host it names a host-side stand-in, not
// device memory); it uses the address cudaGetSymbolAddress returns.
static __device__ __align__(256) double g_noalloc_scratch[ERF_B200_NOALLOC_MAX_DOUBLES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device with that device current.
int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return ERF_B200_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return ERF_B200_EINVAL;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return ERF_B200_ECUDA;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return ERF_B200_OK;
}

}  // namespace

extern "C" int erf_b200_kessler_advance_noalloc(const erf_b200_config* cfg, const erf_b200_fab* cons, double dt,
                                                void* stream) {
    if (!cfg || !cons || !cons->p) return ERF_B200_EINVAL;
    if (cfg->moisture != ERF_MOIST_KESSLER && cfg->moisture != ERF_MOIST_KESSLER_NORAIN) return ERF_B200_ECONFIG;
    if ((cfg->moisture == ERF_MOIST_KESSLER && cfg->ncomp != 8) ||
        (cfg->moisture == ERF_MOIST_KESSLER_NORAIN && cfg->ncomp != 7))
        return ERF_B200_ECONFIG;
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1 || !(cfg->dz > 0.0) || !(cfg->c_p > 0.0)) return ERF_B200_ECONFIG;
    // the caller's view must cover the valid region with all components
    if (cons->lo[0] > 0 || cons->lo[1] > 0 || cons->lo[2] > 0 || cons->hi[0] < cfg->nx - 1 ||
        cons->hi[1] < cfg->ny - 1 || cons->hi[2] < cfg->nz - 1 || cons->ncomp < cfg->ncomp)
        return ERF_B200_EINVAL;
    const int64_t need = (int64_t)cfg->ncomp * cfg->nx * cfg->ny * cfg->nz;
    if (need > (int64_t)ERF_B200_NOALLOC_MAX_DOUBLES) return ERF_B200_EINVAL;

    double* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc != ERF_B200_OK) return rc;

    Geo g{};
    g.nx = cfg->nx; g.ny = cfg->ny; g.nz = cfg->nz;
    g.sk = (int64_t)cfg->nx * cfg->ny;
    g.ncell = g.sk * cfg->nz;
    g.nzf = g.sk * (cfg->nz + 1);
    g.dxi = 1.0 / cfg->dx; g.dyi = 1.0 / cfg->dy; g.dzi = 1.0 / cfg->dz;
    g.zlo_noslip = cfg->zlo_bc == ERF_BC_NO_SLIP_WALL;
    g.zhi_noslip = cfg->zhi_bc == ERF_BC_NO_SLIP_WALL;
    Params P{};
    P.g = g;
    P.ncomp = cfg->ncomp;
    P.nprim = cfg->ncomp - 1;
    P.moist = 1;
    P.kessler_rain = cfg->moisture == ERF_MOIST_KESSLER;
    P.c_p = cfg->c_p;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // every scratch element the column kernel reads is written by the pack
    // kernel first, so nothing in the shared array has to start at zero
    dim3 b(32, 4, 1), gp((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
    k_pack<<<gp, b, 0, st>>>(g, *cons, 0, cfg->ncomp, scratch);
    dim3 gc((g.nx + 31) / 32, (g.ny + 3) / 4, 1);
    k_kessler<<<gc, b, 0, st>>>(P, scratch, dt, cfg->dz);
    int nxb = cons->hi[0] - cons->lo[0] + 1, nyb = cons->hi[1] - cons->lo[1] + 1, nzb = cons->hi[2] - cons->lo[2] + 1;
    dim3 gu((nxb + 31) / 32, (nyb + 3) / 4, nzb);
    k_unpack<<<gu, b, 0, st>>>(g, *cons, 0, cfg->ncomp, scratch, g.zlo_noslip, g.zhi_noslip, 0);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ERF_B200_OK : ERF_B200_ECUDA;
}
