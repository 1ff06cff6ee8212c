// noalloc.cu -- Kessler microphysics for callers that cannot allocate device
// memory.
//
// erf_b200_kessler_advance stages the caller's state (an Array4 view with
// arbitrary ghost widths and strides) in a dense scratch copy owned by the
// context, runs the column kernel on it and writes the result back.  Creating
// a context allocates.  Some callers cannot do that: a host code whose device
// memory is entirely reserved up front by its own pool (AMReX's arenas, for
// example) and which must not see a second allocator next to it.
// erf_b200_kessler_advance_noalloc does the same work with no context and no
// allocation: its scratch is the file-scope device array below, loaded with
// the library.
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
constexpr unsigned kMaxGridYZ = 65535;   // gridDim.y / gridDim.z limit

// Driver entry points, fetched through the runtime so the library does not
// link libcuda directly (it must load on machines without a driver).
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

struct ScratchSlot {
    unsigned long long ctx_id = 0;   // context the address belongs to (0: none)
    double* addr = nullptr;
};

std::mutex g_mutex;
ScratchSlot g_slot[kMaxDevices];
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

// Unique id of the current context (ids are never reused within a process).
int current_context_id(unsigned long long* id) {
    if (!g_ctx_current || !g_ctx_id) {
        void* f0 = nullptr;
        void* f1 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault) != cudaSuccess || !f0)
            return ERF_B200_ECUDA;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault) != cudaSuccess || !f1)
            return ERF_B200_ECUDA;
        g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        g_ctx_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    void* ctx = nullptr;
    if (g_ctx_current(&ctx) != 0 || !ctx) return ERF_B200_ECUDA;
    return g_ctx_id(ctx, id) == 0 ? ERF_B200_OK : ERF_B200_ECUDA;
}

// Device address of g_noalloc_scratch on the current device.  It is looked
// up with that device current the first time a call runs in its context, and
// again whenever the context has changed since (after cudaDeviceReset the
// runtime makes a new primary context, in which the array has a new address).
int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return ERF_B200_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return ERF_B200_EINVAL;
    std::lock_guard<std::mutex> lock(g_mutex);
    ScratchSlot& s = g_slot[dev];
    unsigned long long id = 0;
    // a context the runtime has not made current yet reports no id: the
    // symbol lookup below initialises it, after which the id exists
    int rc = current_context_id(&id);
    if (rc == ERF_B200_OK && s.addr && s.ctx_id == id) {
        *out = s.addr;
        return ERF_B200_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return ERF_B200_ECUDA;
    if (rc != ERF_B200_OK && current_context_id(&id) != ERF_B200_OK) return ERF_B200_ECUDA;
    s.ctx_id = id;
    s.addr = static_cast<double*>(p);
    *out = s.addr;
    return ERF_B200_OK;
}

}  // namespace

extern "C" int erf_b200_kessler_advance_noalloc(const erf_b200_config* cfg, const erf_b200_fab* cons, double dt,
                                                void* stream) {
    if (!cfg || !cons || !cons->p) return ERF_B200_EINVAL;
    // the configuration rules of erf_b200_create, plus Kessler on a flat grid
    // (over terrain the sedimentation needs 1/detJ, which only a context holds)
    int v = validate_config(cfg);
    if (v != ERF_B200_OK) return v;
    if (cfg->moisture != ERF_MOIST_KESSLER && cfg->moisture != ERF_MOIST_KESSLER_NORAIN) return ERF_B200_ECONFIG;
    if (cfg->use_terrain) return ERF_B200_ECONFIG;
    if (!(cfg->c_p > 0.0)) return ERF_B200_ECONFIG;
    // the caller's view must cover the valid region with all components
    if (cons->lo[0] > 0 || cons->lo[1] > 0 || cons->lo[2] > 0 || cons->hi[0] < cfg->nx - 1 ||
        cons->hi[1] < cfg->ny - 1 || cons->hi[2] < cfg->nz - 1 || cons->ncomp < cfg->ncomp)
        return ERF_B200_EINVAL;
    const int64_t need = (int64_t)cfg->ncomp * cfg->nx * cfg->ny * cfg->nz;
    if (need > (int64_t)ERF_B200_NOALLOC_MAX_DOUBLES) return ERF_B200_EINVAL;
    // launch-shape limits: the pack and unpack grids put one level per block
    // in z and four rows per block in y
    const int64_t nxb = (int64_t)cons->hi[0] - cons->lo[0] + 1, nyb = (int64_t)cons->hi[1] - cons->lo[1] + 1,
                  nzb = (int64_t)cons->hi[2] - cons->lo[2] + 1;
    if ((unsigned)cfg->nz > kMaxGridYZ || nzb > kMaxGridYZ || (nyb + 3) / 4 > kMaxGridYZ ||
        (cfg->ny + 3) / 4 > (int)kMaxGridYZ)
        return ERF_B200_EINVAL;
    // an error left pending by earlier work on this thread belongs to that
    // work: leave it in place and launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) return ERF_B200_ECUDA;

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
    if (cudaGetLastError() != cudaSuccess) return ERF_B200_ECUDA;
    dim3 gc((g.nx + 31) / 32, (g.ny + 3) / 4, 1);
    k_kessler<<<gc, b, 0, st>>>(P, scratch, dt, cfg->dz);
    if (cudaGetLastError() != cudaSuccess) return ERF_B200_ECUDA;
    dim3 gu((unsigned)((nxb + 31) / 32), (unsigned)((nyb + 3) / 4), (unsigned)nzb);
    k_unpack<<<gu, b, 0, st>>>(g, *cons, 0, cfg->ncomp, scratch, g.zlo_noslip, g.zhi_noslip, 0);
    if (cudaGetLastError() != cudaSuccess) return ERF_B200_ECUDA;
    return ERF_B200_OK;
}
