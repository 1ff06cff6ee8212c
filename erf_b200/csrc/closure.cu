// closure.cu -- the learned subgrid closure inside the dycore step.
//
// Replaces, for les_type ERF_LES_MLP, the stress pass of the Smagorinsky path
// (erf_make_tau_terms, TimeIntegration/ERF_make_tau_terms.cpp:320-424) and
// the eddy-diffusivity heat flux of theta (DiffusionSrcForState_N,
// Diffusion/ERF_DiffusionSrcForState_N.cpp:196-667):
//
//   k_closure  one persistent kernel per RK stage.  Each CTA takes 128
//              consecutive cells at a time; thread t forms cell t's 13
//              features, checks them against the training envelope, runs the
//              network forward on the tensor cores (mlp::forward_cta) and
//              writes rho * (deviatoric stress, heat flux).  Cells outside
//              the envelope get the Smagorinsky stress and heat flux
//              (nu_t = (Cs Delta)^2 |S|, Pr_t) instead, and cells within
//              ENV_MARGIN of its edge a linear blend of the two, so that
//              the closure is continuous in the state.
//   k_closure_edges  averages the cell-centred off-diagonal stresses to the
//              xy / xz / yz edges where the momentum divergence reads them.
//
// Feature definition (shared with the training-data extraction, k_features):
//   du/dx dv/dy dw/dz   from the face velocities of the cell;
//   the other velocity derivatives and grad(theta): centred differences of
//   cell-centred values, one-sided in z in the first and last cell;
//   filter width Delta = (dx dy dz)^(1/3).
// Order: du/dx du/dy du/dz dv/dx dv/dy dv/dz dw/dx dw/dy dw/dz dT/dx dT/dy
// dT/dz Delta.  Outputs: tau11 tau22 tau33 tau12 tau13 tau23 q1 q2 q3
// (kinematic, stresses deviatoric).
#include "kernels.cuh"
#include "mlp.cuh"

namespace erfb {

using namespace erfb::mlp;

// Share of each feature's training range, at either end, across which the
// network hands over to Smagorinsky.
constexpr float ENV_MARGIN = 0.05f;

template <class R>
__device__ __forceinline__ void closure_features(const Geo& g, const double* __restrict__ u,
                                                 const double* __restrict__ v, const double* __restrict__ w,
                                                 const R* __restrict__ theta, double delta, int i, int j, int k,
                                                 float* f) {
    const int ip = wrap(i + 1, g.nx), im = wrap(i - 1, g.nx), jp = wrap(j + 1, g.ny), jm = wrap(j - 1, g.ny);
    const int kp = min(k + 1, g.nz - 1), km = max(k - 1, 0);
    const double dzf = 1.0 / ((double)(kp - km) / g.dzi);
    auto U = [&](int ii, int jj, int kk) { return 0.5 * (u[cidx(g, ii, jj, kk)] + u[cidx(g, wrap(ii + 1, g.nx), jj, kk)]); };
    auto V = [&](int ii, int jj, int kk) { return 0.5 * (v[cidx(g, ii, jj, kk)] + v[cidx(g, ii, wrap(jj + 1, g.ny), kk)]); };
    auto W = [&](int ii, int jj, int kk) { return 0.5 * (w[cidx(g, ii, jj, kk)] + w[cidx(g, ii, jj, kk + 1)]); };
    auto T = [&](int ii, int jj, int kk) { return (double)theta[cidx(g, ii, jj, kk)]; };
    const double hx = 0.5 * g.dxi, hy = 0.5 * g.dyi;
    f[0] = (float)((u[cidx(g, ip, j, k)] - u[cidx(g, i, j, k)]) * g.dxi);
    f[1] = (float)((U(i, jp, k) - U(i, jm, k)) * hy);
    f[2] = (float)((U(i, j, kp) - U(i, j, km)) * dzf);
    f[3] = (float)((V(ip, j, k) - V(im, j, k)) * hx);
    f[4] = (float)((v[cidx(g, i, jp, k)] - v[cidx(g, i, j, k)]) * g.dyi);
    f[5] = (float)((V(i, j, kp) - V(i, j, km)) * dzf);
    f[6] = (float)((W(ip, j, k) - W(im, j, k)) * hx);
    f[7] = (float)((W(i, jp, k) - W(i, jm, k)) * hy);
    f[8] = (float)((w[cidx(g, i, j, k + 1)] - w[cidx(g, i, j, k)]) * g.dzi);
    f[9] = (float)((T(ip, j, k) - T(im, j, k)) * hx);
    f[10] = (float)((T(i, jp, k) - T(i, jm, k)) * hy);
    f[11] = (float)((T(i, j, kp) - T(i, j, km)) * dzf);
    f[12] = (float)delta;
}

// Smagorinsky stress and heat flux (kinematic) from the same features.
__device__ __forceinline__ void smagorinsky_closure(const float* f, float csd2, float invPr, float* y) {
    float s11 = f[0], s22 = f[4], s33 = f[8];
    float s12 = 0.5f * (f[1] + f[3]), s13 = 0.5f * (f[2] + f[6]), s23 = 0.5f * (f[5] + f[7]);
    float ss = s11 * s11 + s22 * s22 + s33 * s33 + 2.0f * (s12 * s12 + s13 * s13 + s23 * s23);
    float nut = csd2 * sqrtf(2.0f * ss);
    float tr = (s11 + s22 + s33) * (1.0f / 3.0f);
    y[0] = -2.0f * nut * (s11 - tr);
    y[1] = -2.0f * nut * (s22 - tr);
    y[2] = -2.0f * nut * (s33 - tr);
    y[3] = -2.0f * nut * s12;
    y[4] = -2.0f * nut * s13;
    y[5] = -2.0f * nut * s23;
    y[6] = -nut * invPr * f[9];
    y[7] = -nut * invPr * f[10];
    y[8] = -nut * invPr * f[11];
}

template <class R>
// Five CTAs per SM: the register cap (96, no spills) lets one CTA's features
// and GELU overlap the others' MMA waits (124 registers and 4 CTAs without it;
// 1.170 -> 1.150 ms per mixed learned step on the coarse ABL, same results).
__global__ void __launch_bounds__(ROWS, 5) k_closure(Params P, ClosureNet net, const double* __restrict__ cons,
                                                  const double* __restrict__ u, const double* __restrict__ v,
                                                  const double* __restrict__ w, const R* __restrict__ theta,
                                                  R* __restrict__ t11, R* __restrict__ t22, R* __restrict__ t33,
                                                  R* __restrict__ c12, R* __restrict__ c13, R* __restrict__ c23,
                                                  R* __restrict__ hx, R* __restrict__ hy, R* __restrict__ hz) {
    __shared__ __align__(128) unsigned char sW[T_FWD_END];
    __shared__ __align__(128) unsigned char sX[ROWS * KIN * 2];
    __shared__ __align__(128) unsigned char sH[ROWS * HID * 2];
    __shared__ float sB[NBIAS], sN[2 * NIN + 2 * NOUT], sE[2 * NIN];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const Geo& g = P.g;
    const int t = threadIdx.x, warp = t >> 5;
    for (int q = t; q < T_FWD_END / 16; q += ROWS)
        reinterpret_cast<uint4*>(sW)[q] = reinterpret_cast<const uint4*>(net.wpack)[q];
    for (int q = t; q < NBIAS; q += ROWS) sB[q] = net.bias[q];
    for (int q = t; q < 2 * NIN + 2 * NOUT; q += ROWS) sN[q] = net.norm[q];
    for (int q = t; q < 2 * NIN; q += ROWS) sE[q] = net.env[q];
    if (warp == 0) tmem_alloc(&tslot, 64);
    if (t == 0) bar_init(&bar);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = tslot;
    uint32_t phase = 0;
    bool ok = true;
    const double delta = cbrt(1.0 / (g.dxi * g.dyi * g.dzi));
    const float csd2 = (float)P.CsDeltaSqr, invPr = (float)P.invPr;
    const int64_t nblk = (g.ncell + ROWS - 1) / ROWS;
    unsigned int nfb = 0;
    for (int64_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int64_t c = blk * ROWS + t;
        const bool live = c < g.ncell;
        float f[NIN], xn[NIN];
        bool fb = !live;
        // weight of the network: 1 well inside the training envelope, falling
        // linearly to 0 across the outer ENV_MARGIN of each feature's range,
        // so that the closure is continuous where it hands over to Smagorinsky
        float wgt = 1.0f;
        if (live) {
            int k = (int)(c / g.sk), rem = (int)(c - (int64_t)k * g.sk);
            int j = rem / g.nx, i = rem - j * g.nx;
            closure_features<R>(g, u, v, w, theta, delta, i, j, k, f);
            for (int q = 0; q < NIN; ++q) {
                const float lo = sE[q], hi = sE[NIN + q], m = ENV_MARGIN * (hi - lo);
                const float d = fminf(f[q] - lo, hi - f[q]);
                if (m > 0.0f) wgt = fminf(wgt, fmaxf(0.0f, fminf(1.0f, d / m)));
                else if (!(d >= 0.0f)) wgt = 0.0f;
                xn[q] = (f[q] - sN[q]) / sN[NIN + q];
            }
            fb = !(wgt > 0.0f);
        }
        if (fb)
            for (int q = 0; q < NIN; ++q) xn[q] = 0.0f;
        float y[NOUTP];
        ok = forward_cta(sW, sX, sH, sB, &bar, tm, phase, xn, y) && ok;
        if (!live) continue;
        float o[NOUT];
        if (fb) {
            smagorinsky_closure(f, csd2, invPr, o);
            ++nfb;
        } else {
            for (int q = 0; q < NOUT; ++q) o[q] = y[q] * sN[2 * NIN + NOUT + q] + sN[2 * NIN + q];
            if (wgt < 1.0f) {
                float os[NOUT];
                smagorinsky_closure(f, csd2, invPr, os);
                for (int q = 0; q < NOUT; ++q) o[q] = wgt * o[q] + (1.0f - wgt) * os[q];
            }
        }
        const R rho = R(cons[c]);
        t11[c] = rho * R(o[0]); t22[c] = rho * R(o[1]); t33[c] = rho * R(o[2]);
        c12[c] = rho * R(o[3]); c13[c] = rho * R(o[4]); c23[c] = rho * R(o[5]);
        hx[c] = rho * R(o[6]); hy[c] = rho * R(o[7]); hz[c] = rho * R(o[8]);
    }
    for (int o = 16; o > 0; o >>= 1) nfb += __shfl_xor_sync(0xffffffffu, nfb, o);
    if ((t & 31) == 0 && nfb) atomicAdd(net.fallback, nfb);
    if (!ok && t == 0) atomicOr(P.status, ST_TIMEOUT);
    if (warp == 0) tmem_free(tm, 64);
}

// Off-diagonal stresses on the edges the momentum divergence reads:
// tau12 on xy edges (low corner of cell i,j at level k), tau13 / tau23 on
// xz / yz edges at z-face k (first / last cell's value at the walls).
template <class R>
__global__ void k_closure_edges(Params P, const R* __restrict__ c12, const R* __restrict__ c13,
                                const R* __restrict__ c23, R* __restrict__ t12, R* __restrict__ t13,
                                R* __restrict__ t23) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k > g.nz) return;
    const int im = wrap(i - 1, g.nx), jm = wrap(j - 1, g.ny);
    const int ka = max(k - 1, 0), kb = min(k, g.nz - 1);
    if (k < g.nz)
        t12[cidx(g, i, j, k)] = R(0.25) * (c12[cidx(g, im, jm, k)] + c12[cidx(g, i, jm, k)] + c12[cidx(g, im, j, k)] +
                                           c12[cidx(g, i, j, k)]);
    t13[cidx(g, i, j, k)] = R(0.25) * (c13[cidx(g, im, j, ka)] + c13[cidx(g, i, j, ka)] + c13[cidx(g, im, j, kb)] +
                                       c13[cidx(g, i, j, kb)]);
    t23[cidx(g, i, j, k)] = R(0.25) * (c23[cidx(g, i, jm, ka)] + c23[cidx(g, i, j, ka)] + c23[cidx(g, i, jm, kb)] +
                                       c23[cidx(g, i, j, kb)]);
}

// Features of every cell (training-data extraction), theta from the state.
__global__ void k_features(Params P, const double* __restrict__ cons, const double* __restrict__ u,
                           const double* __restrict__ v, const double* __restrict__ w, double* __restrict__ theta,
                           float* __restrict__ out, int pass) {
    const Geo& g = P.g;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz) return;
    int64_t c = cidx(g, i, j, k);
    if (pass == 0) {
        theta[c] = cons[g.ncell + c] / cons[c];
        return;
    }
    const double delta = cbrt(1.0 / (g.dxi * g.dyi * g.dzi));
    float f[NIN];
    closure_features<double>(g, u, v, w, theta, delta, i, j, k, f);
    for (int q = 0; q < NIN; ++q) out[c * NIN + q] = f[q];
}

template <class R>
void launch_closure(const Params& P, const ClosureNet& net, int grid, cudaStream_t st, const double* cons,
                    const double* u, const double* v, const double* w, const R* theta, R* t11, R* t22, R* t33, R* c12,
                    R* c13, R* c23, R* t12, R* t13, R* t23, R* hx, R* hy, R* hz) {
    k_closure<R><<<grid, ROWS, 0, st>>>(P, net, cons, u, v, w, theta, t11, t22, t33, c12, c13, c23, hx, hy, hz);
    const Geo& g = P.g;
    k_closure_edges<R><<<dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz + 1), dim3(32, 4, 1), 0, st>>>(P, c12, c13, c23,
                                                                                                   t12, t13, t23);
}

template <class R>
int closure_grid(const Params& P) {
    int dev = 0, nsm = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_closure<R>, ROWS, 0) != cudaSuccess) per = 0;
    // the same bound from the kernel's registers and shared memory
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_closure<R>) == cudaSuccess && fa.numRegs > 0) {
        int by_regs = 65536 / (fa.numRegs * ROWS);
        int by_smem = (int)(227 * 1024 / (fa.sharedSizeBytes + 1024));
        int est = by_regs < by_smem ? by_regs : by_smem;
        if (est > per) per = est;
    }
    if (per < 1) per = 1;
    per = per > 8 ? 8 : per;   // 8 x 64 TMEM columns per SM
    long nblk = (P.g.ncell + ROWS - 1) / ROWS;
    long grid = (long)per * nsm;
    return (int)(grid < nblk ? grid : nblk);
}

void launch_features(const Params& P, cudaStream_t st, const double* cons, const double* u, const double* v,
                     const double* w, double* theta_scratch, float* out) {
    const Geo& g = P.g;
    dim3 b(32, 4, 1), gr((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
    k_features<<<gr, b, 0, st>>>(P, cons, u, v, w, theta_scratch, out, 0);
    k_features<<<gr, b, 0, st>>>(P, cons, u, v, w, theta_scratch, out, 1);
}

template void launch_closure<double>(const Params&, const ClosureNet&, int, cudaStream_t, const double*, const double*,
                                     const double*, const double*, const double*, double*, double*, double*, double*,
                                     double*, double*, double*, double*, double*, double*, double*, double*);
template void launch_closure<float>(const Params&, const ClosureNet&, int, cudaStream_t, const double*, const double*,
                                    const double*, const double*, const float*, float*, float*, float*, float*, float*,
                                    float*, float*, float*, float*, float*, float*, float*);
template int closure_grid<double>(const Params&);
template int closure_grid<float>(const Params&);

}  // namespace erfb
