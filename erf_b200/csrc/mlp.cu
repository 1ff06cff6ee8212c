// mlp.cu -- learned subgrid closure on the 5th-generation tensor cores.
//
// A 13 -> 64 -> 64 -> 64 -> 9 multilayer perceptron with GELU (tanh form)
// activations maps the resolved velocity gradients (9), the potential
// temperature gradient (3) and the filter width (1) to the six subgrid
// stresses and three subgrid heat fluxes.  Weights and activations are BF16,
// products accumulate in FP32 in tensor memory (TMEM):
//
//   * one CTA of 128 threads owns 128 rows (samples or grid cells); thread t
//     owns row t, which is TMEM lane t of every M = 128 accumulator, so the
//     epilogue of each layer (bias, GELU, BF16 pack) is thread-local;
//   * operands live in shared memory in the no-swizzle K-major canonical
//     layout of tcgen05 (8-row x 16-byte core matrices; 128 B between core
//     matrices along K, K/8 * 128 B between 8-row groups);
//   * one elected thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32)
//     and commits to an mbarrier that the CTA waits on (bounded wait).
//
// Training runs forward and backward in one kernel: dX = dZ W and
// dW = dZ^T H are tcgen05 products as well (dW with the output features as M,
// padded to 128 rows, and the CTA's 128 samples as K).  Per-CTA partial
// gradients are summed in a fixed order by a second kernel, then an Adam step
// updates the FP32 master weights and repacks the BF16 operand tiles.
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "mlp.cuh"

namespace erfb {
namespace mlp {

// ---------------------------------------------------------------------------
// Inference: Y = MLP(X) for rows [blockIdx.x*128, +128).  X is [n][13] FP32
// raw features; the normalisation (mean/std per feature and per output) is
// applied here.  TMEM: 64 columns, reused by every layer.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(ROWS) k_mlp_infer(const float* __restrict__ X, int n, const unsigned char* __restrict__ wpack,
                                                   const float* __restrict__ bias, const float* __restrict__ norm,
                                                   float* __restrict__ Y, int* status) {
    __shared__ __align__(128) unsigned char sW[T_FWD_END];
    __shared__ __align__(128) unsigned char sX[ROWS * KIN * 2];
    __shared__ __align__(128) unsigned char sH[ROWS * HID * 2];
    __shared__ float sB[NBIAS];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x, warp = t >> 5;
    const int row = blockIdx.x * ROWS + t;
    for (int q = t; q < T_FWD_END / 16; q += ROWS)
        reinterpret_cast<uint4*>(sW)[q] = reinterpret_cast<const uint4*>(wpack)[q];
    for (int q = t; q < NBIAS; q += ROWS) sB[q] = bias[q];
    float x[NIN];
    for (int q = 0; q < NIN; ++q) x[q] = row < n ? (X[(int64_t)row * NIN + q] - norm[q]) / norm[NIN + q] : 0.0f;
    if (warp == 0) tmem_alloc(&tslot, 64);
    if (t == 0) bar_init(&bar);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = tslot;
    uint32_t phase = 0;
    float y[NOUTP];
    bool ok = forward_cta(sW, sX, sH, sB, &bar, tm, phase, x, y);
    if (row < n)
        for (int q = 0; q < NOUT; ++q) Y[(int64_t)row * NOUT + q] = y[q] * norm[2 * NIN + NOUT + q] + norm[2 * NIN + q];
    if (!ok && t == 0) atomicOr(status, 1);
    if (warp == 0) tmem_free(tm, 64);
}

// ---------------------------------------------------------------------------
// Training: forward and backward of rows [blockIdx.x*128, +128) of a batch
// of normalised inputs Xn [n][13] and targets Tn [n][9]; loss
// sum (y - t)^2 * inv_count.  Writes this CTA's partial gradient (padded
// parameter layout) and loss.  TMEM columns: z1 [0,64), z2 [64,128),
// z3 [128,192), y [192,208), dW [256,320), dX [320,384).
// ---------------------------------------------------------------------------
struct TrainSmem {
    unsigned char W[T_END];
    unsigned char X0[ROWS * KIN * 2];
    unsigned char H[3][ROWS * HID * 2];
    unsigned char X0T[KIN * ROWS * 2];
    unsigned char HT[3][HID * ROWS * 2];
    unsigned char dZ[ROWS * HID * 2];
    unsigned char dZT[ROWS * ROWS * 2];
    float B[NBIAS];
    float red[4][HID];
    uint64_t bar;
    uint32_t tslot;
};

__global__ void __launch_bounds__(ROWS, 1) k_mlp_train(const float* __restrict__ Xn, const float* __restrict__ Tn, int n,
                                                      float inv_count, const unsigned char* __restrict__ wpack,
                                                      const float* __restrict__ bias, float* __restrict__ gpart,
                                                      float* __restrict__ lpart, int* status) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smraw);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int row = blockIdx.x * ROWS + t;
    const bool live = row < n;
    for (int q = t; q < T_END / 16; q += ROWS) reinterpret_cast<uint4*>(S.W)[q] = reinterpret_cast<const uint4*>(wpack)[q];
    for (int q = t; q < NBIAS; q += ROWS) S.B[q] = bias[q];
    for (int q = t; q < (int)sizeof(S.dZT) / 16; q += ROWS) reinterpret_cast<uint4*>(S.dZT)[q] = make_uint4(0, 0, 0, 0);
    float v[HID];
#pragma unroll
    for (int q = 0; q < HID; ++q) v[q] = 0.0f;
    if (live)
        for (int q = 0; q < NIN; ++q) v[q] = Xn[(int64_t)row * NIN + q];
    put_row(S.X0, KIN, t, v, KIN);
    put_col(S.X0T, t, v, KIN);
    if (warp == 0) tmem_alloc(&S.tslot, 512);
    if (t == 0) bar_init(&S.bar);
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = S.tslot;
    const uint32_t lb = (uint32_t)(warp * 32) << 16;
    uint32_t phase = 0;
    bool ok = true;
    auto sync_mma = [&]() {   // operands written -> visible to the tensor core
        fence_smem_async();
        fence_before();
        __syncthreads();
        fence_after();
    };
    auto wait_mma = [&]() {
        ok = bar_wait(&S.bar, phase) && ok;
        phase ^= 1;
        fence_after();
    };
    // ------------------------------------------------------------- forward
    const int Wf[4] = {T_W1F, T_W2F, T_W3F, T_W4F};
    for (int layer = 0; layer < 4; ++layer) {
        const int N = layer == 3 ? NOUTP : HID, K = layer == 0 ? KIN : HID;
        const unsigned char* A = layer == 0 ? S.X0 : S.H[layer - 1];
        if (t == 0) {
            for (int kk = 0; kk < K / 16; ++kk)
                mma(tm + 64 * layer, sdesc(A, K, kk), sdesc(S.W + Wf[layer], K, kk), idesc(ROWS, N), kk > 0);
            mma_commit(&S.bar);
        }
        wait_mma();
        if (layer < 3) {
            for (int c = 0; c < 4; ++c) tmem_ld16(tm + lb + 64 * layer + c * 16, v + c * 16);
            for (int q = 0; q < HID; ++q) v[q] = gelu(v[q] + S.B[layer * HID + q]);
            put_row(S.H[layer], HID, t, v, HID);
            put_col(S.HT[layer], t, v, HID);
            sync_mma();
        }
    }
    // ------------------------------------------------------------- loss
    float e[NOUTP];
    tmem_ld16(tm + lb + 192, e);
    float loss = 0.0f;
    for (int q = 0; q < NOUTP; ++q) {
        float d = 0.0f;
        if (live && q < NOUT) {
            d = e[q] + S.B[3 * HID + q] - Tn[(int64_t)row * NOUT + q];
            loss += d * d;
        }
        e[q] = 2.0f * d * inv_count;   // dL/dy
    }
    // ------------------------------------------------------------- backward
    // layer l (3..0): dZ known in `e` (l = 3) or computed from dX; then
    // dW_l = dZ^T H_{l-1} and (l > 0) dX_{l-1} = dZ W_l.
    const int Wb[4] = {0, T_W2B, T_W3B, T_W4B};
    float* g = gpart + (int64_t)blockIdx.x * NPAR;
    const int OW[4] = {OW1, OW2, OW3, OW4};
    for (int layer = 3; layer >= 0; --layer) {
        const int nout = layer == 3 ? NOUTP : HID;       // rows of dW (N of this layer)
        const int nin = layer == 0 ? KIN : HID;          // columns of dW (K of this layer)
        float* dz = (layer == 3) ? e : v;
        // bias gradient: column sums of dZ over the CTA's rows
        for (int q = 0; q < nout; ++q) {
            float s = dz[q];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) S.red[warp][q] = s;
        }
        put_row(S.dZ, nout, t, dz, nout);
        put_col(S.dZT, t, dz, nout);
        sync_mma();
        if (t < nout) {
            float s = S.red[0][t] + S.red[1][t] + S.red[2][t] + S.red[3][t];
            g[(layer == 0 ? OB1 : layer == 1 ? OB2 : layer == 2 ? OB3 : OB4) + t] = s;
        }
        if (t == 0) {
            const unsigned char* Hb = layer == 0 ? S.X0T : S.HT[layer - 1];
            for (int kk = 0; kk < ROWS / 16; ++kk)
                mma(tm + 256, sdesc(S.dZT, ROWS, kk), sdesc(Hb, ROWS, kk), idesc(ROWS, nin), kk > 0);
            if (layer > 0)
                for (int kk = 0; kk < nout / 16; ++kk)
                    mma(tm + 320, sdesc(S.dZ, nout, kk), sdesc(S.W + Wb[layer], nout, kk), idesc(ROWS, HID), kk > 0);
            mma_commit(&S.bar);
        }
        wait_mma();
        // dW rows: thread t < nout holds row t (output feature t)
        float w[HID];
        for (int c = 0; c < nin / 16; ++c) tmem_ld16(tm + lb + 256 + c * 16, w + c * 16);
        if (t < nout)
            for (int q = 0; q < nin; ++q) g[OW[layer] + t * nin + q] = w[q];
        if (layer > 0) {
            for (int c = 0; c < 4; ++c) tmem_ld16(tm + lb + 320 + c * 16, w + c * 16);
            float z[HID];
            for (int c = 0; c < 4; ++c) tmem_ld16(tm + lb + 64 * (layer - 1) + c * 16, z + c * 16);
            for (int q = 0; q < HID; ++q) v[q] = live ? w[q] * gelu_grad(z[q] + S.B[(layer - 1) * HID + q]) : 0.0f;
        }
        fence_before();
        __syncthreads();
        fence_after();
    }
    // CTA loss
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) S.red[warp][0] = loss;
    __syncthreads();
    if (t == 0) lpart[blockIdx.x] = S.red[0][0] + S.red[1][0] + S.red[2][0] + S.red[3][0];
    if (!ok && t == 0) atomicOr(status, 1);
    if (warp == 0) tmem_free(tm, 512);
}

// Sum of the per-CTA partials in a fixed order (deterministic).
__global__ void k_mlp_reduce(const float* __restrict__ gpart, const float* __restrict__ lpart, int nblk,
                             float* __restrict__ grad, float* __restrict__ loss) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < NPAR) {
        float s = 0.0f;
        for (int b = 0; b < nblk; ++b) s += gpart[(int64_t)b * NPAR + p];
        grad[p] = s;
    }
    if (p == 0) {
        float s = 0.0f;
        for (int b = 0; b < nblk; ++b) s += lpart[b];
        *loss = s;
    }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; padded entries have
// zero gradient and stay zero.
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v2,
                           const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPAR) return;
    float gr = grad[p];
    float mm = b1 * m[p] + (1.0f - b1) * gr;
    float vv = b2 * v2[p] + (1.0f - b2) * gr * gr;
    m[p] = mm;
    v2[p] = vv;
    w[p] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
}

// FP32 master parameters -> BF16 operand tiles (forward and transposed) and
// the FP32 bias vector.
__global__ void k_mlp_pack(const float* __restrict__ w, unsigned char* __restrict__ wpack, float* __restrict__ bias) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    auto put = [&](int tile, int r, int k, int K, float x) {
        *reinterpret_cast<__nv_bfloat16*>(wpack + tile + kmaj(r, k, K)) = __float2bfloat16_rn(x);
    };
    if (p < HID * KIN) { int r = p / KIN, k = p % KIN; put(T_W1F, r, k, KIN, w[OW1 + p]); }
    if (p < HID * HID) {
        int r = p / HID, k = p % HID;
        put(T_W2F, r, k, HID, w[OW2 + p]);
        put(T_W3F, r, k, HID, w[OW3 + p]);
        put(T_W2B, k, r, HID, w[OW2 + p]);
        put(T_W3B, k, r, HID, w[OW3 + p]);
    }
    if (p < NOUTP * HID) {
        int r = p / HID, k = p % HID;
        put(T_W4F, r, k, HID, w[OW4 + p]);
        put(T_W4B, k, r, NOUTP, w[OW4 + p]);
    }
    if (p < NBIAS) bias[p] = w[OB1 + p];
}

}  // namespace mlp
}  // namespace erfb

using namespace erfb::mlp;

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
namespace {
int mlp_fail(cudaError_t e) { return e == cudaSuccess ? ERF_B200_OK : (e == cudaErrorMemoryAllocation ? ERF_B200_ENOMEM : ERF_B200_ECUDA); }
template <class T>
int mlp_alloc(T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return mlp_fail(e);
    cudaMemset(q, 0, n * sizeof(T));
    *p = (T*)q;
    return ERF_B200_OK;
}
int ensure_blocks(erf_b200_mlp* M, int nblk) {
    if (nblk <= M->max_blocks) return ERF_B200_OK;
    cudaFree(M->gpart); cudaFree(M->lpart);
    M->gpart = nullptr; M->lpart = nullptr;
    int rc = mlp_alloc(&M->gpart, (size_t)nblk * NPAR);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->lpart, (size_t)nblk);
    M->max_blocks = rc == ERF_B200_OK ? nblk : 0;
    return rc;
}

// Failure-detection self-test: an mbarrier that expects one arrival which
// never comes, waited on with the bounded poll of the tensor-core kernels;
// the wait must end by its limit and report, never hang.
__global__ void k_selftest_wait(int limit, int* timed_out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) bar_init(&bar);
    __syncthreads();
    const bool done = bar_wait(&bar, 0u, limit);
    if (threadIdx.x == 0) *timed_out = done ? 0 : 1;
}
}  // namespace

extern "C" {

int erf_b200_mlp_num_params(void) { return NPAR; }

int erf_b200_mlp_create(erf_b200_mlp** out, void* stream) {
    if (!out) return ERF_B200_EINVAL;
    *out = nullptr;
    erf_b200_mlp* M = new (std::nothrow) erf_b200_mlp();
    if (!M) return ERF_B200_ENOMEM;
    M->stream = (cudaStream_t)stream;
    int rc = ERF_B200_OK;
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->w, NPAR);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->m, NPAR);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->v, NPAR);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->grad, NPAR);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->bias, NBIAS);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->norm, 2 * NIN + 2 * NOUT);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->loss, 1);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->wpack, T_END);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->status, 1);
    if (rc == ERF_B200_OK) rc = mlp_alloc(&M->env, 2 * NIN);
    if (rc == ERF_B200_OK && cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)sizeof(TrainSmem)) != cudaSuccess)
        rc = ERF_B200_ECUDA;
    for (int q = 0; q < NIN; ++q) { M->lo[q] = -3.0e38f; M->hi[q] = 3.0e38f; }
    if (rc != ERF_B200_OK) { erf_b200_mlp_destroy(M); return rc; }
    *out = M;
    return ERF_B200_OK;
}

int erf_b200_mlp_destroy(erf_b200_mlp* M) {
    if (!M) return ERF_B200_EINVAL;
    float* fs[] = {M->w, M->m, M->v, M->grad, M->bias, M->norm, M->gpart, M->lpart, M->loss};
    for (float* f : fs) cudaFree(f);
    cudaFree(M->wpack);
    cudaFree(M->status);
    cudaFree(M->env);
    delete M;
    return ERF_B200_OK;
}

int erf_b200_mlp_set_params(erf_b200_mlp* M, const float* host_params) {
    if (!M || !host_params) return ERF_B200_EINVAL;
    int rc = mlp_fail(cudaMemcpyAsync(M->w, host_params, NPAR * sizeof(float), cudaMemcpyHostToDevice, M->stream));
    if (rc) return rc;
    cudaMemsetAsync(M->m, 0, NPAR * sizeof(float), M->stream);
    cudaMemsetAsync(M->v, 0, NPAR * sizeof(float), M->stream);
    M->step = 0;
    k_mlp_pack<<<(HID * HID + 255) / 256, 256, 0, M->stream>>>(M->w, M->wpack, M->bias);
    return mlp_fail(cudaStreamSynchronize(M->stream));
}

int erf_b200_mlp_get_params(erf_b200_mlp* M, float* host_params) {
    if (!M || !host_params) return ERF_B200_EINVAL;
    int rc = mlp_fail(cudaMemcpyAsync(host_params, M->w, NPAR * sizeof(float), cudaMemcpyDeviceToHost, M->stream));
    if (rc) return rc;
    return mlp_fail(cudaStreamSynchronize(M->stream));
}

int erf_b200_mlp_set_normalization(erf_b200_mlp* M, const float* in_mean, const float* in_std, const float* out_mean,
                                   const float* out_std, const float* in_lo, const float* in_hi) {
    if (!M || !in_mean || !in_std || !out_mean || !out_std) return ERF_B200_EINVAL;
    float h[2 * NIN + 2 * NOUT];
    for (int q = 0; q < NIN; ++q) {
        if (!(in_std[q] > 0.0f)) return ERF_B200_EINVAL;
        h[q] = in_mean[q]; h[NIN + q] = in_std[q];
    }
    for (int q = 0; q < NOUT; ++q) { h[2 * NIN + q] = out_mean[q]; h[2 * NIN + NOUT + q] = out_std[q]; }
    for (int q = 0; q < NIN; ++q) {
        M->lo[q] = in_lo ? in_lo[q] : -3.0e38f;
        M->hi[q] = in_hi ? in_hi[q] : 3.0e38f;
    }
    float env[2 * NIN];
    for (int q = 0; q < NIN; ++q) { env[q] = M->lo[q]; env[NIN + q] = M->hi[q]; }
    int rc = mlp_fail(cudaMemcpyAsync(M->norm, h, sizeof(h), cudaMemcpyHostToDevice, M->stream));
    if (rc == ERF_B200_OK) rc = mlp_fail(cudaMemcpyAsync(M->env, env, sizeof(env), cudaMemcpyHostToDevice, M->stream));
    if (rc) return rc;
    return mlp_fail(cudaStreamSynchronize(M->stream));
}

// Loss and gradient of one batch (normalised inputs/targets on the device);
// host_grad receives NPAR floats (padded layout), host_loss the loss.
int erf_b200_mlp_gradient(erf_b200_mlp* M, const float* xn, const float* tn, int n, float* host_grad, float* host_loss) {
    if (!M || !xn || !tn || n <= 0) return ERF_B200_EINVAL;
    int nblk = (n + ROWS - 1) / ROWS;
    int rc = ensure_blocks(M, nblk);
    if (rc) return rc;
    k_mlp_train<<<nblk, ROWS, sizeof(TrainSmem), M->stream>>>(xn, tn, n, 1.0f / (float)(n * NOUT), M->wpack, M->bias,
                                                              M->gpart, M->lpart, M->status);
    k_mlp_reduce<<<(NPAR + 255) / 256, 256, 0, M->stream>>>(M->gpart, M->lpart, nblk, M->grad, M->loss);
    if ((rc = mlp_fail(cudaGetLastError()))) return rc;
    if (host_grad) cudaMemcpyAsync(host_grad, M->grad, NPAR * sizeof(float), cudaMemcpyDeviceToHost, M->stream);
    if (host_loss) cudaMemcpyAsync(host_loss, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->stream);
    rc = mlp_fail(cudaStreamSynchronize(M->stream));
    if (rc) return rc;
    if (host_loss) *host_loss /= (float)(n * NOUT);
    int st = 0;
    cudaMemcpy(&st, M->status, sizeof(int), cudaMemcpyDeviceToHost);
    return st ? ERF_B200_ETIMEOUT : ERF_B200_OK;
}

// `iters` Adam steps over consecutive minibatches of `batch` rows of the
// device arrays xn [n][13], tn [n][9] (wrapping around); host_loss (optional)
// receives the mean loss of the last minibatch.
int erf_b200_mlp_train(erf_b200_mlp* M, const float* xn, const float* tn, int n, int batch, int iters, float lr,
                       float* host_loss) {
    if (!M || !xn || !tn || n <= 0 || batch <= 0 || batch > n || iters <= 0) return ERF_B200_EINVAL;
    int nblk = (batch + ROWS - 1) / ROWS;
    int rc = ensure_blocks(M, nblk);
    if (rc) return rc;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    long off = 0;
    for (int it = 0; it < iters; ++it) {
        if (off + batch > n) off = 0;
        k_mlp_train<<<nblk, ROWS, sizeof(TrainSmem), M->stream>>>(xn + off * NIN, tn + off * NOUT, batch,
                                                                  1.0f / (float)(batch * NOUT), M->wpack, M->bias,
                                                                  M->gpart, M->lpart, M->status);
        k_mlp_reduce<<<(NPAR + 255) / 256, 256, 0, M->stream>>>(M->gpart, M->lpart, nblk, M->grad, M->loss);
        M->step += 1;
        float c1 = 1.0f / (1.0f - powf(b1, (float)M->step)), c2 = 1.0f / (1.0f - powf(b2, (float)M->step));
        k_mlp_adam<<<(NPAR + 255) / 256, 256, 0, M->stream>>>(M->w, M->m, M->v, M->grad, lr, b1, b2, eps, c1, c2);
        k_mlp_pack<<<(HID * HID + 255) / 256, 256, 0, M->stream>>>(M->w, M->wpack, M->bias);
        off += batch;
    }
    if ((rc = mlp_fail(cudaGetLastError()))) return rc;
    if (host_loss) cudaMemcpyAsync(host_loss, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->stream);
    rc = mlp_fail(cudaStreamSynchronize(M->stream));
    if (rc) return rc;
    if (host_loss) *host_loss /= (float)(batch * NOUT);
    int st = 0;
    cudaMemcpy(&st, M->status, sizeof(int), cudaMemcpyDeviceToHost);
    return st ? ERF_B200_ETIMEOUT : ERF_B200_OK;
}

// Y [n][9] (raw units) = MLP(X [n][13] raw units), device arrays.
int erf_b200_mlp_infer(erf_b200_mlp* M, const float* x, int n, float* y) {
    if (!M || !x || !y || n <= 0) return ERF_B200_EINVAL;
    k_mlp_infer<<<(n + ROWS - 1) / ROWS, ROWS, 0, M->stream>>>(x, n, M->wpack, M->bias, M->norm, y, M->status);
    int rc = mlp_fail(cudaGetLastError());
    if (rc) return rc;
    rc = mlp_fail(cudaStreamSynchronize(M->stream));
    if (rc) return rc;
    int st = 0;
    cudaMemcpy(&st, M->status, sizeof(int), cudaMemcpyDeviceToHost);
    return st ? ERF_B200_ETIMEOUT : ERF_B200_OK;
}

int erf_b200_selftest_bounded_wait(int limit, int* timed_out) {
    if (limit < 1 || !timed_out) return ERF_B200_EINVAL;
    int* d = nullptr;
    if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return ERF_B200_ENOMEM;
    cudaMemset(d, 0xff, sizeof(int));
    k_selftest_wait<<<1, 32>>>(limit, d);
    int h = -1;
    cudaError_t e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess || h < 0) return ERF_B200_ECUDA;
    *timed_out = h;
    return ERF_B200_OK;
}

}  // extern "C"
