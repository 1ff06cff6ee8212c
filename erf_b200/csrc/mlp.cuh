// mlp.cuh -- the learned subgrid closure network (13 -> 64 -> 64 -> 64 -> 9,
// GELU in tanh form, BF16 operands, FP32 accumulation on tcgen05): parameter and
// operand-tile layouts, the CTA forward pass shared by inference and the
// dycore's closure kernel, and the network object behind the C-ABI handle.
#pragma once
#include "tcgen05.cuh"
#include "../../include/erf_b200.h"

namespace erfb {
namespace mlp {

using namespace erfb::tc;

constexpr int NIN = 13, KIN = 16, HID = 64, NOUT = 9, NOUTP = 16;

// Master parameter vector (FP32, padded layout):
//   W1[64][16] W2[64][64] W3[64][64] W4[16][64] b1[64] b2[64] b3[64] b4[16]
constexpr int OW1 = 0, OW2 = OW1 + HID * KIN, OW3 = OW2 + HID * HID, OW4 = OW3 + HID * HID;
constexpr int OB1 = OW4 + NOUTP * HID, OB2 = OB1 + HID, OB3 = OB2 + HID, OB4 = OB3 + HID;
constexpr int NPAR = OB4 + NOUTP;  // 10448
constexpr int NBIAS = 3 * HID + NOUTP;

// Packed BF16 operand tiles (bytes): forward W (N = out, K = in) and
// backward W^T (N = in, K = out).
constexpr int T_W1F = 0, T_W2F = T_W1F + HID * KIN * 2, T_W3F = T_W2F + HID * HID * 2, T_W4F = T_W3F + HID * HID * 2;
constexpr int T_W4B = T_W4F + NOUTP * HID * 2, T_W3B = T_W4B + HID * NOUTP * 2, T_W2B = T_W3B + HID * HID * 2;
constexpr int T_FWD_END = T_W4B, T_END = T_W2B + HID * HID * 2;  // 20480, 38912

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
// (Hendrycks & Gimpel 2016), with tanh from the hardware approximation
// instruction; its derivative for the backward pass.
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float GELU_C = 0.7978845608028654f, GELU_A = 0.044715f;
// The same function in nested form: sqrt(2/pi) (z + a z^3) = z (C + C a z^2)
// and 0.5 z (1 + t) = h + h t with h = z / 2, so a value costs five
// multiply / fused multiply-add operations and one tanh.
__device__ __forceinline__ float gelu(float z) {
    const float u = z * z;
    const float t = tanh_fast(z * fmaf(GELU_C * GELU_A, u, GELU_C));
    const float h = 0.5f * z;
    return fmaf(h, t, h);
}
// Bias plus GELU of two values with the paired FP32 instructions of sm_100
// (one instruction per operation for both lanes, each lane rounded as the
// scalar operation above, so the values are the same as gelu(z + b)).
__device__ __forceinline__ float2 bias_gelu2(float2 z, float2 b) {
    const float2 CA = make_float2(GELU_C * GELU_A, GELU_C * GELU_A), C = make_float2(GELU_C, GELU_C);
    const float2 half = make_float2(0.5f, 0.5f);
    z = __fadd2_rn(z, b);
    const float2 u = __fmul2_rn(z, z);
    const float2 a = __fmul2_rn(z, __ffma2_rn(CA, u, C));
    const float2 t = make_float2(tanh_fast(a.x), tanh_fast(a.y));
    const float2 h = __fmul2_rn(half, z);
    return __ffma2_rn(h, t, h);
}
__device__ __forceinline__ float gelu_grad(float z) {
    float t = tanh_fast(GELU_C * (z + GELU_A * z * z * z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * GELU_C * (1.0f + 3.0f * GELU_A * z * z);
}


// Forward pass of the CTA's 128 rows (thread t = row t).  xn: this row's 13
// normalised inputs; returns y[16] = last-layer output + bias (padded).
// sW holds the forward weight tiles, sB the biases; TMEM columns [tm, tm+64)
// are reused by every layer.  Returns false if an MMA wait ran out.
__device__ __forceinline__ bool forward_cta(const unsigned char* sW, unsigned char* sX, unsigned char* sH,
                                            const float* sB, uint64_t* bar, uint32_t tm, uint32_t& phase,
                                            const float* xn, float* y) {
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    put_row(sX, KIN, t, xn, NIN);
    fence_smem_async();
    fence_before();
    __syncthreads();
    fence_after();
    bool ok = true;
    float z[HID];
#pragma unroll
    for (int layer = 0; layer < 4; ++layer) {
        const int N = layer == 3 ? NOUTP : HID;
        const int K = layer == 0 ? KIN : HID;
        const unsigned char* A = layer == 0 ? sX : sH;
        const unsigned char* B = sW + (layer == 0 ? T_W1F : layer == 1 ? T_W2F : layer == 2 ? T_W3F : T_W4F);
        if (t == 0) {
            for (int kk = 0; kk < K / 16; ++kk) mma(tm, sdesc(A, K, kk), sdesc(B, K, kk), idesc(ROWS, N), kk > 0);
            mma_commit(bar);
        }
        ok = bar_wait(bar, phase) && ok;
        phase ^= 1;
        fence_after();
#pragma unroll
        for (int c = 0; c < N / 16; ++c) tmem_ld16(tm + lane_base + c * 16, z + c * 16);
        const float* b = sB + layer * HID;
        if (layer < 3) {
#pragma unroll
            for (int q = 0; q < HID; q += 2) {
                const float2 r = bias_gelu2(make_float2(z[q], z[q + 1]), make_float2(b[q], b[q + 1]));
                z[q] = r.x;
                z[q + 1] = r.y;
            }
            put_row(sH, HID, t, z, HID);
        } else {
            for (int q = 0; q < NOUTP; ++q) y[q] = z[q] + b[q];
        }
        fence_smem_async();
        fence_before();
        __syncthreads();
        fence_after();
    }
    return ok;
}

}  // namespace mlp
}  // namespace erfb

// The network object behind the C-ABI handle.
struct erf_b200_mlp {
    cudaStream_t stream = nullptr;
    float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *bias = nullptr, *norm = nullptr;
    float *gpart = nullptr, *lpart = nullptr, *loss = nullptr;
    unsigned char* wpack = nullptr;
    int* status = nullptr;
    int max_blocks = 0;
    long step = 0;
    float lo[erfb::mlp::NIN], hi[erfb::mlp::NIN];   // training envelope of the raw inputs
    float* env = nullptr;        // the envelope on the device (lo[13], hi[13])
};

