// tcgen05.cuh -- helpers for the 5th-generation tensor cores (sm_100a):
// K-major no-swizzle operand tiles in shared memory, shared-memory matrix and
// instruction descriptors, tcgen05.mma / commit / ld, tensor-memory
// allocation, mbarrier waits with an iteration limit, and the proxy fences
// between thread-written shared memory and the tensor core.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace erfb {
namespace tc {

constexpr int ROWS = 128;   // M of every product: one CTA row per thread

// Byte offset of element (r, k) of a K-major tile with K columns.
__host__ __device__ constexpr uint32_t kmaj(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// tcgen05 instruction descriptor: D = F32, A = B = BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a K-major tile (K columns), starting at
// K-chunk pair `kk` (16 elements per MMA step).
__device__ __forceinline__ uint64_t sdesc(const void* tile, int K, int kk) {
    uint32_t a = saddr(tile) + (uint32_t)kk * 256u;
    uint64_t d = (uint64_t)((a >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;                        // leading byte offset (K)
    d |= (uint64_t)(((uint32_t)(K >> 3) * 128u >> 4) & 0x3FFFu) << 32;   // stride byte offset (M/N)
    d |= (uint64_t)1 << 46;                                              // descriptor version
    return d;
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(id), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}
__device__ __forceinline__ void bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait on the mbarrier phase; false if the limit (polls) ran out.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, int limit = 1 << 22) {
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(saddr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Row r of a K-major tile with K columns from n FP32 values (columns >= n are 0).
__device__ __forceinline__ void put_row(unsigned char* tile, int K, int r, const float* v, int n) {
#pragma unroll
    for (int c = 0; c < K / 8; ++c) {
        __align__(16) __nv_bfloat162 h[4];   // pairs: one round-to-nearest conversion per two values
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = c * 8 + 2 * q;
            h[q] = __floats2bfloat162_rn(k < n ? v[k] : 0.0f, k + 1 < n ? v[k + 1] : 0.0f);
        }
        *reinterpret_cast<uint4*>(tile + kmaj(r, c * 8, K)) = *reinterpret_cast<const uint4*>(h);
    }
}
// Column r (as K index) of a K-major tile with ROWS columns: element (f, r)
// for f < n.
__device__ __forceinline__ void put_col(unsigned char* tile, int r, const float* v, int n) {
    for (int f = 0; f < n; ++f)
        *reinterpret_cast<__nv_bfloat16*>(tile + kmaj(f, r, ROWS)) = __float2bfloat16_rn(v[f]);
}


}  // namespace tc
}  // namespace erfb
