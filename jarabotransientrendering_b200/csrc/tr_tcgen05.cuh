// tr_tcgen05.cuh - 5th-generation tensor-core building blocks of the proposal network: PTX
// wrappers (mbarrier, tcgen05 alloc/mma/commit/ld, fences), the UMMA shared-memory and
// instruction descriptors for BF16 128x64x16 tiles in the canonical K-major layout, one bounded
// 64x64 layer MMA and the shared-memory layout of a CTA that keeps all four weight tiles
// resident.  Used by the training kernels (tr_guide.cu) and by the renderer's fused
// guided-sampling kernel (tr_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

#include "tr_guide.cuh"

namespace trg {

// ---------------------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// UMMA shared-memory descriptor, K-major, no swizzle: core matrices of 8 rows x 16 bytes,
// LBO = distance between the two K-halves of one K=16 step (128 B), SBO = distance between
// 8-row groups (1024 B for a 64-wide K tile); bits 46-47 = 1 (sm100 descriptor version).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    const uint64_t start = (addr >> 4) & 0x3FFFu;
    const uint64_t lbo = 128u >> 4;
    const uint64_t sbo = 1024u >> 4;
    return start | (lbo << 16) | (sbo << 32) | (1ull << 46);
}
// instruction descriptor: D = F32, A = B = BF16, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

// byte offset of element (row, k) of a [rows][64] bf16 tile in the canonical layout
__host__ __device__ __forceinline__ uint32_t canon_off(uint32_t row, uint32_t k) {
    return (row >> 3) * 1024u + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// mbarrier polls before a wait for the CTA's own MMAs counts as timed out: the default wait
// limit of the kernels' completion waits (host-settable per guide) and the fixed bound of the
// drain wait that always lets in-flight MMAs land before tensor memory is freed
constexpr uint32_t kSpin = kWaitPolls;

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
// bf16x2 {relu(a) low, relu(b) high} rounded to nearest in one conversion (cvt.rn.relu.bf16x2.f32):
// the same bits as pack2(fmaxf(a, 0), fmaxf(b, 0)) for every non-NaN input
__device__ __forceinline__ uint32_t pack2_relu(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
}
__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }

// Issues the four K=16 MMAs of one layer and waits for them, polling the mbarrier at most `spin`
// times (0: no wait at all - the wait times out at once); returns false on timeout.  Called by
// all threads; thread 0 issues and waits, the others meet it at the barrier.
__device__ __forceinline__ bool layer_mma(uint32_t taddr, uint32_t a_addr, uint32_t b_addr, uint64_t* bar,
                                          uint32_t& phase, volatile int* s_ok, uint32_t spin) {
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        tc_fence_after();
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k)
            umma_bf16(taddr, smem_desc(a_addr + k * 256u), smem_desc(b_addr + k * 256u), kIdesc, k > 0 ? 1u : 0u);
        umma_commit(bar);
        bool done = false;
        for (uint32_t it = 0; it < spin && !done; ++it) done = mbar_try_wait(bar, phase);
        *s_ok = done ? 1 : 0;
    }
    __syncthreads();
    phase ^= 1u;
    tc_fence_after();
    return *s_ok != 0;
}

__device__ __forceinline__ void drain_and_free(uint32_t taddr, uint64_t* bar, uint32_t phase, bool ok) {
    if (!ok && threadIdx.x == 0) {               // let in-flight MMAs land before freeing TMEM
        uint32_t it = 0;
        while (!mbar_try_wait(bar, phase ^ 1u) && ++it < kSpin) {}
    }
    tc_fence_before();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) tmem_dealloc(taddr, 64);
}

// shared memory: 4 weight tiles (32 KB) | A tile (16 KB) | bias (1 KB) | mbarrier | tmem slot | flag
constexpr uint32_t kSmemW = 0, kSmemA = 32768, kSmemBias = 49152, kSmemBar = 50176, kSmemSlot = 50184,
                   kSmemOk = 50188, kSmemBytes = 50192;

// Two-tile variant (the renderer's fused guided-sampling kernel): 4 weight tiles (32 KB) | A
// tiles of two 128-row tiles (16 KB each) | bias (1 KB) | two mbarriers | tmem slot | flag.  The
// two tiles' MMA chains are interleaved: both layers' MMAs are issued back to back, so one
// tile's MMAs run while the CTA turns the other tile's accumulators into the next A operand.
constexpr uint32_t kG2W = 0, kG2A0 = 32768, kG2A1 = 49152, kG2Bias = 65536, kG2Bar = 66560, kG2Slot = 66576,
                   kG2Ok = 66580, kG2Bytes = 66592;

// Thread 0 polls `bar` for completion of `phase` at most `spin` times; the result is made
// CTA-uniform through shared memory and a barrier (every thread must call this).
__device__ __forceinline__ bool wait_uniform(uint64_t* bar, uint32_t phase, volatile int* s_ok, uint32_t spin) {
    if (threadIdx.x == 0) {
        bool done = false;
        for (uint32_t it = 0; it < spin && !done; ++it) done = mbar_try_wait(bar, phase);
        *s_ok = done ? 1 : 0;
    }
    __syncthreads();
    const bool ok = *s_ok != 0;
    tc_fence_after();
    return ok;
}

// Issues one layer's four K=16 MMAs (A tile x weight tile -> 128 x 64 FP32 accumulator in tensor
// memory) and commits them to `bar`.  Thread 0 only; the caller fences and synchronises first.
__device__ __forceinline__ void issue_layer(uint32_t taddr, uint32_t a_addr, uint32_t b_addr, uint64_t* bar) {
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k)
        umma_bf16(taddr, smem_desc(a_addr + k * 256u), smem_desc(b_addr + k * 256u), kIdesc, k > 0 ? 1u : 0u);
    umma_commit(bar);
}

__device__ __forceinline__ void stage_weights(uint8_t* smem, const uint4* w, const float* bias) {
    uint4* sw = reinterpret_cast<uint4*>(smem + kSmemW);
    for (uint32_t i = threadIdx.x; i < 2048u; i += blockDim.x) sw[i] = __ldg(&w[i]);
    float* sb = reinterpret_cast<float*>(smem + kSmemBias);
    for (uint32_t i = threadIdx.x; i < 256u; i += blockDim.x) sb[i] = __ldg(&bias[i]);
}

__device__ __forceinline__ void store_row_a(uint8_t* sA, uint32_t row, const uint4* v) {
#pragma unroll
    for (uint32_t c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(sA + (row >> 3) * 1024u + c * 128u + (row & 7u) * 16u) = v[c];
}

}  // namespace trg
