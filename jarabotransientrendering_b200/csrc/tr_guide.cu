// tr_guide.cu - kernels of the learned directional proposal (no reference counterpart).
//
// The network is 64 -> 64 -> 64 -> 64 -> 40 (ReLU on the three hidden layers), BF16 operands,
// FP32 accumulation.  Forward and the hidden-layer backward run on the 5th-generation tensor
// cores: one CTA of 128 threads owns a 128-row tile; all four weight tiles stay resident in
// shared memory in the UMMA canonical K-major layout (8x16-byte core matrices, no swizzle);
// one elected thread issues tcgen05.mma (M=128, N=64, K=16, four per layer) into a 128x64 FP32
// accumulator in tensor memory; tcgen05.commit arrives on an mbarrier; every thread then reads
// its row back with tcgen05.ld, adds the bias, applies ReLU and writes the BF16 row as the next
// layer's A operand.  The weight gradients (a reduction over the batch, 2 GFLOP per 65,536-row
// step) run on the tensor cores too (k_dw_tc).  Every wait on an mbarrier is bounded (the
// guide's wait limit); on expiry the kernel records an error, waits (bounded) for its MMAs,
// frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>

#include "tr_guide.cuh"
#include "tr_guide_math.cuh"
#include "tr_tcgen05.cuh"

namespace trg {


// ---------------------------------------------------------------------------------------------
// forward: out[m][0..40) = L4(relu(L3(relu(L2(relu(L1(x)))))));  act (optional) = H1, H2, H3
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) k_mlp_fwd(GuideDev g, const uint4* __restrict__ x, uint32_t m,
                                                    const uint32_t* __restrict__ m_dev, float* __restrict__ out,
                                                    uint4* __restrict__ act, int* err) {
    if (m_dev) m = min(m, *m_dev);      // row count produced on the device (guided rendering)
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem + kSmemA;
    const float* sB = reinterpret_cast<const float*>(smem + kSmemBias);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSmemBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kSmemSlot);
    volatile int* s_ok = reinterpret_cast<volatile int*>(smem + kSmemOk);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    stage_weights(smem, g.w_fwd, g.bias);
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    if (warp == 0) { tmem_alloc(slot, 64); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *slot;
    const uint32_t lane_addr = taddr + ((32u * warp) << 16);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile * kTile < m && ok; tile += gridDim.x) {
        const uint32_t row = tile * kTile + tid;
        uint4 v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = row < m ? __ldg(&x[(size_t)row * 8 + c]) : make_uint4(0, 0, 0, 0);
        store_row_a(sA, tid, v);
        for (uint32_t l = 0; l < 4 && ok; ++l) {
            ok = layer_mma(taddr, smem_u32(sA), smem_u32(smem + kSmemW + l * 8192u), bar, phase, s_ok, g.spin);
            if (!ok) break;
            float acc[64];
#pragma unroll
            for (int j = 0; j < 4; ++j) tmem_ld16(lane_addr + 16u * j, acc + 16 * j);
            tmem_wait_ld();
            if (l < 3) {
                uint4 h[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    float t[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) t[e] = acc[8 * c + e] + sB[l * 64 + 8 * c + e];
                    h[c] = make_uint4(pack2_relu(t[0], t[1]), pack2_relu(t[2], t[3]), pack2_relu(t[4], t[5]),
                                      pack2_relu(t[6], t[7]));
                }
                store_row_a(sA, tid, h);
                if (act && row < m) {
#pragma unroll
                    for (int c = 0; c < 8; ++c) act[((size_t)l * m + row) * 8 + c] = h[c];
                }
            } else if (row < m) {
#pragma unroll
                for (int j = 0; j < kOut; ++j) out[(size_t)row * kOut + j] = acc[j] + sB[3 * 64 + j];
            }
        }
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    drain_and_free(taddr, bar, phase, ok);
}

// ---------------------------------------------------------------------------------------------
// backward through the hidden layers: given dY = dL/d(out) (bf16, cols >= 40 zero) and the
// stored activations, dh[2] = dH3 = (dY W4^T) * 1[H3>0], dh[1] = dH2, dh[0] = dH1 (BF16, the
// weight-gradient kernel's B operands).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) k_mlp_bwd(GuideDev g, const uint4* __restrict__ dy,
                                                    const uint4* __restrict__ act, uint32_t m,
                                                    uint4* __restrict__ dh, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA = smem + kSmemA;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSmemBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kSmemSlot);
    volatile int* s_ok = reinterpret_cast<volatile int*>(smem + kSmemOk);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    stage_weights(smem, g.w_bwd, g.bias);
    if (tid == 0) { mbar_init(bar, 1); fence_mbar_init(); }
    if (warp == 0) { tmem_alloc(slot, 64); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *slot;
    const uint32_t lane_addr = taddr + ((32u * warp) << 16);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile * kTile < m && ok; tile += gridDim.x) {
        const uint32_t row = tile * kTile + tid;
        uint4 v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = row < m ? __ldg(&dy[(size_t)row * 8 + c]) : make_uint4(0, 0, 0, 0);
        store_row_a(sA, tid, v);
        // layer index of the weights used: 3 (W4), 2 (W3), 1 (W2); activation masks H3, H2, H1
        for (int l = 3; l >= 1 && ok; --l) {
            ok = layer_mma(taddr, smem_u32(sA), smem_u32(smem + kSmemW + (uint32_t)l * 8192u), bar, phase, s_ok, g.spin);
            if (!ok) break;
            float acc[64];
#pragma unroll
            for (int j = 0; j < 4; ++j) tmem_ld16(lane_addr + 16u * j, acc + 16 * j);
            tmem_wait_ld();
            uint4 h[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint4 a = row < m ? __ldg(&act[((size_t)(l - 1) * m + row) * 8 + c]) : make_uint4(0, 0, 0, 0);
                const uint32_t aw[4] = {a.x, a.y, a.z, a.w};
                float t[8];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    t[2 * e] = bf_lo(aw[e]) > 0.0f ? acc[8 * c + 2 * e] : 0.0f;
                    t[2 * e + 1] = bf_hi(aw[e]) > 0.0f ? acc[8 * c + 2 * e + 1] : 0.0f;
                }
                h[c] = make_uint4(pack2(t[0], t[1]), pack2(t[2], t[3]), pack2(t[4], t[5]), pack2(t[6], t[7]));
                if (row < m) dh[((size_t)(l - 1) * m + row) * 8 + c] = h[c];
            }
            store_row_a(sA, tid, h);
        }
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    drain_and_free(taddr, bar, phase, ok);
}

int resident_grid(int device, const void* kernel, int threads, size_t dyn_smem, int tmem_cols) {
    int sms = 1, smem_sm = 0, regs_sm = 0, warps_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device);
    cudaDeviceGetAttribute(&warps_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device);
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return sms > 0 ? sms : 1;
    const int per_cta_smem = (int)dyn_smem + (int)fa.sharedSizeBytes + 1024;     // 1 KB reserved per CTA
    const int regs = fa.numRegs > 0 ? ((fa.numRegs + 7) / 8) * 8 : 1;
    int per_sm = std::min(smem_sm / per_cta_smem, regs_sm / (regs * threads));
    per_sm = std::min(per_sm, warps_sm / threads);
    per_sm = std::min(per_sm, 512 / tmem_cols);                                   // TMEM columns each
    if (per_sm < 1) per_sm = 1;
    return (sms > 0 ? sms : 1) * per_sm;
}

int mlp_grid(int device) {
    static int grid = 0;
    if (!grid) grid = resident_grid(device, reinterpret_cast<const void*>(k_mlp_fwd), 128, kSmemBytes);
    return grid;
}

static int mlp_bwd_grid(int device) {
    static int grid = 0;
    if (!grid) grid = resident_grid(device, reinterpret_cast<const void*>(k_mlp_bwd), 128, kSmemBytes);
    return grid;
}

cudaError_t mlp_forward(const GuideDev& g, const uint4* x, uint32_t m, float* out, uint4* act, int* err,
                        cudaStream_t s, const uint32_t* m_dev) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_mlp_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        attr = true;
    }
    if (m == 0) return cudaSuccess;
    int dev = 0;
    cudaGetDevice(&dev);
    const uint32_t tiles = (m + kTile - 1) / kTile;
    const uint32_t grid = tiles < (uint32_t)mlp_grid(dev) ? tiles : (uint32_t)mlp_grid(dev);
    k_mlp_fwd<<<grid, 128, kSmemBytes, s>>>(g, x, m, m_dev, out, act, err);
    return cudaGetLastError();
}

cudaError_t mlp_backward(const GuideDev& g, const uint4* dy, const uint4* act, uint32_t m, uint4* dh, int* err,
                         cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_mlp_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
        attr = true;
    }
    if (m == 0) return cudaSuccess;
    int dev = 0;
    cudaGetDevice(&dev);
    const uint32_t tiles = (m + kTile - 1) / kTile;
    const uint32_t grid = tiles < (uint32_t)mlp_bwd_grid(dev) ? tiles : (uint32_t)mlp_bwd_grid(dev);
    k_mlp_bwd<<<grid, 128, kSmemBytes, s>>>(g, dy, act, m, dh, err);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// parameters: master FP32 [4][64 in][64 out] weights + [4][64] biases; packed BF16 tiles
// ---------------------------------------------------------------------------------------------
__global__ void k_pack_weights(const float* __restrict__ params, uint8_t* __restrict__ w_fwd, uint8_t* __restrict__ w_bwd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;          // one weight element
    if (i >= 4u * 4096u) return;
    const uint32_t l = i >> 12, in = (i >> 6) & 63u, o = i & 63u;
    const __nv_bfloat16 v = __float2bfloat16_rn(params[i]);
    // forward B tile: rows = output, K = input;  backward B tile: rows = input, K = output
    *reinterpret_cast<__nv_bfloat16*>(w_fwd + l * 8192u + canon_off(o, in)) = v;
    *reinterpret_cast<__nv_bfloat16*>(w_bwd + l * 8192u + canon_off(in, o)) = v;
}

// training loss -(w/W) log q(dir) and its gradient w.r.t. the 40 raw outputs; dy bf16
// [m][64], columns >= 40 zero.  wsum = sum of weights over the batch.
__global__ void k_mix_grad(const float* __restrict__ out, const float* __restrict__ dirs, const float* __restrict__ w,
                           uint32_t m, const float* __restrict__ wsum, uint4* __restrict__ dy_bf,
                           float* __restrict__ loss) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float l_i = 0.0f;
    if (i < m) {
        const float* o = out + (size_t)i * kOut;
        Lobe L[kLobes];
        decode_mixture(o, L);
        const float dx = dirs[3 * i], dyy = dirs[3 * i + 1], dz = dirs[3 * i + 2];
        float lg[kLobes], cs[kLobes];
        float lmax = -3.4e38f;
#pragma unroll
        for (int j = 0; j < kLobes; ++j) {
            cs[j] = L[j].mx * dx + L[j].my * dyy + L[j].mz * dz;
            lg[j] = logf(fmaxf(L[j].pi, 1e-30f)) + log_vmf(L[j].kappa, cs[j]);
            lmax = fmaxf(lmax, lg[j]);
        }
        float se = 0.0f;
#pragma unroll
        for (int j = 0; j < kLobes; ++j) se += expf(lg[j] - lmax);
        const float logq = lmax + logf(se);
        const float scale = w[i] / fmaxf(*wsum, 1e-30f);
        l_i = -scale * logq;
        float g[64];
#pragma unroll
        for (int k = 0; k < 64; ++k) g[k] = 0.0f;
#pragma unroll
        for (int j = 0; j < kLobes; ++j) {
            const float r = expf(lg[j] - logq);                 // responsibility
            const float kap = L[j].kappa;
            g[5 * j] = -scale * (r - L[j].pi);                  // d(-log q)/d logit
            const float c = r * kap / L[j].mnorm;
            g[5 * j + 1] = -scale * c * (dx - cs[j] * L[j].mx);
            g[5 * j + 2] = -scale * c * (dyy - cs[j] * L[j].my);
            g[5 * j + 3] = -scale * c * (dz - cs[j] * L[j].mz);
            const float e2 = expf(-2.0f * kap);
            const float dlogv = 1.0f / kap - 2.0f * e2 / (1.0f - e2) + (cs[j] - 1.0f);
            g[5 * j + 4] = -scale * r * dlogv * L[j].sig;
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            dy_bf[(size_t)i * 8 + c] = make_uint4(pack2(g[8 * c], g[8 * c + 1]), pack2(g[8 * c + 2], g[8 * c + 3]),
                                                  pack2(g[8 * c + 4], g[8 * c + 5]), pack2(g[8 * c + 6], g[8 * c + 7]));
        }
    }
    // block-reduce the loss
    for (int off = 16; off > 0; off >>= 1) l_i += __shfl_down_sync(0xffffffffu, l_i, off);
    if ((threadIdx.x & 31u) == 0 && l_i != 0.0f) atomicAdd(loss, l_i);
}

__global__ void k_sum(const float* __restrict__ w, uint32_t m, float* __restrict__ out) {
    float s = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) s += w[i];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31u) == 0) atomicAdd(out, s);
}

// Weight gradients of all four layers on the tensor cores (blockIdx.y = layer):
//   gw[l][in][out] = sum_rows prev[row][in] * grad[row][out],  gb[l][out] = sum_rows grad[row][out]
// with BF16 operands and FP32 accumulation in tensor memory.  One MMA chain per CTA computes
// D (128 x 64) += A (128 x K) * B (64 x K)^T over the CTA's rows, in K-tiles of 64 rows:
//   A rows 0..63 = prev^T (m = input unit, k = batch row); row 64 = 1 for every valid row, so
//   D row 64 is the bias gradient; rows 65..127 = 0;
//   B rows = grad^T (n = output unit, k = batch row).
// Both operands are staged transposed into the canonical K-major layout (the same layout as
// the forward's A tile), double-buffered: tile i + 1 is staged while the MMAs of tile i run
// (one mbarrier per stage, each wait bounded).  The CTA then reads D rows 0..64 back from
// tensor memory and adds them to gw / gb with coalesced atomics.
constexpr uint32_t kDwK = 64;                                  // batch rows per K-tile
constexpr uint32_t kDwA = 16384, kDwB = 8192;                  // bytes per stage
constexpr uint32_t kDwSmemA0 = 0, kDwSmemB0 = 2 * kDwA, kDwSmemBar = 2 * kDwA + 2 * kDwB,
                   kDwSmemSlot = kDwSmemBar + 16, kDwSmemOk = kDwSmemSlot + 4, kDwSmemBytes = kDwSmemOk + 12;
constexpr uint32_t kIdescM128N64 = kIdesc;                     // BF16 x BF16 -> FP32, M = 128, N = 64

__global__ void __launch_bounds__(128) k_dw_tc(DwLayers L, uint32_t m, uint32_t tiles_per_cta, uint32_t spin,
                                               int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kDwSmemBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kDwSmemSlot);
    volatile int* s_ok = reinterpret_cast<volatile int*>(smem + kDwSmemOk);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, l = blockIdx.y;
    // constant-index selects keep the parameter arrays out of local memory
    auto pick = [l](auto a0, auto a1, auto a2, auto a3) { return l == 0 ? a0 : l == 1 ? a1 : l == 2 ? a2 : a3; };
    const uint4* __restrict__ prev = pick(L.prev[0], L.prev[1], L.prev[2], L.prev[3]);
    const uint4* __restrict__ grad = pick(L.grad_bf[0], L.grad_bf[1], L.grad_bf[2], L.grad_bf[3]);
    const uint32_t ntiles = (m + kDwK - 1) / kDwK;
    const uint32_t t0 = blockIdx.x * tiles_per_cta;
    const uint32_t t1 = min(ntiles, t0 + tiles_per_cta);
    if (t0 >= t1) return;
    // zero both A stages (rows 65..127 stay zero; rows 0..64 are rewritten per tile)
    for (uint32_t i = tid; i < 2 * kDwA / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(smem + kDwSmemA0)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) { mbar_init(&bar[0], 1); mbar_init(&bar[1], 1); fence_mbar_init(); }
    if (warp == 0) { tmem_alloc(tslot, 64); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *tslot;
    uint32_t phases = 0u;              // bit s = parity of the next completion of stage s
    bool ok = true;
    // thread -> (row r of the tile, half h of the 8 16-byte chunks of a 64-wide row)
    const uint32_t r = tid & 63u, h = tid >> 6;
    for (uint32_t t = t0; t < t1 && ok; ++t) {
        const uint32_t st = (t - t0) & 1u;
        uint8_t* sA = smem + kDwSmemA0 + st * kDwA;
        uint8_t* sB = smem + kDwSmemB0 + st * kDwB;
        // the MMAs that last read this stage (two tiles ago) must have completed
        if (t - t0 >= 2u) {
            if (tid == 0) {
                bool done = false;
                for (uint32_t it = 0; it < spin && !done; ++it) done = mbar_try_wait(&bar[st], (phases >> st) & 1u);
                *s_ok = done ? 1 : 0;
            }
            __syncthreads();
            ok = *s_ok != 0;
            if (!ok) break;
            phases ^= 1u << st;
        }
        const uint32_t row = t * kDwK + r;
        const bool valid = row < m;
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            const uint32_t c = 4u * h + q;                  // chunk: units 8c .. 8c + 7
            const uint4 a = valid ? __ldg(&prev[(size_t)row * 8 + c]) : make_uint4(0u, 0u, 0u, 0u);
            const uint4 b = valid ? __ldg(&grad[(size_t)row * 8 + c]) : make_uint4(0u, 0u, 0u, 0u);
            const uint32_t aw[4] = {a.x, a.y, a.z, a.w}, bw[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (uint32_t e = 0; e < 4; ++e) {
                *reinterpret_cast<uint16_t*>(sA + canon_off(8u * c + 2u * e, r)) = (uint16_t)(aw[e] & 0xffffu);
                *reinterpret_cast<uint16_t*>(sA + canon_off(8u * c + 2u * e + 1u, r)) = (uint16_t)(aw[e] >> 16);
                *reinterpret_cast<uint16_t*>(sB + canon_off(8u * c + 2u * e, r)) = (uint16_t)(bw[e] & 0xffffu);
                *reinterpret_cast<uint16_t*>(sB + canon_off(8u * c + 2u * e + 1u, r)) = (uint16_t)(bw[e] >> 16);
            }
        }
        if (h == 0) *reinterpret_cast<uint16_t*>(sA + canon_off(64u, r)) = valid ? (uint16_t)0x3f80u : (uint16_t)0u;
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (uint32_t k = 0; k < 4; ++k)
                umma_bf16(taddr, smem_desc(smem_u32(sA) + k * 256u), smem_desc(smem_u32(sB) + k * 256u),
                          kIdescM128N64, (t > t0 || k > 0) ? 1u : 0u);
            umma_commit(&bar[st]);
        }
    }
    // the last one or two tiles' MMAs
    if (ok) {
        const uint32_t n = t1 - t0;
        if (tid == 0) {
            bool done = true;
            for (uint32_t back = (n >= 2u ? 2u : 1u); back >= 1u && done; --back) {
                const uint32_t st = (n - back) & 1u;
                done = false;
                for (uint32_t it = 0; it < spin && !done; ++it) done = mbar_try_wait(&bar[st], (phases >> st) & 1u);
                if (done) phases ^= 1u << st;
            }
            *s_ok = done ? 1 : 0;
        }
        __syncthreads();
        ok = *s_ok != 0;
    }
    tc_fence_after();
    if (ok) {
        // D rows 0..64 -> shared memory (stage-0 A buffer, free now) -> coalesced atomics
        float* sD = reinterpret_cast<float*>(smem + kDwSmemA0);       // [65][64]
        if (warp < 3) {
            float v[64];
            const uint32_t lane_addr = taddr + ((32u * warp) << 16);
#pragma unroll
            for (int j = 0; j < 4; ++j) tmem_ld16(lane_addr + 16u * j, v + 16 * j);
            tmem_wait_ld();
            const uint32_t drow = 32u * warp + (tid & 31u);
            if (drow <= 64u) {
#pragma unroll
                for (int j = 0; j < 64; ++j) sD[drow * 64u + j] = v[j];
            }
        }
        __syncthreads();
        float* gw = pick(L.gw[0], L.gw[1], L.gw[2], L.gw[3]);
        float* gb = pick(L.gb[0], L.gb[1], L.gb[2], L.gb[3]);
        for (uint32_t i = tid; i < 64u * 64u; i += blockDim.x) atomicAdd(&gw[i], sD[i]);
        if (tid < 64u) atomicAdd(&gb[tid], sD[64u * 64u + tid]);
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    // every MMA this CTA issued must have landed before its tensor memory is freed
    if (!ok && tid == 0) {
        for (uint32_t st = 0; st < 2; ++st) {
            uint32_t it = 0;
            while (!mbar_try_wait(&bar[st], (phases >> st) & 1u) && ++it < kSpin) {}
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, 64);
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters
__global__ void k_adam(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m1,
                       float* __restrict__ m2, uint32_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grads[i];
    const float a = b1 * m1[i] + (1.0f - b1) * g;
    const float b = b2 * m2[i] + (1.0f - b2) * g * g;
    m1[i] = a;
    m2[i] = b;
    params[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

cudaError_t pack_weights(const float* params, uint8_t* w_fwd, uint8_t* w_bwd, cudaStream_t s) {
    k_pack_weights<<<(4 * 4096 + 255) / 256, 256, 0, s>>>(params, w_fwd, w_bwd);
    return cudaGetLastError();
}
cudaError_t mix_grad(const float* out, const float* dirs, const float* w, uint32_t m, float* wsum, uint4* dy_bf,
                     float* loss, cudaStream_t s) {
    if (m == 0) return cudaSuccess;
    k_sum<<<256, 256, 0, s>>>(w, m, wsum);
    k_mix_grad<<<(m + 127) / 128, 128, 0, s>>>(out, dirs, w, m, wsum, dy_bf, loss);
    return cudaGetLastError();
}
cudaError_t weight_grad(const DwLayers& L, uint32_t m, uint32_t spin, int* err, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_dw_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDwSmemBytes);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    if (m == 0) return cudaSuccess;
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // two CTAs per SM over the four layers; each CTA walks a contiguous run of K-tiles
    const uint32_t ntiles = (m + kDwK - 1) / kDwK;
    const uint32_t per_layer = std::max<uint32_t>(1u, (uint32_t)sms / 2u);
    const uint32_t tiles_per_cta = (ntiles + per_layer - 1) / per_layer;
    const uint32_t gx = (ntiles + tiles_per_cta - 1) / tiles_per_cta;
    k_dw_tc<<<dim3(gx, 4), 128, kDwSmemBytes, s>>>(L, m, tiles_per_cta, spin, err);
    return cudaGetLastError();
}
cudaError_t adam(float* params, const float* grads, float* m1, float* m2, uint32_t n, float lr, uint32_t step,
                 cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, s>>>(params, grads, m1, m2, n, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

}  // namespace trg
