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
// step) run on the CUDA cores.  Every wait on the mbarrier is bounded; on expiry the kernel
// records an error, waits (bounded) for its MMAs, frees its tensor memory and returns.
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
            ok = layer_mma(taddr, smem_u32(sA), smem_u32(smem + kSmemW + l * 8192u), bar, phase, s_ok);
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
                    for (int e = 0; e < 8; ++e) t[e] = fmaxf(acc[8 * c + e] + sB[l * 64 + 8 * c + e], 0.0f);
                    h[c] = make_uint4(pack2(t[0], t[1]), pack2(t[2], t[3]), pack2(t[4], t[5]), pack2(t[6], t[7]));
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
// stored activations, dh[2] = dH3 = (dY W4^T) * 1[H3>0], dh[1] = dH2, dh[0] = dH1 (FP32).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) k_mlp_bwd(GuideDev g, const uint4* __restrict__ dy,
                                                    const uint4* __restrict__ act, uint32_t m,
                                                    float* __restrict__ dh, int* err) {
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
            ok = layer_mma(taddr, smem_u32(sA), smem_u32(smem + kSmemW + (uint32_t)l * 8192u), bar, phase, s_ok);
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
                if (row < m) {
                    float4* d = reinterpret_cast<float4*>(dh + ((size_t)(l - 1) * m + row) * 64 + 8 * c);
                    d[0] = make_float4(t[0], t[1], t[2], t[3]);
                    d[1] = make_float4(t[4], t[5], t[6], t[7]);
                }
                h[c] = make_uint4(pack2(t[0], t[1]), pack2(t[2], t[3]), pack2(t[4], t[5]), pack2(t[6], t[7]));
            }
            store_row_a(sA, tid, h);
        }
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    drain_and_free(taddr, bar, phase, ok);
}

int resident_grid(int device, const void* kernel, int threads, size_t dyn_smem) {
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
    per_sm = std::min(per_sm, 512 / 64);                                          // 64 TMEM columns each
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

cudaError_t mlp_backward(const GuideDev& g, const uint4* dy, const uint4* act, uint32_t m, float* dh, int* err,
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

// training loss -(w/W) log q(dir) and its gradient w.r.t. the 40 raw outputs; dy bf16 (and
// FP32 copy) [m][64], columns >= 40 zero.  wsum = sum of weights over the batch.
__global__ void k_mix_grad(const float* __restrict__ out, const float* __restrict__ dirs, const float* __restrict__ w,
                           uint32_t m, const float* __restrict__ wsum, uint4* __restrict__ dy_bf,
                           float* __restrict__ dy_f, float* __restrict__ loss) {
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
            float4* d = reinterpret_cast<float4*>(dy_f + (size_t)i * 64 + 8 * c);
            d[0] = make_float4(g[8 * c], g[8 * c + 1], g[8 * c + 2], g[8 * c + 3]);
            d[1] = make_float4(g[8 * c + 4], g[8 * c + 5], g[8 * c + 6], g[8 * c + 7]);
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

// weight gradients of all four layers in one launch (blockIdx.y = layer):
// gw[in][out] = sum_rows prev[row][in] * grad[row][out], gb[out] = sum_rows grad[row][out];
// prev is bf16 (x or a stored activation), grad FP32.  256 threads per block; each thread
// owns a 4x4 patch of the 64x64 gradient and keeps it in registers while the block walks its
// 64-row chunks (grid-stride), so each block adds its partial sums to global memory once.
constexpr uint32_t kDwRows = 64;
__global__ void __launch_bounds__(256) k_dw(DwLayers L, uint32_t m) {
    __shared__ float sp[kDwRows][65];
    __shared__ float sg[kDwRows][65];
    const uint32_t l = blockIdx.y;
    const uint4* __restrict__ prev = L.prev[l];
    const float* __restrict__ grad = L.grad[l];
    const uint32_t ti = (threadIdx.x >> 4) * 4u, to = (threadIdx.x & 15u) * 4u;
    float acc[4][4] = {};
    float sb = 0.0f;
    for (uint32_t r0 = blockIdx.x * kDwRows; r0 < m; r0 += gridDim.x * kDwRows) {
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < kDwRows * 8u; e += blockDim.x) {
            const uint32_t r = e >> 3, c = e & 7u, row = r0 + r;
            const uint4 v = row < m ? __ldg(&prev[(size_t)row * 8 + c]) : make_uint4(0, 0, 0, 0);
            const uint32_t vw[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) { sp[r][8 * c + 2 * q] = bf_lo(vw[q]); sp[r][8 * c + 2 * q + 1] = bf_hi(vw[q]); }
        }
        for (uint32_t e = threadIdx.x; e < kDwRows * 16u; e += blockDim.x) {
            const uint32_t r = e >> 4, c = (e & 15u) * 4u, row = r0 + r;
            const float4 v = row < m ? __ldg(reinterpret_cast<const float4*>(grad + (size_t)row * 64 + c))
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
            sg[r][c] = v.x; sg[r][c + 1] = v.y; sg[r][c + 2] = v.z; sg[r][c + 3] = v.w;
        }
        __syncthreads();
#pragma unroll 4
        for (uint32_t r = 0; r < kDwRows; ++r) {
            float a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) { a[q] = sp[r][ti + q]; b[q] = sg[r][to + q]; }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
        }
        if (threadIdx.x < 64u)
            for (uint32_t r = 0; r < kDwRows; ++r) sb += sg[r][threadIdx.x];
    }
    float* gw = L.gw[l];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) atomicAdd(&gw[(ti + u) * 64u + to + v], acc[u][v]);
    if (threadIdx.x < 64u) atomicAdd(&L.gb[l][threadIdx.x], sb);
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
                     float* dy_f, float* loss, cudaStream_t s) {
    if (m == 0) return cudaSuccess;
    k_sum<<<256, 256, 0, s>>>(w, m, wsum);
    k_mix_grad<<<(m + 127) / 128, 128, 0, s>>>(out, dirs, w, m, wsum, dy_bf, dy_f, loss);
    return cudaGetLastError();
}
cudaError_t weight_grad(const DwLayers& L, uint32_t m, cudaStream_t s) {
    if (m == 0) return cudaSuccess;
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // four blocks per SM over the four layers
    uint32_t gx = (uint32_t)sms;
    const uint32_t chunks = (m + kDwRows - 1) / kDwRows;
    if (gx > chunks) gx = chunks;
    k_dw<<<dim3(gx, 4), 256, 0, s>>>(L, m);
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
