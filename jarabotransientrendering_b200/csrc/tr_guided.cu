// tr_guided.cu - guided path sampling with the learned proposal (no reference counterpart):
// the fused proposal-inference + one-sample-MIS kernel of each depth and the gathering of
// training targets.  Built with FMA contraction (-fmad=true): unlike the plain path, nothing
// here has to reproduce the oracle's operation sequence bit for bit.
#include <cuda_bf16.h>

#include "tr_bsdf.cuh"
#include "tr_device.cuh"
#include "tr_guide_math.cuh"
#include "tr_kernels.cuh"
#include "tr_tcgen05.cuh"

namespace trk {
using namespace trd;

// Features of a surface vertex for the learned proposal (64 BF16 values, 46 used):
// sin/cos(2^k pi p_d) for k = 0..5 (index 6k + 2d + {0,1}), p normalised to the scene box,
// geometric normal, outgoing direction, path length / film time length; in multi-scene mode
// [46 + scene] = 1 (one network serves up to 16 scenes).  Octave k+1 follows
// from octave k by the double-angle identities (sin 2x = 2 sin x cos x, cos 2x = 1 - 2 sin^2 x);
// the rounding error doubles per octave, about 3e-6 at k = 5, far below BF16 resolution.
__device__ __forceinline__ void write_features(uint4* row, const SceneDev& sc, f3 pos, f3 nrm, f3 wo, float tn,
                                               int scene_onehot = -1) {
    float v[64];
    const float pn[3] = {(pos.x - sc.bmin[0]) * sc.binv[0], (pos.y - sc.bmin[1]) * sc.binv[1],
                         (pos.z - sc.bmin[2]) * sc.binv[2]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float sv, cv;
        sincospif(pn[d], &sv, &cv);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            v[6 * k + 2 * d] = sv;
            v[6 * k + 2 * d + 1] = cv;
            const float s2 = (2.0f * sv) * cv;
            cv = fmaf(-2.0f * sv, sv, 1.0f);
            sv = s2;
        }
    }
    v[36] = pn[0]; v[37] = pn[1]; v[38] = pn[2];
    v[39] = nrm.x; v[40] = nrm.y; v[41] = nrm.z;
    v[42] = wo.x; v[43] = wo.y; v[44] = wo.z;
    v[45] = tn;
#pragma unroll
    for (int k = 46; k < 64; ++k) v[k] = k - 46 == scene_onehot ? 1.0f : 0.0f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        __nv_bfloat162 a = __floats2bfloat162_rn(v[8 * c], v[8 * c + 1]);
        __nv_bfloat162 b = __floats2bfloat162_rn(v[8 * c + 2], v[8 * c + 3]);
        __nv_bfloat162 e = __floats2bfloat162_rn(v[8 * c + 4], v[8 * c + 5]);
        __nv_bfloat162 h = __floats2bfloat162_rn(v[8 * c + 6], v[8 * c + 7]);
        row[c] = make_uint4(*reinterpret_cast<uint32_t*>(&a), *reinterpret_cast<uint32_t*>(&b),
                            *reinterpret_cast<uint32_t*>(&e), *reinterpret_cast<uint32_t*>(&h));
    }
}

// -----------------------------------------------------------------------------------------
// guided direction sampling (no reference counterpart): one-sample multiple importance
// sampling (Veach & Guibas 1995, balance heuristic) between the learned vMF mixture (chosen
// with probability mix_prob) and the BSDF sampler, so the estimator stays unbiased whatever
// the network predicts.  Directions below the surface carry no reflectance and end the path.
// -----------------------------------------------------------------------------------------

// Fast-math GGX for the guided path: the same formulas as ggx_sample / ggx_eval_cos /
// ggx_pdf (Walter et al. 2007, Heitz 2018), evaluated in a local frame built once per vertex and
// with hardware reciprocal square roots and divisions.  Sampling and density come from the same
// formulas, so the MIS weights stay consistent.
__device__ __forceinline__ f3 fnormalize(f3 v) { return v * rsqrtf(dot(v, v)); }

struct GgxVertex {
    Frame3 F;
    f3 wo;              // outgoing direction in the local frame
    float a2, alpha, lo, g1, inv4wz;
};

__device__ __forceinline__ float ggx_lambda_fast(float a2, f3 w) {
    const float t2 = __fdividef(w.x * w.x + w.y * w.y, w.z * w.z);
    return 0.5f * (sqrtf(1.0f + a2 * t2) - 1.0f);
}

// returns false when wo lies below the surface (every direction then carries zero reflectance)
__device__ __forceinline__ bool ggx_vertex(GgxVertex& g, float alpha, f3 n, f3 wo_w) {
    g.F = make_frame(n);
    g.wo = to_local(g.F, wo_w);
    if (!(g.wo.z > 0.0f)) return false;
    g.alpha = alpha;
    g.a2 = alpha * alpha;
    g.lo = ggx_lambda_fast(g.a2, g.wo);
    g.g1 = __frcp_rn(1.0f + g.lo);
    g.inv4wz = __fdividef(0.25f, g.wo.z);
    return true;
}

// f cos and visible-normal sampling density at the local direction wi
__device__ __forceinline__ float ggx_eval_pdf_fast(const GgxVertex& g, f3 kd, f3 wi, f3& fcos) {
    if (!(wi.z > 0.0f)) { fcos = mk(0.0f, 0.0f, 0.0f); return 0.0f; }
    const f3 h = fnormalize(g.wo + wi);
    const float d = h.z * h.z * (g.a2 - 1.0f) + 1.0f;
    const float D = __fdividef(g.a2, 3.14159274f * d * d);
    const float G2 = __frcp_rn(1.0f + g.lo + ggx_lambda_fast(g.a2, wi));
    const float c = fmaxf(dot(g.wo, h), 0.0f);
    const float common = D * G2 * g.inv4wz;
    fcos = mk(schlick(kd.x, c) * common, schlick(kd.y, c) * common, schlick(kd.z, c) * common);
    return g.g1 * D * g.inv4wz;
}

// visible-normal sample (Heitz 2018) in the local frame; false if the reflection leaves the
// upper hemisphere
__device__ __forceinline__ bool ggx_sample_fast(const GgxVertex& g, float sp, float cp, float x2, f3& wi) {
    const f3 Vh = fnormalize(mk(g.alpha * g.wo.x, g.alpha * g.wo.y, g.wo.z));
    const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    const f3 T1 = lensq > 0.0f ? mk(-Vh.y, Vh.x, 0.0f) * rsqrtf(lensq) : mk(1.0f, 0.0f, 0.0f);
    const f3 T2 = cross(Vh, T1);
    const float r = sqrtf(x2);
    const float t1 = r * cp;
    const float s = 0.5f * (1.0f + Vh.z);
    const float t2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + s * (r * sp);
    const float tz = sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2));
    const f3 Nh = T1 * t1 + T2 * t2 + Vh * tz;
    const f3 h = fnormalize(mk(g.alpha * Nh.x, g.alpha * Nh.y, fmaxf(Nh.z, 0.0f)));
    wi = h * (2.0f * dot(g.wo, h)) - g.wo;
    return wi.z > 0.0f;
}

// Fused proposal inference and sampling: one CTA of 128 threads owns two tiles of 128 guided
// vertices at a time.  Each thread gathers its vertex of both tiles and writes their 64 BF16
// features as row `tid` of the two A tiles in shared memory; the four layers run on the tensor
// cores with the two tiles' MMAs issued back to back (accumulators in tensor-memory columns 0-63
// and 64-127), so one tile's MMAs run while the CTA applies bias + ReLU to the other's; the
// epilogue decodes the thread's mixture from the last layer's accumulator row in registers and
// samples the direction, tile by tile.  Neither features nor mixtures touch HBM.  Three CTAs per
// SM (65 KB shared memory, 128 TMEM columns each) give six tiles in flight per SM.
// Training-pool tag of the current batch (0: untagged).  Single-scene launches carry theirs in
// the parameters; multi-scene launches, replayed from one graph for every batch, use the batch
// index + 1 (the pool's tags are cleared before each render).
__device__ __forceinline__ uint32_t pool_tag(const Params& p) {
    if (!p.guide.tag) return 0u;
    return p.multi.scenes ? *p.multi.cur + 1u : p.guide.tag;
}

template <bool kMulti>
__global__ void __launch_bounds__(128, 3) k_guide(const __grid_constant__ Params p, int depth, uint32_t* pool_count) {
    const GuideWave& G = p.guide;
    const uint32_t n = p.wave.counters[cnt_guide(depth)];
    constexpr uint32_t kPair = 2u * (uint32_t)trg::kTile;
    if (blockIdx.x * kPair >= n) return;     // no tile pair for this CTA
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sA0 = smem + trg::kG2A0;
    uint8_t* sA1 = smem + trg::kG2A1;
    const float* sB = reinterpret_cast<const float*>(smem + trg::kG2Bias);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + trg::kG2Bar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + trg::kG2Slot);
    volatile int* s_ok = reinterpret_cast<volatile int*>(smem + trg::kG2Ok);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    {
        uint4* sw = reinterpret_cast<uint4*>(smem + trg::kG2W);
        for (uint32_t i = tid; i < 2048u; i += blockDim.x) sw[i] = __ldg(&G.net.w_fwd[i]);
        float* sb = reinterpret_cast<float*>(smem + trg::kG2Bias);
        for (uint32_t i = tid; i < 256u; i += blockDim.x) sb[i] = __ldg(&G.net.bias[i]);
    }
    if (tid == 0) { trg::mbar_init(&bar[0], 1); trg::mbar_init(&bar[1], 1); trg::fence_mbar_init(); }
    if (warp == 0) { trg::tmem_alloc(tslot, 128); trg::tmem_relinquish(); }
    trg::tc_fence_before();
    __syncthreads();
    trg::tc_fence_after();
    const uint32_t taddr = *tslot;
    const uint32_t lane_off = (32u * warp) << 16;
    uint32_t ph0 = 0, ph1 = 0;            // parity of the next completion of each tile's mbarrier
    bool pend0 = false, pend1 = false;    // MMAs committed and not yet waited for
    bool ok = true;

    uint32_t* qout = p.wave.q[(depth + 1) & 1];
    const float c = G.mix_prob;
    // scene, film length and scene feature of a slot: the launch's own in single-scene mode
    struct SlotScene { const SceneDev* sc; float total_time; int onehot; };
    auto scene_of = [&](uint32_t slot) {
        SlotScene r{&p.scene, (float)p.film.T * p.film.exposure + p.film.offset, -1};
        if constexpr (kMulti) {
            const Batch& Bs = seg_of_slot(cur_batch(p), slot);
            const SceneSlot& S = p.multi.scenes[Bs.scene];
            r.sc = &S.scene;
            r.total_time = (float)S.film.T * S.film.exposure + S.film.offset;
            r.onehot = (int)Bs.scene;
        }
        return r;
    };
    // features of vertex idx as row tid of an A tile (zeros past the queue's end)
    auto stage = [&](uint8_t* sA, uint32_t idx) {
        uint4 feat[8];
        if (idx < n) {
            const uint4* rec = G.vrec + (size_t)idx * 5;
            const float4 r0 = __ldg(reinterpret_cast<const float4*>(rec));
            const float4 r1 = __ldg(reinterpret_cast<const float4*>(rec + 1));
            const float4 r3 = __ldg(reinterpret_cast<const float4*>(rec + 3));
            const SlotScene ss = scene_of(__float_as_uint(r3.w));
            write_features(feat, *ss.sc, mk(r0.x, r0.y, r0.z), mk(r3.x, r3.y, r3.z), mk(-r1.x, -r1.y, -r1.z),
                           r0.w / ss.total_time, ss.onehot);
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) feat[q] = make_uint4(0u, 0u, 0u, 0u);
        }
        trg::store_row_a(sA, tid, feat);
    };
    // bias + ReLU of layer l's accumulator row, written back as the next layer's A row
    auto hidden = [&](uint32_t tcol, uint8_t* sA, uint32_t l) {
        float a[64];
#pragma unroll
        for (int j = 0; j < 4; ++j) trg::tmem_ld16(taddr + tcol + lane_off + 16u * j, a + 16 * j);
        trg::tmem_wait_ld();
        uint4 h[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            float t[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) t[e] = a[8 * q + e] + sB[l * 64 + 8 * q + e];
            h[q] = make_uint4(trg::pack2_relu(t[0], t[1]), trg::pack2_relu(t[2], t[3]), trg::pack2_relu(t[4], t[5]),
                              trg::pack2_relu(t[6], t[7]));
        }
        trg::store_row_a(sA, tid, h);
    };
    const unsigned lane = tid & 31u;
    for (uint32_t pair = blockIdx.x; pair * kPair < n && ok; pair += gridDim.x) {
        const uint32_t base = pair * kPair;
        stage(sA0, base + tid);
        stage(sA1, base + (uint32_t)trg::kTile + tid);
        for (uint32_t l = 0; l < 4 && ok; ++l) {
            trg::fence_proxy_async();
            trg::tc_fence_before();
            __syncthreads();
            if (tid == 0) {
                trg::tc_fence_after();
                const uint32_t w = trg::smem_u32(smem + trg::kG2W + l * 8192u);
                trg::issue_layer(taddr, trg::smem_u32(sA0), w, &bar[0]);
                trg::issue_layer(taddr + 64u, trg::smem_u32(sA1), w, &bar[1]);
            }
            pend0 = pend1 = true;
            if (l == 3) break;                // the output layer's accumulators are read per tile below
            ok = trg::wait_uniform(&bar[0], ph0, s_ok, G.net.spin);
            if (!ok) break;
            ph0 ^= 1u; pend0 = false;
            hidden(0u, sA0, l);
            ok = trg::wait_uniform(&bar[1], ph1, s_ok, G.net.spin);
            if (!ok) break;
            ph1 ^= 1u; pend1 = false;
            hidden(64u, sA1, l);
        }
        if (!ok) break;

        for (uint32_t t = 0; t < 2u; ++t) {
            ok = trg::wait_uniform(t ? &bar[1] : &bar[0], t ? ph1 : ph0, s_ok, G.net.spin);
            if (!ok) break;
            if (t) { ph1 ^= 1u; pend1 = false; } else { ph0 ^= 1u; pend0 = false; }
            float o[48];
#pragma unroll
            for (int j = 0; j < 3; ++j) trg::tmem_ld16(taddr + 64u * t + lane_off + 16u * j, o + 16 * j);
            trg::tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < trg::kOut; ++j) o[j] += sB[3 * 64 + j];
            const uint32_t idx = base + t * (uint32_t)trg::kTile + tid;
            const bool active = idx < n;
            const uint4* rec = G.vrec + (size_t)idx * 5;

            // ---- one-sample MIS between the mixture and the BSDF ----
            bool want_next = false;
            uint32_t slot = 0;
            if (active) {
                const float4 ro = __ldg(reinterpret_cast<const float4*>(rec));
                const float4 rd = __ldg(reinterpret_cast<const float4*>(rec + 1));
                const float4 th = __ldg(reinterpret_cast<const float4*>(rec + 2));
                const float4 rn = __ldg(reinterpret_cast<const float4*>(rec + 3));
                const uint4 rr = __ldg(rec + 4);
                slot = __float_as_uint(rn.w);
                const SlotScene ss = scene_of(slot);
                const SceneDev& sc = *ss.sc;
                const bool medium = sc.medium != 0;
                const uint32_t mi = __float_as_uint(th.w);
                const f3 nrm = mk(rn.x, rn.y, rn.z);
                const float4 m = __ldg(&sc.mats[mi]);
                const f3 kd = mk(m.x, m.y, m.z);
                const bool ggx = __float_as_uint(m.w) == 1u;
                const float alpha = ggx ? __ldg(&sc.mats2[mi]).x : 0.0f;
                const f3 pos = mk(ro.x, ro.y, ro.z);
                const f3 wo = mk(-rd.x, -rd.y, -rd.z);
                const f3 f = mk(th.x, th.y, th.z);
                const float albedo = rd.w, time = ro.w;
                Pcg rng;
                rng.state = ((unsigned long long)rr.y << 32) | rr.x;
                rng.inc = ((unsigned long long)rr.w << 32) | rr.z;
                trg::SampLobe L[trg::kLobes];
                const float esum = trg::decode_sampling(o, L);
                GgxVertex gv;
                bool alive = !ggx || ggx_vertex(gv, alpha, nrm, wo);
                f3 wi = mk(0.f, 0.f, 1.f), wl = wi;      // world and (GGX) local direction
                if (pcg_float(rng) < c) {
                    const float u0 = pcg_float(rng), u1 = pcg_float(rng), u2 = pcg_float(rng);
                    float d[3];
                    trg::sampling_draw(L, esum, u0, u1, u2, d);
                    wi = fnormalize(mk(d[0], d[1], d[2]));
                    if (ggx) wl = to_local(gv.F, wi);
                } else {
                    const float x1 = pcg_float(rng), x2 = pcg_float(rng);
                    float sp, cp;
                    __sincosf(6.28318531f * x1, &sp, &cp);
                    if (ggx) {
                        alive = alive && ggx_sample_fast(gv, sp, cp, x2, wl);
                        wi = fnormalize(to_world(gv.F, wl));
                    } else {
                        const float ct = sqrtf(x2);
                        const float stt = sqrtf(1.0f - ct * ct);
                        wi = to_world(make_frame(nrm), mk(cp * stt, sp * stt, ct));
                    }
                }
                if (alive) {
                    f3 fcos;
                    float pb;
                    if (ggx) {
                        pb = ggx_eval_pdf_fast(gv, kd, wl, fcos);
                    } else {
                        const float cl = fmaxf(dot(nrm, wi), 0.0f);
                        fcos = mk((kd.x * kInvPi) * cl, (kd.y * kInvPi) * cl, (kd.z * kInvPi) * cl);
                        pb = cl * kInvPi;
                    }
                    const float pdf = c * trg::sampling_pdf(L, wi.x, wi.y, wi.z) + (1.0f - c) * pb;
                    if (pdf > 0.0f && (fcos.x > 0.0f || fcos.y > 0.0f || fcos.z > 0.0f) && isfinite(pdf)) {
                        const f3 fn = mulv(f, fcos);
                        const bool keep = G.pool_cap > 0 && pcg_float(rng) < G.keep_prob;
                        float nds = __int_as_float(0x7f800000);
                        if (medium) nds = -tr_log(pcg_float(rng)) / sc.lambda;
                        p.wave.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, nds);
                        p.wave.ray_d[slot] = make_float4(wi.x, wi.y, wi.z, time);
                        p.wave.thr[slot] = make_float4(fn.x, fn.y, fn.z, albedo * pdf);
                        want_next = true;
                        if (keep) {
                            const uint32_t k = atomicAdd(pool_count, 1u);
                            if (k < G.pool_cap) {
                                write_features(G.pool_feat + (size_t)k * 8, sc, pos, nrm, wo, time / ss.total_time,
                                               ss.onehot);
                                G.pool_dir[3 * (size_t)k] = wi.x;
                                G.pool_dir[3 * (size_t)k + 1] = wi.y;
                                G.pool_dir[3 * (size_t)k + 2] = wi.z;
                                G.pool_meta[k] = make_uint4(slot, (uint32_t)depth, __float_as_uint(avg3(f)), pool_tag(p));
                            }
                        }
                    }
                }
                p.wave.rng[slot] = rng.state;
            }
            const unsigned mn = __ballot_sync(kFull, want_next);
            uint32_t bn = 0;
            if (lane == 0 && mn) bn = atomicAdd(&p.wave.counters[cnt_ext(depth + 1)], (uint32_t)__popc(mn));
            bn = __shfl_sync(kFull, bn, 0);
            if (want_next) qout[bn + (uint32_t)__popc(mn & lanemask_lt())] = slot;
        }
    }
    if (!ok && tid == 0) {
        atomicExch(G.err, 1);
        // the MMAs this CTA issued must land before its tensor memory is freed
        uint32_t it = 0;
        if (pend0) while (!trg::mbar_try_wait(&bar[0], ph0) && ++it < trg::kSpin) {}
        it = 0;
        if (pend1) while (!trg::mbar_try_wait(&bar[1], ph1) && ++it < trg::kSpin) {}
    }
    trg::tc_fence_before();
    __syncthreads();
    if (warp == 0) trg::tmem_dealloc(taddr, 128);
}

// Training targets of this batch's pool entries: the luminance reaching the film through the
// rest of the path (splat records of later bounces) relative to the throughput at the vertex,
// i.e. an estimate of (incident radiance x f cos / sampling pdf) along the sampled direction.
// pool_state[0] = entries filled, pool_state[1] = entries already given a target.  A tagged
// batch (batches in flight on several wave lanes fill the pool interleaved) scans every
// filled entry and takes those carrying its tag.
__global__ void k_train_gather(Params p, const uint32_t* pool_state) {
    const GuideWave& G = p.guide;
    const uint32_t end = min(pool_state[0], G.pool_cap);
    const uint32_t tag = pool_tag(p);
    const uint32_t begin = tag ? 0u : pool_state[1];
    const size_t rs = p.wave.capacity;
    for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const uint4 meta = G.pool_meta[i];
        if (meta.w != tag) continue;
        const uint32_t slot = meta.x, d = meta.y;
        const float lumf = __uint_as_float(meta.z);
        const uint32_t cnt = p.wave.rec_n[slot];
        float sum = 0.0f;
        for (uint32_t k = 0; k < cnt; ++k) {
            const float4 r = p.wave.rec[(size_t)k * rs + slot];
            if ((__float_as_uint(r.w) >> 24) > d) sum += ((r.x + r.y) + r.z) / 3.0f;
        }
        G.pool_w[i] = lumf > 0.0f && isfinite(sum / lumf) ? sum / lumf : 0.0f;
    }
}

__global__ void k_train_mark(uint32_t* pool_state, uint32_t cap) {
    pool_state[1] = min(pool_state[0], cap);
}

// -----------------------------------------------------------------------------------------
// host launchers
// -----------------------------------------------------------------------------------------
cudaError_t launch_guide(const Params& p, int depth, uint32_t* pool_state, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_guide<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trg::kG2Bytes);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_guide<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trg::kG2Bytes);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    if (p.multi.scenes) {
        static int grid = 0;
        if (!grid) grid = trg::resident_grid(dev, reinterpret_cast<const void*>(k_guide<true>), 128, trg::kG2Bytes, 128);
        k_guide<true><<<grid, 128, trg::kG2Bytes, s>>>(p, depth, pool_state);
    } else {
        static int grid = 0;
        if (!grid) grid = trg::resident_grid(dev, reinterpret_cast<const void*>(k_guide<false>), 128, trg::kG2Bytes, 128);
        k_guide<false><<<grid, 128, trg::kG2Bytes, s>>>(p, depth, pool_state);
    }
    return cudaGetLastError();
}

cudaError_t launch_train_gather(const Params& p, uint32_t* pool_state, cudaStream_t s) {
    k_train_gather<<<256, 256, 0, s>>>(p, pool_state);
    if (!p.guide.tag) k_train_mark<<<1, 1, 0, s>>>(pool_state, p.guide.pool_cap);
    return cudaGetLastError();
}

}  // namespace trk
