// tr_kernels.cu - wavefront transient path tracing kernels for sm_100a.
//
// Pipeline per batch of path slots (one slot = one camera sample x incoming sample):
//   raygen  -> camera ray, per-path PCG32 stream, optional free-flight distance
//   for depth in [0, max_bounces):
//     extend  (persistent, closest hit, shared-memory stack)
//     shade   (vertex, next-event estimate -> shadow queue, Russian roulette, new direction
//              -> next extend queue; queues compacted with warp ballots)
//     shadow  (persistent, any hit) -> splat record per surviving connection
//   splat   (per group of pixels: records -> shared-memory FP32 (pixel, bin) tile with
//            warp-aggregated atomics -> FP64 film in HBM)
// Reference path: src/Integrator/BidirectionalPathTracing.h:485-692,975-1140 and
// src/Film/StreakCameraFilm.h:139-192 (details at each kernel).
#include <cuda_bf16.h>

#include "tr_device.cuh"
#include "tr_guide_math.cuh"
#include "tr_tcgen05.cuh"
#include "tr_kernels.cuh"

namespace trk {
using namespace trd;

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// -----------------------------------------------------------------------------------------
// BVH traversal: two-child 64-byte nodes, near-first, conservative slab test (Ize 2013),
// watertight triangle test, per-thread stack in shared memory (strided by block size).
// Closest hit: smallest t in (tnear, tfar], ties -> lower triangle id (order independent).
// -----------------------------------------------------------------------------------------
template <bool kAnyHit>
__device__ __forceinline__ uint32_t traverse(const SceneDev& sc, const WRay& r, float tfar,
                                             float& t_out, float& u_out, float& v_out,
                                             int* __restrict__ stack, int stride) {
    float best = tfar;
    uint32_t bid = kInvalid;
    float bu = 0.f, bv = 0.f;
    int sp = 0;
    int node = 0;
    const float ox = r.o.x, oy = r.o.y, oz = r.o.z;
    const float ix = r.inv.x, iy = r.inv.y, iz = r.inv.z;
    for (;;) {
        while (node >= 0) {
            const float4* np = sc.nodes + 4 * node;
            const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2);
            const int4 d = __ldg(reinterpret_cast<const int4*>(np + 3));
            float lx0 = (a.x - ox) * ix, hx0 = (a.y - ox) * ix;
            float ly0 = (a.z - oy) * iy, hy0 = (a.w - oy) * iy;
            float lz0 = (c.x - oz) * iz, hz0 = (c.y - oz) * iz;
            float lx1 = (b.x - ox) * ix, hx1 = (b.y - ox) * ix;
            float ly1 = (b.z - oy) * iy, hy1 = (b.w - oy) * iy;
            float lz1 = (c.z - oz) * iz, hz1 = (c.w - oz) * iz;
            float tmin0 = fmaxf(fmaxf(fminf(lx0, hx0), fminf(ly0, hy0)), fmaxf(fminf(lz0, hz0), r.tnear));
            float tmax0 = fminf(fminf(fmaxf(lx0, hx0), fmaxf(ly0, hy0)), fminf(fmaxf(lz0, hz0), best)) * 1.00000036f;
            float tmin1 = fmaxf(fmaxf(fminf(lx1, hx1), fminf(ly1, hy1)), fmaxf(fminf(lz1, hz1), r.tnear));
            float tmax1 = fminf(fminf(fmaxf(lx1, hx1), fmaxf(ly1, hy1)), fminf(fmaxf(lz1, hz1), best)) * 1.00000036f;
            const bool h0 = tmin0 <= tmax0, h1 = tmin1 <= tmax1;
            if (h0 && h1) {
                const bool first0 = tmin0 <= tmin1;
                stack[sp * stride] = first0 ? d.y : d.x;
                ++sp;
                node = first0 ? d.x : d.y;
            } else if (h0) {
                node = d.x;
            } else if (h1) {
                node = d.y;
            } else {
                if (sp == 0) goto done;
                --sp;
                node = stack[sp * stride];
            }
        }
        {
            const uint32_t ref = (uint32_t)(~node);
            const uint32_t first = ref >> 3, cnt = ref & 7u;
            for (uint32_t k = 0; k < cnt; ++k) {
                const float4* tp = sc.tris + 3 * (first + k);
                const float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
                const uint32_t id = __float_as_uint(q0.w);
                float t, u, v;
                if (wt_hit(r, f3of(q0), f3of(q1), f3of(q2), best, t, u, v)) {
                    if (t < best || bid == kInvalid || id < bid) {
                        best = t; bid = id; bu = u; bv = v;
                        if (kAnyHit) goto done;
                    }
                }
            }
        }
        if (sp == 0) break;
        --sp;
        node = stack[sp * stride];
    }
done:
    t_out = bid == kInvalid ? tfar : best;
    u_out = bu; v_out = bv;
    return bid;
}

// -----------------------------------------------------------------------------------------
// raygen: StratifiedSampler::get_next_sample (StratifiedSampler.h:47-89),
// Film::window_coords2image_coords (Film.h:222-225), PinholeCamera::get_ray_direction
// (PinholeCamera.h:82-91); per-path PCG32 stream; free flight in a world medium
// (BidirectionalPathTracing.h:240-268).
// -----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_raygen(Params p) {
    const Batch& B = p.batch;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B.n_slots) return;
    const uint32_t per_pix = B.ns * B.ninc;
    const uint32_t pl = i / per_pix;
    const uint32_t rem = i - pl * per_pix;
    const uint32_t sl = rem / B.ninc;
    const uint32_t j = rem - sl * B.ninc;
    const uint32_t wpix = B.pix_begin + pl;
    const uint32_t py = B.win_y0 + wpix / B.win_w;
    const uint32_t px = B.win_x0 + wpix % B.win_w;
    const unsigned long long s = B.s0 + sl;
    const uint32_t W = p.film.W, H = p.film.H;
    const uint32_t pixel = py * W + px;

    const uint32_t strata = p.sqrt_spp;
    const uint32_t spp = strata * strata;
    const uint32_t st = (uint32_t)(s % spp);
    const uint32_t subx = st % strata, suby = st / strata;
    Pcg cr;
    pcg_seed(cr, p.seed, cam_id(pixel, s));
    const float inv = 1.0f / (float)strata;
    const float shx = ((float)subx + pcg_float(cr)) * inv;
    const float shy = ((float)suby + pcg_float(cr)) * inv;
    const float posx = fminf((float)px + shx, nextafterf((float)(px + 1), 0.0f));
    const float posy = fminf((float)py + shy, nextafterf((float)(py + 1), 0.0f));
    const float Wf = (float)W, Hf = (float)H;
    const float ratio = Wf / Hf;
    const float imx = (posx - Wf / 2.0f) / Wf;
    const float imy = ((posy - Hf / 2.0f) / Hf) / ratio;
    const CameraDev& c = p.cam;
    const f3 nv = mk(c.nv[0], c.nv[1], c.nv[2]);
    const f3 uv = mk(c.uv[0], c.uv[1], c.uv[2]);
    const f3 vv = mk(c.vv[0], c.vv[1], c.vv[2]);
    const f3 dd = ((nv * c.fd) + ((uv * 2.0f) * imx)) - ((vv * 2.0f) * imy);
    const f3 d = normalize(dd);

    Pcg r;
    pcg_seed(r, p.seed + (unsigned long long)(j + 1) * kGolden64, cam_id(pixel, s));
    float dsamp = __int_as_float(0x7f800000);
    if (p.scene.medium) dsamp = -tr_log(pcg_float(r)) / p.scene.lambda;

    p.wave.ray_o[i] = make_float4(c.pos[0], c.pos[1], c.pos[2], dsamp);
    p.wave.ray_d[i] = make_float4(d.x, d.y, d.z, 0.0f);
    p.wave.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    p.wave.rng[i] = r.state;
    p.wave.rec_n[i] = 0;
}

// -----------------------------------------------------------------------------------------
// extend / shadow: persistent warps fetch 32 queue entries at a time.
// -----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_extend(Params p, int depth) {
    extern __shared__ int stack[];     // [bvh depth + 1][kTraceBlock]
    const uint32_t n = depth == 0 ? p.batch.n_slots : p.wave.counters[cnt_ext(depth)];
    const uint32_t* q = p.wave.q[depth & 1];
    const unsigned lane = threadIdx.x & 31u;
    uint32_t* cursor = &p.wave.counters[cur_ext(depth)];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.wave.stats[0], (unsigned long long)n);
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(cursor, 32u);
        base = __shfl_sync(kFull, base, 0);
        if (base >= n) break;
        const uint32_t idx = base + lane;
        if (idx < n) {
            const uint32_t slot = depth == 0 ? idx : q[idx];
            const float4 o = p.wave.ray_o[slot];
            const float4 d = p.wave.ray_d[slot];
            WRay r;
            wray_setup(r, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), kSigmaVis);
            float t, u, v;
            const uint32_t id = traverse<false>(p.scene, r, o.w, t, u, v, stack + threadIdx.x, kTraceBlock);
            p.wave.hit[slot] = make_float4(t, __uint_as_float(id), u, v);
        }
    }
}

__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_shadow(Params p, int depth) {
    extern __shared__ int stack[];     // [bvh depth + 1][kTraceBlock]
    const uint32_t n = p.wave.counters[cnt_sh(depth)];
    const unsigned lane = threadIdx.x & 31u;
    uint32_t* cursor = &p.wave.counters[cur_sh(depth)];
    const size_t rs = p.wave.capacity;          // record stride: records are [bounce][slot]
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.wave.stats[1], (unsigned long long)n);
    unsigned long long splats = 0;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(cursor, 32u);
        base = __shfl_sync(kFull, base, 0);
        if (base >= n) break;
        const uint32_t idx = base + lane;
        if (idx < n) {
            const float4 o = p.wave.sh_o[idx];
            const float4 d = p.wave.sh_d[idx];
            WRay r;
            wray_setup(r, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), kSigmaVis);
            float t, u, v;
            const uint32_t id = traverse<true>(p.scene, r, o.w, t, u, v, stack + threadIdx.x, kTraceBlock);
            if (id == kInvalid) {
                const float4 L = p.wave.sh_L[idx];
                const uint32_t slot = __float_as_uint(L.w);
                const uint32_t k = p.wave.rec_n[slot];
                p.wave.rec[(size_t)k * rs + slot] = make_float4(L.x, L.y, L.z, d.w);
                p.wave.rec_n[slot] = (uint8_t)(k + 1);
                ++splats;
            }
        }
    }
    if (splats) atomicAdd(&p.wave.stats[2], splats);
}

// -----------------------------------------------------------------------------------------
// shade: one path vertex.  Follows generate_path (BidirectionalPathTracing.h:485-644) for the
// free-flight correction (:273-307), throughput and time update (:588-615) and termination
// (:447-481); connect_paths/connect_vertex_with_light (:975-1045, :649-692) for the
// next-event estimate with Path::Vertex::compute_scattering / compute_attenuation
// (Path.h:183-256); Lambertian cosine sampling in the Intersection frame (Lambertian.h:106-122,
// Intersection.h:167-178) or Henyey-Greenstein sampling (HenyeyGreensteinPhaseFunction.h:218-276).
// -----------------------------------------------------------------------------------------
__device__ __forceinline__ float hg_eval(float g, float cs) {
    const float gg = g * g;
    const float b = (1.0f + gg) - (2.0f * g) * cs;
    return ((1.0f - gg) * kInv4Pi) / (b * sqrtf(b));
}

// GGX microfacet reflection (no reference counterpart): D, height-correlated Smith G2 and
// Schlick F of Walter et al. 2007; visible-normal sampling of Heitz 2018 (JCGT 7(4)); local
// frame around the geometric normal by Duff et al. 2017.  Reflection only; the back side absorbs.
struct Frame3 { f3 t1, t2, n; };
__device__ __forceinline__ Frame3 make_frame(f3 n) {
    const float sg = copysignf(1.0f, n.z);
    const float a = -1.0f / (sg + n.z);
    const float b = n.x * n.y * a;
    return Frame3{mk(1.0f + sg * n.x * n.x * a, sg * b, -sg * n.x), mk(b, sg + n.y * n.y * a, -n.y), n};
}
__device__ __forceinline__ f3 to_local(const Frame3& F, f3 w) { return mk(dot(w, F.t1), dot(w, F.t2), dot(w, F.n)); }
__device__ __forceinline__ f3 to_world(const Frame3& F, f3 l) { return ((F.t1 * l.x) + (F.t2 * l.y)) + (F.n * l.z); }
__device__ __forceinline__ float ggx_D(float a2, float hz) {
    const float c = hz * hz;
    const float d = c * (a2 - 1.0f) + 1.0f;
    return a2 / ((3.14159274f * d) * d);
}
__device__ __forceinline__ float ggx_lambda(float a2, f3 w) {
    const float t2 = (w.x * w.x + w.y * w.y) / (w.z * w.z);
    return (-1.0f + sqrtf(1.0f + a2 * t2)) * 0.5f;
}
__device__ __forceinline__ float schlick(float f0, float c) {
    const float m = 1.0f - c;
    const float m2 = m * m;
    return f0 + (1.0f - f0) * ((m2 * m2) * m);
}
// f(wo, wi) * max(0, n.wi)
__device__ __forceinline__ f3 ggx_eval_cos(f3 kd, float alpha, f3 n, f3 wo_w, f3 wi_w) {
    const Frame3 F = make_frame(n);
    const f3 wo = to_local(F, wo_w), wi = to_local(F, wi_w);
    if (!(wo.z > 0.0f) || !(wi.z > 0.0f)) return mk(0.0f, 0.0f, 0.0f);
    const f3 h = normalize(wo + wi);
    const float a2 = alpha * alpha;
    const float D = ggx_D(a2, h.z);
    const float G2 = 1.0f / ((1.0f + ggx_lambda(a2, wo)) + ggx_lambda(a2, wi));
    float c = dot(wo, h);
    if (c < 0.0f) c = 0.0f;
    const float common = (D * G2) / (4.0f * wo.z);
    return mk(schlick(kd.x, c) * common, schlick(kd.y, c) * common, schlick(kd.z, c) * common);
}
__device__ __forceinline__ bool ggx_sample(f3 kd, float alpha, f3 n, f3 wo_w, float sp, float cp, float x2,
                                           f3& wi_w, f3& fa, float& pa) {
    const Frame3 F = make_frame(n);
    const f3 wo = to_local(F, wo_w);
    if (!(wo.z > 0.0f)) return false;
    const f3 Vh = normalize(mk(alpha * wo.x, alpha * wo.y, wo.z));
    const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    const f3 T1 = lensq > 0.0f ? divs(mk(-Vh.y, Vh.x, 0.0f), sqrtf(lensq)) : mk(1.0f, 0.0f, 0.0f);
    const f3 T2 = cross(Vh, T1);
    const float r = sqrtf(x2);
    const float t1 = r * cp;
    float t2 = r * sp;
    const float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    const float tz2 = (1.0f - t1 * t1) - t2 * t2;
    const float tz = sqrtf(tz2 > 0.0f ? tz2 : 0.0f);
    const f3 Nh = ((T1 * t1) + (T2 * t2)) + (Vh * tz);
    const f3 h = normalize(mk(alpha * Nh.x, alpha * Nh.y, Nh.z > 0.0f ? Nh.z : 0.0f));
    float c = dot(wo, h);
    const f3 wi = (h * (2.0f * c)) - wo;
    if (!(wi.z > 0.0f)) return false;
    const float a2 = alpha * alpha;
    const float Lo = ggx_lambda(a2, wo), Li = ggx_lambda(a2, wi);
    const float G1 = 1.0f / (1.0f + Lo);
    const float G2 = 1.0f / ((1.0f + Lo) + Li);
    const float pdf = (G1 * ggx_D(a2, h.z)) / (4.0f * wo.z);
    const float w = G2 / G1;
    if (c < 0.0f) c = 0.0f;
    fa = mk((schlick(kd.x, c) * w) * pdf, (schlick(kd.y, c) * w) * pdf, (schlick(kd.z, c) * w) * pdf);
    pa = pdf;
    wi_w = normalize(to_world(F, wi));
    return true;
}

__device__ __forceinline__ bool finite3(float a, float b, float c) {
    return isfinite(a) && isfinite(b) && isfinite(c);
}

// Features of a surface vertex for the learned proposal (64 BF16 values, 46 used):
// sin/cos(2^k pi p_d) for k = 0..5 (index 6k + 2d + {0,1}), p normalised to the scene box,
// geometric normal, outgoing direction, path length / film time length.
__device__ __forceinline__ void write_features(uint4* row, const SceneDev& sc, f3 pos, f3 nrm, f3 wo, float tn) {
    float v[64];
    const float pn[3] = {(pos.x - sc.bmin[0]) * sc.binv[0], (pos.y - sc.bmin[1]) * sc.binv[1],
                         (pos.z - sc.bmin[2]) * sc.binv[2]};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float f = (float)(1 << k);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            float sv, cv;
            sincospif(f * pn[d], &sv, &cv);
            v[6 * k + 2 * d] = sv;
            v[6 * k + 2 * d + 1] = cv;
        }
    }
    v[36] = pn[0]; v[37] = pn[1]; v[38] = pn[2];
    v[39] = nrm.x; v[40] = nrm.y; v[41] = nrm.z;
    v[42] = wo.x; v[43] = wo.y; v[44] = wo.z;
    v[45] = tn;
#pragma unroll
    for (int k = 46; k < 64; ++k) v[k] = 0.0f;
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

template <bool kGuided>
__global__ void __launch_bounds__(256) k_shade(Params p, int depth) {
    const SceneDev& sc = p.scene;
    const uint32_t n = depth == 0 ? p.batch.n_slots : p.wave.counters[cnt_ext(depth)];
    const uint32_t* qin = p.wave.q[depth & 1];
    uint32_t* qout = p.wave.q[(depth + 1) & 1];
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const bool medium = sc.medium != 0;
    const f3 sig_s = mk(sc.sig_s[0], sc.sig_s[1], sc.sig_s[2]);
    const f3 sig_t = mk(sc.sig_t[0], sc.sig_t[1], sc.sig_t[2]);
    const float lambda = sc.lambda;
    const float g = sc.g;
    const float total_time = (float)p.film.T * p.film.exposure + p.film.offset;
    const float inv_inc = 1.0f / (float)p.batch.ninc;
    const uint32_t per_pix = p.batch.ns * p.batch.ninc;

    for (uint32_t base = warp_global * 32u; base < n; base += nwarps * 32u) {
        const uint32_t idx = base + lane;
        bool want_shadow = false, want_next = false, want_guide = false;
        uint32_t slot = 0;
        float4 sh_o = make_float4(0, 0, 0, 0), sh_d = make_float4(0, 0, 0, 0), sh_L = make_float4(0, 0, 0, 0);
        if (idx < n) {
            slot = depth == 0 ? idx : qin[idx];
            const float4 h = p.wave.hit[slot];
            const float4 ro = p.wave.ray_o[slot];
            const float4 rd = p.wave.ray_d[slot];
            const float4 th = p.wave.thr[slot];
            const uint32_t id = __float_as_uint(h.y);
            const bool hit = id != kInvalid;
            const float dsamp = ro.w;
            const bool surface = hit && (!medium || h.x < dsamp);
            if (medium || hit) {
                // per-path RNG: state in memory, increment from the camera sample
                const uint32_t pl = slot / per_pix;
                const uint32_t sl = (slot - pl * per_pix) / p.batch.ninc;
                const uint32_t wpix = p.batch.pix_begin + pl;
                const uint32_t pixel = (p.batch.win_y0 + wpix / p.batch.win_w) * p.film.W +
                                       (p.batch.win_x0 + wpix % p.batch.win_w);
                Pcg rng;
                rng.state = p.wave.rng[slot];
                rng.inc = (cam_id(pixel, p.batch.s0 + sl) << 1u) | 1ull;

                float dist, pd;
                if (surface) { dist = h.x; pd = medium ? tr_exp(-(dist * lambda)) : 1.0f; }
                else { dist = dsamp; pd = tr_exp(-(dist * lambda)) * lambda; }
                const float ptot = th.w * pd;
                f3 f;
                if (medium) {
                    f = mk((th.x * tr_exp(-(dist * sig_t.x))) / ptot, (th.y * tr_exp(-(dist * sig_t.y))) / ptot,
                           (th.z * tr_exp(-(dist * sig_t.z))) / ptot);
                } else {
                    f = mk(th.x / ptot, th.y / ptot, th.z / ptot);
                }
                const float time = rd.w + dist;
                const f3 org = mk(ro.x, ro.y, ro.z), dir = mk(rd.x, rd.y, rd.z);
                const f3 pos = org + dir * dist;
                if (!(time > total_time)) {
                    f3 nrm = mk(0.f, 0.f, 0.f), kd = mk(0.f, 0.f, 0.f);
                    bool ggx = false;
                    float alpha = 0.0f;
                    if (surface) {
                        const float4 ng = __ldg(&sc.tri_ng[id]);
                        nrm = mk(ng.x, ng.y, ng.z);
                        const uint32_t mi = __float_as_uint(ng.w);
                        const float4 m = __ldg(&sc.mats[mi]);
                        kd = mk(m.x, m.y, m.z);
                        ggx = __float_as_uint(m.w) == 1u;
                        if (ggx) alpha = __ldg(&sc.mats2[mi]).x;
                    }
                    const f3 wo = mk(-dir.x, -dir.y, -dir.z);
                    // ---- next-event estimate ----
                    {
                        const float xl = pcg_float(rng);
                        uint32_t li = (uint32_t)(xl * (float)sc.num_lights);
                        if (li >= sc.num_lights) li = sc.num_lights - 1;
                        const float4* L = sc.lights + 5 * li;
                        const float4 L0 = __ldg(L), L1 = __ldg(L + 1);
                        const bool rect = __float_as_uint(L0.w) == 1u;
                        float pl_ = 1.0f / (float)sc.num_lights;
                        f3 lp = mk(L0.x, L0.y, L0.z);
                        if (rect) {
                            const float xu = pcg_float(rng), xv = pcg_float(rng);
                            const float4 L2 = __ldg(L + 2), L3 = __ldg(L + 3);
                            lp = (lp + f3of(L2) * xu) + f3of(L3) * xv;
                            pl_ = pl_ * (1.0f / L1.w);
                        }
                        f3 ld = pos - lp;
                        const float d2 = dot(ld, ld);
                        const float dl = sqrtf(d2);
                        ld = divs(ld, dl);
                        bool ok = true;
                        f3 irr;
                        if (rect) {
                            const float4 L4 = __ldg(L + 4);
                            const float dot_l = dot(ld, f3of(L4));
                            if (!(dot_l > 0.0f)) ok = false;
                            const float a = dot_l / (dl * dl);
                            irr = mk(L1.x * a, L1.y * a, L1.z * a);
                        } else {
                            irr = mk(L1.x / d2, L1.y / d2, L1.z / d2);
                        }
                        if (ok) {
                            const f3 wl = mk(-ld.x, -ld.y, -ld.z);
                            f3 fe;
                            if (surface && ggx) {
                                fe = ggx_eval_cos(kd, alpha, nrm, wo, wl);
                            } else if (surface) {
                                const float cs = dot(wl, nrm);
                                const float cl = cs > 0.0f ? cs : 0.0f;
                                fe = mk((kd.x * kInvPi) * cl, (kd.y * kInvPi) * cl, (kd.z * kInvPi) * cl);
                            } else {
                                const float ph = hg_eval(g, dot(dir, wl));
                                fe = mk(ph * sig_s.x, ph * sig_s.y, ph * sig_s.z);
                            }
                            f3 att = mk(1.0f, 1.0f, 1.0f);
                            if (medium)
                                att = mk(tr_exp(-(sig_t.x * dl)), tr_exp(-(sig_t.y * dl)), tr_exp(-(sig_t.z * dl)));
                            const float scale = inv_inc / pl_;
                            const float Lr = (f.x * (fe.x * (irr.x * att.x))) * scale;
                            const float Lg = (f.y * (fe.y * (irr.y * att.y))) * scale;
                            const float Lb = (f.z * (fe.z * (irr.z * att.z))) * scale;
                            const float tt = time + dl;
                            const float ps = (tt - p.film.offset) / p.film.exposure;
                            if (ps < (float)p.film.T && ps >= 0.0f && finite3(Lr, Lg, Lb) &&
                                (Lr != 0.0f || Lg != 0.0f || Lb != 0.0f)) {
                                want_shadow = true;
                                sh_o = make_float4(lp.x, lp.y, lp.z, dl - kSigmaVis);
                                sh_d = make_float4(ld.x, ld.y, ld.z,
                                                   __uint_as_float((uint32_t)floorf(ps) | ((uint32_t)depth << 24)));
                                sh_L = make_float4(Lr, Lg, Lb, __uint_as_float(slot));
                            }
                        }
                    }
                    if ((uint32_t)depth + 1u < p.max_bounces) {
                        // ---- Russian roulette ----
                        const float albedo = surface ? avg3(kd)
                            : avg3(mk(sig_s.x / sig_t.x, sig_s.y / sig_t.y, sig_s.z / sig_t.z));
                        if (kGuided && surface && !(pcg_float(rng) > albedo)) {
                            // ---- direction deferred to the learned proposal (k_guide_sample) ----
                            p.wave.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, 0.0f);
                            p.wave.ray_d[slot] = make_float4(dir.x, dir.y, dir.z, time);
                            p.wave.thr[slot] = make_float4(f.x, f.y, f.z, albedo);
                            want_guide = true;
                        } else if ((!kGuided || !surface) && !(pcg_float(rng) > albedo)) {
                            // ---- outgoing direction ----
                            const float x1 = pcg_float(rng), x2 = pcg_float(rng);
                            float sp, cp;
                            tr_sincos2pi(x1, &sp, &cp);
                            f3 fa, nd;
                            float pa;
                            bool alive = true;
                            if (surface && ggx) {
                                alive = ggx_sample(kd, alpha, nrm, wo, sp, cp, x2, nd, fa, pa);
                            } else if (surface && (p.flags & kFlagOrthoFrame)) {
                                // cosine sampling in an orthonormal frame (Duff et al. 2017)
                                const float ct = sqrtf(x2);
                                const float stt = sqrtf(1.0f - ct * ct);
                                const Frame3 Fr = make_frame(nrm);
                                nd = to_world(Fr, mk(cp * stt, sp * stt, ct));
                                fa = mk((kd.x * kInvPi) * ct, (kd.y * kInvPi) * ct, (kd.z * kInvPi) * ct);
                                pa = ct * kInvPi;
                            } else if (surface) {
                                const float ct = sqrtf(x2);
                                const float stt = sqrtf(1.0f - ct * ct);
                                const f3 aux = fabsf(nrm.x) > fabsf(nrm.z) ? mk(-nrm.y, nrm.x, nrm.z)
                                                                           : mk(0.0f, -nrm.z, nrm.y);
                                const f3 tv = normalize(aux);
                                const f3 tu = cross(nrm, tv);
                                const f3 w = ((tu * (cp * stt)) + (nrm * ct)) + (tv * (sp * stt));
                                nd = normalize(w);
                                const float ca = fabsf(dot(nrm, nd));
                                fa = mk((kd.x * kInvPi) * ca, (kd.y * kInvPi) * ca, (kd.z * kInvPi) * ca);
                                pa = ct * kInvPi;
                            } else {
                                float ct;
                                if (fabsf(g) < 1e-4f) {
                                    ct = 1.0f - 2.0f * x2;
                                } else {
                                    const float gg = g * g;
                                    const float a = (1.0f - gg) / ((1.0f - g) + (2.0f * g) * x2);
                                    ct = ((1.0f + gg) - a * a) / (2.0f * g);
                                    if (ct < -1.0f) ct = -1.0f;
                                    if (ct > 1.0f) ct = 1.0f;
                                }
                                const float stt = sqrtf(1.0f - ct * ct);
                                // orthonormal frame around the propagation direction (Duff et al. 2017)
                                const float sg = copysignf(1.0f, dir.z);
                                const float aa = -1.0f / (sg + dir.z);
                                const float bb = dir.x * dir.y * aa;
                                const f3 t1 = mk(1.0f + sg * dir.x * dir.x * aa, sg * bb, -sg * dir.x);
                                const f3 t2 = mk(bb, sg + dir.y * dir.y * aa, -dir.y);
                                nd = ((t1 * (cp * stt)) + (t2 * (sp * stt))) + (dir * ct);
                                const float ph = hg_eval(g, ct);
                                fa = mk(ph * sig_s.x, ph * sig_s.y, ph * sig_s.z);
                                pa = ph;
                            }
                            if (alive) {
                                const f3 fn = mulv(f, fa);
                                float nds = __int_as_float(0x7f800000);
                                if (medium) nds = -tr_log(pcg_float(rng)) / lambda;
                                p.wave.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, nds);
                                p.wave.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, time);
                                p.wave.thr[slot] = make_float4(fn.x, fn.y, fn.z, albedo * pa);
                                want_next = true;
                            }
                        }
                    }
                }
                p.wave.rng[slot] = rng.state;
            }
        }
        // ---- warp-aggregated queue appends (order preserved within the warp) ----
        const unsigned ms = __ballot_sync(kFull, want_shadow);
        const unsigned mn = __ballot_sync(kFull, want_next);
        uint32_t bs = 0, bn = 0;
        if (lane == 0) {
            if (ms) bs = atomicAdd(&p.wave.counters[cnt_sh(depth)], (uint32_t)__popc(ms));
            if (mn) bn = atomicAdd(&p.wave.counters[cnt_ext(depth + 1)], (uint32_t)__popc(mn));
        }
        bs = __shfl_sync(kFull, bs, 0);
        bn = __shfl_sync(kFull, bn, 0);
        const unsigned lt = lanemask_lt();
        if (want_shadow) {
            const uint32_t k = bs + (uint32_t)__popc(ms & lt);
            p.wave.sh_o[k] = sh_o;
            p.wave.sh_d[k] = sh_d;
            p.wave.sh_L[k] = sh_L;
        }
        if (want_next) qout[bn + (uint32_t)__popc(mn & lt)] = slot;
        if (kGuided) {
            const unsigned mg = __ballot_sync(kFull, want_guide);
            uint32_t bg = 0;
            if (lane == 0 && mg) bg = atomicAdd(&p.wave.counters[cnt_guide(depth)], (uint32_t)__popc(mg));
            bg = __shfl_sync(kFull, bg, 0);
            if (want_guide) p.guide.gq[bg + (uint32_t)__popc(mg & lt)] = slot;
        }
    }
}

// -----------------------------------------------------------------------------------------
// guided direction sampling (no reference counterpart): one-sample multiple importance
// sampling (Veach & Guibas 1995, balance heuristic) between the learned vMF mixture (chosen
// with probability mix_prob) and the BSDF sampler, so the estimator stays unbiased whatever
// the network predicts.  Directions below the surface carry no reflectance and end the path.
// -----------------------------------------------------------------------------------------
__device__ __forceinline__ float ggx_pdf(float alpha, f3 n, f3 wo_w, f3 wi_w) {
    const Frame3 F = make_frame(n);
    const f3 wo = to_local(F, wo_w), wi = to_local(F, wi_w);
    if (!(wo.z > 0.0f) || !(wi.z > 0.0f)) return 0.0f;
    const f3 h = normalize(wo + wi);
    const float a2 = alpha * alpha;
    const float G1 = 1.0f / (1.0f + ggx_lambda(a2, wo));
    return (G1 * ggx_D(a2, h.z)) / (4.0f * wo.z);
}

// Fused proposal inference and sampling: one CTA of 128 threads owns 128 guided vertices at a
// time.  Each thread gathers its vertex, writes its 64 BF16 features as row `tid` of the A tile
// in shared memory, the four layers run on the tensor cores (trg::layer_mma, accumulators in
// tensor memory), and the epilogue decodes the thread's mixture from the last layer's
// accumulator row in registers and samples the direction.  Neither features nor mixtures touch
// HBM.  Four CTAs per SM (50 KB shared memory, 64 TMEM columns each) overlap one CTA's MMA waits
// with the others' gathers.
__global__ void __launch_bounds__(128, 4) k_guide(Params p, int depth, uint32_t* pool_count) {
    const GuideWave& G = p.guide;
    const uint32_t n = p.wave.counters[cnt_guide(depth)];
    if (blockIdx.x * (uint32_t)trg::kTile >= n) return;     // no tile for this CTA
    extern __shared__ __align__(1024) uint8_t smem[];
    const SceneDev& sc = p.scene;
    uint8_t* sA = smem + trg::kSmemA;
    const float* sB = reinterpret_cast<const float*>(smem + trg::kSmemBias);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + trg::kSmemBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + trg::kSmemSlot);
    volatile int* s_ok = reinterpret_cast<volatile int*>(smem + trg::kSmemOk);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    trg::stage_weights(smem, G.net.w_fwd, G.net.bias);
    if (tid == 0) { trg::mbar_init(bar, 1); trg::fence_mbar_init(); }
    if (warp == 0) { trg::tmem_alloc(tslot, 64); trg::tmem_relinquish(); }
    trg::tc_fence_before();
    __syncthreads();
    trg::tc_fence_after();
    const uint32_t taddr = *tslot;
    const uint32_t lane_addr = taddr + ((32u * warp) << 16);
    uint32_t phase = 0;
    bool ok = true;

    uint32_t* qout = p.wave.q[(depth + 1) & 1];
    const bool medium = sc.medium != 0;
    const uint32_t per_pix = p.batch.ns * p.batch.ninc;
    const float total_time = (float)p.film.T * p.film.exposure + p.film.offset;
    const float c = G.mix_prob;
    const unsigned lane = tid & 31u;
    for (uint32_t tile = blockIdx.x; tile * (uint32_t)trg::kTile < n && ok; tile += gridDim.x) {
        const uint32_t idx = tile * (uint32_t)trg::kTile + tid;
        const bool active = idx < n;
        uint32_t slot = 0, mi = 0;
        float4 ro = make_float4(0.f, 0.f, 0.f, 0.f), rd = ro, th = ro;
        f3 nrm = mk(0.f, 0.f, 1.f);
        {
            uint4 feat[8];
            if (active) {
                slot = G.gq[idx];
                ro = p.wave.ray_o[slot];
                rd = p.wave.ray_d[slot];
                th = p.wave.thr[slot];
                const float4 ng = __ldg(&sc.tri_ng[__float_as_uint(p.wave.hit[slot].y)]);
                nrm = mk(ng.x, ng.y, ng.z);
                mi = __float_as_uint(ng.w);
                write_features(feat, sc, mk(ro.x, ro.y, ro.z), nrm, mk(-rd.x, -rd.y, -rd.z), rd.w / total_time);
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) feat[q] = make_uint4(0u, 0u, 0u, 0u);
            }
            trg::store_row_a(sA, tid, feat);
        }
        float o[48];
        for (uint32_t l = 0; l < 4; ++l) {
            ok = trg::layer_mma(taddr, trg::smem_u32(sA), trg::smem_u32(smem + trg::kSmemW + l * 8192u), bar, phase, s_ok);
            if (!ok) break;
            if (l < 3) {
                float a[64];
#pragma unroll
                for (int j = 0; j < 4; ++j) trg::tmem_ld16(lane_addr + 16u * j, a + 16 * j);
                trg::tmem_wait_ld();
                uint4 h[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    float t[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) t[e] = fmaxf(a[8 * q + e] + sB[l * 64 + 8 * q + e], 0.0f);
                    h[q] = make_uint4(trg::pack2(t[0], t[1]), trg::pack2(t[2], t[3]), trg::pack2(t[4], t[5]),
                                      trg::pack2(t[6], t[7]));
                }
                trg::store_row_a(sA, tid, h);
            } else {
#pragma unroll
                for (int j = 0; j < 3; ++j) trg::tmem_ld16(lane_addr + 16u * j, o + 16 * j);
                trg::tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < trg::kOut; ++j) o[j] += sB[3 * 64 + j];
            }
        }
        if (!ok) break;

        // ---- one-sample MIS between the mixture and the BSDF ----
        bool want_next = false;
        if (active) {
            const float4 m = __ldg(&sc.mats[mi]);
            const f3 kd = mk(m.x, m.y, m.z);
            const bool ggx = __float_as_uint(m.w) == 1u;
            const float alpha = ggx ? __ldg(&sc.mats2[mi]).x : 0.0f;
            const f3 pos = mk(ro.x, ro.y, ro.z);
            const f3 wo = mk(-rd.x, -rd.y, -rd.z);
            const f3 f = mk(th.x, th.y, th.z);
            const uint32_t pl = slot / per_pix;
            const uint32_t sl = (slot - pl * per_pix) / p.batch.ninc;
            const uint32_t wpix = p.batch.pix_begin + pl;
            const uint32_t pixel = (p.batch.win_y0 + wpix / p.batch.win_w) * p.film.W +
                                   (p.batch.win_x0 + wpix % p.batch.win_w);
            Pcg rng;
            rng.state = p.wave.rng[slot];
            rng.inc = (cam_id(pixel, p.batch.s0 + sl) << 1u) | 1ull;
            trg::Lobe L[trg::kLobes];
            trg::decode_mixture(o, L);
            f3 wi = mk(0.f, 0.f, 1.f);
            bool alive = true;
            if (pcg_float(rng) < c) {
                const float u0 = pcg_float(rng), u1 = pcg_float(rng), u2 = pcg_float(rng);
                float d[3];
                trg::mixture_sample(L, u0, u1, u2, d);
                wi = normalize(mk(d[0], d[1], d[2]));
            } else {
                const float x1 = pcg_float(rng), x2 = pcg_float(rng);
                float sp, cp;
                tr_sincos2pi(x1, &sp, &cp);
                if (ggx) {
                    f3 fa;
                    float pa;
                    alive = ggx_sample(kd, alpha, nrm, wo, sp, cp, x2, wi, fa, pa);
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
                    fcos = ggx_eval_cos(kd, alpha, nrm, wo, wi);
                    pb = ggx_pdf(alpha, nrm, wo, wi);
                } else {
                    const float cs = dot(nrm, wi);
                    const float cl = cs > 0.0f ? cs : 0.0f;
                    fcos = mk((kd.x * kInvPi) * cl, (kd.y * kInvPi) * cl, (kd.z * kInvPi) * cl);
                    pb = cl * kInvPi;
                }
                const float pdf = c * trg::mixture_pdf(L, wi.x, wi.y, wi.z) + (1.0f - c) * pb;
                if (pdf > 0.0f && (fcos.x > 0.0f || fcos.y > 0.0f || fcos.z > 0.0f) && isfinite(pdf)) {
                    const f3 fn = mulv(f, fcos);
                    const bool keep = G.pool_cap > 0 && pcg_float(rng) < G.keep_prob;
                    float nds = __int_as_float(0x7f800000);
                    if (medium) nds = -tr_log(pcg_float(rng)) / sc.lambda;
                    p.wave.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, nds);
                    p.wave.ray_d[slot] = make_float4(wi.x, wi.y, wi.z, rd.w);
                    p.wave.thr[slot] = make_float4(fn.x, fn.y, fn.z, th.w * pdf);
                    want_next = true;
                    if (keep) {
                        const uint32_t k = atomicAdd(pool_count, 1u);
                        if (k < G.pool_cap) {
                            write_features(G.pool_feat + (size_t)k * 8, sc, pos, nrm, wo, rd.w / total_time);
                            G.pool_dir[3 * (size_t)k] = wi.x;
                            G.pool_dir[3 * (size_t)k + 1] = wi.y;
                            G.pool_dir[3 * (size_t)k + 2] = wi.z;
                            G.pool_meta[k] = make_uint4(slot, (uint32_t)depth, __float_as_uint(avg3(f)), 0u);
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
    if (!ok && tid == 0) atomicExch(G.err, 1);
    trg::drain_and_free(taddr, bar, phase, ok);
}

// Training targets of this batch's pool entries: the luminance reaching the film through the
// rest of the path (splat records of later bounces) relative to the throughput at the vertex,
// i.e. an estimate of (incident radiance x f cos / sampling pdf) along the sampled direction.
// pool_state[0] = entries filled, pool_state[1] = entries already given a target.
__global__ void k_train_gather(Params p, const uint32_t* pool_state) {
    const GuideWave& G = p.guide;
    const uint32_t end = min(pool_state[0], G.pool_cap);
    const uint32_t begin = pool_state[1];
    const size_t rs = p.wave.capacity;
    for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        const uint4 meta = G.pool_meta[i];
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
// splat: StreakCameraFilm::add_samples / add_temporal_sample (StreakCameraFilm.h:139-192,
// 279-315) with the box filter of size 1: bin = floor((t - offset) / exposure) (computed in
// shade), streak(pixel, bin) += L, steady(pixel) += L, weight(pixel) += 1 per camera sample.
// A CTA owns `G` whole pixels of the batch, accumulates their records in an FP32 shared-memory
// tile (warp-aggregated atomics on equal (pixel, bin) keys) and adds the tile to the FP64 film.
// -----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kSplatBlock) k_splat(Params p, int G) {
    extern __shared__ __align__(16) float tile[];
    const uint32_t T = p.film.T;
    const uint32_t TT = T * 3u;
    const Batch& B = p.batch;
    const uint32_t pix0 = blockIdx.x * (uint32_t)G;
    if (pix0 >= B.npix) return;
    const uint32_t gp = min((uint32_t)G, B.npix - pix0);
    float* steady = tile + (size_t)G * TT;
    {
        float4* t4 = reinterpret_cast<float4*>(tile);
        const uint32_t n4 = ((uint32_t)G * TT + 3u * G + 3u) / 4u;
        for (uint32_t e = threadIdx.x; e < n4; e += blockDim.x) t4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    const uint32_t per_pix = B.ns * B.ninc;
    const uint32_t nslots = gp * per_pix;
    const uint32_t slot0 = pix0 * per_pix;
    const size_t rs = p.wave.capacity;           // records are [bounce][slot]
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt = lanemask_lt();
    // per-lane running steady-image sums, flushed when the lane moves to another pixel
    uint32_t acc_pl = 0xffffffffu;
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (uint32_t base = (threadIdx.x & ~31u); base < nslots; base += blockDim.x) {
        const uint32_t ls = base + lane;
        const bool act = ls < nslots;
        const uint32_t slot = slot0 + (act ? ls : 0u);
        const uint32_t cnt = act ? (uint32_t)p.wave.rec_n[slot] : 0u;
        const uint32_t pl = act ? ls / per_pix : 0u;
        if (act && pl != acc_pl) {
            if (acc_pl != 0xffffffffu) {
                float* sd = steady + acc_pl * 3u;
                atomicAdd(sd, ax); atomicAdd(sd + 1, ay); atomicAdd(sd + 2, az);
            }
            acc_pl = pl; ax = ay = az = 0.f;
        }
        const uint32_t kmax = __reduce_max_sync(kFull, cnt);
        for (uint32_t k = 0; k < kmax; ++k) {
            const bool valid = k < cnt;
            float4 rc = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid) rc = __ldcs(&p.wave.rec[(size_t)k * rs + slot]);     // streamed, read once
            const uint32_t key = valid ? pl * T + (__float_as_uint(rc.w) & 0x00ffffffu) : 0xffffffffu;
            // lanes holding the same (pixel, bin) are summed with shuffles; the group's
            // lowest lane issues one shared-memory atomic per channel
            const unsigned peers = __match_any_sync(kFull, key);
            const int rank = __popc(peers & lt);
            const int gsize = __popc(peers);
            float vx = rc.x, vy = rc.y, vz = rc.z;
            const uint32_t maxg = __reduce_max_sync(kFull, valid ? (uint32_t)gsize : 1u);
            for (int step = 1; step < (int)maxg; step <<= 1) {
                const int src_rank = rank + step;
                const int src = src_rank < gsize ? (int)__fns(peers, 0, src_rank + 1) : (int)lane;
                const float ox = __shfl_sync(kFull, vx, src);
                const float oy = __shfl_sync(kFull, vy, src);
                const float oz = __shfl_sync(kFull, vz, src);
                if ((rank & (2 * step - 1)) == 0 && src_rank < gsize) { vx += ox; vy += oy; vz += oz; }
            }
            if (valid && rank == 0) {
                float* cell = tile + (size_t)key * 3u;
                atomicAdd(cell, vx); atomicAdd(cell + 1, vy); atomicAdd(cell + 2, vz);
            }
            if (valid) { ax += rc.x; ay += rc.y; az += rc.z; }
        }
    }
    if (acc_pl != 0xffffffffu) {
        float* sd = steady + acc_pl * 3u;
        atomicAdd(sd, ax); atomicAdd(sd + 1, ay); atomicAdd(sd + 2, az);
    }
    __syncthreads();
    // flush: FP64 read-add-write of the touched bins (the film starts zeroed); four
    // independent loads in flight per thread
    for (uint32_t pl = 0; pl < gp; ++pl) {
        const uint32_t wpix = B.pix_begin + pix0 + pl;
        const size_t pixel = (size_t)(B.win_y0 + wpix / B.win_w) * p.film.W + (B.win_x0 + wpix % B.win_w);
        double* dst = p.film.streak + pixel * TT;
        const float* src = tile + (size_t)pl * TT;
        for (uint32_t e0 = threadIdx.x; e0 < TT; e0 += 4u * blockDim.x) {
            float v[4];
            double o[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t e = e0 + (uint32_t)u * blockDim.x;
                v[u] = e < TT ? src[e] : 0.0f;
                o[u] = v[u] != 0.0f ? dst[e] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t e = e0 + (uint32_t)u * blockDim.x;
                if (v[u] != 0.0f) dst[e] = o[u] + (double)v[u];
            }
        }
        if (threadIdx.x == 0) {
            p.film.weight[pixel] += (double)B.ns;
            for (int c = 0; c < 3; ++c) p.film.steady[pixel * 3 + c] += (double)steady[pl * 3 + c];
        }
    }
}

// -----------------------------------------------------------------------------------------
// ray-batch queries (World::first_intersection / World::intersects on user rays)
// -----------------------------------------------------------------------------------------
struct HitOut { float t; uint32_t id; float u, v; };

__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_trace_user(SceneDev sc, const float* __restrict__ rays,
                                                            uint32_t n, int any_hit, HitOut* out,
                                                            uint32_t* cursor) {
    extern __shared__ int stack[];     // [bvh depth + 1][kTraceBlock]
    const unsigned lane = threadIdx.x & 31u;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(cursor, 32u);
        base = __shfl_sync(kFull, base, 0);
        if (base >= n) break;
        const uint32_t i = base + lane;
        if (i < n) {
            const float4 a = reinterpret_cast<const float4*>(rays)[2 * (size_t)i];
            const float4 b = reinterpret_cast<const float4*>(rays)[2 * (size_t)i + 1];
            WRay r;
            wray_setup(r, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w);
            float t, u, v;
            uint32_t id = any_hit ? traverse<true>(sc, r, b.w, t, u, v, stack + threadIdx.x, kTraceBlock)
                                  : traverse<false>(sc, r, b.w, t, u, v, stack + threadIdx.x, kTraceBlock);
            out[i] = HitOut{t, id, u, v};
        }
    }
}

// -----------------------------------------------------------------------------------------
// launchers
// -----------------------------------------------------------------------------------------
size_t trace_smem_bytes(uint32_t bvh_depth) { return (size_t)(bvh_depth + 1u) * kTraceBlock * sizeof(int); }

cudaError_t launch_guide(const Params& p, int depth, uint32_t* pool_state, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_guide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trg::kSmemBytes);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    const int grid = trg::resident_grid(dev, reinterpret_cast<const void*>(k_guide), 128, trg::kSmemBytes);
    k_guide<<<grid, 128, trg::kSmemBytes, s>>>(p, depth, pool_state);
    return cudaGetLastError();
}

cudaError_t launch_train_gather(const Params& p, uint32_t* pool_state, cudaStream_t s) {
    k_train_gather<<<256, 256, 0, s>>>(p, pool_state);
    k_train_mark<<<1, 1, 0, s>>>(pool_state, p.guide.pool_cap);
    return cudaGetLastError();
}

int trace_grid_size(int device, uint32_t bvh_depth) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extend, kTraceBlock, trace_smem_bytes(bvh_depth));
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

size_t splat_smem_bytes(uint32_t T, int G) {
    // tile [G][T][3] + steady [G][3] floats, rounded up to whole float4 (zeroed as float4)
    return (((size_t)G * T * 3u + 3u * (size_t)G) * sizeof(float) + 15u) & ~size_t(15);
}

cudaError_t launch_raygen(const Params& p, cudaStream_t s) {
    const uint32_t n = p.batch.n_slots;
    k_raygen<<<(n + 255) / 256, 256, 0, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launch_extend(const Params& p, int depth, int grid, cudaStream_t s) {
    k_extend<<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    return cudaGetLastError();
}
cudaError_t launch_shade(const Params& p, int depth, cudaStream_t s) {
    int dev = 0, grid = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&grid, cudaDevAttrMultiProcessorCount, dev);
    grid *= 8;
    const uint32_t need = (p.batch.n_slots + 255) / 256;
    if ((uint32_t)grid > need) grid = (int)need;
    if (grid < 1) grid = 1;
    if (p.guide.gq) k_shade<true><<<grid, 256, 0, s>>>(p, depth);
    else k_shade<false><<<grid, 256, 0, s>>>(p, depth);
    return cudaGetLastError();
}
cudaError_t launch_shadow(const Params& p, int depth, int grid, cudaStream_t s) {
    k_shadow<<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    return cudaGetLastError();
}
cudaError_t launch_splat(const Params& p, int G, cudaStream_t s) {
    const size_t smem = splat_smem_bytes(p.film.T, G);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_splat, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_set = true;
    }
    const uint32_t blocks = (p.batch.npix + (uint32_t)G - 1) / (uint32_t)G;
    k_splat<<<blocks, kSplatBlock, smem, s>>>(p, G);
    return cudaGetLastError();
}
cudaError_t launch_trace_user(const SceneDev& sc, const float* rays, uint32_t n, int any_hit, void* out,
                              uint32_t* cursor, int grid, cudaStream_t s) {
    k_trace_user<<<grid, kTraceBlock, trace_smem_bytes(sc.bvh_depth), s>>>(sc, rays, n, any_hit,
                                                                          reinterpret_cast<HitOut*>(out), cursor);
    return cudaGetLastError();
}

}  // namespace trk
