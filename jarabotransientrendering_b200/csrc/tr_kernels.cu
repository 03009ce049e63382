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
#include "tr_bsdf.cuh"
#include "tr_device.cuh"
#include "tr_kernels.cuh"

#include <algorithm>

namespace trk {
using namespace trd;


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
template <bool kMulti>
__global__ void __launch_bounds__(256) k_raygen(const __grid_constant__ Params p) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const Batch* Bp = &p.batch;
    const SceneSlot* SS = nullptr;
    if constexpr (kMulti) {
        const BatchDesc& BD = cur_batch(p);
        if (i >= BD.n_slots) return;
        Bp = &seg_of_slot(BD, i);
        SS = p.multi.scenes + Bp->scene;
    } else {
        if (i >= p.batch.n_slots) return;
    }
    const Batch& B = *Bp;
    const FilmDev& film = kMulti ? SS->film : p.film;
    const CameraDev& c = kMulti ? SS->cam : p.cam;
    const unsigned long long seed = kMulti ? SS->seed : p.seed;
    const uint32_t per_pix = B.ns * B.ninc;
    const uint32_t li = i - B.slot_begin;
    const uint32_t pl = li / per_pix;
    const uint32_t rem = li - pl * per_pix;
    const uint32_t sl = rem / B.ninc;
    const uint32_t j = rem - sl * B.ninc;
    const uint32_t wpix = B.pix_begin + pl;
    const uint32_t py = B.win_y0 + wpix / B.win_w;
    const uint32_t px = B.win_x0 + wpix % B.win_w;
    const unsigned long long s = B.s0 + sl;
    const uint32_t W = film.W, H = film.H;
    const uint32_t pixel = py * W + px;

    const uint32_t strata = kMulti ? SS->sqrt_spp : p.sqrt_spp;
    const uint32_t spp = strata * strata;
    const uint32_t st = (uint32_t)(s % spp);
    const uint32_t subx = st % strata, suby = st / strata;
    Pcg cr;
    pcg_seed(cr, seed, cam_id(pixel, s));
    const float inv = 1.0f / (float)strata;
    const float shx = ((float)subx + pcg_float(cr)) * inv;
    const float shy = ((float)suby + pcg_float(cr)) * inv;
    const float posx = fminf((float)px + shx, nextafterf((float)(px + 1), 0.0f));
    const float posy = fminf((float)py + shy, nextafterf((float)(py + 1), 0.0f));
    const float Wf = (float)W, Hf = (float)H;
    const float ratio = Wf / Hf;
    const float imx = (posx - Wf / 2.0f) / Wf;
    const float imy = ((posy - Hf / 2.0f) / Hf) / ratio;
    const f3 nv = mk(c.nv[0], c.nv[1], c.nv[2]);
    const f3 uv = mk(c.uv[0], c.uv[1], c.uv[2]);
    const f3 vv = mk(c.vv[0], c.vv[1], c.vv[2]);
    const f3 dd = ((nv * c.fd) + ((uv * 2.0f) * imx)) - ((vv * 2.0f) * imy);
    const f3 d = normalize(dd);

    const SceneDev& sc = kMulti ? SS->scene : p.scene;
    Pcg r;
    pcg_seed(r, seed + (unsigned long long)(j + 1) * kGolden64, cam_id(pixel, s));
    float dsamp = __int_as_float(0x7f800000);
    if (sc.medium) dsamp = -tr_log(pcg_float(r)) / sc.lambda;

    p.wave.ray_o[i] = make_float4(c.pos[0], c.pos[1], c.pos[2], dsamp);
    p.wave.ray_d[i] = make_float4(d.x, d.y, d.z, 0.0f);
    p.wave.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    p.wave.rng[i] = r.state;
    p.wave.rec_n[i] = 0;
}

// -----------------------------------------------------------------------------------------
// extend / shadow: persistent warps fetch 32 queue entries at a time.
// -----------------------------------------------------------------------------------------
template <bool kMulti>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_extend(const __grid_constant__ Params p, int depth) {
    extern __shared__ int stack[];     // [bvh depth + 1][kTraceBlock]
    uint32_t n0 = p.batch.n_slots;
    if constexpr (kMulti) n0 = cur_batch(p).n_slots;
    const uint32_t n = depth == 0 ? n0 : p.wave.counters[cnt_ext(depth)];
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
            const SceneDev* sc = &p.scene;
            const FilmDev* film = &p.film;
            if constexpr (kMulti) {
                const SceneSlot& S = p.multi.scenes[seg_of_slot(cur_batch(p), slot).scene];
                sc = &S.scene;
                film = &S.film;
            }
            const float4 o = p.wave.ray_o[slot];
            const float4 d = p.wave.ray_d[slot];
            WRay r;
            wray_setup(r, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), kSigmaVis);
            float t, u, v;
            // camera unwarp and the film components need the camera ray's closest surface at any
            // distance (World::Li's record, World.h:749-766); shade still
            // decides surface vs medium event by comparing with the sampled distance (o.w)
            const float tfar = depth == 0 && (film->unwarp || film->comps) ? __int_as_float(0x7f800000) : o.w;
            const uint32_t id = traverse<false>(*sc, r, tfar, t, u, v, stack + threadIdx.x, kTraceBlock);
            p.wave.hit[slot] = make_float4(t, __uint_as_float(id), u, v);
        }
    }
}

template <bool kMulti>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_shadow(const __grid_constant__ Params p, int depth) {
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
            const SceneDev* sc = &p.scene;
            if constexpr (kMulti)
                sc = &p.multi.scenes[seg_of_slot(cur_batch(p), __float_as_uint(p.wave.sh_L[idx].w)).scene].scene;
            WRay r;
            wray_setup(r, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), kSigmaVis);
            float t, u, v;
            const uint32_t id = traverse<true>(*sc, r, o.w, t, u, v, stack + threadIdx.x, kTraceBlock);
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

template <bool kGuided, bool kMulti>
__global__ void __launch_bounds__(256) k_shade(const __grid_constant__ Params p, int depth) {
    uint32_t n0 = p.batch.n_slots;
    if constexpr (kMulti) n0 = cur_batch(p).n_slots;
    const uint32_t n = depth == 0 ? n0 : p.wave.counters[cnt_ext(depth)];
    const uint32_t* qin = p.wave.q[depth & 1];
    uint32_t* qout = p.wave.q[(depth + 1) & 1];
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;

    for (uint32_t base = warp_global * 32u; base < n; base += nwarps * 32u) {
        const uint32_t idx = base + lane;
        bool want_shadow = false, want_next = false, want_guide = false;
        uint4 gv[5];                     // guided-vertex record (kGuided only)
        uint32_t slot = 0;
        float4 sh_o = make_float4(0, 0, 0, 0), sh_d = make_float4(0, 0, 0, 0), sh_L = make_float4(0, 0, 0, 0);
        if (idx < n) {
            slot = depth == 0 ? idx : qin[idx];
            // the slot's segment (pixels, samples) and scene: the launch's own in single-scene
            // mode, looked up in the current batch descriptor in multi-scene mode
            const Batch* Bp = &p.batch;
            const SceneSlot* SS = nullptr;
            if constexpr (kMulti) {
                Bp = &seg_of_slot(cur_batch(p), slot);
                SS = p.multi.scenes + Bp->scene;
            }
            const Batch& B = *Bp;
            const SceneDev& sc = kMulti ? SS->scene : p.scene;
            const FilmDev& film = kMulti ? SS->film : p.film;
            const uint32_t max_bounces = kMulti ? SS->max_bounces : p.max_bounces;
            const uint32_t flags = kMulti ? SS->flags : p.flags;
            const bool medium = sc.medium != 0;
            const f3 sig_s = mk(sc.sig_s[0], sc.sig_s[1], sc.sig_s[2]);
            const f3 sig_t = mk(sc.sig_t[0], sc.sig_t[1], sc.sig_t[2]);
            const float lambda = sc.lambda;
            const float g = sc.g;
            const float total_time = (float)film.T * film.exposure + film.offset;
            const float inv_inc = 1.0f / (float)B.ninc;
            const uint32_t per_pix = B.ns * B.ninc;
            const uint32_t lslot = slot - B.slot_begin;
            const float4 h = p.wave.hit[slot];
            const float4 ro = p.wave.ray_o[slot];
            const float4 rd = p.wave.ray_d[slot];
            const float4 th = p.wave.thr[slot];
            const uint32_t id = __float_as_uint(h.y);
            const bool hit = id != kInvalid;
            const float dsamp = ro.w;
            const bool surface = hit && (!medium || h.x < dsamp);
            if (depth == 0 && film.comps && lslot % B.ninc == 0) {
                // film components: one camera-ray record per camera sample (Film.h:127-145)
                const uint32_t pl = lslot / per_pix;
                const uint32_t wpix = B.pix_begin + pl;
                const size_t pixel = (size_t)(B.win_y0 + wpix / B.win_w) * film.W + (B.win_x0 + wpix % B.win_w);
                f3 cp = mk(0.f, 0.f, 0.f), cn = cp;
                if (hit) {
                    cp = mk(ro.x, ro.y, ro.z) + mk(rd.x, rd.y, rd.z) * h.x;
                    const float4 ng = __ldg(&sc.tri_ng[id]);
                    cn = mk(ng.x, ng.y, ng.z);
                }
                if (film.comps & 2u) atomicAdd(&film.cdepth[pixel], (double)(hit ? h.x : 3.40282347e+38f));
                if (film.comps & 8u) {
                    atomicAdd(&film.cpos[pixel * 3], (double)cp.x);
                    atomicAdd(&film.cpos[pixel * 3 + 1], (double)cp.y);
                    atomicAdd(&film.cpos[pixel * 3 + 2], (double)cp.z);
                }
                if (film.comps & 16u) {
                    atomicAdd(&film.cnorm[pixel * 3], (double)cn.x);
                    atomicAdd(&film.cnorm[pixel * 3 + 1], (double)cn.y);
                    atomicAdd(&film.cnorm[pixel * 3 + 2], (double)cn.z);
                }
            }
            if (medium || hit) {
                // per-path RNG: state in memory, increment from the camera sample
                const uint32_t pl = lslot / per_pix;
                const uint32_t sl = (lslot - pl * per_pix) / B.ninc;
                const uint32_t wpix = B.pix_begin + pl;
                const uint32_t pixel = (B.win_y0 + wpix / B.win_w) * film.W + (B.win_x0 + wpix % B.win_w);
                Pcg rng;
                rng.state = p.wave.rng[slot];
                rng.inc = (cam_id(pixel, B.s0 + sl) << 1u) | 1ull;

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
                // camera unwarp: World::Li's record distance = closest surface along the camera
                // ray, FLT_MAX when there is none (World.h:749-766, Ray.h:74-84)
                float cam_d = 0.0f;
                if (film.unwarp) {
                    if (depth == 0) {
                        cam_d = hit ? h.x : 3.40282347e+38f;
                        p.wave.cam_dist[slot] = cam_d;
                    } else {
                        cam_d = p.wave.cam_dist[slot];
                    }
                }
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
                            const float tc = film.unwarp ? tt - cam_d : tt;      // StreakCameraFilm.h:167
                            const float ps = (tc - film.offset) / film.exposure;
                            const bool inside = ps < (float)film.T && ps >= 0.0f;
                            const bool fin = finite3(Lr, Lg, Lb);
                            // with bounce films every visible light connection is a sample (its
                            // time and radiance aside; non-finite radiance becomes 0 as in
                            // TransientRenderer.h:165-169); otherwise only useful ones are traced
                            if ((inside && fin && (Lr != 0.0f || Lg != 0.0f || Lb != 0.0f)) || film.nbounce) {
                                want_shadow = true;
                                const uint32_t bin = inside ? (uint32_t)floorf(ps) : kBinOutside;
                                sh_o = make_float4(lp.x, lp.y, lp.z, dl - kSigmaVis);
                                sh_d = make_float4(ld.x, ld.y, ld.z, __uint_as_float(bin | ((uint32_t)depth << 24)));
                                sh_L = fin ? make_float4(Lr, Lg, Lb, __uint_as_float(slot))
                                           : make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(slot));
                            }
                        }
                    }
                    if ((uint32_t)depth + 1u < max_bounces) {
                        // ---- Russian roulette ----
                        const float albedo = surface ? avg3(kd)
                            : avg3(mk(sig_s.x / sig_t.x, sig_s.y / sig_t.y, sig_s.z / sig_t.z));
                        if (kGuided && surface && !(pcg_float(rng) > albedo)) {
                            // ---- direction deferred to the learned proposal (k_guide) ----
                            want_guide = true;
                            gv[0] = make_uint4(__float_as_uint(pos.x), __float_as_uint(pos.y), __float_as_uint(pos.z),
                                               __float_as_uint(time));
                            gv[1] = make_uint4(__float_as_uint(dir.x), __float_as_uint(dir.y), __float_as_uint(dir.z),
                                               __float_as_uint(albedo));
                            gv[2] = make_uint4(__float_as_uint(f.x), __float_as_uint(f.y), __float_as_uint(f.z),
                                               __float_as_uint(__ldg(&sc.tri_ng[id]).w));
                            gv[3] = make_uint4(__float_as_uint(nrm.x), __float_as_uint(nrm.y), __float_as_uint(nrm.z), slot);
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
                            } else if (surface && (flags & kFlagOrthoFrame)) {
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
                if (kGuided && want_guide)
                    gv[4] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), (uint32_t)rng.inc,
                                       (uint32_t)(rng.inc >> 32));
                else
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
            if (want_guide) {
                uint4* r = p.guide.vrec + (size_t)(bg + (uint32_t)__popc(mg & lt)) * 5;
#pragma unroll
                for (int q = 0; q < 5; ++q) r[q] = gv[q];
            }
        }
    }
}

// -----------------------------------------------------------------------------------------
// splat: StreakCameraFilm::add_samples / add_temporal_sample (StreakCameraFilm.h:139-192,
// 279-315) with the box filter of size 1: bin = floor((t - offset) / exposure) (computed in
// shade), streak(pixel, bin) += L, steady(pixel) += L, weight(pixel) += 1 per camera sample.
// A CTA owns `G` whole pixels of the batch, accumulates their records in an FP32 shared-memory
// tile (warp-aggregated atomics on equal (pixel, bin) keys) and adds the tile to the FP64 film.
// -----------------------------------------------------------------------------------------
template <bool kMulti>
__global__ void __launch_bounds__(kSplatBlock) k_splat(const __grid_constant__ Params p, int G_launch, int bsel) {
    extern __shared__ __align__(16) float tile[];
    // the block's segment and film: the launch's own in single-scene mode; in multi-scene mode
    // from the current batch's block table, each segment with its own film-tile width
    const Batch* Bp = &p.batch;
    const FilmDev* Fp = &p.film;
    uint32_t G = (uint32_t)G_launch, blk = blockIdx.x;
    if constexpr (kMulti) {
        const BatchDesc& BD = cur_batch(p);
        if (blockIdx.x >= BD.n_blocks) return;
        Bp = &seg_of_block(BD, blockIdx.x);
        Fp = &p.multi.scenes[Bp->scene].film;
        G = Bp->splat_g;
        blk = blockIdx.x - Bp->blk_begin;
    }
    const Batch& B = *Bp;
    const FilmDev& film = *Fp;
    const uint32_t T = film.T;
    const uint32_t TT = T * 3u;
    const uint32_t pix0 = blk * G;
    if (pix0 >= B.npix) return;
    if (bsel >= (int)film.nbounce) return;                // this scene has no such bounce film
    const uint32_t gp = min((uint32_t)G, B.npix - pix0);
    // bsel < 0: the film; with bounce films its steady image is the base Film's (all samples).
    // bsel = b: bounce film b, fed by the records of bounce min(depth, N-1) == b.
    const size_t npix_film = (size_t)film.W * film.H;
    double* out_streak = bsel < 0 ? film.streak : film.bstreak + (size_t)bsel * npix_film * TT;
    double* out_steady = bsel < 0 ? film.steady : film.bsteady + (size_t)bsel * npix_film * 3u;
    const bool steady_all = bsel < 0 && film.nbounce > 0;
    const uint32_t nb_last = film.nbounce ? film.nbounce - 1u : 0u;
    float* steady = tile + (size_t)G * TT;
    {
        float4* t4 = reinterpret_cast<float4*>(tile);
        const uint32_t n4 = ((uint32_t)G * TT + 3u * G + 3u) / 4u;
        for (uint32_t e = threadIdx.x; e < n4; e += blockDim.x) t4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    const uint32_t per_pix = B.ns * B.ninc;
    const uint32_t nslots = gp * per_pix;
    const uint32_t slot0 = B.slot_begin + pix0 * per_pix;
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
            const uint32_t bin = __float_as_uint(rc.w) & 0x00ffffffu;
            const uint32_t rdepth = __float_as_uint(rc.w) >> 24;
            const bool mine = valid && (bsel < 0 || min(rdepth, nb_last) == (uint32_t)bsel);
            const bool inwin = mine && bin != kBinOutside;
            const uint32_t key = inwin ? pl * T + bin : 0xffffffffu;
            // lanes holding the same (pixel, bin) are summed with shuffles; the group's
            // lowest lane issues one shared-memory atomic per channel
            const unsigned peers = __match_any_sync(kFull, key);
            const int rank = __popc(peers & lt);
            const int gsize = __popc(peers);
            float vx = rc.x, vy = rc.y, vz = rc.z;
            const uint32_t maxg = __reduce_max_sync(kFull, inwin ? (uint32_t)gsize : 1u);
            for (int step = 1; step < (int)maxg; step <<= 1) {
                const int src_rank = rank + step;
                const int src = src_rank < gsize ? (int)__fns(peers, 0, src_rank + 1) : (int)lane;
                const float ox = __shfl_sync(kFull, vx, src);
                const float oy = __shfl_sync(kFull, vy, src);
                const float oz = __shfl_sync(kFull, vz, src);
                if ((rank & (2 * step - 1)) == 0 && src_rank < gsize) { vx += ox; vy += oy; vz += oz; }
            }
            if (inwin && rank == 0) {
                float* cell = tile + (size_t)key * 3u;
                atomicAdd(cell, vx); atomicAdd(cell + 1, vy); atomicAdd(cell + 2, vz);
            }
            if (inwin || (steady_all && valid)) { ax += rc.x; ay += rc.y; az += rc.z; }
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
        const size_t pixel = (size_t)(B.win_y0 + wpix / B.win_w) * film.W + (B.win_x0 + wpix % B.win_w);
        double* dst = out_streak + pixel * TT;
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
            if (bsel < 0) film.weight[pixel] += (double)B.ns;
            for (int c = 0; c < 3; ++c) out_steady[pixel * 3 + c] += (double)steady[pl * 3 + c];
        }
    }
}

// Per-bounce film weights (MultibounceStreakCameraFilm.h:151-171 with StreakCameraFilm.h:139-160):
// bounce film b's weight grows by one per camera sample (all its incoming paths together) that
// has at least one radiance sample of bounce min(depth, N-1) == b, inside the time window or not.
__global__ void __launch_bounds__(256) k_bounce_weights(const __grid_constant__ Params p) {
    const Batch& B = p.batch;
    const FilmDev& film = p.film;
    const uint32_t ncs = B.npix * B.ns;
    const size_t rs = p.wave.capacity;
    const size_t npix_film = (size_t)film.W * film.H;
    const uint32_t nb_last = film.nbounce - 1u;
    for (uint32_t cs = blockIdx.x * blockDim.x + threadIdx.x; cs < ncs; cs += gridDim.x * blockDim.x) {
        const uint32_t pl = cs / B.ns;
        const uint32_t slot0 = cs * B.ninc;              // ((pl * ns) + s) * ninc
        uint32_t mask = 0;
        for (uint32_t j = 0; j < B.ninc; ++j) {
            const uint32_t slot = slot0 + j;
            const uint32_t cnt = p.wave.rec_n[slot];
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t d = __float_as_uint(p.wave.rec[(size_t)k * rs + slot].w) >> 24;
                mask |= 1u << min(d, nb_last);
            }
        }
        if (!mask) continue;
        const uint32_t wpix = B.pix_begin + pl;
        const size_t pixel = (size_t)(B.win_y0 + wpix / B.win_w) * film.W + (B.win_x0 + wpix % B.win_w);
        for (uint32_t b = 0; b <= nb_last; ++b)
            if (mask >> b & 1u) atomicAdd(&film.bweight[(size_t)b * npix_film + pixel], 1.0);
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

int trace_grid_size(int device, uint32_t bvh_depth, bool multi) {
    int sms = 0, per_sm = 0, per_sm_sh = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (multi) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extend<true>, kTraceBlock, trace_smem_bytes(bvh_depth));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_sh, k_shadow<true>, kTraceBlock, trace_smem_bytes(bvh_depth));
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extend<false>, kTraceBlock, trace_smem_bytes(bvh_depth));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_sh, k_shadow<false>, kTraceBlock, trace_smem_bytes(bvh_depth));
    }
    per_sm = per_sm_sh < per_sm ? per_sm_sh : per_sm;
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

size_t splat_smem_bytes(uint32_t T, int G) {
    // tile [G][T][3] + steady [G][3] floats, rounded up to whole float4 (zeroed as float4)
    return (((size_t)G * T * 3u + 3u * (size_t)G) * sizeof(float) + 15u) & ~size_t(15);
}

// Kernel variants: multi-scene when the parameters carry a scene table (tr_batch), else the
// single-scene kernels.  Multi-scene grids cover the wave's capacity / the plan's largest batch,
// because the per-batch counts live in device memory (the launches are replayed from a graph).
cudaError_t launch_raygen(const Params& p, cudaStream_t s) {
    if (p.multi.scenes) {
        k_raygen<true><<<(p.wave.capacity + 255) / 256, 256, 0, s>>>(p);
    } else {
        const uint32_t n = p.batch.n_slots;
        k_raygen<false><<<(n + 255) / 256, 256, 0, s>>>(p);
    }
    return cudaGetLastError();
}
cudaError_t launch_extend(const Params& p, int depth, int grid, cudaStream_t s) {
    if (p.multi.scenes) k_extend<true><<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    else k_extend<false><<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    return cudaGetLastError();
}
cudaError_t launch_shade(const Params& p, int depth, cudaStream_t s) {
    int dev = 0, grid = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&grid, cudaDevAttrMultiProcessorCount, dev);
    const bool multi = p.multi.scenes != nullptr;
    const int block = multi && p.multi.shade_block ? (int)p.multi.shade_block : 256;
    grid *= 8 * 256 / block;
    const uint32_t need = ((multi ? p.wave.capacity : p.batch.n_slots) + block - 1) / block;
    if ((uint32_t)grid > need) grid = (int)need;
    if (grid < 1) grid = 1;
    if (multi) {
        if (p.guide.vrec) k_shade<true, true><<<grid, block, 0, s>>>(p, depth);
        else k_shade<false, true><<<grid, block, 0, s>>>(p, depth);
    } else {
        if (p.guide.vrec) k_shade<true, false><<<grid, block, 0, s>>>(p, depth);
        else k_shade<false, false><<<grid, block, 0, s>>>(p, depth);
    }
    return cudaGetLastError();
}
cudaError_t launch_shadow(const Params& p, int depth, int grid, cudaStream_t s) {
    if (p.multi.scenes) k_shadow<true><<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    else k_shadow<false><<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    return cudaGetLastError();
}
cudaError_t launch_splat(const Params& p, int G, cudaStream_t s, int bsel) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_splat<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(k_splat<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_set = true;
    }
    if (p.multi.scenes) {
        k_splat<true><<<p.multi.max_splat_blocks, kSplatBlock, p.multi.splat_smem, s>>>(p, 0, bsel);
    } else {
        const size_t smem = splat_smem_bytes(p.film.T, G);
        const uint32_t blocks = (p.batch.npix + (uint32_t)G - 1) / (uint32_t)G;
        k_splat<false><<<blocks, kSplatBlock, smem, s>>>(p, G, bsel);
    }
    return cudaGetLastError();
}
cudaError_t launch_bounce_weights(const Params& p, cudaStream_t s) {
    const uint32_t ncs = p.batch.npix * p.batch.ns;
    k_bounce_weights<<<std::max(1u, std::min(4096u, (ncs + 255) / 256)), 256, 0, s>>>(p);
    return cudaGetLastError();
}

// last node of a multi-scene batch: the next replay renders the next batch descriptor
__global__ void k_advance(uint32_t* cur) { *cur += 1u; }
cudaError_t launch_advance(uint32_t* cur, cudaStream_t s) {
    k_advance<<<1, 1, 0, s>>>(cur);
    return cudaGetLastError();
}
cudaError_t launch_trace_user(const SceneDev& sc, const float* rays, uint32_t n, int any_hit, void* out,
                              uint32_t* cursor, int grid, cudaStream_t s) {
    k_trace_user<<<grid, kTraceBlock, trace_smem_bytes(sc.bvh_depth), s>>>(sc, rays, n, any_hit,
                                                                          reinterpret_cast<HitOut*>(out), cursor);
    return cudaGetLastError();
}

}  // namespace trk
