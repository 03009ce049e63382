// tr_kernels.cu - wavefront transient path tracing kernels for sm_100a.
//
// Pipeline per batch of path slots (one slot = one camera sample x incoming sample):
//   raygen  -> camera ray, per-path PCG32 stream, optional free-flight distance
//   for depth in [0, max_bounces):
//     extend  (persistent warps, closest hit, shared-memory stack, lane refill from the queue)
//     shade   (vertex, next-event estimate -> shadow queue, Russian roulette, new direction
//              -> next extend queue, appended per block grouped by direction octant)
//     shadow  (persistent, any hit) -> splat record per surviving connection
//   splat   (per group of whole pixels: records read bounce-major; lanes with equal
//            (pixel, bin) keys found with __match_any_sync, summed in FP32 by a shuffle tree,
//            one native FP64 atomicAdd per group into the film in HBM)
// Reference path: src/Integrator/BidirectionalPathTracing.h:485-692,975-1140 and
// src/Film/StreakCameraFilm.h:139-192 (details at each kernel).
#include "tr_bsdf.cuh"
#include "tr_device.cuh"
#include "tr_kernels.cuh"

#include <algorithm>

namespace trk {
using namespace trd;


// -----------------------------------------------------------------------------------------
// BVH traversal: four-child 128-byte nodes (one conservative slab test for the four children,
// after Ize 2013), hit children visited nearest first (a five-exchange sorting network), the
// others pushed on a per-thread stack in shared memory (strided by block size); watertight
// triangle test.  Closest hit: smallest t in (tnear, tfar], ties -> lower triangle id (order
// independent, so the result does not depend on the tree).
// -----------------------------------------------------------------------------------------
__device__ __forceinline__ void slab4(float lo_x, float hi_x, float lo_y, float hi_y, float lo_z, float hi_z, int ref,
                                      float ox, float oy, float oz, float ix, float iy, float iz, float tnear,
                                      float best, float& key) {
    const float lx = (lo_x - ox) * ix, hx = (hi_x - ox) * ix;
    const float ly = (lo_y - oy) * iy, hy = (hi_y - oy) * iy;
    const float lz = (lo_z - oz) * iz, hz = (hi_z - oz) * iz;
    const float tmin = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), tnear));
    const float tmax = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fminf(fmaxf(lz, hz), best)) * 1.00000036f;
    // empty slots are leaves of 0 triangles
    const bool use = ref >= 0 || ((~ref) & 7) != 0;
    key = (use && tmin <= tmax) ? tmin : __int_as_float(0x7f800000);
}
// 32 bytes in one load (sm_100: 256-bit global loads); p must be 32-byte aligned (the launchers
// check the node buffer).  A node's bounds arrive in three such loads instead of six 128-bit
// ones: the divergent lanes of a warp each cost their own L1 request per load instruction.
__device__ __forceinline__ void ldg256(const float4* p, float4& a, float4& b) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}
__device__ __forceinline__ void order2(float& ka, int& ra, float& kb, int& rb) {
    if (kb < ka) {
        const float tk = ka; ka = kb; kb = tk;
        const int tr = ra; ra = rb; rb = tr;
    }
}

// Traversal state of one ray between calls of trav_run: next node (or the triangles left in a
// leaf), stack depth, closest hit so far.
struct Trav {
    int node, sp;
    float best, bu, bv;
    uint32_t bid;
};
__device__ __forceinline__ void trav_init(Trav& st, float tfar) {
    st.node = 0; st.sp = 0; st.best = tfar; st.bu = 0.f; st.bv = 0.f; st.bid = kInvalid;
}

// Runs at most `budget` node or triangle visits of the ray's traversal; returns true once the
// traversal is complete (closest hit, or any hit with kAnyHit, in st).  The stack lives in
// shared memory at stack[k * stride].
template <bool kAnyHit>
__device__ __forceinline__ bool trav_run(const SceneDev& sc, const WRay& r, Trav& st, int* __restrict__ stack,
                                         int stride, int budget) {
    const float ox = r.o.x, oy = r.o.y, oz = r.o.z;
    const float ix = r.inv.x, iy = r.inv.y, iz = r.inv.z;
    const float kInf = __int_as_float(0x7f800000);
    for (;;) {
        if (budget-- == 0) return false;
        if (st.node >= 0) {
            const float4* np = sc.nodes + 8 * st.node;
            float4 lx, hx, ly, hy, lz, hz;
            ldg256(np, lx, hx);
            ldg256(np + 2, ly, hy);
            ldg256(np + 4, lz, hz);
            const int4 ch = __ldg(reinterpret_cast<const int4*>(np + 6));
            float k0, k1, k2, k3;
            int c0 = ch.x, c1 = ch.y, c2 = ch.z, c3 = ch.w;
            slab4(lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, c0, ox, oy, oz, ix, iy, iz, r.tnear, st.best, k0);
            slab4(lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, c1, ox, oy, oz, ix, iy, iz, r.tnear, st.best, k1);
            slab4(lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, c2, ox, oy, oz, ix, iy, iz, r.tnear, st.best, k2);
            slab4(lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, c3, ox, oy, oz, ix, iy, iz, r.tnear, st.best, k3);
            if constexpr (!kAnyHit) {
                order2(k0, c0, k1, c1);
                order2(k2, c2, k3, c3);
                order2(k0, c0, k2, c2);
                order2(k1, c1, k3, c3);
                order2(k1, c1, k2, c2);
                if (k0 == kInf) {
                    if (st.sp == 0) return true;
                    --st.sp;
                    st.node = stack[st.sp * stride];
                    continue;
                }
                // farthest first, so the nearest of the others is popped next
                if (k3 != kInf) { stack[st.sp * stride] = c3; ++st.sp; }
                if (k2 != kInf) { stack[st.sp * stride] = c2; ++st.sp; }
                if (k1 != kInf) { stack[st.sp * stride] = c1; ++st.sp; }
                st.node = c0;
            } else {
                // any hit ends the query: children in slot order, no sorting
                int next = -1;
                if (k3 != kInf) { next = c3; }
                if (k2 != kInf) { if (next != -1) { stack[st.sp * stride] = next; ++st.sp; } next = c2; }
                if (k1 != kInf) { if (next != -1) { stack[st.sp * stride] = next; ++st.sp; } next = c1; }
                if (k0 != kInf) { if (next != -1) { stack[st.sp * stride] = next; ++st.sp; } next = c0; }
                if (next == -1) {
                    if (st.sp == 0) return true;
                    --st.sp;
                    st.node = stack[st.sp * stride];
                    continue;
                }
                st.node = next;
            }
            continue;
        }
        // one triangle per visit: the leaf's remaining triangles stay in st.node, so a lane in
        // a leaf and a lane at an inner node each advance by one step per loop iteration
        const uint32_t ref = (uint32_t)(~st.node);
        const uint32_t first = ref >> 3, cnt = ref & 7u;
        {
            const float4* tp = sc.tris + 3 * first;
            const float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
            const uint32_t id = __float_as_uint(q0.w);
            float t, u, v;
            if (wt_hit(r, f3of(q0), f3of(q1), f3of(q2), st.best, t, u, v)) {
                if (t < st.best || st.bid == kInvalid || id < st.bid) {
                    st.best = t; st.bid = id; st.bu = u; st.bv = v;
                    if (kAnyHit) return true;
                }
            }
        }
        if (cnt > 1u) {
            st.node = (int)~(((first + 1u) << 3) | (cnt - 1u));
            continue;
        }
        if (st.sp == 0) return true;
        --st.sp;
        st.node = stack[st.sp * stride];
    }
}

// Whole traversal in one call (used where one thread owns a fixed set of rays).
template <bool kAnyHit>
__device__ __forceinline__ uint32_t traverse(const SceneDev& sc, const WRay& r, float tfar,
                                             float& t_out, float& u_out, float& v_out,
                                             int* __restrict__ stack, int stride) {
    Trav st;
    trav_init(st, tfar);
    trav_run<kAnyHit>(sc, r, st, stack, stride, 0x7fffffff);
    t_out = st.bid == kInvalid ? tfar : st.best;
    u_out = st.bu; v_out = st.bv;
    return st.bid;
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
    if ((kMulti ? SS->flags : p.flags) & kFlagTimeSampling) {
        // time sampling: one light point per path, the target of the time-angular sampler
        // (World::sample_light + LightSource::sample, BidirectionalPathTracing.h:1107-1113;
        // PointLightSource.h:174-183, RectangularAreaLightSource.h:252-276)
        const float xl = pcg_float(r);
        uint32_t lsel = (uint32_t)(xl * (float)sc.num_lights);
        if (lsel >= sc.num_lights) lsel = sc.num_lights - 1;
        const float4* L = sc.lights + 5 * lsel;
        const float4 L0 = __ldg(L);
        f3 tg = mk(L0.x, L0.y, L0.z);
        if (__float_as_uint(L0.w) == 1u) {
            const float xu = pcg_float(r), xv = pcg_float(r);
            tg = (tg + f3of(__ldg(L + 2)) * xu) + f3of(__ldg(L + 3)) * xv;
        }
        p.wave.target[i] = make_float4(tg.x, tg.y, tg.z, __uint_as_float(lsel));
    }
    if (p.bd.ne) p.bd.ne[i] = 0;
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
// Node and triangle visits a lane makes between two refills of the warp's finished lanes.
constexpr int kTravBudget = 8;

// Warp-aggregated refill from a queue: every lane with busy == false takes the next entry
// index (one atomic per warp); lanes left without an entry get idx >= n.  `drained` (warp
// uniform) records that the queue is exhausted.
__device__ __forceinline__ uint32_t refill(bool busy, uint32_t* cursor, uint32_t n, bool& drained) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned idle = __ballot_sync(kFull, !busy);
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(cursor, (uint32_t)__popc(idle));
    base = __shfl_sync(kFull, base, 0);
    if (base + (uint32_t)__popc(idle) >= n) drained = true;
    return base + (uint32_t)__popc(idle & lanemask_lt());
}

// Closest hit of each queued ray.  Persistent warps; a lane whose ray is done takes the next
// queued ray at the warp's next refill point, so the lanes stay busy while rays of very
// different traversal lengths share a warp.
template <bool kMulti>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_extend(const __grid_constant__ Params p, int depth) {
    extern __shared__ int stack[];     // [stack entries][kTraceBlock]
    uint32_t n0 = p.batch.n_slots;
    if constexpr (kMulti) n0 = cur_batch(p).n_slots;
    const uint32_t n = depth == 0 ? n0 : p.wave.counters[cnt_ext(depth)];
    const uint32_t* q = p.wave.q[depth & 1];
    uint32_t* cursor = &p.wave.counters[cur_ext(depth)];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.wave.stats[0], (unsigned long long)n);
    bool busy = false, drained = false;
    uint32_t slot = 0;
    float tfar = 0.f;
    const SceneDev* sc = &p.scene;
    WRay r;
    Trav st;
    for (;;) {
        if (!drained && __any_sync(kFull, !busy)) {
            const uint32_t idx = refill(busy, cursor, n, drained);
            if (!busy && idx < n) {
                slot = depth == 0 ? idx : q[idx];
                const FilmDev* film = &p.film;
                if constexpr (kMulti) {
                    const SceneSlot& S = p.multi.scenes[seg_of_slot(cur_batch(p), slot).scene];
                    sc = &S.scene;
                    film = &S.film;
                }
                const float4 o = p.wave.ray_o[slot];
                const float4 d = p.wave.ray_d[slot];
                wray_setup(r, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), kSigmaVis);
                // camera unwarp and the film components need the camera ray's closest surface
                // at any distance (World::Li's record, World.h:749-766); shade still decides
                // surface vs medium event by comparing with the sampled distance (o.w)
                tfar = depth == 0 && (film->unwarp || film->comps) ? __int_as_float(0x7f800000) : o.w;
                trav_init(st, tfar);
                busy = true;
            }
        }
        if (!__any_sync(kFull, busy)) break;
        if (busy && trav_run<false>(*sc, r, st, stack + threadIdx.x, kTraceBlock, kTravBudget)) {
            const float t = st.bid == kInvalid ? tfar : st.best;
            p.wave.hit[slot] = make_float4(t, __uint_as_float(st.bid), st.bu, st.bv);
            busy = false;
        }
    }
}

// Any hit of each queued shadow ray; a record for the unoccluded ones.  Same lane refill as
// k_extend.
template <bool kMulti>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_shadow(const __grid_constant__ Params p, int depth) {
    extern __shared__ int stack[];     // [stack entries][kTraceBlock]
    const uint32_t n = p.wave.counters[cnt_sh(depth)];
    uint32_t* cursor = &p.wave.counters[cur_sh(depth)];
    const size_t rs = p.wave.capacity;          // record stride: records are [bounce][slot]
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.wave.stats[1], (unsigned long long)n);
    unsigned long long splats = 0;
    bool busy = false, drained = false;
    uint32_t idx = 0;
    const SceneDev* sc = &p.scene;
    WRay r;
    Trav st;
    for (;;) {
        if (!drained && __any_sync(kFull, !busy)) {
            const uint32_t k = refill(busy, cursor, n, drained);
            if (!busy && k < n) {
                idx = k;
                const float4 o = p.wave.sh_o[idx];
                const float4 d = p.wave.sh_d[idx];
                if constexpr (kMulti)
                    sc = &p.multi.scenes[seg_of_slot(cur_batch(p), __float_as_uint(p.wave.sh_L[idx].w)).scene].scene;
                wray_setup(r, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), kSigmaVis);
                trav_init(st, o.w);
                busy = true;
            }
        }
        if (!__any_sync(kFull, busy)) break;
        if (busy && trav_run<true>(*sc, r, st, stack + threadIdx.x, kTraceBlock, kTravBudget)) {
            const float4 d = p.wave.sh_d[idx];
            const uint32_t dw = __float_as_uint(d.w);
            if (dw & kConnRay) {
                // eye-light vertex connection: the reference records it when the segment is
                // blocked (World::intersects returns true on a hit); fixed record index
                if (st.bid != kInvalid && !(dw & kConnNoRecord)) {
                    const float4 L = p.wave.sh_L[idx];
                    const uint32_t lw = __float_as_uint(L.w);
                    const uint32_t slot = lw & 0xffffffu, kk = lw >> 24;
                    p.wave.rec[(size_t)kk * rs + slot] = make_float4(L.x, L.y, L.z, __uint_as_float(dw & 0x1fffffffu));
                    p.bd.valid[(size_t)kk * rs + slot] = 1;
                }
            } else if (st.bid == kInvalid) {
                const float4 L = p.wave.sh_L[idx];
                const uint32_t slot = __float_as_uint(L.w);
                const uint32_t kk = p.wave.rec_n[slot];
                p.wave.rec[(size_t)kk * rs + slot] = make_float4(L.x, L.y, L.z, d.w);
                p.wave.rec_n[slot] = (uint8_t)(kk + 1);
                ++splats;
            }
            busy = false;
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

// The vector-to-vector matrix of Moeller & Hughes ("Efficiently building a matrix to rotate
// one vector to another", JGT 4(4), 1999) from +y to `to`, applied to d and normalised, as
// VectorN::transform_matrix_to (VectorN.h:427-521) builds it.  The time-angular sampler passes
// the unnormalised target offset as `to` (BidirectionalPathTracing.h:392), for which the matrix
// is not a rotation; the same construction keeps the sampled directions those of the reference.
__device__ __forceinline__ f3 mh_from_y(f3 to, f3 d) {
    // (0,1,0) x to and (0,1,0) . to, every product written out so zero signs match a plain
    // evaluation of the cross and dot products
    const f3 v = mk(1.0f * to.z - 0.0f * to.y, 0.0f * to.x - 0.0f * to.z, 0.0f * to.y - 1.0f * to.x);
    const float e = (0.0f * to.x + 1.0f * to.y) + 0.0f * to.z;
    float m[3][3];
    if (fabsf(e) > 1.0f - 1e-4f) {
        // near-parallel: reflections through the coordinate axis least aligned with +y (z)
        const f3 u = mk(0.0f, -1.0f, 1.0f);                      // z - y
        const f3 w = mk(0.0f - to.x, 0.0f - to.y, 1.0f - to.z);  // z - to
        const float c1 = 2.0f / dot(u, u), c2 = 2.0f / dot(w, w);
        const float c3 = (c1 * c2) * dot(u, w);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                m[i][j] = ((-c1 * comp(u, i)) * comp(u, j) - (c2 * comp(w, i)) * comp(w, j)) + (c3 * comp(w, i)) * comp(u, j);
                if (i == j) m[i][j] += 1.0f;
            }
    } else {
        const float h = 1.0f / (1.0f + e);
        const float hvx = h * v.x, hvz = h * v.z, hvxy = hvx * v.y, hvxz = hvx * v.z, hvyz = hvz * v.y;
        m[0][0] = e + hvx * v.x; m[0][1] = hvxy - v.z;           m[0][2] = hvxz + v.y;
        m[1][0] = hvxy + v.z;    m[1][1] = e + (h * v.y) * v.y;   m[1][2] = hvyz - v.x;
        m[2][0] = hvxz - v.y;    m[2][1] = hvyz + v.x;           m[2][2] = e + hvz * v.z;
    }
    const f3 r = mk((m[0][0] * d.x + m[0][1] * d.y) + m[0][2] * d.z, (m[1][0] * d.x + m[1][1] * d.y) + m[1][2] * d.z,
                    (m[2][0] * d.x + m[2][1] * d.y) + m[2][2] * d.z);
    return normalize(r);
}

// One direction of the time-angular sampler (SamplingTechniques.h:170-247 TimeAngular;
// BidirectionalPathTracing.h:365-405 with p_ts = 1): the time t is uniform on the sampler's
// bounds [t_a, t_b], theta is the angle to the target at which a scattering after `r` reaches
// the target at time t, phi is uniform.  Operand types follow the reference (the cosine in
// double, stored as a float; float products).  When the bounds are inverted (the current delay
// exceeds 2r) the cosine clamps to -1, theta is the float nearest pi (above pi), its sine the
// small negative number pi - (float)pi, and the density dtdtheta / (t_b - t_a) / (2 pi) a small
// positive number; the caller keeps the direction when that density is >= 1e-5 (rare huge
// weights, as in the reference).  e, e2: the theta and phi draws.
struct TaSample { f3 nd; float ph; float pa; };
__device__ __noinline__ TaSample time_angular_sample(f3 l, float mod, float r, float t_a, float t_b, float e, float e2,
                                                     f3 dir, float g) {
    const float t = e * (t_b - t_a) + t_a;
    float ct = (float)((((double)(mod * mod) + ((2.0 * (double)t) * (double)r)) - (double)(t * t)) /
                       ((2.0 * (double)r) * (double)mod));
    ct = ct < -1.0f ? -1.0f : (ct > 1.0f ? 1.0f : ct);
    constexpr float kSinFloatPi = (float)(3.14159265358979323846 - (double)3.14159265358979323846f);
    const float st = ct == -1.0f ? kSinFloatPi : (float)sqrt(1.0 - (double)ct * (double)ct);
    float sp2, cp2;
    tr_sincos2pi(e2, &sp2, &cp2);
    TaSample o;
    o.nd = mh_from_y(l, mk(cp2 * st, ct, sp2 * st));
    o.ph = hg_eval(g, dot(dir, o.nd));
    const float dtdth = (float)((double)((mod * r) * st) /
                                sqrt((double)(r * r + mod * mod) - ((2.0 * (double)r) * (double)mod) * (double)ct));
    const float pdf_theta = dtdth / (t_b - t_a);
    o.pa = (float)((double)pdf_theta / (2.0 * 3.14159265358979323846));
    return o;
}

// kTimeSampling: compiled with the time-sampling branches (a launch whose context, or some
// context of whose batch, has TR_FLAG_TIME_SAMPLING; the flag is still read per slot).
// Register budgets (the kernel is latency-bound, so resident warps matter more than a few
// spilled values, which stay in L1): the plain variant 64 registers (4 CTAs per SM); the guided
// and time-sampling variants 80 (3 CTAs per SM; unbounded they took 146-172 registers and ran
// one CTA of 8 warps per SM); the multi-scene variants 128 (2 CTAs, no spills).
template <bool kGuided, bool kMulti, bool kTimeSampling>
__global__ void __launch_bounds__(256, kMulti ? 3 : (kTimeSampling ? 3 : 4))
    k_shade(const __grid_constant__ Params p, int depth) {
    uint32_t n0 = p.batch.n_slots;
    if constexpr (kMulti) n0 = cur_batch(p).n_slots;
    const uint32_t n = depth == 0 ? n0 : p.wave.counters[cnt_ext(depth)];
    const uint32_t* qin = p.wave.q[depth & 1];
    uint32_t* qout = p.wave.q[(depth + 1) & 1];
    const unsigned lane = threadIdx.x & 31u;
    // block-uniform iterations (the next-ray queue is filled per block, below)
    __shared__ uint32_t oc[8], ob[8], sc8[8], sb8[8];
    for (uint32_t bbase = blockIdx.x * blockDim.x; bbase < n; bbase += gridDim.x * blockDim.x) {
        const uint32_t base = bbase + (threadIdx.x & ~31u);
        const uint32_t idx = base + lane;
        uint32_t oct = 0, soct = 0;
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
                                soct = (ld.x < 0.0f ? 1u : 0u) | (ld.y < 0.0f ? 2u : 0u) | (ld.z < 0.0f ? 4u : 0u);
                                const uint32_t bin = inside ? (uint32_t)floorf(ps) : kBinOutside;
                                sh_o = make_float4(lp.x, lp.y, lp.z, dl - kSigmaVis);
                                sh_d = make_float4(ld.x, ld.y, ld.z, __uint_as_float(bin | ((uint32_t)depth << 24)));
                                sh_L = fin ? make_float4(Lr, Lg, Lb, __uint_as_float(slot))
                                           : make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(slot));
                            }
                        }
                    }
                    if constexpr (kTimeSampling) {
                        // ---- bidirectional connections: keep the eye vertex (value, pdf,
                        // delay) for the connection passes (connect_paths, BidirectionalPathTracing.h:
                        // 1018-1041); scenes without a medium, so every vertex is a surface ----
                        if ((flags & kFlagBidirectional) && surface && (uint32_t)depth + 2u <= max_bounces) {
                            const size_t cap = p.wave.capacity;
                            float4* v = p.bd.evert + (size_t)depth * 4 * cap + slot;
                            v[0] = make_float4(pos.x, pos.y, pos.z, time);
                            v[cap] = make_float4(nrm.x, nrm.y, nrm.z, ptot);
                            v[2 * cap] = make_float4(kd.x, kd.y, kd.z, 0.0f);
                            v[3 * cap] = make_float4(f.x, f.y, f.z, 0.0f);
                            p.bd.ne[slot] = (uint8_t)(depth + 1);
                        }
                    }
                    if ((uint32_t)depth + 1u < max_bounces) {
                        // ---- Russian roulette (none in time-sampling mode: the walk ends when
                        // its time passes the film's, above) ----
                        const float albedo = surface ? avg3(kd)
                            : avg3(mk(sig_s.x / sig_t.x, sig_s.y / sig_t.y, sig_s.z / sig_t.z));
                        const bool tsm = kTimeSampling && (flags & kFlagTimeSampling) != 0;
                        const bool survive = tsm || !(pcg_float(rng) > albedo);
                        const float prr = tsm ? 1.0f : albedo;
                        if (kGuided && surface && survive && !(ggx && alpha < p.guide.min_alpha)) {
                            // ---- direction deferred to the learned proposal (k_guide) ----
                            want_guide = true;
                            gv[0] = make_uint4(__float_as_uint(pos.x), __float_as_uint(pos.y), __float_as_uint(pos.z),
                                               __float_as_uint(time));
                            gv[1] = make_uint4(__float_as_uint(dir.x), __float_as_uint(dir.y), __float_as_uint(dir.z),
                                               __float_as_uint(prr));
                            gv[2] = make_uint4(__float_as_uint(f.x), __float_as_uint(f.y), __float_as_uint(f.z),
                                               __float_as_uint(__ldg(&sc.tri_ng[id]).w));
                            gv[3] = make_uint4(__float_as_uint(nrm.x), __float_as_uint(nrm.y), __float_as_uint(nrm.z), slot);
                        } else if (survive) {
                            // ---- outgoing direction ----
                            f3 fa, nd;
                            float pa;
                            bool alive = true;
                            bool angular = false;
                            float nds_first = 0.0f;
                            if (tsm && !surface) {
                                // time sampling in the medium: the next free flight r first
                                // (generate_path, BidirectionalPathTracing.h:530-545), then the
                                // time-angular sampler towards the path's light point with
                                // probability 1 when its bounds leave at least one exposure
                                // (:365-405), else (or when its density is < 1e-5) the phase
                                // function (:408-418)
                                nds_first = -tr_log(pcg_float(rng)) / lambda;
                                const float4 tg = p.wave.target[slot];
                                const f3 l = mk(tg.x, tg.y, tg.z) - pos;
                                const float mod = sqrtf(dot(l, l));
                                const float ta = mod + time;
                                float t_a = ta, t_b = total_time;
                                if (nds_first > mod) t_a = fmaxf(t_a, 2.0f * nds_first - mod);
                                else t_a = fmaxf(t_a, mod);
                                t_b = fminf(t_b, 2.0f * nds_first + mod);
                                const bool use_ts = !((total_time - (ta + nds_first)) < film.exposure);
                                (void)pcg_float(rng);                          // the choice xi < p_ts
                                if (use_ts) {
                                    const float e = pcg_float(rng), e2 = pcg_float(rng);
                                    const TaSample ts = time_angular_sample(l, mod, nds_first, t_a, t_b, e, e2, dir, g);
                                    if (ts.pa >= 1e-5f) {
                                        angular = true;
                                        nd = ts.nd;
                                        fa = mk(ts.ph * sig_s.x, ts.ph * sig_s.y, ts.ph * sig_s.z);
                                        pa = ts.pa;
                                    }
                                }
                            }
                            const float x1 = angular ? 0.0f : pcg_float(rng);
                            const float x2 = angular ? 0.0f : pcg_float(rng);
                            float sp, cp;
                            tr_sincos2pi(x1, &sp, &cp);
                            if (angular) {
                            } else if (surface && ggx) {
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
                                if (medium) nds = (tsm && !surface) ? nds_first : -tr_log(pcg_float(rng)) / lambda;
                                p.wave.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, nds);
                                p.wave.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, time);
                                p.wave.thr[slot] = make_float4(fn.x, fn.y, fn.z, prr * pa);
                                want_next = true;
                                oct = (nd.x < 0.0f ? 1u : 0u) | (nd.y < 0.0f ? 2u : 0u) | (nd.z < 0.0f ? 4u : 0u);
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
        // ---- shadow queue: warp-aggregated appends (order preserved within the warp) ----
        const unsigned lt = lanemask_lt();
        // ---- shadow and next-ray queues: the block's rays grouped by direction octant (one
        // atomic per queue and block), so a warp of k_shadow / k_extend takes rays heading the
        // same way; the shadow rays of a light also share their origin ----
        if (threadIdx.x < 8) { oc[threadIdx.x] = 0; sc8[threadIdx.x] = 0; }
        __syncthreads();
        uint32_t rk = 0, rs = 0;
        if (want_next) rk = atomicAdd(&oc[oct], 1u);
        if (want_shadow) rs = atomicAdd(&sc8[soct], 1u);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tot = 0, tsh = 0;
            for (int o = 0; o < 8; ++o) { ob[o] = tot; tot += oc[o]; sb8[o] = tsh; tsh += sc8[o]; }
            const uint32_t g0 = tot ? atomicAdd(&p.wave.counters[cnt_ext(depth + 1)], tot) : 0u;
            const uint32_t s0 = tsh ? atomicAdd(&p.wave.counters[cnt_sh(depth)], tsh) : 0u;
            for (int o = 0; o < 8; ++o) { ob[o] += g0; sb8[o] += s0; }
        }
        __syncthreads();
        if (want_shadow) {
            const uint32_t k = sb8[soct] + rs;
            p.wave.sh_o[k] = sh_o;
            p.wave.sh_d[k] = sh_d;
            p.wave.sh_L[k] = sh_L;
        }
        if (want_next) qout[ob[oct] + rk] = slot;
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
// A CTA owns `G` whole pixels of the batch.  A warp reads one record per lane and step; lanes
// holding the same (pixel, bin) sum their radiance with shuffles and the group's lowest lane
// adds the sum to the FP64 film with native double atomics (resolved in L2, so the film cells
// of a pixel's hot bins stay on chip while its warps add to them).  Steady sums are kept per
// lane and added the same way once per pass over the slots.
// -----------------------------------------------------------------------------------------

// Averaged film cells in the reference's .hdr encoding (the host writer's rgbe_encode of
// avg_nan0(sum, weight), tr_film_io.cpp; ImageIO.h:146-193): the average in double rounded to
// float (NaN -> 0), then the largest channel v = m 2^e (frexp, m in [0.5, 1)), scale m 256 / v,
// each channel truncated to [0, 255], exponent e + 128; 0 for v < 1e-32.
__device__ __forceinline__ float film_avg(double v, double w) {
    const double t = v / w;
    return isnan(t) ? 0.0f : (float)t;
}
__device__ __forceinline__ unsigned char rgbe_q(float c, float scale) {
    const float s = c * scale;
    return (unsigned char)(s > 0.f ? (s < 255.f ? s : 255.f) : 0.f);
}
// cell c (three FP64 sums, read through L2: just written by this block's atomics)
__device__ __forceinline__ uchar4 rgbe_cell(const double* c, double w) {
    const float r = film_avg(__ldcg(c), w), g = film_avg(__ldcg(c + 1), w), b = film_avg(__ldcg(c + 2), w);
    float v = r > g ? r : g;
    v = v > b ? v : b;
    if (!(v >= 1e-32f)) return make_uchar4(0, 0, 0, 0);
    int e = 0;
    const float m = frexpf(v, &e);
    const float scale = m * 256.0f / v;
    return make_uchar4(rgbe_q(r, scale), rgbe_q(g, scale), rgbe_q(b, scale), (unsigned char)(e + 128));
}

// Sum (x, y, z) over the lanes of `peers` (the calling lane's group, all lanes active); the
// group's lowest lane receives the total.  Tree over the group's ranks: at step s the member of
// rank r (r a multiple of 2s) adds the partial sum of rank r + s.  Each lane keeps the lane
// index of the member s ranks above it (32: none) and doubles that distance per step by
// pointer jumping.  `steps_to` is the largest group size that has to be summed.
__device__ __forceinline__ void group_sum3(unsigned peers, unsigned lane, uint32_t steps_to, float& x, float& y,
                                          float& z) {
    const int rank = __popc(peers & lanemask_lt());
    const unsigned above = peers & ~((2u << lane) - 1u);      // lane 31: 2u << 31 == 0
    int up = above ? __ffs(above) - 1 : 32;
    for (int step = 1; step < (int)steps_to; step <<= 1) {
        const int src = up < 32 ? up : (int)lane;
        const float ox = __shfl_sync(kFull, x, src);
        const float oy = __shfl_sync(kFull, y, src);
        const float oz = __shfl_sync(kFull, z, src);
        const int up2 = __shfl_sync(kFull, up, src);
        if ((rank & (2 * step - 1)) == 0 && up < 32) { x += ox; y += oy; z += oz; }
        up = up < 32 ? up2 : 32;
    }
}

template <bool kMulti>
__global__ void __launch_bounds__(kSplatBlock) k_splat(const __grid_constant__ Params p, int G_launch, int bsel) {
    // the block's segment and film: the launch's own in single-scene mode; in multi-scene mode
    // from the current batch's block table, each segment with its own pixels per block
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
    // film pixel of the block's pixel `pl`
    auto film_pixel = [&](uint32_t pl) {
        const uint32_t wpix = B.pix_begin + pix0 + pl;
        return (size_t)(B.win_y0 + wpix / B.win_w) * film.W + (B.win_x0 + wpix % B.win_w);
    };
    const uint32_t per_pix = B.ns * B.ninc;
    const uint32_t nslots = gp * per_pix;
    const uint32_t slot0 = B.slot_begin + pix0 * per_pix;
    const size_t rs = p.wave.capacity;           // records are [bounce][slot]
    const unsigned lane = threadIdx.x & 31u;
    // RGBE images of a fresh film: one bit per (pixel, bin) cell this block adds to (dynamic
    // shared memory, sized by the launcher)
    extern __shared__ uint32_t touched[];
    const bool mark = !kMulti && bsel < 0 && film.rgbe_streak != nullptr && film.rgbe_fresh != 0u;
    if (mark) {
        for (uint32_t i = threadIdx.x; i < (gp * T + 31u) / 32u; i += blockDim.x) touched[i] = 0u;
        __syncthreads();
    }
    for (uint32_t base = (threadIdx.x & ~31u); base < nslots; base += blockDim.x) {
        const uint32_t ls = base + lane;
        const bool act = ls < nslots;
        const uint32_t slot = slot0 + (act ? ls : 0u);
        const uint32_t cnt = act ? (uint32_t)p.wave.rec_n[slot] : 0u;
        const uint32_t pl = act ? ls / per_pix : 0u;
        // a warp's 32 slots span at most 32 pixels: keys (pixel - the warp's first) * T + bin
        // stay below 32 * 2^24 and never reach the out-of-window key
        const uint32_t pl_rel = pl - __shfl_sync(kFull, pl, 0);
        float ax = 0.f, ay = 0.f, az = 0.f;              // this lane's steady-image sum
        const uint32_t kmax = __reduce_max_sync(kFull, cnt);
        // records are streamed (read once); the next one is in flight while this one is summed
        float4 next = make_float4(0.f, 0.f, 0.f, 0.f);
        if (cnt > 0u) next = __ldcs(&p.wave.rec[slot]);
        for (uint32_t k = 0; k < kmax; ++k) {
            const bool valid = k < cnt;
            const float4 rc = next;
            if (k + 1u < cnt) next = __ldcs(&p.wave.rec[(size_t)(k + 1u) * rs + slot]);
            const uint32_t bin = __float_as_uint(rc.w) & 0x00ffffffu;
            const uint32_t rdepth = __float_as_uint(rc.w) >> 24;
            const bool mine = valid && (bsel < 0 || min(rdepth, nb_last) == (uint32_t)bsel);
            const bool inwin = mine && bin != kBinOutside;
            const uint32_t key = inwin ? pl_rel * T + bin : 0xffffffffu;
            const unsigned peers = __match_any_sync(kFull, key);
            const uint32_t maxg = __reduce_max_sync(kFull, inwin ? (uint32_t)__popc(peers) : 1u);
            float vx = rc.x, vy = rc.y, vz = rc.z;
            group_sum3(peers, lane, maxg, vx, vy, vz);
            if (inwin && (peers & lanemask_lt()) == 0u) {
                double* cell = out_streak + film_pixel(pl) * TT + (size_t)bin * 3u;
                atomicAdd(cell, (double)vx); atomicAdd(cell + 1, (double)vy); atomicAdd(cell + 2, (double)vz);
                if (mark) {
                    const uint32_t c = pl * T + bin;
                    atomicOr(&touched[c >> 5], 1u << (c & 31u));
                }
            }
            if (inwin || (steady_all && valid)) { ax += rc.x; ay += rc.y; az += rc.z; }
        }
        // steady image: lanes of the same pixel sum, the group's lowest lane adds
        const bool has = act && (ax != 0.f || ay != 0.f || az != 0.f);
        const unsigned peers = __match_any_sync(kFull, has ? pl_rel : 0xffffffffu);
        const uint32_t maxg = __reduce_max_sync(kFull, has ? (uint32_t)__popc(peers) : 1u);
        group_sum3(peers, lane, maxg, ax, ay, az);
        if (has && (peers & lanemask_lt()) == 0u) {
            double* sd = out_steady + film_pixel(pl) * 3u;
            atomicAdd(sd, (double)ax); atomicAdd(sd + 1, (double)ay); atomicAdd(sd + 2, (double)az);
        }
    }
    // weight: one per camera sample (atomic: batches on different lanes can hold different
    // sample chunks of the same pixels)
    if (bsel < 0)
        for (uint32_t pl = threadIdx.x; pl < gp; pl += blockDim.x) atomicAdd(&film.weight[film_pixel(pl)], (double)B.ns);
    if constexpr (!kMulti) {
        if (bsel < 0 && film.rgbe_streak) {
            // the block's pixels are final: their images, cell by cell (the block's own atomics
            // are visible to it after the barrier)
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < gp * (T + 1u); i += blockDim.x) {
                if (i < gp * T) {
                    const uint32_t pl = i / T, t = i - pl * T;
                    const size_t fp = film_pixel(pl);
                    // a cell of a fresh film that this block did not add to is zero: RGBE 0
                    const bool any = !mark || ((touched[i >> 5] >> (i & 31u)) & 1u) != 0u;
                    film.rgbe_streak[fp * T + t] =
                        any ? rgbe_cell(out_streak + fp * TT + (size_t)t * 3u, __ldcg(&film.weight[fp]))
                            : make_uchar4(0, 0, 0, 0);
                } else {
                    const size_t fp = film_pixel(i - gp * T);
                    film.rgbe_steady[fp] = rgbe_cell(out_steady + fp * 3u, __ldcg(&film.weight[fp]));
                }
            }
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
// Bidirectional connections (BidirectionalPathTracing with set_path_tracing_only(false)) in
// time-sampling mode, scenes without a medium.  Per batch: k_raygen draws the path's light
// point (as for time sampling); k_light_raygen emits the light subpath from it on the light
// wave (its own rays, queues, counters and PCG32 stream); k_extend + k_light_shade walk it,
// storing its vertices; the eye walk (k_extend / k_shade / k_shadow) stores the eye vertices
// next to its next-event estimates; per eye depth k_connect_gen queues the connection rays,
// k_shadow traces them and records the pairs the reference connects, and k_connect_compact
// appends those records after the slot's next-event records.
// -----------------------------------------------------------------------------------------

// slot -> (pixel, camera sample, incoming sample) of a single-scene batch
struct SlotId { uint32_t pixel; unsigned long long s; uint32_t j; };
__device__ __forceinline__ SlotId slot_id(const Params& p, uint32_t i) {
    const Batch& B = p.batch;
    const uint32_t per_pix = B.ns * B.ninc;
    const uint32_t li = i - B.slot_begin;
    const uint32_t pl = li / per_pix;
    const uint32_t rem = li - pl * per_pix;
    const uint32_t sl = rem / B.ninc;
    const uint32_t wpix = B.pix_begin + pl;
    SlotId r;
    r.pixel = (B.win_y0 + wpix / B.win_w) * p.film.W + (B.win_x0 + wpix % B.win_w);
    r.s = B.s0 + sl;
    r.j = rem - sl * B.ninc;
    return r;
}

// Lambertian direction at a surface vertex, in the frame the eye walk uses (orthonormal frame
// with TR_FLAG_ORTHONORMAL_FRAME, else Intersection::set_coordinate_system's, Intersection.h:
// 167-178); same operations as k_shade's.
__device__ __forceinline__ void lambert_sample(uint32_t flags, f3 nrm, f3 kd, float x1, float x2, f3& nd, f3& fa,
                                               float& pa) {
    float sp, cp;
    tr_sincos2pi(x1, &sp, &cp);
    const float ct = sqrtf(x2);
    const float stt = sqrtf(1.0f - ct * ct);
    if (flags & kFlagOrthoFrame) {
        const Frame3 Fr = make_frame(nrm);
        nd = to_world(Fr, mk(cp * stt, sp * stt, ct));
        fa = mk((kd.x * kInvPi) * ct, (kd.y * kInvPi) * ct, (kd.z * kInvPi) * ct);
    } else {
        const f3 aux = fabsf(nrm.x) > fabsf(nrm.z) ? mk(-nrm.y, nrm.x, nrm.z) : mk(0.0f, -nrm.z, nrm.y);
        const f3 tv = normalize(aux);
        const f3 tu = cross(nrm, tv);
        const f3 w = ((tu * (cp * stt)) + (nrm * ct)) + (tv * (sp * stt));
        nd = normalize(w);
        const float ca = fabsf(dot(nrm, nd));
        fa = mk((kd.x * kInvPi) * ca, (kd.y * kInvPi) * ca, (kd.z * kInvPi) * ca);
    }
    pa = ct * kInvPi;
}

// light subpath emission (generate_path FROM_LIGHT started at BidirectionalPathTracing.h:
// 1121-1124): direction from PointLightSource::sample (uniform sphere, PointLightSource.h:
// 174-183, Sampling.h:80-94) or RectangularAreaLightSource::sample (cosine lobe about the
// normal, RectangularAreaLightSource.h:252-276, Sampling.h:131-143); initial pdf (1 / lights) x
// emission pdf; subpath value = emitted intensity (times cos for the rectangle).
__global__ void __launch_bounds__(256) k_light_raygen(const __grid_constant__ Params pl) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pl.batch.n_slots) return;
    const SlotId id = slot_id(pl, i);
    Pcg rl;
    pcg_seed(rl, pl.seed + (unsigned long long)(id.j + 1) * kGolden64 + kLightStateSalt,
             cam_id(id.pixel, id.s) ^ kLightSeqSalt);
    const float4 tg = pl.wave.target[i];
    const SceneDev& sc = pl.scene;
    const float4* L = sc.lights + 5 * __float_as_uint(tg.w);
    const float4 L0 = __ldg(L), L1 = __ldg(L + 1);
    const float e1 = pcg_float(rl), e2 = pcg_float(rl);
    float sp, cp;
    tr_sincos2pi(e1, &sp, &cp);
    f3 dir, val;
    float pdf_dir;
    if (__float_as_uint(L0.w) == 1u) {
        const float ct = sqrtf(e2);
        const float stt = sqrtf(1.0f - ct * ct);
        const f3 ln = f3of(__ldg(L + 4));
        dir = mh_from_y(ln, mk(cp * stt, ct, sp * stt));
        pdf_dir = ct * kInvPi;
        const float dl = dot(dir, ln);
        val = mk(L1.x * dl, L1.y * dl, L1.z * dl);
        pdf_dir = (1.0f / L1.w) * pdf_dir;
    } else {
        const float ct = (float)(1.0 - 2.0 * (double)e2);
        const float stt = sqrtf(1.0f - ct * ct);
        dir = mk(cp * stt, ct, sp * stt);
        pdf_dir = kInv4Pi;
        val = mk(L1.x, L1.y, L1.z);
    }
    const float pi = (1.0f / (float)sc.num_lights) * pdf_dir;
    pl.wave.ray_o[i] = make_float4(tg.x, tg.y, tg.z, __int_as_float(0x7f800000));
    pl.wave.ray_d[i] = make_float4(dir.x, dir.y, dir.z, 0.0f);
    pl.wave.thr[i] = make_float4(1.0f, 1.0f, 1.0f, pi);
    pl.wave.rng[i] = rl.state;
    pl.bd.L0[i] = make_float4(val.x, val.y, val.z, 0.0f);
    pl.bd.nl[i] = 0;
}

// one light subpath vertex per queued slot: throughput over the step's pdf, delay, stored
// while within the film (TotalTime termination, no Russian roulette); then the next Lambertian
// direction.  The walk is in vacuum (the reference's light ray carries no medium).
__global__ void __launch_bounds__(256) k_light_shade(const __grid_constant__ Params pl, int depth) {
    const uint32_t n = depth == 0 ? pl.batch.n_slots : pl.wave.counters[cnt_ext(depth)];
    const uint32_t* qin = pl.wave.q[depth & 1];
    uint32_t* qout = pl.wave.q[(depth + 1) & 1];
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const SceneDev& sc = pl.scene;
    const float total_time = (float)pl.film.T * pl.film.exposure + pl.film.offset;
    const size_t cap = pl.wave.capacity;
    for (uint32_t base = warp_global * 32u; base < n; base += nwarps * 32u) {
        const uint32_t idx = base + lane;
        bool want_next = false;
        uint32_t slot = 0;
        if (idx < n) {
            slot = depth == 0 ? idx : qin[idx];
            const float4 h = pl.wave.hit[slot];
            const uint32_t tid = __float_as_uint(h.y);
            if (tid != kInvalid) {
                const float4 ro = pl.wave.ray_o[slot], rd = pl.wave.ray_d[slot], th = pl.wave.thr[slot];
                const float dist = h.x;
                const f3 f = mk(th.x / th.w, th.y / th.w, th.z / th.w);
                const float time = rd.w + dist;
                if (!(time > total_time)) {
                    const f3 pos = mk(ro.x, ro.y, ro.z) + mk(rd.x, rd.y, rd.z) * dist;
                    const float4 ng = __ldg(&sc.tri_ng[tid]);
                    const float4 m = __ldg(&sc.mats[__float_as_uint(ng.w)]);
                    const f3 nrm = mk(ng.x, ng.y, ng.z), kd = mk(m.x, m.y, m.z);
                    float4* v = pl.bd.lvert + (size_t)depth * 4 * cap + slot;
                    v[0] = make_float4(pos.x, pos.y, pos.z, time);
                    v[cap] = make_float4(nrm.x, nrm.y, nrm.z, th.w);
                    v[2 * cap] = make_float4(kd.x, kd.y, kd.z, 0.0f);
                    v[3 * cap] = make_float4(f.x, f.y, f.z, 0.0f);
                    pl.bd.nl[slot] = (uint8_t)(depth + 1);
                    if ((uint32_t)depth + 1u < pl.bd.nvert) {
                        const SlotId id = slot_id(pl, slot);
                        Pcg rl;
                        rl.state = pl.wave.rng[slot];
                        rl.inc = ((cam_id(id.pixel, id.s) ^ kLightSeqSalt) << 1u) | 1ull;
                        const float x1 = pcg_float(rl), x2 = pcg_float(rl);
                        f3 nd, fa;
                        float pa;
                        lambert_sample(pl.flags, nrm, kd, x1, x2, nd, fa, pa);
                        const f3 fn = mulv(f, fa);
                        pl.wave.ray_o[slot] = make_float4(pos.x, pos.y, pos.z, __int_as_float(0x7f800000));
                        pl.wave.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, time);
                        pl.wave.thr[slot] = make_float4(fn.x, fn.y, fn.z, 1.0f * pa);
                        pl.wave.rng[slot] = rl.state;
                        want_next = true;
                    }
                }
            }
        }
        const unsigned mn = __ballot_sync(kFull, want_next);
        uint32_t bn = 0;
        if (lane == 0 && mn) bn = atomicAdd(&pl.wave.counters[cnt_ext(depth + 1)], (uint32_t)__popc(mn));
        bn = __shfl_sync(kFull, bn, 0);
        if (want_next) qout[bn + (uint32_t)__popc(mn & lanemask_lt())] = slot;
    }
}

struct BVert { f3 pos; float time; f3 n; float pdf; f3 kd; f3 f; };
__device__ __forceinline__ BVert load_vert(const float4* base, uint32_t v, size_t cap, uint32_t slot) {
    const float4* q = base + (size_t)v * 4 * cap + slot;
    const float4 a = q[0], b = q[cap], c = q[2 * cap], d = q[3 * cap];
    BVert r;
    r.pos = mk(a.x, a.y, a.z); r.time = a.w;
    r.n = mk(b.x, b.y, b.z); r.pdf = b.w;
    r.kd = mk(c.x, c.y, c.z);
    r.f = mk(d.x, d.y, d.z);
    return r;
}
__device__ __forceinline__ f3 load_pos(const float4* base, uint32_t v, size_t cap, uint32_t slot) {
    const float4 a = base[(size_t)v * 4 * cap + slot];
    return mk(a.x, a.y, a.z);
}
__device__ __forceinline__ float4 load_npdf(const float4* base, uint32_t v, size_t cap, uint32_t slot) {
    return base[((size_t)v * 4 + 1) * cap + slot];
}

// PathMIS::connection_probability (PathMIS.h:49-60) for Lambertian vertices: the density with
// which the vertex at `from` (normal nf) samples the direction towards `to`.
__device__ __forceinline__ float conn_prob(f3 from, f3 nf, f3 to) {
    const f3 d = normalize(to - from);
    const float c = dot(d, nf);
    return (c > 0.0f ? c : 0.0f) * kInvPi;
}

// PathMIS::compute_weight with beta = 1 (PathMIS.h:63-111): ratios accumulated by addition
// along each subpath, as the reference does; the caller divides by the result
// (BidirectionalPathTracing.h:1034).  t = eye vertex index, s = light vertex index.
__device__ float mis_quantity(const Params& p, uint32_t slot, uint32_t t, uint32_t s, f3 et_pos, float4 et_npdf,
                              f3 ls_pos, float4 ls_npdf) {
    const size_t cap = p.wave.capacity;
    float iw = 1.0f;
    if (s > 1) {
        const float p_s_1 = conn_prob(et_pos, mk(et_npdf.x, et_npdf.y, et_npdf.z), ls_pos) / ls_npdf.w;
        iw = iw + p_s_1;
        float p_i_0 = p_s_1;
        f3 nxt_pos = ls_pos;
        f3 nxt_n = mk(ls_npdf.x, ls_npdf.y, ls_npdf.z);
        for (uint32_t i = s - 1; i > 0; --i) {
            const f3 pos_i = load_pos(p.bd.lvert, i, cap, slot);
            const float4 np_i = load_npdf(p.bd.lvert, i, cap, slot);
            float p_i = conn_prob(nxt_pos, nxt_n, pos_i);
            p_i = p_i_0 + p_i / np_i.w;
            iw = iw + p_i;
            p_i_0 = p_i;
            nxt_pos = pos_i;
            nxt_n = mk(np_i.x, np_i.y, np_i.z);
        }
    }
    if (t > 1) {
        const float p_t_1 = conn_prob(ls_pos, mk(ls_npdf.x, ls_npdf.y, ls_npdf.z), et_pos) / et_npdf.w;
        iw = iw + p_t_1;
        float p_i_0 = p_t_1;
        f3 nxt_pos = et_pos;
        f3 nxt_n = mk(et_npdf.x, et_npdf.y, et_npdf.z);
        for (uint32_t i = t - 1; i > 0; --i) {
            const f3 pos_i = load_pos(p.bd.evert, i, cap, slot);
            const float4 np_i = load_npdf(p.bd.evert, i, cap, slot);
            float p_i = conn_prob(nxt_pos, nxt_n, pos_i);
            p_i = p_i_0 + p_i / np_i.w;
            iw = iw + p_i;
            p_i_0 = p_i;
            nxt_pos = pos_i;
            nxt_n = mk(np_i.x, np_i.y, np_i.z);
        }
    }
    return (float)(1.0 / (double)iw);
}

// Eye-light vertex connections of eye depth ie (transient connect_paths,
// BidirectionalPathTracing.h:1018-1041; connect_vertices' shadow connection, :840-871): for every
// slot, the pairs (ie, il) with ie + il + 2 <= max_bounces whose delays fit the film each get a
// connection ray from the light vertex to the eye vertex in the connection queue, with the
// sample the pair contributes -- value fe * (fv * (f_l * L0)) / w, time = distance + both
// delays, bounce ie + il + 1 -- and its fixed record index (after the slot's next-event
// records, in (ie, il) order).  k_shadow then records the pairs whose segment is blocked (the
// reference connects when World::intersects returns true, World.h:617-639 / 693-697).
// One slot per thread; the warp appends its rays with one atomic.
__global__ void __launch_bounds__(256) k_connect_gen(const __grid_constant__ Params p, int ie) {
    const FilmDev& film = p.film;
    const size_t cap = p.wave.capacity;
    const float total_time = (float)film.T * film.exposure + film.offset;
    const float inv_inc = 1.0f / (float)p.batch.ninc;
    const uint32_t maxb = p.max_bounces;
    const uint32_t uie = (uint32_t)ie;
    const uint32_t off = uie * (maxb - 1u) - uie * (uie - 1u) / 2u;      // records of eye depths < ie
    uint32_t* counter = &p.wave.counters[cnt_sh((int)maxb + ie)];
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < p.batch.n_slots; base += gridDim.x * blockDim.x) {
        const uint32_t slot = base + threadIdx.x;
        const bool have = slot < p.batch.n_slots && uie < p.bd.ne[slot] && p.bd.nl[slot] > 0;
        uint32_t nl = 0;
        BVert E;
        if (have) {
            nl = p.bd.nl[slot];
            E = load_vert(p.bd.evert, uie, cap, slot);
        }
        // the pairs that get a ray (the reference's delay tests, :1020-1024 and :705-711)
        auto traced = [&](uint32_t il, f3& l2e, float& dd) -> int {        // 1 ray, 0 skip, -1 stop
            if (uie + il + 2u > maxb) return -1;
            const float4 a = p.bd.lvert[(size_t)il * 4 * cap + slot];
            if (E.time + a.w > total_time) return -1;
            l2e = E.pos - mk(a.x, a.y, a.z);
            dd = sqrtf(dot(l2e, l2e));
            l2e = divs(l2e, dd);
            return ((dd + E.time) + a.w > total_time) ? 0 : 1;
        };
        uint32_t cnt = 0;
        if (have) {
            for (uint32_t il = 0; il < nl; ++il) {
                f3 l2e; float dd;
                const int t = traced(il, l2e, dd);
                if (t < 0) break;
                cnt += (uint32_t)t;
            }
        }
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        uint32_t wbase = 0;
        if (lane == 0 && total) wbase = atomicAdd(counter, total);
        wbase = __shfl_sync(kFull, wbase, 0);
        if (!have || cnt == 0) continue;
        uint32_t q = wbase + incl - cnt;
        const uint32_t n0 = p.wave.rec_n[slot];
        const float4 L0 = p.bd.L0[slot];
        const float cam_d = film.unwarp ? p.wave.cam_dist[slot] : 0.0f;
        const float4 e_npdf = make_float4(E.n.x, E.n.y, E.n.z, E.pdf);
        for (uint32_t il = 0; il < nl; ++il) {
            f3 l2e; float dd;
            const int t = traced(il, l2e, dd);
            if (t < 0) break;
            if (t == 0) continue;
            const BVert Lv = load_vert(p.bd.lvert, il, cap, slot);
            float ce = -dot(l2e, E.n), cl = dot(l2e, Lv.n);
            ce = ce > 0.0f ? ce : 0.0f;
            cl = cl > 0.0f ? cl : 0.0f;
            const f3 fe = mk((E.kd.x * kInvPi) * ce, (E.kd.y * kInvPi) * ce, (E.kd.z * kInvPi) * ce);
            const f3 fl = mk((Lv.kd.x * kInvPi) * cl, (Lv.kd.y * kInvPi) * cl, (Lv.kd.z * kInvPi) * cl);
            const float att = 1.0f / (dd * dd);
            const f3 fv = mk((fe.x * fl.x) * att, (fe.y * fl.y) * att, (fe.z * fl.z) * att);
            const float w = mis_quantity(p, slot, uie, il, E.pos, e_npdf, Lv.pos,
                                         make_float4(Lv.n.x, Lv.n.y, Lv.n.z, Lv.pdf));
            const float Lr = ((E.f.x * (fv.x * (Lv.f.x * L0.x))) / w) * inv_inc;
            const float Lg = ((E.f.y * (fv.y * (Lv.f.y * L0.y))) / w) * inv_inc;
            const float Lb = ((E.f.z * (fv.z * (Lv.f.z * L0.z))) / w) * inv_inc;
            const float tt = dd + (E.time + Lv.time);
            const float tc = film.unwarp ? tt - cam_d : tt;
            const float ps = (tc - film.offset) / film.exposure;
            const bool inside = ps < (float)film.T && ps >= 0.0f;
            const bool fin = finite3(Lr, Lg, Lb);
            const uint32_t bin = inside ? (uint32_t)floorf(ps) : kBinOutside;
            const uint32_t bounce = uie + il + 1u;
            uint32_t bw = bin | (bounce << 24) | kConnRay;
            if (!(inside || film.nbounce)) bw |= kConnNoRecord;
            const uint32_t k = n0 + off + il;
            p.bd.co_o[q] = make_float4(Lv.pos.x, Lv.pos.y, Lv.pos.z, dd - kSigmaVis);
            p.bd.co_d[q] = make_float4(l2e.x, l2e.y, l2e.z, __uint_as_float(bw));
            p.bd.co_L[q] = fin ? make_float4(Lr, Lg, Lb, __uint_as_float(slot | (k << 24)))
                               : make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(slot | (k << 24)));
            ++q;
        }
    }
}

// After the connection passes: a slot's recorded connections moved, in (ie, il) order, right
// after its next-event records, for k_splat.
__global__ void __launch_bounds__(256) k_connect_compact(const __grid_constant__ Params p) {
    const size_t cap = p.wave.capacity;
    unsigned long long splats = 0;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < p.batch.n_slots;
         slot += gridDim.x * blockDim.x) {
        const uint32_t n0 = p.wave.rec_n[slot];
        uint32_t j = n0;
        for (uint32_t c = 0; c < p.bd.ncand; ++c) {
            const size_t k = (size_t)(n0 + c) * cap + slot;
            if (!p.bd.valid[k]) continue;
            if (j != n0 + c) p.wave.rec[(size_t)j * cap + slot] = p.wave.rec[k];
            ++j;
        }
        splats += j - n0;
        p.wave.rec_n[slot] = (uint8_t)j;
    }
    if (splats) atomicAdd(&p.wave.stats[2], splats);
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

uint32_t splat_pixels_per_block(uint32_t per_pix) {
    // whole pixels that fill one splat block with one slot per thread
    return per_pix >= (uint32_t)kSplatBlock ? 1u : (uint32_t)kSplatBlock / (per_pix ? per_pix : 1u);
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
    if (reinterpret_cast<uintptr_t>(p.scene.nodes) & 31u) return cudaErrorMisalignedAddress;
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
    const bool tsm = multi ? p.wave.target != nullptr : (p.flags & kFlagTimeSampling) != 0;
    const bool guided = p.guide.vrec != nullptr;
    if (multi) {
        if (tsm) {
            if (guided) k_shade<true, true, true><<<grid, block, 0, s>>>(p, depth);
            else k_shade<false, true, true><<<grid, block, 0, s>>>(p, depth);
        } else {
            if (guided) k_shade<true, true, false><<<grid, block, 0, s>>>(p, depth);
            else k_shade<false, true, false><<<grid, block, 0, s>>>(p, depth);
        }
    } else {
        if (tsm) {
            if (guided) k_shade<true, false, true><<<grid, block, 0, s>>>(p, depth);
            else k_shade<false, false, true><<<grid, block, 0, s>>>(p, depth);
        } else {
            if (guided) k_shade<true, false, false><<<grid, block, 0, s>>>(p, depth);
            else k_shade<false, false, false><<<grid, block, 0, s>>>(p, depth);
        }
    }
    return cudaGetLastError();
}
cudaError_t launch_shadow(const Params& p, int depth, int grid, cudaStream_t s) {
    if (reinterpret_cast<uintptr_t>(p.scene.nodes) & 31u) return cudaErrorMisalignedAddress;
    if (p.multi.scenes) k_shadow<true><<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    else k_shadow<false><<<grid, kTraceBlock, trace_smem_bytes(p.bvh_depth), s>>>(p, depth);
    return cudaGetLastError();
}
cudaError_t launch_splat(const Params& p, cudaStream_t s, int bsel) {
    if (p.multi.scenes) {
        k_splat<true><<<p.multi.max_splat_blocks, kSplatBlock, 0, s>>>(p, 0, bsel);
    } else {
        const uint32_t G = splat_pixels_per_block(p.batch.ns * p.batch.ninc);
        const uint32_t blocks = (p.batch.npix + G - 1) / G;
        // a fresh film's RGBE images: the cells each block adds to, one bit each (up to 32 KB;
        // beyond that every cell is read back)
        const size_t bits = (size_t)G * p.film.T;
        const bool mark = bsel < 0 && p.film.rgbe_streak && p.film.rgbe_fresh && bits <= 32u * 8192u;
        if (p.film.rgbe_fresh && !mark) {
            Params q = p;
            q.film.rgbe_fresh = 0;
            k_splat<false><<<blocks, kSplatBlock, 0, s>>>(q, (int)G, bsel);
        } else {
            k_splat<false><<<blocks, kSplatBlock, mark ? (bits + 31u) / 32u * 4u : 0u, s>>>(p, (int)G, bsel);
        }
    }
    return cudaGetLastError();
}
cudaError_t launch_bounce_weights(const Params& p, cudaStream_t s) {
    const uint32_t ncs = p.batch.npix * p.batch.ns;
    k_bounce_weights<<<std::max(1u, std::min(4096u, (ncs + 255) / 256)), 256, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_light_raygen(const Params& pl, cudaStream_t s) {
    const uint32_t n = pl.batch.n_slots;
    k_light_raygen<<<std::max(1u, (n + 255) / 256), 256, 0, s>>>(pl);
    return cudaGetLastError();
}
cudaError_t launch_light_shade(const Params& pl, int depth, cudaStream_t s) {
    int dev = 0, grid = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&grid, cudaDevAttrMultiProcessorCount, dev);
    grid *= 8;
    const uint32_t need = (pl.batch.n_slots + 255) / 256;
    if ((uint32_t)grid > need) grid = (int)need;
    k_light_shade<<<std::max(1, grid), 256, 0, s>>>(pl, depth);
    return cudaGetLastError();
}
cudaError_t launch_connect_gen(const Params& p, int ie, cudaStream_t s) {
    const uint32_t n = p.batch.n_slots;
    k_connect_gen<<<std::max(1u, std::min(4096u, (n + 255) / 256)), 256, 0, s>>>(p, ie);
    return cudaGetLastError();
}
cudaError_t launch_connect_compact(const Params& p, cudaStream_t s) {
    const uint32_t n = p.batch.n_slots;
    k_connect_compact<<<std::max(1u, std::min(4096u, (n + 255) / 256)), 256, 0, s>>>(p);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_build_tris(const float* __restrict__ v, const uint32_t* __restrict__ t,
                                                    const uint32_t* __restrict__ mat, const uint32_t* __restrict__ order,
                                                    uint32_t nt, float4* __restrict__ tris, float4* __restrict__ tri_ng) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        const uint32_t id = order[i];
        const uint32_t a = t[3 * (size_t)id], b = t[3 * (size_t)id + 1], c = t[3 * (size_t)id + 2];
        const f3 p0 = mk(v[3 * (size_t)a], v[3 * (size_t)a + 1], v[3 * (size_t)a + 2]);
        const f3 p1 = mk(v[3 * (size_t)b], v[3 * (size_t)b + 1], v[3 * (size_t)b + 2]);
        const f3 p2 = mk(v[3 * (size_t)c], v[3 * (size_t)c + 1], v[3 * (size_t)c + 2]);
        tris[3 * (size_t)i] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(id));
        tris[3 * (size_t)i + 1] = make_float4(p1.x, p1.y, p1.z, 0.0f);
        tris[3 * (size_t)i + 2] = make_float4(p2.x, p2.y, p2.z, 0.0f);
        const f3 n = normalize(cross(p2 - p0, p1 - p0));
        tri_ng[id] = make_float4(n.x, n.y, n.z, __uint_as_float(mat[id]));
    }
}
cudaError_t launch_build_tris(const float* vertices, const uint32_t* triangles, const uint32_t* material,
                              const uint32_t* order, uint32_t nt, float4* tris, float4* tri_ng, cudaStream_t s) {
    k_build_tris<<<std::max(1u, std::min(8192u, (nt + 255) / 256)), 256, 0, s>>>(vertices, triangles, material,
                                                                                   order, nt, tris, tri_ng);
    return cudaGetLastError();
}

// FP64 film sums to FP32 (round to nearest); grid-stride, streaming loads
__global__ void __launch_bounds__(256) k_to_f32(const double* __restrict__ src, float* __restrict__ dst, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (float)__ldcs(&src[i]);
}
cudaError_t launch_to_f32(const double* src, float* dst, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t need = (n + 255) / 256;
    const int grid = (int)std::min<size_t>(need, (size_t)sms * 8);
    k_to_f32<<<std::max(1, grid), 256, 0, s>>>(src, dst, n);
    return cudaGetLastError();
}

// last node of a multi-scene batch: the next replay renders the next batch descriptor
__global__ void k_advance(uint32_t* cur, uint32_t step) { *cur += step; }
cudaError_t launch_advance(uint32_t* cur, uint32_t step, cudaStream_t s) {
    k_advance<<<1, 1, 0, s>>>(cur, step);
    return cudaGetLastError();
}
cudaError_t launch_trace_user(const SceneDev& sc, const float* rays, uint32_t n, int any_hit, void* out,
                              uint32_t* cursor, int grid, cudaStream_t s) {
    if (reinterpret_cast<uintptr_t>(sc.nodes) & 31u) return cudaErrorMisalignedAddress;
    k_trace_user<<<grid, kTraceBlock, trace_smem_bytes(sc.bvh_depth), s>>>(sc, rays, n, any_hit,
                                                                          reinterpret_cast<HitOut*>(out), cursor);
    return cudaGetLastError();
}

}  // namespace trk
