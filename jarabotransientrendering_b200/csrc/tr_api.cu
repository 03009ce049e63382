// tr_api.cu - the C ABI (include/transient_b200.h): context, scene upload, wavefront batch
// scheduling and film read-out.  Host code; kernels live in tr_kernels.cu.
#include "transient_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "tr_device.cuh"
#include "tr_film_io.h"
#include "tr_internal.h"

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace tri {
tr_status fail(tr_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}
}  // namespace tri

using namespace tri;


namespace {

tr_status validate(const tr_scene* s, const tr_camera* c, const tr_film* f, const tr_integrator* it) {
    if (!s || !c || !f || !it) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    if (!s->vertices || !s->triangles || !s->triangle_material || s->num_triangles == 0)
        return fail(TR_ERR_INVALID_ARGUMENT, "scene has no triangles");
    if (s->num_materials == 0 || !s->materials) return fail(TR_ERR_INVALID_ARGUMENT, "scene has no materials");
    if (s->num_materials > (uint32_t)trk::kMaxMaterials) return fail(TR_ERR_INVALID_ARGUMENT, "too many materials");
    if (s->num_lights == 0 || !s->lights)
        return fail(TR_ERR_INVALID_ARGUMENT, "scene has no light source (next-event estimation needs one)");
    if (s->num_lights > (uint32_t)trk::kMaxLights) return fail(TR_ERR_INVALID_ARGUMENT, "too many lights");
    for (uint32_t i = 0; i < s->num_triangles; ++i)
        if (s->triangle_material[i] >= s->num_materials)
            return fail(TR_ERR_INVALID_ARGUMENT, "triangle " + std::to_string(i) + " has material index out of range");
    for (uint32_t i = 0; i < s->num_materials; ++i) {
        const tr_material& m = s->materials[i];
        if (m.kind != TR_MAT_LAMBERTIAN && m.kind != TR_MAT_GGX)
            return fail(TR_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + " has unknown kind");
        if (m.kind == TR_MAT_GGX && !(m.alpha >= 1e-3f && m.alpha <= 1.0f))
            return fail(TR_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + ": GGX alpha must be in [0.001, 1]");
        for (float v : m.kd)
            if (!std::isfinite(v)) return fail(TR_ERR_INVALID_ARGUMENT, "material " + std::to_string(i) + " albedo is not finite");
    }
    for (uint32_t i = 0; i < s->num_lights; ++i) {
        const tr_light& L = s->lights[i];
        if (L.kind != TR_LIGHT_POINT && L.kind != TR_LIGHT_RECT)
            return fail(TR_ERR_INVALID_ARGUMENT, "light " + std::to_string(i) + " has unknown kind");
        if (L.kind == TR_LIGHT_RECT && !(L.area > 0.0f))
            return fail(TR_ERR_INVALID_ARGUMENT, "rectangular light " + std::to_string(i) + " has zero area");
    }
    if (s->medium.enabled) {
        for (int k = 0; k < 3; ++k) {
            if (!(s->medium.sigma_a[k] >= 0.0f) || !(s->medium.sigma_s[k] >= 0.0f))
                return fail(TR_ERR_INVALID_ARGUMENT, "medium coefficients must be >= 0");
        }
        float st = (s->medium.sigma_a[0] + s->medium.sigma_s[0]) + (s->medium.sigma_a[1] + s->medium.sigma_s[1]) +
                   (s->medium.sigma_a[2] + s->medium.sigma_s[2]);
        if (!(st > 0.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "medium extinction must be > 0");
        if (!(std::fabs(s->medium.g) < 1.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "HG g must be in (-1, 1)");
    }
    if (f->width == 0 || f->height == 0 || f->time_bins == 0)
        return fail(TR_ERR_INVALID_ARGUMENT, "film has zero size");
    if (!(f->exposure > 0.0f) || !std::isfinite(f->offset))
        return fail(TR_ERR_INVALID_ARGUMENT, "film exposure must be > 0");
    if ((uint64_t)f->width * f->height >= (1ull << 32)) return fail(TR_ERR_INVALID_ARGUMENT, "film too large");
    if (f->camera_unwarp > 1) return fail(TR_ERR_INVALID_ARGUMENT, "camera_unwarp must be 0 or 1");
    if (f->bounce_films > 32) return fail(TR_ERR_INVALID_ARGUMENT, "at most 32 bounce films");
    if (f->components & ~(TR_COMP_DEPTH | TR_COMP_POSITIONS | TR_COMP_NORMALS))
        return fail(TR_ERR_INVALID_ARGUMENT, "unknown film component bits");
    if (f->time_bins >= trk::kBinOutside)     // bin indices are 24-bit fields of the splat records
        return fail(TR_ERR_INVALID_ARGUMENT, "time_bins must be below 16777215");
    if (it->sqrt_spp == 0 || it->incoming_samples == 0)
        return fail(TR_ERR_INVALID_ARGUMENT, "sqrt_spp and incoming_samples must be >= 1");
    if (it->max_bounces > kMaxBounces) return fail(TR_ERR_INVALID_ARGUMENT, "max_bounces must be <= 63");
    if (it->flags & ~(TR_FLAG_ORTHONORMAL_FRAME | TR_FLAG_TIME_SAMPLING | TR_FLAG_BIDIRECTIONAL))
        return fail(TR_ERR_INVALID_ARGUMENT, "unknown integrator flags");
    if (it->flags & TR_FLAG_BIDIRECTIONAL) {
        if (!(it->flags & TR_FLAG_TIME_SAMPLING))
            return fail(TR_ERR_NOT_SUPPORTED, "bidirectional connections need TR_FLAG_TIME_SAMPLING (without it the "
                                              "reference's light subpath starts from an uninitialised light sample "
                                              "and all its connections are dropped: render without the flag)");
        if (s->medium.enabled)
            return fail(TR_ERR_NOT_SUPPORTED, "bidirectional connections in a medium are not defined by the reference "
                                              "(its time-sampled connections dereference a null medium)");
        if (it->max_bounces > TR_BIDIR_MAX_BOUNCES)
            return fail(TR_ERR_NOT_SUPPORTED, "bidirectional connections support max_bounces <= 16");
        for (uint32_t m = 0; m < s->num_materials; ++m)
            if (s->materials[m].kind != TR_MAT_LAMBERTIAN)
                return fail(TR_ERR_NOT_SUPPORTED, "bidirectional connections support Lambertian materials only");
    }
    if (!std::isfinite(c->focal_distance)) return fail(TR_ERR_INVALID_ARGUMENT, "camera focal distance not finite");
    return TR_OK;
}

// Host-to-device copy ordered on `s`, the stream whose kernels read the data.  (A plain
// cudaMemcpy runs on the legacy default stream, which does not order with the library's
// non-blocking streams, and from pageable memory it may return before the data has landed.)
void upload(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    TR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    TR_CUDA(cudaStreamSynchronize(s));        // the host buffer may be released after return
}

}  // namespace

namespace tri {

cudaMemPool_t device_pool(int device) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0) throw CudaError(cudaErrorInvalidDevice, "device_pool");
    if ((size_t)device >= pools.size()) pools.resize((size_t)device + 1, nullptr);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        TR_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = ~0ull;
        TR_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[device] = pool;
    }
    return pools[device];
}

size_t pool_idle_bytes(int device) {
    uint64_t reserved = 0, used = 0;
    cudaMemPool_t pool = device_pool(device);
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess) return 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) return 0;
    return reserved > used ? (size_t)(reserved - used) : 0;
}

void ensure_wave(tr_ctx* x, uint32_t capacity) {
    if (x->wave.capacity >= capacity) return;
    // grow: drop the old buffers (they are only scratch between calls)
    auto drop = [&](void* p) {
        if (!p) return;
        cudaFree(p);
        x->allocs.erase(std::remove(x->allocs.begin(), x->allocs.end(), p), x->allocs.end());
    };
    trk::Wave& w = x->wave;
    drop(w.ray_o); drop(w.ray_d); drop(w.thr); drop(w.rng); drop(w.hit); drop(w.q[0]); drop(w.q[1]);
    drop(w.sh_o); drop(w.sh_d); drop(w.sh_L); drop(w.rec); drop(w.rec_n);
    size_t R = std::max<uint32_t>(1u, x->integ.max_bounces);
    // records per slot: one next-event estimate per bounce, plus with light subpaths one per
    // eye-light vertex pair with ie + il + 2 <= max_bounces
    if (x->integ.flags & TR_FLAG_BIDIRECTIONAL) R += R * (R - 1) / 2;
    w.ray_o = x->alloc<float4>(capacity);
    w.ray_d = x->alloc<float4>(capacity);
    w.thr = x->alloc<float4>(capacity);
    w.rng = x->alloc<unsigned long long>(capacity);
    w.hit = x->alloc<float4>(capacity);
    w.q[0] = x->alloc<uint32_t>(capacity);
    w.q[1] = x->alloc<uint32_t>(capacity);
    w.sh_o = x->alloc<float4>(capacity);
    w.sh_d = x->alloc<float4>(capacity);
    w.sh_L = x->alloc<float4>(capacity);
    w.rec = x->alloc<float4>((size_t)capacity * R);
    w.rec_n = x->alloc<uint8_t>(capacity);
    drop(w.cam_dist);
    w.cam_dist = x->alloc<float>(capacity);
    drop(w.target);
    w.target = (x->integ.flags & TR_FLAG_TIME_SAMPLING) ? x->alloc<float4>(capacity) : nullptr;
    if (x->integ.flags & TR_FLAG_BIDIRECTIONAL) {
        // light wave (own rays, queues, counters; shares target and ray counts) and the
        // subpath vertex arrays
        trk::Wave& lw = x->lwave;
        trk::BidirWave& bd = x->bd;
        drop(lw.ray_o); drop(lw.ray_d); drop(lw.thr); drop(lw.rng); drop(lw.hit); drop(lw.q[0]); drop(lw.q[1]);
        drop(bd.lvert); drop(bd.evert); drop(bd.nl); drop(bd.ne); drop(bd.L0);
        lw = trk::Wave{};
        lw.ray_o = x->alloc<float4>(capacity);
        lw.ray_d = x->alloc<float4>(capacity);
        lw.thr = x->alloc<float4>(capacity);
        lw.rng = x->alloc<unsigned long long>(capacity);
        lw.hit = x->alloc<float4>(capacity);
        lw.q[0] = x->alloc<uint32_t>(capacity);
        lw.q[1] = x->alloc<uint32_t>(capacity);
        if (!x->d_lcounters) x->d_lcounters = x->alloc<uint32_t>(trk::kCounters);
        lw.counters = x->d_lcounters;
        bd.nvert = std::max<uint32_t>(1u, x->integ.max_bounces) - 1u;
        const size_t nv = std::max<uint32_t>(1u, bd.nvert);
        bd.lvert = x->alloc<float4>(nv * 4 * capacity);
        bd.evert = x->alloc<float4>(nv * 4 * capacity);
        bd.nl = x->alloc<uint8_t>(capacity);
        bd.ne = x->alloc<uint8_t>(capacity);
        bd.L0 = x->alloc<float4>(capacity);
        // connection queue of one eye depth (up to nvert rays per slot) and the record flags
        drop(bd.co_o); drop(bd.co_d); drop(bd.co_L); drop(bd.valid);
        bd.co_o = x->alloc<float4>(nv * capacity);
        bd.co_d = x->alloc<float4>(nv * capacity);
        bd.co_L = x->alloc<float4>(nv * capacity);
        bd.ncand = x->integ.max_bounces * (std::max<uint32_t>(1u, x->integ.max_bounces) - 1u) / 2u;
        bd.valid = x->alloc<uint8_t>(R * capacity);
    }
    if (!w.counters) w.counters = x->alloc<uint32_t>(trk::kCounters);
    if (!w.stats) {
        w.stats = x->alloc<unsigned long long>(8);
        TR_CUDA(cudaMemsetAsync(w.stats, 0, 8 * sizeof(unsigned long long), x->s()));
    }
    w.capacity = capacity;
}

// Per-kind kernel times of the pending timed launches and the union of the traversal (extend,
// shadow) launch intervals, into the context's statistics; one cudaEventElapsedTime per event,
// relative to the first pending event.  Clears the pending launches.
// Reads the pending launch events out and adds their kernel times to x->prof_sum (each
// read-out's traversal union is over its own launches, which end before the next read-out's
// begin, so the sums stay exact unions).
cudaError_t prof_readout(tr_ctx* x) {
    if (x->prof_marks.empty()) { x->prof_next = 0; return cudaSuccess; }
    std::vector<float> t(x->prof_next, 0.f);
    for (size_t i = 0; i < x->prof_next; ++i) {
        const cudaError_t e = cudaEventElapsedTime(&t[i], x->prof_events[0], x->prof_events[i]);
        if (e != cudaSuccess) return e;
    }
    std::vector<std::pair<float, float>> trace_iv;
    for (const tr_ctx::ProfMark& m : x->prof_marks) {
        x->prof_sum[m.kind] += t[m.ev + 1] - t[m.ev];
        if (m.kind == 1 || m.kind == 3) trace_iv.push_back({t[m.ev], t[m.ev + 1]});
    }
    std::sort(trace_iv.begin(), trace_iv.end());
    for (size_t i = 0; i < trace_iv.size();) {
        float a = trace_iv[i].first, b = trace_iv[i].second;
        for (++i; i < trace_iv.size() && trace_iv[i].first <= b; ++i) b = std::max(b, trace_iv[i].second);
        x->prof_sum[6] += b - a;
    }
    x->prof_marks.clear();
    x->prof_next = 0;
    x->prof_dirty = true;
    return cudaSuccess;
}

// Moves the accumulated kernel times into x->stats and starts a new sum.
void prof_publish(tr_ctx* x) {
    x->stats.raygen_ms = x->prof_sum[0]; x->stats.extend_ms = x->prof_sum[1]; x->stats.shade_ms = x->prof_sum[2];
    x->stats.shadow_ms = x->prof_sum[3]; x->stats.splat_ms = x->prof_sum[4]; x->stats.guide_ms = x->prof_sum[5];
    x->stats.trace_ms = x->prof_sum[6];
    for (double& v : x->prof_sum) v = 0.0;
    x->prof_dirty = false;
}

// Lane k + 1's buffers: the per-slot arrays of the first wave at its capacity, its own queue
// counters, the first wave's statistics counters.
void ensure_lane_wave(tr_ctx* x, int k) {
    trk::Wave& w = x->lane_wave[k];
    const uint32_t capacity = x->wave.capacity;
    if (w.capacity >= capacity && w.counters) return;
    auto drop = [&](void* p) {
        if (!p) return;
        cudaFree(p);
        x->allocs.erase(std::remove(x->allocs.begin(), x->allocs.end(), p), x->allocs.end());
    };
    drop(w.ray_o); drop(w.ray_d); drop(w.thr); drop(w.rng); drop(w.hit); drop(w.q[0]); drop(w.q[1]);
    drop(w.sh_o); drop(w.sh_d); drop(w.sh_L); drop(w.rec); drop(w.rec_n); drop(w.cam_dist); drop(w.target);
    const size_t R = std::max<uint32_t>(1u, x->integ.max_bounces);
    w.ray_o = x->alloc<float4>(capacity);
    w.ray_d = x->alloc<float4>(capacity);
    w.thr = x->alloc<float4>(capacity);
    w.rng = x->alloc<unsigned long long>(capacity);
    w.hit = x->alloc<float4>(capacity);
    w.q[0] = x->alloc<uint32_t>(capacity);
    w.q[1] = x->alloc<uint32_t>(capacity);
    w.sh_o = x->alloc<float4>(capacity);
    w.sh_d = x->alloc<float4>(capacity);
    w.sh_L = x->alloc<float4>(capacity);
    w.rec = x->alloc<float4>((size_t)capacity * R);
    w.rec_n = x->alloc<uint8_t>(capacity);
    w.cam_dist = x->alloc<float>(capacity);
    w.target = (x->integ.flags & TR_FLAG_TIME_SAMPLING) ? x->alloc<float4>(capacity) : nullptr;
    if (!w.counters) w.counters = x->alloc<uint32_t>(trk::kCounters);
    w.stats = x->wave.stats;
    w.capacity = capacity;
}

// Lane k + 1's guided-vertex records (the training pool and its counters are shared: the
// batches of all lanes fill it, each entry tagged with its batch).
void ensure_lane_guided(tr_ctx* x, int k) {
    const uint32_t capacity = x->wave.capacity;
    if (x->lane_vrec_cap[k] >= capacity && x->lane_vrec[k]) return;
    if (x->lane_vrec[k]) {
        cudaFree(x->lane_vrec[k]);
        x->allocs.erase(std::remove(x->allocs.begin(), x->allocs.end(), (void*)x->lane_vrec[k]), x->allocs.end());
    }
    x->lane_vrec[k] = x->alloc<uint4>((size_t)capacity * 5);
    x->lane_vrec_cap[k] = capacity;
}

void ensure_guided(tr_ctx* x, uint32_t capacity) {
    if (x->gw_capacity >= capacity && x->gw.pool_cap == x->guide_pool && x->pool_state && x->pool_alt.state) return;
    auto drop = [&](void* p) {
        if (!p) return;
        cudaFree(p);
        x->allocs.erase(std::remove(x->allocs.begin(), x->allocs.end(), p), x->allocs.end());
    };
    trk::GuideWave& g = x->gw;
    tr_ctx::PoolBuf& a = x->pool_alt;
    drop(g.vrec); drop(g.pool_feat); drop(g.pool_dir); drop(g.pool_w); drop(g.pool_meta);
    drop(a.feat); drop(a.dir); drop(a.w); drop(a.meta);
    g.vrec = x->alloc<uint4>((size_t)capacity * 5);
    const uint32_t pc = std::max<uint32_t>(1u, x->guide_pool);
    g.pool_feat = x->alloc<uint4>((size_t)pc * 8);
    g.pool_dir = x->alloc<float>((size_t)pc * 3);
    g.pool_w = x->alloc<float>(pc);
    g.pool_meta = x->alloc<uint4>(pc);
    a.feat = x->alloc<uint4>((size_t)pc * 8);
    a.dir = x->alloc<float>((size_t)pc * 3);
    a.w = x->alloc<float>(pc);
    a.meta = x->alloc<uint4>(pc);
    g.pool_cap = x->guide_pool;
    if (!x->pool_state) x->pool_state = x->alloc<uint32_t>(2);
    if (!a.state) a.state = x->alloc<uint32_t>(2);
    if (!x->w_snap) x->w_snap = x->alloc<uint4>(4 * 8192 / 16);
    if (!x->bias_snap) x->bias_snap = x->alloc<float>(4 * 64);
    if (!x->ev_snap) TR_CUDA(cudaEventCreateWithFlags(&x->ev_snap, cudaEventDisableTiming));
    if (!x->ev_train) TR_CUDA(cudaEventCreateWithFlags(&x->ev_train, cudaEventDisableTiming));
    x->pool_pending = 0;                 // a reallocated pool holds nothing to train on
    x->gw_capacity = capacity;
}

trk::Params make_params(tr_ctx* x) {
    trk::Params p{};
    p.scene = x->scene;
    for (int k = 0; k < 3; ++k) {
        p.cam.pos[k] = x->cam.position[k]; p.cam.nv[k] = x->cam.nv[k];
        p.cam.uv[k] = x->cam.uv[k]; p.cam.vv[k] = x->cam.vv[k];
    }
    p.cam.fd = x->cam.focal_distance;
    p.film.streak = x->d_streak; p.film.steady = x->d_steady; p.film.weight = x->d_weight;
    p.film.unwarp = x->film.camera_unwarp;
    p.film.nbounce = x->film.bounce_films;
    p.film.bstreak = x->d_bstreak; p.film.bsteady = x->d_bsteady; p.film.bweight = x->d_bweight;
    p.film.comps = x->film.components;
    p.film.cdepth = x->d_cdepth; p.film.cpos = x->d_cpos; p.film.cnorm = x->d_cnorm;
    p.film.W = x->film.width; p.film.H = x->film.height; p.film.T = x->film.time_bins;
    p.film.exposure = x->film.exposure; p.film.offset = x->film.offset;
    p.wave = x->wave;
    p.bd = x->bd;
    p.seed = x->integ.seed;
    p.max_bounces = x->integ.max_bounces;
    p.sqrt_spp = x->integ.sqrt_spp;
    p.bvh_depth = x->bvh_depth;
    p.flags = x->integ.flags;
    if (x->guide) {
        p.guide = x->gw;
        p.guide.net = guide_dev(x->guide);
        if (x->w_snap) {                 // the render samples with the snapshot taken at its start
            p.guide.net.w_fwd = x->w_snap;
            p.guide.net.bias = x->bias_snap;
        }
        p.guide.err = guide_err(x->guide);
        p.guide.min_alpha = x->guide_min_alpha;
    }
    return p;
}

}  // namespace tri

namespace {

// Guided renders: guide_begin_render snapshots the network for the render and starts training on
// the previous render's samples beside it; guide_end_render waits for that training, reports
// tensor-core timeouts and hands this render's pool to the next call.
tr_status guide_begin_render(tr_ctx* x, cudaStream_t s);
tr_status guide_end_render(tr_ctx* x, cudaStream_t s);

// Host buffers the film is streamed into while rendering (tr_render_film): FP64 or FP32 sums,
// or RGBE images, of the whole frame.
struct FilmSink { int type; void* streak; void* steady; void* weight; };

tr_status render_region(tr_ctx* x, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                        uint64_t s0, uint32_t ns_total, const FilmSink* sink = nullptr) {
    if (x1 > x->film.width || y1 > x->film.height || x0 >= x1 || y0 >= y1)
        return fail(TR_ERR_INVALID_ARGUMENT, "pixel window out of range or empty");
    if (ns_total == 0) return TR_OK;
    if (s0 + ns_total > (1ull << 32)) return fail(TR_ERR_INVALID_ARGUMENT, "camera sample index must stay below 2^32");
    const uint32_t ninc = x->integ.incoming_samples;
    const uint32_t win_w = x1 - x0, win_h = y1 - y0;
    const uint64_t win_pix = (uint64_t)win_w * win_h;
    const uint64_t total_slots = win_pix * (uint64_t)ns_total * ninc;
    // with light subpaths a slot also holds two subpaths' vertices and its connection records
    const uint32_t cap_max = (x->integ.flags & TR_FLAG_BIDIRECTIONAL) ? kDefaultCapacity / 2 : kDefaultCapacity;
    uint32_t cap = (uint32_t)std::min<uint64_t>(total_slots, cap_max);
    cap = std::max<uint32_t>(cap, ninc);
    ensure_wave(x, cap);
    const bool guided = x->guide != nullptr;
    const bool bidir = (x->integ.flags & TR_FLAG_BIDIRECTIONAL) != 0;
    if (guided) {
        ensure_guided(x, cap);
        // about 1.5 guided vertices per path; keep enough of them to fill the training pool
        x->gw.keep_prob = x->guide_pool ? std::min(1.0f, (float)x->guide_pool / (1.5f * (float)total_slots)) : 0.0f;
        x->gw.mix_prob = x->guide_mix;
        TR_CUDA(cudaMemsetAsync(x->pool_state, 0, 2 * sizeof(uint32_t), x->s()));
        tr_status ts = guide_begin_render(x, x->s());
        if (ts != TR_OK) return ts;
    }
    // samples per pixel per batch, and pixels per batch
    uint32_t ns_chunk = std::max<uint32_t>(1u, std::min<uint32_t>(ns_total, cap / ninc));
    const bool film_was_clean = x->film_clean;
    x->film_clean = false;
    cudaStream_t strm = x->s();
    // per-kernel timing: an event before and after each launch, kind-tagged.  Read out at the
    // end of the render (profiling 1) or at tr_stats_get (profiling 2; a long series of renders
    // is read out once 2^16 events are pending)
    if (x->profiling == 2 && x->prof_next > (1u << 16)) TR_CUDA(prof_readout(x));
    if (x->profiling != 2) { x->prof_marks.clear(); x->prof_next = 0; }
    size_t& next_ev = x->prof_next;
    auto ev_get = [&]() -> cudaEvent_t {
        if (next_ev == x->prof_events.size()) {
            cudaEvent_t e;
            TR_CUDA(cudaEventCreate(&e));
            x->prof_events.push_back(e);
        }
        return x->prof_events[next_ev++];
    };
    auto timed_on = [&](int kind, cudaStream_t st, auto&& launch) {
        if (!x->profiling) { TR_CUDA(launch()); return; }
        size_t a = next_ev;
        TR_CUDA(cudaEventRecord(ev_get(), st));
        TR_CUDA(launch());
        TR_CUDA(cudaEventRecord(ev_get(), st));
        x->prof_marks.push_back({kind, a});
    };
    // `to` waits for the work queued on `from` so far
    auto order = [&](cudaStream_t from, cudaStream_t to) -> cudaError_t {
        if (x->dep_events.size() < 4) {
            cudaEvent_t e;
            cudaError_t err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
            if (err != cudaSuccess) return err;
            x->dep_events.push_back(e);
        }
        cudaEvent_t e = x->dep_events[x->next_dep++ % x->dep_events.size()];
        cudaError_t err = cudaEventRecord(e, from);
        return err != cudaSuccess ? err : cudaStreamWaitEvent(to, e, 0);
    };
    // Shadow rays of depth d and closest-hit rays of depth d + 1 both only read what shade(d)
    // wrote, so the shadow launch runs on a second stream and the two persistent traversal
    // kernels fill each other's drain tails.  shade(d + 1) refills the shadow queue and waits
    // for shadow(d); the batch's later work waits for the last shadow launch.
    if (!x->shadow_stream) TR_CUDA(cudaStreamCreateWithFlags(&x->shadow_stream, cudaStreamNonBlocking));
    const cudaStream_t s_sh = x->shadow_stream;
    uint64_t launches = 0, ext_l = 0, sh_l = 0;
    // film streaming: once a pixel batch of the last sample chunk is splatted its film rows are
    // final; the copy stream waits for that point and copies them (FP32: converted on the
    // device first, into a staging buffer the copy stream reuses in order)
    const uint32_t T = x->film.time_bins;
    const bool f32 = sink && sink->type == TR_FILM_F32;
    const bool rgbe = sink && sink->type == TR_FILM_RGBE;
    if (sink) {
        if (!x->copy_stream) {
            // highest priority: its FP32 conversions get SMs as soon as a traversal launch's
            // blocks retire, so the host copies start without waiting behind the other lanes
            int lo = 0, hi = 0;
            TR_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            TR_CUDA(cudaStreamCreateWithPriority(&x->copy_stream, cudaStreamNonBlocking, hi));
        }
        // only the last sample chunk's batches deliver rows; a shorter last chunk packs more
        // pixels into a batch, so the staging buffer is sized by that chunk
        const uint32_t ns_last = ns_total - ((ns_total - 1u) / ns_chunk) * ns_chunk;
        const size_t ppb_last = std::min<uint64_t>(win_pix, std::max<uint32_t>(1u, cap / (ns_last * ninc)));
        const size_t stage = ppb_last * ((size_t)T * 3u + 4u);
        if (f32 && x->stage_floats < stage) {
            x->d_stage = x->alloc<float>(stage);
            x->stage_floats = stage;
        }
        // RGBE: the images of the whole film in device memory (a third of the FP32 bytes), so each
        // batch is encoded on its own lane right after its splat and the copy stream only copies
        const size_t cells = (size_t)x->film.width * x->film.height * ((size_t)T + 1u);
        if (rgbe && x->rgbe_cells < cells) {
            x->d_rgbe = x->alloc<uchar4>(cells);
            x->rgbe_cells = cells;
        }
    }
    // Wave lanes: with more than one pixel batch and each pixel in one batch only (a single
    // sample chunk), consecutive batches alternate between kWaveLanes sets of wave buffers and
    // pairs of streams, so one batch's last, nearly empty depths run beside the next batch's
    // first ones.  The batches share no pixels; with the learned proposal they share the
    // training pool (entries tagged by batch).  Light subpaths (one light wave) keep a single
    // lane.
    const uint64_t n_pix_batches = (win_pix + std::max<uint32_t>(1u, cap / (ns_chunk * ninc)) - 1) /
                                   std::max<uint32_t>(1u, cap / (ns_chunk * ninc));
    const int lanes = (!bidir && ns_chunk >= ns_total)
                          ? (int)std::min<uint64_t>((uint64_t)kWaveLanes, n_pix_batches) : 1;
    uint32_t batch_no = 0;
    for (int k = 0; k + 1 < lanes; ++k) {
        ensure_lane_wave(x, k);
        if (guided) ensure_lane_guided(x, k);
        if (!x->lane_stream[k]) TR_CUDA(cudaStreamCreateWithFlags(&x->lane_stream[k], cudaStreamNonBlocking));
        if (!x->lane_shadow_stream[k])
            TR_CUDA(cudaStreamCreateWithFlags(&x->lane_shadow_stream[k], cudaStreamNonBlocking));
    }
    TR_CUDA(cudaEventRecord(x->ev0, strm));
    for (int k = 0; k + 1 < lanes; ++k) TR_CUDA(order(strm, x->lane_stream[k]));
    for (uint64_t sb = 0; sb < ns_total; sb += ns_chunk) {
        const uint32_t ns = (uint32_t)std::min<uint64_t>(ns_chunk, ns_total - sb);
        const uint32_t per_pix = ns * ninc;
        const uint32_t ppb = std::max<uint32_t>(1u, cap / per_pix);
        for (uint64_t pb = 0; pb < win_pix; pb += ppb) {
            const uint32_t npix = (uint32_t)std::min<uint64_t>(ppb, win_pix - pb);
            trk::Params p = make_params(x);
            const int lane = (int)(batch_no++ % (uint32_t)lanes);
            const cudaStream_t ls = lane ? x->lane_stream[lane - 1] : strm;
            const cudaStream_t lsh = lane ? x->lane_shadow_stream[lane - 1] : s_sh;
            if (lane) p.wave = x->lane_wave[lane - 1];
            if (guided && lanes > 1) {
                // several batches fill the training pool at once: each tags its entries
                if (++x->guide_tag == 0) ++x->guide_tag;
                p.guide.tag = x->guide_tag;
                if (lane) p.guide.vrec = x->lane_vrec[lane - 1];
            }
            auto tl = [&](int kind, auto&& launch) { timed_on(kind, ls, launch); };
            p.batch.win_x0 = x0; p.batch.win_y0 = y0; p.batch.win_w = win_w;
            p.batch.pix_begin = (uint32_t)pb; p.batch.npix = npix;
            p.batch.s0 = s0 + sb; p.batch.ns = ns; p.batch.ninc = ninc;
            p.batch.n_slots = npix * per_pix;
            TR_CUDA(cudaMemsetAsync(p.wave.counters, 0, trk::kCounters * sizeof(uint32_t), ls));
            tl(0, [&] { return trk::launch_raygen(p, ls); });
            if (bidir) {
                // the light subpaths, on the light wave, from the light points raygen drew.
                // They share nothing with the eye walks until the connections (own rays,
                // queues, counters and vertex store), so they run on a third stream beside
                // them; the connection passes wait for both.
                if (!x->light_stream) TR_CUDA(cudaStreamCreateWithFlags(&x->light_stream, cudaStreamNonBlocking));
                const cudaStream_t slt = x->light_stream;
                TR_CUDA(order(ls, slt));
                trk::Params pl = p;
                pl.wave = x->lwave;
                pl.wave.target = x->wave.target;
                pl.wave.stats = x->wave.stats;
                pl.wave.capacity = x->wave.capacity;
                TR_CUDA(cudaMemsetAsync(pl.wave.counters, 0, trk::kCounters * sizeof(uint32_t), slt));
                timed_on(0, slt, [&] { return trk::launch_light_raygen(pl, slt); });
                for (uint32_t d = 0; d < x->bd.nvert; ++d) {
                    timed_on(1, slt, [&] { return trk::launch_extend(pl, (int)d, x->trace_grid, slt); });
                    timed_on(2, slt, [&] { return trk::launch_light_shade(pl, (int)d, slt); });
                }
                launches += 1 + 2ull * x->bd.nvert;
                ext_l += x->bd.nvert;
            }
            for (uint32_t d = 0; d < x->integ.max_bounces; ++d) {
                tl(1, [&] { return trk::launch_extend(p, (int)d, x->trace_grid, ls); });
                if (d > 0) TR_CUDA(order(lsh, ls));
                if (guided && d < x->guide_depth) {
                    tl(2, [&] { return trk::launch_shade(p, (int)d, ls); });
                    tl(5, [&] { return trk::launch_guide(p, (int)d, x->pool_state, ls); });
                    launches += 1;
                } else if (guided) {
                    // deeper vertices sample their BSDF in the shading kernel (unguided)
                    trk::Params pu = p;
                    pu.guide.vrec = nullptr;
                    tl(2, [&] { return trk::launch_shade(pu, (int)d, ls); });
                } else {
                    tl(2, [&] { return trk::launch_shade(p, (int)d, ls); });
                }
                TR_CUDA(order(ls, lsh));
                timed_on(3, lsh, [&] { return trk::launch_shadow(p, (int)d, x->trace_grid, lsh); });
            }
            if (x->integ.max_bounces) TR_CUDA(order(lsh, ls));
            if (guided && x->guide_pool) {
                TR_CUDA(trk::launch_train_gather(p, x->pool_state, ls));
                launches += 2;
            }
            if (bidir) TR_CUDA(order(x->light_stream, ls));
            if (bidir && x->bd.nvert) {
                // eye-light vertex connections, one eye depth at a time: rays with their samples
                // into the connection queue, traced by k_shadow (records on blocked pairs),
                // then compacted after the next-event records
                const size_t R = (size_t)x->integ.max_bounces + x->bd.ncand;
                TR_CUDA(cudaMemsetAsync(x->bd.valid, 0, R * x->wave.capacity, ls));
                trk::Params pc = p;
                pc.wave.sh_o = x->bd.co_o;
                pc.wave.sh_d = x->bd.co_d;
                pc.wave.sh_L = x->bd.co_L;
                for (uint32_t ie = 0; ie < x->bd.nvert; ++ie) {
                    tl(3, [&] { return trk::launch_connect_gen(p, (int)ie, ls); });
                    const int dq = (int)(x->integ.max_bounces + ie);
                    tl(3, [&] { return trk::launch_shadow(pc, dq, x->trace_grid, ls); });
                }
                tl(3, [&] { return trk::launch_connect_compact(p, ls); });
                launches += 1 + 2ull * x->bd.nvert;
                sh_l += x->bd.nvert;
            }
            if (rgbe && sb + ns >= ns_total) {
                // final pixels: the splat blocks encode their images as they finish them
                trk::Params ps = p;
                ps.film.rgbe_streak = x->d_rgbe;
                ps.film.rgbe_steady = x->d_rgbe + (size_t)x->film.width * x->film.height * T;
                ps.film.rgbe_fresh = (film_was_clean && ns_chunk >= ns_total) ? 1u : 0u;
                tl(4, [&] { return trk::launch_splat(ps, ls); });
            } else {
                tl(4, [&] { return trk::launch_splat(p, ls); });
            }
            for (uint32_t b = 0; b < x->film.bounce_films; ++b)
                tl(4, [&] { return trk::launch_splat(p, ls, (int)b); });
            if (x->film.bounce_films) {
                tl(4, [&] { return trk::launch_bounce_weights(p, ls); });
                launches += 1ull + x->film.bounce_films;
            }
            launches += 2 + 3ull * x->integ.max_bounces;
            ext_l += x->integ.max_bounces;
            sh_l += x->integ.max_bounces;
            if (sink && sb + ns >= ns_total) {
                // window = whole frame: the batch's pixels are contiguous film rows
                const size_t p0 = pb, np = npix;
                const size_t npix_all = (size_t)x->film.width * x->film.height;
                uchar4* rst = rgbe ? x->d_rgbe + p0 * T : nullptr;
                uchar4* rsd = rgbe ? x->d_rgbe + npix_all * T + p0 : nullptr;
                cudaEvent_t done = ev_get();
                TR_CUDA(cudaEventRecord(done, ls));
                TR_CUDA(cudaStreamWaitEvent(x->copy_stream, done, 0));
                const size_t es = f32 ? sizeof(float) : sizeof(double);
                const size_t n_st = np * T * 3u, n_sd = np * 3u;
                if (rgbe) {
                    if (sink->streak)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->streak) + p0 * T * 4u, rst, np * T * 4u,
                                                cudaMemcpyDeviceToHost, x->copy_stream));
                    if (sink->steady)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->steady) + p0 * 4u, rsd, np * 4u,
                                                cudaMemcpyDeviceToHost, x->copy_stream));
                } else if (f32) {
                    float* st = x->d_stage;
                    float* sd = st + n_st;
                    float* wt = sd + n_sd;
                    TR_CUDA(trk::launch_to_f32(x->d_streak + p0 * T * 3u, st, n_st, x->copy_stream));
                    TR_CUDA(trk::launch_to_f32(x->d_steady + p0 * 3u, sd, n_sd, x->copy_stream));
                    TR_CUDA(trk::launch_to_f32(x->d_weight + p0, wt, np, x->copy_stream));
                    launches += 3;
                    if (sink->streak)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->streak) + p0 * T * 3u * es, st, n_st * es,
                                                cudaMemcpyDeviceToHost, x->copy_stream));
                    if (sink->steady)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->steady) + p0 * 3u * es, sd, n_sd * es,
                                                cudaMemcpyDeviceToHost, x->copy_stream));
                    if (sink->weight)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->weight) + p0 * es, wt, np * es,
                                                cudaMemcpyDeviceToHost, x->copy_stream));
                } else {
                    if (sink->streak)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->streak) + p0 * T * 3u * es,
                                                x->d_streak + p0 * T * 3u, n_st * es, cudaMemcpyDeviceToHost,
                                                x->copy_stream));
                    if (sink->steady)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->steady) + p0 * 3u * es, x->d_steady + p0 * 3u,
                                                n_sd * es, cudaMemcpyDeviceToHost, x->copy_stream));
                    if (sink->weight)
                        TR_CUDA(cudaMemcpyAsync(static_cast<char*>(sink->weight) + p0 * es, x->d_weight + p0,
                                                np * es, cudaMemcpyDeviceToHost, x->copy_stream));
                }
            }
        }
    }
    for (int k = 0; k + 1 < lanes; ++k) TR_CUDA(order(x->lane_stream[k], strm));
    if (sink) TR_CUDA(cudaStreamSynchronize(x->copy_stream));
    TR_CUDA(cudaEventRecord(x->ev1, strm));
    TR_CUDA(cudaEventSynchronize(x->ev1));
    float ms = 0.f;
    TR_CUDA(cudaEventElapsedTime(&ms, x->ev0, x->ev1));
    if (x->profiling == 1) {
        TR_CUDA(prof_readout(x));
        prof_publish(x);
    }
    x->stats.kernel_launches = launches;
    x->stats.extend_launches = ext_l;
    x->stats.shadow_launches = sh_l;
    unsigned long long st[8];
    TR_CUDA(cudaMemcpy(st, x->wave.stats, sizeof(st), cudaMemcpyDeviceToHost));
    x->stats.closest_rays = st[0];
    x->stats.shadow_rays = st[1];
    x->stats.splats = st[2];
    x->stats.paths += total_slots;
    x->stats.camera_samples += win_pix * ns_total;
    x->stats.render_ms = ms;
    if (guided) return guide_end_render(x, strm);
    return TR_OK;
}

}  // namespace

namespace {
void noalloc_prepare(int device);
}  // namespace

extern "C" {

int tr_abi_version(void) { return TR_ABI_VERSION; }

const char* tr_status_string(tr_status s) {
    switch (s) {
        case TR_OK: return "ok";
        case TR_ERR_INVALID_ARGUMENT: return "invalid argument";
        case TR_ERR_CUDA: return "CUDA error";
        case TR_ERR_OUT_OF_MEMORY: return "out of device memory";
        case TR_ERR_NOT_SUPPORTED: return "not supported";
        case TR_ERR_TIMEOUT: return "device wait timed out";
        case TR_ERR_NO_DEVICE: return "no usable CUDA device";
        case TR_ERR_IO: return "I/O error";
    }
    return "unknown status";
}

const char* tr_last_error(void) { return g_last_error.c_str(); }

tr_status tr_create(const tr_scene* s, const tr_camera* c, const tr_film* f, const tr_integrator* it,
                    int device, tr_ctx** out) {
    if (!out) return fail(TR_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    tr_status v = validate(s, c, f, it);
    if (v != TR_OK) return v;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(TR_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(TR_ERR_NO_DEVICE, "device index out of range");
    // one attribute query (cudaGetDeviceProperties reads every property and costs milliseconds)
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) {
        cudaDeviceProp prop{};
        cudaGetDeviceProperties(&prop, device);
        return fail(TR_ERR_NO_DEVICE, std::string("this build targets sm_100a; device is ") + prop.name);
    }
    tr_ctx* x = new (std::nothrow) tr_ctx();
    if (!x) return fail(TR_ERR_OUT_OF_MEMORY, "host allocation failed");
    try {
        x->device = device;
        TR_CUDA(cudaSetDevice(device));
        TR_CUDA(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
        TR_CUDA(cudaEventCreate(&x->ev0));
        TR_CUDA(cudaEventCreate(&x->ev1));
        x->cam = *c; x->film = *f; x->integ = *it;
        x->nt = s->num_triangles;

        // film: [H][W][T][3] + steady + weights, double precision, zeroed.  Allocated first, so
        // the largest block is taken from the memory pool before any scratch (a film freed by an
        // earlier context is reused whole instead of mapped again)
        const size_t nstreak = (size_t)f->width * f->height * f->time_bins * 3u;
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        free_b += tri::pool_idle_bytes(device);      // kept by the pool for reuse
        const size_t nb = f->bounce_films;
        if ((1 + nb) * nstreak * sizeof(double) + ((size_t)2 << 30) > free_b) {
            x->release();
            delete x;
            return fail(TR_ERR_OUT_OF_MEMORY, "streak film of " + std::to_string(nstreak * 8 >> 20) +
                                                  " MiB does not fit in free device memory");
        }
        x->d_streak = x->alloc<double>(nstreak);
        x->d_steady = x->alloc<double>((size_t)f->width * f->height * 3u);
        x->d_weight = x->alloc<double>((size_t)f->width * f->height);
        TR_CUDA(cudaMemsetAsync(x->d_streak, 0, nstreak * sizeof(double), x->stream));
        TR_CUDA(cudaMemsetAsync(x->d_steady, 0, (size_t)f->width * f->height * 3u * sizeof(double), x->stream));
        TR_CUDA(cudaMemsetAsync(x->d_weight, 0, (size_t)f->width * f->height * sizeof(double), x->stream));
        if (nb) {
            const size_t npix = (size_t)f->width * f->height;
            x->d_bstreak = x->alloc<double>(nb * nstreak);
            x->d_bsteady = x->alloc<double>(nb * npix * 3u);
            x->d_bweight = x->alloc<double>(nb * npix);
            TR_CUDA(cudaMemsetAsync(x->d_bstreak, 0, nb * nstreak * sizeof(double), x->stream));
            TR_CUDA(cudaMemsetAsync(x->d_bsteady, 0, nb * npix * 3u * sizeof(double), x->stream));
            TR_CUDA(cudaMemsetAsync(x->d_bweight, 0, nb * npix * sizeof(double), x->stream));
        }
        {
            const size_t npix = (size_t)f->width * f->height;
            if (f->components & TR_COMP_DEPTH) x->d_cdepth = x->alloc<double>(npix);
            if (f->components & TR_COMP_POSITIONS) x->d_cpos = x->alloc<double>(npix * 3u);
            if (f->components & TR_COMP_NORMALS) x->d_cnorm = x->alloc<double>(npix * 3u);
            if (x->d_cdepth) TR_CUDA(cudaMemsetAsync(x->d_cdepth, 0, npix * sizeof(double), x->stream));
            if (x->d_cpos) TR_CUDA(cudaMemsetAsync(x->d_cpos, 0, npix * 3u * sizeof(double), x->stream));
            if (x->d_cnorm) TR_CUDA(cudaMemsetAsync(x->d_cnorm, 0, npix * 3u * sizeof(double), x->stream));
        }
        // the context's ray and splat counters (every render entry point adds to them) and,
        // for tr_render_region_noalloc, the scratch array's device address: both at set-up, so
        // that entry point allocates nothing and loads no module when it is called
        x->wave.stats = x->alloc<unsigned long long>(8);
        TR_CUDA(cudaMemsetAsync(x->wave.stats, 0, 8 * sizeof(unsigned long long), x->stream));
        noalloc_prepare(device);

        // the scene's own arrays go to the device first (the BVH is built there from them)
        const size_t ntri = s->num_triangles;
        float* d_v = x->alloc<float>(3 * (size_t)s->num_vertices);
        uint32_t* d_t = x->alloc<uint32_t>(3 * ntri);
        uint32_t* d_m = x->alloc<uint32_t>(ntri);
        uint32_t* d_o = x->alloc<uint32_t>(ntri);
        TR_CUDA(cudaMemcpyAsync(d_v, s->vertices, sizeof(float) * 3 * (size_t)s->num_vertices,
                                cudaMemcpyHostToDevice, x->stream));
        TR_CUDA(cudaMemcpyAsync(d_t, s->triangles, sizeof(uint32_t) * 3 * ntri, cudaMemcpyHostToDevice, x->stream));
        TR_CUDA(cudaMemcpyAsync(d_m, s->triangle_material, sizeof(uint32_t) * ntri, cudaMemcpyHostToDevice, x->stream));

        // BVH (replaces World::freeze -> rtcCommit): built on the device from the uploaded arrays,
        // nodes and leaf order left there; the host builder takes one-leaf scenes and names the
        // offending index or vertex of invalid input
        trh::DeviceBvh dbv;
        float4* dnodes = nullptr;
        const bool on_device = trh::build_bvh_device(
            d_v, s->num_vertices, d_t, s->num_triangles, 4, x->stream,
            [&](size_t n) { dnodes = x->alloc<float4>(n * 8); return reinterpret_cast<trh::GpuNode*>(dnodes); },
            d_o, dbv);
        trh::BvhBuildResult bvh;
        if (!on_device) {
            std::string msg;
            if (!trh::build_bvh(s->vertices, s->num_vertices, s->triangles, s->num_triangles, 4, bvh, &msg,
                                /*write_tris*/ false)) {
                cudaStreamSynchronize(x->stream);
                x->release();
                delete x;
                return fail(TR_ERR_INVALID_ARGUMENT, msg);
            }
            dbv.nodes = (uint32_t)bvh.nodes.size();
            dbv.depth = bvh.depth;
            dbv.stack = bvh.stack;
            dbv.build_ms = bvh.build_ms;
            dnodes = x->alloc<float4>(bvh.nodes.size() * 8);
            upload(dnodes, bvh.nodes.data(), bvh.nodes.size() * sizeof(trh::GpuNode), x->stream);
            TR_CUDA(cudaMemcpyAsync(d_o, bvh.order.data(), sizeof(uint32_t) * ntri, cudaMemcpyHostToDevice, x->stream));
        }
        if (dbv.stack > (uint32_t)trk::kStack) {
            cudaStreamSynchronize(x->stream);
            x->release();
            delete x;
            return fail(TR_ERR_NOT_SUPPORTED, "BVH deeper than the traversal stack");
        }
        if (reinterpret_cast<uintptr_t>(dnodes) & 31u) {
            // the traversal fetches a node's bounds with 256-bit loads (32-byte aligned)
            cudaStreamSynchronize(x->stream);
            x->release();
            delete x;
            return fail(TR_ERR_CUDA, "BVH node buffer not 32-byte aligned");
        }
        x->bvh_nodes = dbv.nodes;
        x->bvh_depth = dbv.stack - 1;               // sizes the shared-memory traversal stack
        x->bvh_levels = dbv.depth;
        x->bvh_ms = dbv.build_ms;
        x->d_nodes = dnodes;
        // the leaf-ordered triangle records and the per-triangle normals, built on the device
        // (World.h:449 normals, the same IEEE operations as a host evaluation)
        x->d_tris = x->alloc<float4>(ntri * 3);
        x->d_tri_ng = x->alloc<float4>(ntri);
        TR_CUDA(trk::launch_build_tris(d_v, d_t, d_m, d_o, (uint32_t)ntri, x->d_tris, x->d_tri_ng, x->stream));
        TR_CUDA(cudaStreamSynchronize(x->stream));      // bvh.order is released on return

        std::vector<float4> mats(s->num_materials), mats2(s->num_materials);
        for (uint32_t i = 0; i < s->num_materials; ++i) {
            const tr_material& m = s->materials[i];
            float kf;
            std::memcpy(&kf, &m.kind, 4);
            mats[i] = make_float4(m.kd[0], m.kd[1], m.kd[2], kf);
            mats2[i] = make_float4(m.alpha, 0.f, 0.f, 0.f);
        }
        x->d_mats = x->alloc<float4>(mats.size());
        upload(x->d_mats, mats.data(), mats.size() * sizeof(float4), x->stream);
        x->d_mats2 = x->alloc<float4>(mats2.size());
        upload(x->d_mats2, mats2.data(), mats2.size() * sizeof(float4), x->stream);

        std::vector<float4> lights(5 * (size_t)s->num_lights);
        for (uint32_t i = 0; i < s->num_lights; ++i) {
            const tr_light& L = s->lights[i];
            float kf;
            std::memcpy(&kf, &L.kind, 4);
            lights[5 * i + 0] = make_float4(L.position[0], L.position[1], L.position[2], kf);
            lights[5 * i + 1] = make_float4(L.intensity[0], L.intensity[1], L.intensity[2], L.area);
            lights[5 * i + 2] = make_float4(L.left[0], L.left[1], L.left[2], 0.f);
            lights[5 * i + 3] = make_float4(L.up[0], L.up[1], L.up[2], 0.f);
            lights[5 * i + 4] = make_float4(L.normal[0], L.normal[1], L.normal[2], 0.f);
        }
        x->d_lights = x->alloc<float4>(lights.size());
        upload(x->d_lights, lights.data(), lights.size() * sizeof(float4), x->stream);

        trk::SceneDev& sc = x->scene;
        sc.nodes = x->d_nodes; sc.tris = x->d_tris; sc.tri_ng = x->d_tri_ng;
        sc.mats = x->d_mats; sc.mats2 = x->d_mats2; sc.lights = x->d_lights;
        sc.num_lights = s->num_lights;
        sc.bvh_depth = x->bvh_depth;
        {
            float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
            for (uint32_t i = 0; i < s->num_vertices; ++i)
                for (int k = 0; k < 3; ++k) {
                    lo[k] = std::min(lo[k], s->vertices[3 * (size_t)i + k]);
                    hi[k] = std::max(hi[k], s->vertices[3 * (size_t)i + k]);
                }
            for (int k = 0; k < 3; ++k) {
                sc.bmin[k] = lo[k];
                sc.binv[k] = hi[k] > lo[k] ? 1.0f / (hi[k] - lo[k]) : 1.0f;
            }
        }
        sc.medium = s->medium.enabled ? 1u : 0u;
        if (sc.medium) {
            trd::f3 st = trd::mk(s->medium.sigma_a[0] + s->medium.sigma_s[0], s->medium.sigma_a[1] + s->medium.sigma_s[1],
                                 s->medium.sigma_a[2] + s->medium.sigma_s[2]);
            for (int k = 0; k < 3; ++k) { sc.sig_s[k] = s->medium.sigma_s[k]; sc.sig_t[k] = trd::comp(st, k); }
            sc.lambda = trd::avg3(st);
            // time sampling: free flights at the rate m_avg_nb_vertices_path (4) per film
            // duration (BidirectionalPathTracing.h:189-206, :240-307)
            if (it->flags & TR_FLAG_TIME_SAMPLING) sc.lambda = 4.0f / ((float)f->time_bins * f->exposure);
            sc.g = s->medium.g;
        }

        x->trace_grid = trk::trace_grid_size(device, x->bvh_depth);
        x->d_cursor = x->alloc<uint32_t>(1);
        TR_CUDA(cudaStreamSynchronize(x->stream));

        x->stats.bvh_build_ms = x->bvh_ms;
        x->stats.bvh_nodes = x->bvh_nodes;
        x->stats.bvh_depth = x->bvh_levels;
    } catch (const CudaError& e) {
        x->release();
        delete x;
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        x->release();
        delete x;
        return fail(TR_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    *out = x;
    return TR_OK;
}

tr_status tr_render_region(tr_ctx* x, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                           uint64_t sample_begin, uint32_t sample_count) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        return render_region(x, x0, y0, x1, y1, sample_begin, sample_count);
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
}

tr_status tr_release_cached_memory(int device) {
    try {
        int n = 0;
        TR_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) return fail(TR_ERR_INVALID_ARGUMENT, "no such device");
        TR_CUDA(cudaSetDevice(device));
        TR_CUDA(cudaDeviceSynchronize());
        TR_CUDA(cudaMemPoolTrimTo(tri::device_pool(device), 0));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status tr_render(tr_ctx* x, uint64_t sample_begin, uint32_t sample_count) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    return tr_render_region(x, 0, 0, x->film.width, x->film.height, sample_begin, sample_count);
}

static tr_status copy_film(tr_ctx* x, double* streak, double* steady, double* weight, cudaMemcpyKind kind);

tr_status tr_render_film(tr_ctx* x, uint64_t sample_begin, uint32_t sample_count, int type, void* streak,
                         void* steady, void* weight) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if (type != TR_FILM_F64 && type != TR_FILM_F32 && type != TR_FILM_RGBE)
        return fail(TR_ERR_INVALID_ARGUMENT, "unknown film type");
    if (type == TR_FILM_RGBE && weight) return fail(TR_ERR_INVALID_ARGUMENT, "RGBE delivery has no weight array");
    if (sample_count == 0) {
        // nothing to render: deliver the current sums
        if (type == TR_FILM_F64) return copy_film(x, (double*)streak, (double*)steady, (double*)weight, cudaMemcpyDeviceToHost);
        return fail(TR_ERR_INVALID_ARGUMENT, "sample_count must be >= 1 for FP32 and RGBE delivery");
    }
    try {
        TR_CUDA(cudaSetDevice(x->device));
        FilmSink sink{type, streak, steady, weight};
        return render_region(x, 0, 0, x->film.width, x->film.height, sample_begin, sample_count, &sink);
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
}

tr_status tr_clear_film(tr_ctx* x) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        x->film_clean = true;
        const size_t npix = (size_t)x->film.width * x->film.height;
        TR_CUDA(cudaMemsetAsync(x->d_streak, 0, npix * x->film.time_bins * 3u * sizeof(double), x->s()));
        TR_CUDA(cudaMemsetAsync(x->d_steady, 0, npix * 3u * sizeof(double), x->s()));
        TR_CUDA(cudaMemsetAsync(x->d_weight, 0, npix * sizeof(double), x->s()));
        if (const size_t nb = x->film.bounce_films) {
            TR_CUDA(cudaMemsetAsync(x->d_bstreak, 0, nb * npix * x->film.time_bins * 3u * sizeof(double), x->s()));
            TR_CUDA(cudaMemsetAsync(x->d_bsteady, 0, nb * npix * 3u * sizeof(double), x->s()));
            TR_CUDA(cudaMemsetAsync(x->d_bweight, 0, nb * npix * sizeof(double), x->s()));
        }
        if (x->d_cdepth) TR_CUDA(cudaMemsetAsync(x->d_cdepth, 0, npix * sizeof(double), x->s()));
        if (x->d_cpos) TR_CUDA(cudaMemsetAsync(x->d_cpos, 0, npix * 3u * sizeof(double), x->s()));
        if (x->d_cnorm) TR_CUDA(cudaMemsetAsync(x->d_cnorm, 0, npix * 3u * sizeof(double), x->s()));
        TR_CUDA(cudaStreamSynchronize(x->s()));
        x->stats.camera_samples = 0;
        x->stats.paths = 0;
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

static tr_status copy_film(tr_ctx* x, double* streak, double* steady, double* weight, cudaMemcpyKind kind) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        // on the context's stream (after its renders), and complete before returning: a
        // device-to-device cudaMemcpy would return early and could race with a later
        // tr_clear_film on the context's stream
        cudaStream_t s = x->s();
        const size_t npix = (size_t)x->film.width * x->film.height;
        if (streak) TR_CUDA(cudaMemcpyAsync(streak, x->d_streak, npix * x->film.time_bins * 3u * sizeof(double), kind, s));
        if (steady) TR_CUDA(cudaMemcpyAsync(steady, x->d_steady, npix * 3u * sizeof(double), kind, s));
        if (weight) TR_CUDA(cudaMemcpyAsync(weight, x->d_weight, npix * sizeof(double), kind, s));
        TR_CUDA(cudaStreamSynchronize(s));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status tr_get_film(tr_ctx* x, double* streak, double* steady, double* weight) {
    return copy_film(x, streak, steady, weight, cudaMemcpyDeviceToHost);
}

tr_status tr_get_film_device(tr_ctx* x, double* streak, double* steady, double* weight) {
    return copy_film(x, streak, steady, weight, cudaMemcpyDeviceToDevice);
}

tr_status tr_get_film_components(tr_ctx* x, double* depth, double* positions, double* normals) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if ((depth && !x->d_cdepth) || (positions && !x->d_cpos) || (normals && !x->d_cnorm))
        return fail(TR_ERR_INVALID_ARGUMENT, "the film does not have that component");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        cudaStream_t s = x->s();
        const size_t npix = (size_t)x->film.width * x->film.height;
        if (depth) TR_CUDA(cudaMemcpyAsync(depth, x->d_cdepth, npix * sizeof(double), cudaMemcpyDefault, s));
        if (positions) TR_CUDA(cudaMemcpyAsync(positions, x->d_cpos, npix * 3u * sizeof(double), cudaMemcpyDefault, s));
        if (normals) TR_CUDA(cudaMemcpyAsync(normals, x->d_cnorm, npix * 3u * sizeof(double), cudaMemcpyDefault, s));
        TR_CUDA(cudaStreamSynchronize(s));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status tr_get_film_bounce(tr_ctx* x, uint32_t b, double* streak, double* steady, double* weight) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if (b >= x->film.bounce_films) return fail(TR_ERR_INVALID_ARGUMENT, "bounce film index out of range");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        cudaStream_t s = x->s();
        const size_t npix = (size_t)x->film.width * x->film.height;
        const size_t ns = npix * x->film.time_bins * 3u;
        if (streak) TR_CUDA(cudaMemcpyAsync(streak, x->d_bstreak + b * ns, ns * sizeof(double), cudaMemcpyDefault, s));
        if (steady) TR_CUDA(cudaMemcpyAsync(steady, x->d_bsteady + b * npix * 3u, npix * 3u * sizeof(double), cudaMemcpyDefault, s));
        if (weight) TR_CUDA(cudaMemcpyAsync(weight, x->d_bweight + b * npix, npix * sizeof(double), cudaMemcpyDefault, s));
        TR_CUDA(cudaStreamSynchronize(s));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status tr_write_film(tr_ctx* x, const char* name) {
    if (!x || !name) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    const size_t npix = (size_t)x->film.width * x->film.height;
    const uint32_t nb = x->film.bounce_films;
    std::vector<double> streak, steady(npix * 3), weight(npix);
    try {
        streak.resize(npix * x->film.time_bins * 3u);
    } catch (const std::bad_alloc&) {
        return fail(TR_ERR_OUT_OF_MEMORY, "host film buffer");
    }
    std::string err;
    // with bounce films: the base steady image (Film::write) and the per-bounce streak images
    // named as MultibounceStreakFilm::set_name does (MultibounceStreakCameraFilm.h:130-141)
    tr_status st = tr_get_film(x, nb ? nullptr : streak.data(), steady.data(), weight.data());
    if (st != TR_OK) return st;
    if (!trio::write_streak_film(name, x->film.width, x->film.height, x->film.time_bins, nb ? nullptr : streak.data(),
                                 steady.data(), weight.data(), &err))
        return fail(TR_ERR_IO, err);
    // film components, averaged by the film weight (Film::average_and_write, Film.h:357-471)
    if (x->film.components) {
        std::vector<double> cd(npix), cp(npix * 3), cn(npix * 3);
        st = tr_get_film_components(x, x->d_cdepth ? cd.data() : nullptr, x->d_cpos ? cp.data() : nullptr,
                                    x->d_cnorm ? cn.data() : nullptr);
        if (st != TR_OK) return st;
        const std::string base(name);
        if (x->d_cdepth && !trio::write_component(base + "_depth.hdr", x->film.width, x->film.height, 1, cd.data(),
                                                  weight.data(), &err))
            return fail(TR_ERR_IO, err);
        if (x->d_cpos && !trio::write_component(base + "_positions.raw", x->film.width, x->film.height, 3, cp.data(),
                                                weight.data(), &err))
            return fail(TR_ERR_IO, err);
        if (x->d_cnorm && !trio::write_component(base + "_normals.raw", x->film.width, x->film.height, 3, cn.data(),
                                                 weight.data(), &err))
            return fail(TR_ERR_IO, err);
    }
    for (uint32_t b = 0; b < nb; ++b) {
        st = tr_get_film_bounce(x, b, streak.data(), nullptr, weight.data());
        if (st != TR_OK) return st;
        char bname[4096];
        std::snprintf(bname, sizeof(bname), "%s_b%02u", name, b + 1);
        if (!trio::write_streak_film(bname, x->film.width, x->film.height, x->film.time_bins, streak.data(), nullptr,
                                     weight.data(), &err))
            return fail(TR_ERR_IO, err);
    }
    return TR_OK;
}

tr_status tr_trace_rays_device(tr_ctx* x, const float* d_rays, uint32_t n, int any_hit, tr_hit* d_out, void* stream) {
    if (!x || (!d_rays && n) || (!d_out && n)) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return TR_OK;
    if ((reinterpret_cast<uintptr_t>(d_rays) & 15u) != 0) return fail(TR_ERR_INVALID_ARGUMENT, "rays must be 16-byte aligned");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : x->s();
        TR_CUDA(cudaMemsetAsync(x->d_cursor, 0, sizeof(uint32_t), s));
        TR_CUDA(trk::launch_trace_user(x->scene, d_rays, n, any_hit, d_out, x->d_cursor, x->trace_grid, s));
        x->stats.closest_rays += any_hit ? 0 : n;
        x->stats.shadow_rays += any_hit ? n : 0;
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status tr_trace_rays(tr_ctx* x, const float* rays, uint32_t n, int any_hit, tr_hit* out) {
    if (!x || (!rays && n) || (!out && n)) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return TR_OK;
    try {
        TR_CUDA(cudaSetDevice(x->device));
        if (x->ray_cap < n) {
            auto drop = [&](void* p) {
                if (!p) return;
                cudaFree(p);
                x->allocs.erase(std::remove(x->allocs.begin(), x->allocs.end(), p), x->allocs.end());
            };
            drop(x->d_rays); drop(x->d_hits);
            x->d_rays = x->alloc<float>((size_t)n * 8);
            x->d_hits = x->alloc<tr_hit>(n);
            x->ray_cap = n;
        }
        cudaStream_t strm = x->s();
        TR_CUDA(cudaMemcpyAsync(x->d_rays, rays, (size_t)n * 8 * sizeof(float), cudaMemcpyHostToDevice, strm));
        tr_status st = tr_trace_rays_device(x, x->d_rays, n, any_hit, static_cast<tr_hit*>(x->d_hits), strm);
        if (st != TR_OK) return st;
        TR_CUDA(cudaMemcpyAsync(out, x->d_hits, (size_t)n * sizeof(tr_hit), cudaMemcpyDeviceToHost, strm));
        TR_CUDA(cudaStreamSynchronize(strm));
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status tr_stats_get(tr_ctx* x, tr_stats* out) {
    if (!x || !out) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    if (x->profiling == 2 && (x->prof_dirty || !x->prof_marks.empty())) {
        // the sums over every render since the previous read (unchanged if none ran since)
        cudaSetDevice(x->device);
        const cudaError_t e = prof_readout(x);
        if (e != cudaSuccess) return fail(TR_ERR_CUDA, cudaGetErrorString(e));
        prof_publish(x);
    }
    if (x->wave.stats) {                // counters of every render, tr_render_region_noalloc's included
        cudaSetDevice(x->device);
        unsigned long long st[8];
        cudaError_t e = cudaStreamSynchronize(x->s());
        if (e == cudaSuccess) e = cudaMemcpy(st, x->wave.stats, sizeof(st), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return fail(TR_ERR_CUDA, cudaGetErrorString(e));
        x->stats.closest_rays = st[0];
        x->stats.shadow_rays = st[1];
        x->stats.splats = st[2];
    }
    *out = x->stats;
    out->device_bytes = x->bytes;
    return TR_OK;
}

}  // extern "C"

// -----------------------------------------------------------------------------------------
// tr_render_region_noalloc: the same wavefront kernels, with every per-path buffer carved out
// of one file-scope device array instead of cudaMalloc'd memory.
// -----------------------------------------------------------------------------------------
namespace {

constexpr size_t na_align(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kNaSlots = TR_NOALLOC_MAX_PATHS;
constexpr size_t kNaF4 = na_align(sizeof(float4) * kNaSlots);
constexpr size_t kNaBytes = 7 * kNaF4                                            // ray_o ray_d thr hit sh_o sh_d sh_L
                          + na_align(sizeof(unsigned long long) * kNaSlots)       // rng
                          + 2 * na_align(sizeof(uint32_t) * kNaSlots)             // extend queues
                          + na_align(sizeof(float4) * kNaSlots * TR_NOALLOC_MAX_BOUNCES)  // records
                          + na_align(kNaSlots)                                    // records per slot
                          + na_align(sizeof(uint32_t) * trk::kCounters)           // queue counters
                          + na_align(sizeof(float) * kNaSlots)                    // camera distances
                          + kNaF4;                                                // light points (time sampling)

// The scratch itself.  Its name is only a host-side handle: host code must use the device
// address from cudaGetSymbolAddress, never &g_noalloc_scratch.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};     // device address of the array, per device ordinal

// Looks the array up once per device, with that device current.
tr_status noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= 64) return fail(TR_ERR_NO_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(TR_ERR_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
    return TR_OK;
}

// Set-up half of the look-up, run by tr_create with `device` current: loads the array on this
// device once, so that tr_render_region_noalloc's calls only read the cached address.  A
// failure here is not fatal to the context; the entry point then retries and reports it.
void noalloc_prepare(int device) {
    unsigned char* p = nullptr;
    if (noalloc_scratch(device, &p) != TR_OK) cudaGetLastError();
}

}  // namespace

extern "C" {

extern "C" tr_status tr_render_region_noalloc(tr_ctx* x, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                                              uint64_t s0, uint32_t ns, void* stream) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if (x1 > x->film.width || y1 > x->film.height || x0 >= x1 || y0 >= y1)
        return fail(TR_ERR_INVALID_ARGUMENT, "pixel window out of range or empty");
    if (ns == 0) return TR_OK;
    if (s0 + ns > (1ull << 32)) return fail(TR_ERR_INVALID_ARGUMENT, "camera sample index must stay below 2^32");
    if (x->integ.flags & TR_FLAG_BIDIRECTIONAL)
        return fail(TR_ERR_NOT_SUPPORTED, "light subpaths need their vertex arrays: render with tr_render");
    x->film_clean = false;
    if (x->integ.max_bounces > TR_NOALLOC_MAX_BOUNCES)
        return fail(TR_ERR_INVALID_ARGUMENT, "tr_render_region_noalloc supports max_bounces <= " +
                                                 std::to_string(TR_NOALLOC_MAX_BOUNCES) + " (scene has " +
                                                 std::to_string(x->integ.max_bounces) + ")");
    const uint64_t npix = (uint64_t)(x1 - x0) * (y1 - y0);
    const uint64_t paths = npix * ns * x->integ.incoming_samples;
    if (paths > TR_NOALLOC_MAX_PATHS)
        return fail(TR_ERR_INVALID_ARGUMENT, "tr_render_region_noalloc renders at most " +
                                                 std::to_string(TR_NOALLOC_MAX_PATHS) + " paths per call (asked for " +
                                                 std::to_string(paths) + "); split the window or the samples");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        unsigned char* base = nullptr;
        tr_status st = noalloc_scratch(x->device, &base);
        if (st != TR_OK) return st;
        cudaStream_t strm = stream ? static_cast<cudaStream_t>(stream) : x->s();
        trk::Params p = make_params(x);
        p.guide = trk::GuideWave{};      // the fixed array holds no proposal buffers: plain sampling
        trk::Wave& w = p.wave;
        unsigned char* c = base;
        auto take = [&](size_t bytes) { unsigned char* r = c; c += na_align(bytes); return r; };
        w.ray_o = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.ray_d = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.thr = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.hit = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.sh_o = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.sh_d = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.sh_L = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.rng = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long) * kNaSlots));
        w.q[0] = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * kNaSlots));
        w.q[1] = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * kNaSlots));
        w.rec = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots * TR_NOALLOC_MAX_BOUNCES));
        w.rec_n = take(kNaSlots);
        w.counters = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * trk::kCounters));
        w.stats = x->wave.stats;         // the context's own ray / splat counters (from tr_create)
        w.cam_dist = reinterpret_cast<float*>(take(sizeof(float) * kNaSlots));
        w.target = reinterpret_cast<float4*>(take(sizeof(float4) * kNaSlots));
        w.capacity = (uint32_t)kNaSlots;
        // what the kernels expect to start at zero: queue counters / fetch cursors (records per
        // slot are reset by the ray generation kernel; the ray counters keep adding up)
        TR_CUDA(cudaMemsetAsync(w.counters, 0, sizeof(uint32_t) * trk::kCounters, strm));
        p.batch.win_x0 = x0; p.batch.win_y0 = y0; p.batch.win_w = x1 - x0;
        p.batch.pix_begin = 0; p.batch.npix = (uint32_t)npix;
        p.batch.s0 = s0; p.batch.ns = ns; p.batch.ninc = x->integ.incoming_samples;
        p.batch.n_slots = (uint32_t)paths;
        TR_CUDA(trk::launch_raygen(p, strm));
        for (uint32_t d = 0; d < x->integ.max_bounces; ++d) {
            TR_CUDA(trk::launch_extend(p, (int)d, x->trace_grid, strm));
            TR_CUDA(trk::launch_shade(p, (int)d, strm));
            TR_CUDA(trk::launch_shadow(p, (int)d, x->trace_grid, strm));
        }
        TR_CUDA(trk::launch_splat(p, strm));
        for (uint32_t b = 0; b < x->film.bounce_films; ++b) TR_CUDA(trk::launch_splat(p, strm, (int)b));
        if (x->film.bounce_films) TR_CUDA(trk::launch_bounce_weights(p, strm));
        x->stats.paths += paths;
        x->stats.camera_samples += npix * ns;
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

}  // extern "C"

// -----------------------------------------------------------------------------------------
// learned proposal network
// -----------------------------------------------------------------------------------------

namespace tri {
tr_status guide_check_err(tr_guide* g, cudaStream_t s) {
    int e = 0;
    TR_CUDA(cudaMemcpyAsync(&e, g->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaStreamSynchronize(s));
    if (e) {
        TR_CUDA(cudaMemsetAsync(g->err, 0, sizeof(int), s));
        return fail(TR_ERR_TIMEOUT, "tensor-core MMA completion wait timed out");
    }
    return TR_OK;
}
}  // namespace tri

extern "C" tr_status tr_guide_create(int device, uint64_t seed, tr_guide** out) {
    if (!out) return fail(TR_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(TR_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(TR_ERR_NO_DEVICE, "device index out of range");
    // one attribute query (cudaGetDeviceProperties reads every property and costs milliseconds)
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) {
        cudaDeviceProp prop{};
        cudaGetDeviceProperties(&prop, device);
        return fail(TR_ERR_NO_DEVICE, std::string("this build targets sm_100a; device is ") + prop.name);
    }
    tr_guide* g = new (std::nothrow) tr_guide();
    if (!g) return fail(TR_ERR_OUT_OF_MEMORY, "host allocation failed");
    try {
        g->device = device;
        TR_CUDA(cudaSetDevice(device));
        // highest priority: training steps that run beside a render get SMs as soon as the
        // render's traversal blocks retire, instead of queueing behind its later launches
        int lo = 0, hi = 0;
        TR_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        TR_CUDA(cudaStreamCreateWithPriority(&g->stream, cudaStreamNonBlocking, hi));
        g->params = g->alloc<float>(TR_GUIDE_PARAMS);
        g->grads = g->alloc<float>(TR_GUIDE_PARAMS);
        g->m1 = g->alloc<float>(TR_GUIDE_PARAMS);
        g->m2 = g->alloc<float>(TR_GUIDE_PARAMS);
        g->w_fwd = g->alloc<uint8_t>(4 * 8192);
        g->w_bwd = g->alloc<uint8_t>(4 * 8192);
        g->err = g->alloc<int>(1);
        g->scalars = g->alloc<float>(4);
        // He-uniform hidden layers; a small output layer so the first mixture is broad
        std::vector<float> p(TR_GUIDE_PARAMS, 0.0f);
        unsigned long long st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
        auto uni = [&]() {
            st = st * 6364136223846793005ULL + 1442695040888963407ULL;
            return (float)((st >> 40) & 0xFFFFFFull) / 16777216.0f * 2.0f - 1.0f;
        };
        for (int l = 0; l < 4; ++l) {
            const float a = l < 3 ? std::sqrt(6.0f / 64.0f) : 0.05f;
            for (int i = 0; i < 4096; ++i) p[(size_t)l * 4096 + i] = a * uni();
        }
        // everything ordered on the guide's stream (see upload)
        TR_CUDA(cudaMemcpyAsync(g->params, p.data(), sizeof(float) * TR_GUIDE_PARAMS, cudaMemcpyHostToDevice, g->stream));
        TR_CUDA(cudaMemsetAsync(g->m1, 0, sizeof(float) * TR_GUIDE_PARAMS, g->stream));
        TR_CUDA(cudaMemsetAsync(g->m2, 0, sizeof(float) * TR_GUIDE_PARAMS, g->stream));
        TR_CUDA(cudaMemsetAsync(g->grads, 0, sizeof(float) * TR_GUIDE_PARAMS, g->stream));
        TR_CUDA(cudaMemsetAsync(g->err, 0, sizeof(int), g->stream));
        TR_CUDA(trg::pack_weights(g->params, g->w_fwd, g->w_bwd, g->stream));
        TR_CUDA(cudaStreamSynchronize(g->stream));
    } catch (const CudaError& e) {
        for (void* q : g->allocs) cudaFree(q);
        delete g;
        return fail(TR_ERR_CUDA, e.what());
    }
    *out = g;
    return TR_OK;
}

extern "C" tr_status tr_guide_set_params(tr_guide* g, const float* params) {
    if (!g || !params) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    try {
        TR_CUDA(cudaSetDevice(g->device));
        TR_CUDA(cudaMemcpyAsync(g->params, params, sizeof(float) * TR_GUIDE_PARAMS, cudaMemcpyHostToDevice, g->stream));
        TR_CUDA(trg::pack_weights(g->params, g->w_fwd, g->w_bwd, g->stream));
        TR_CUDA(cudaStreamSynchronize(g->stream));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

extern "C" tr_status tr_guide_get_params(tr_guide* g, float* params) {
    if (!g || !params) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    try {
        TR_CUDA(cudaSetDevice(g->device));
        TR_CUDA(cudaStreamSynchronize(g->stream));
        TR_CUDA(cudaMemcpy(params, g->params, sizeof(float) * TR_GUIDE_PARAMS, cudaMemcpyDeviceToHost));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

extern "C" tr_status tr_guide_get_grads(tr_guide* g, float* grads) {
    if (!g || !grads) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    try {
        TR_CUDA(cudaSetDevice(g->device));
        TR_CUDA(cudaStreamSynchronize(g->stream));
        TR_CUDA(cudaMemcpy(grads, g->grads, sizeof(float) * TR_GUIDE_PARAMS, cudaMemcpyDeviceToHost));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

extern "C" tr_status tr_guide_forward(tr_guide* g, const uint16_t* d_features, uint32_t n, float* d_out, void* stream) {
    if (!g || (n && (!d_features || !d_out))) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    if (n == 0) return TR_OK;
    if ((reinterpret_cast<uintptr_t>(d_features) & 15u) != 0) return fail(TR_ERR_INVALID_ARGUMENT, "features must be 16-byte aligned");
    try {
        TR_CUDA(cudaSetDevice(g->device));
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
        TR_CUDA(trg::mlp_forward(g->dev(), reinterpret_cast<const uint4*>(d_features), n, d_out, nullptr, g->err, s));
        return guide_check_err(g, s);
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
}

namespace tri {
// Enqueues one training step (forward, loss gradient, backward, weight gradients, Adam, weight
// repacking) on stream s without waiting for it; the loss lands in g->scalars[1].
void train_enqueue(tr_guide* g, const uint4* x, const float* d_dirs, const float* d_weights, uint32_t n, float lr,
                   cudaStream_t s) {
    g->ensure(n);
    TR_CUDA(trg::mlp_forward(g->dev(), x, n, g->out, g->act, g->err, s));
    TR_CUDA(cudaMemsetAsync(g->scalars, 0, 4 * sizeof(float), s));
    TR_CUDA(trg::mix_grad(g->out, d_dirs, d_weights, n, g->scalars, g->dy_bf, g->scalars + 1, s));
    TR_CUDA(trg::mlp_backward(g->dev(), g->dy_bf, g->act, n, g->dh, g->err, s));
    TR_CUDA(cudaMemsetAsync(g->grads, 0, sizeof(float) * TR_GUIDE_PARAMS, s));
    float* gb = g->grads + 4 * 4096;
    const size_t mrow = (size_t)n * 8;
    trg::DwLayers dw{};
    dw.prev[0] = x;                  dw.grad_bf[0] = g->dh;
    dw.prev[1] = g->act;             dw.grad_bf[1] = g->dh + mrow;
    dw.prev[2] = g->act + mrow;      dw.grad_bf[2] = g->dh + 2 * mrow;
    dw.prev[3] = g->act + 2 * mrow;  dw.grad_bf[3] = g->dy_bf;                // output layer
    for (int l = 0; l < 4; ++l) { dw.gw[l] = g->grads + 4096 * l; dw.gb[l] = gb + 64 * l; }
    TR_CUDA(trg::weight_grad(dw, n, g->spin, g->err, s));
    if (lr > 0.0f) {
        g->step += 1;
        TR_CUDA(trg::adam(g->params, g->grads, g->m1, g->m2, TR_GUIDE_PARAMS, lr, g->step, s));
        TR_CUDA(trg::pack_weights(g->params, g->w_fwd, g->w_bwd, s));
    }
}
}  // namespace tri

extern "C" tr_status tr_guide_train_step(tr_guide* g, const uint16_t* d_features, const float* d_dirs,
                                         const float* d_weights, uint32_t n, float lr, float* loss, void* stream) {
    if (!g || !n || !d_features || !d_dirs || !d_weights) return fail(TR_ERR_INVALID_ARGUMENT, "null argument or empty batch");
    if ((reinterpret_cast<uintptr_t>(d_features) & 15u) != 0) return fail(TR_ERR_INVALID_ARGUMENT, "features must be 16-byte aligned");
    try {
        TR_CUDA(cudaSetDevice(g->device));
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : g->stream;
        train_enqueue(g, reinterpret_cast<const uint4*>(d_features), d_dirs, d_weights, n, lr, s);
        if (loss) TR_CUDA(cudaMemcpyAsync(loss, g->scalars + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
        return guide_check_err(g, s);
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
}

extern "C" tr_status tr_guide_set_wait_limit(tr_guide* g, uint32_t polls) {
    if (!g) return fail(TR_ERR_INVALID_ARGUMENT, "null guide");
    g->spin = polls;
    return TR_OK;
}

extern "C" tr_status tr_guide_destroy(tr_guide* g) {
    if (!g) return TR_OK;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (void* q : g->allocs) cudaFree(q);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return TR_OK;
}

namespace tri {
trg::GuideDev guide_dev(tr_guide* g) { return g->dev(); }
int* guide_err(tr_guide* g) { return g->err; }

tr_status train_on_pool(tr_guide* g, const trk::GuideWave& gw, const uint32_t* pool_state, uint32_t pool, float lr,
                        cudaStream_t s, tr_stats& stats) {
    stats.train_steps = 0;
    if (!pool) return guide_check_err(g, s);
    // one synchronisation for the render's MMA status and the pool fill ...
    int e = 0;
    uint32_t fill = 0;
    TR_CUDA(cudaMemcpyAsync(&e, g->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaMemcpyAsync(&fill, pool_state, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TR_CUDA(cudaStreamSynchronize(s));
    if (e) return guide_check_err(g, s);
    // ... the training steps are enqueued back to back, and one more for their status and loss
    const uint32_t n = std::min(fill, pool);
    const uint32_t batch = 65536;
    try {
        for (uint32_t off = 0; off + 1024 <= n; off += batch) {
            const uint32_t m = std::min(batch, n - off);
            train_enqueue(g, gw.pool_feat + (size_t)off * 8, gw.pool_dir + (size_t)off * 3, gw.pool_w + off, m, lr, s);
            stats.train_steps += 1;
        }
    } catch (const CudaError& err) {
        return fail(err.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, err.what());
    }
    if (stats.train_steps) {
        TR_CUDA(cudaMemcpyAsync(&stats.train_loss, g->scalars + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
        return guide_check_err(g, s);
    }
    return TR_OK;
}
}  // namespace tri

namespace {
tr_status guide_begin_render(tr_ctx* x, cudaStream_t s) {
    tr_guide* g = x->guide;
    x->stats.train_steps = 0;
    try {
        // the snapshot must not catch a training step of another render half-way
        TR_CUDA(cudaEventRecord(x->ev_train, g->stream));
        TR_CUDA(cudaStreamWaitEvent(s, x->ev_train, 0));
        TR_CUDA(cudaMemcpyAsync(x->w_snap, g->w_fwd, 4 * 8192, cudaMemcpyDeviceToDevice, s));
        TR_CUDA(cudaMemcpyAsync(x->bias_snap, g->params + 4 * 4096, 4 * 64 * sizeof(float), cudaMemcpyDeviceToDevice, s));
        if (x->pool_pending == 0 || x->guide_lr <= 0.0f) return TR_OK;
        // training on the previous render's pool runs on the guide's stream, after the snapshot
        TR_CUDA(cudaEventRecord(x->ev_snap, s));
        TR_CUDA(cudaStreamWaitEvent(g->stream, x->ev_snap, 0));
        const uint32_t n = x->pool_pending, batch = 65536;
        const tr_ctx::PoolBuf& a = x->pool_alt;
        for (uint32_t off = 0; off + 1024 <= n; off += batch) {
            const uint32_t m = std::min(batch, n - off);
            train_enqueue(g, a.feat + (size_t)off * 8, a.dir + (size_t)off * 3, a.w + off, m, x->guide_lr, g->stream);
            x->stats.train_steps += 1;
        }
        if (x->stats.train_steps)
            TR_CUDA(cudaMemcpyAsync(&x->last_train_loss, g->scalars + 1, sizeof(float), cudaMemcpyDeviceToHost,
                                    g->stream));
        x->pool_pending = 0;
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
    return TR_OK;
}

tr_status guide_end_render(tr_ctx* x, cudaStream_t s) {
    tr_guide* g = x->guide;
    uint32_t fill = 0;
    try {
        // the render has completed (render_region waited for it): its pool fill is final
        TR_CUDA(cudaMemcpyAsync(&fill, x->pool_state, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TR_CUDA(cudaStreamSynchronize(s));
        TR_CUDA(cudaStreamSynchronize(g->stream));     // the training that ran beside the render
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    if (x->stats.train_steps) x->stats.train_loss = x->last_train_loss;
    // this render's pool is trained during the next call; the other pool is filled next
    trk::GuideWave& w = x->gw;
    tr_ctx::PoolBuf& a = x->pool_alt;
    std::swap(w.pool_feat, a.feat);
    std::swap(w.pool_dir, a.dir);
    std::swap(w.pool_w, a.w);
    std::swap(w.pool_meta, a.meta);
    std::swap(x->pool_state, a.state);
    x->pool_pending = std::min(fill, x->guide_pool);
    return guide_check_err(g, g->stream);             // tensor-core timeouts of render or training
}
}  // namespace

extern "C" tr_status tr_set_guide(tr_ctx* x, tr_guide* g, float mix_prob, float lr, uint32_t train_pool) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if (!g) { x->guide = nullptr; x->pool_pending = 0; return TR_OK; }
    if (!(x->integ.flags & TR_FLAG_ORTHONORMAL_FRAME))
        return fail(TR_ERR_INVALID_ARGUMENT, "guided rendering needs TR_FLAG_ORTHONORMAL_FRAME (MIS needs the exact BSDF density)");
    if (x->integ.flags & TR_FLAG_BIDIRECTIONAL)
        return fail(TR_ERR_NOT_SUPPORTED, "the learned proposal is not combined with light subpaths");
    if (g->device != x->device) return fail(TR_ERR_INVALID_ARGUMENT, "guide and context are on different devices");
    if (!(mix_prob > 0.0f && mix_prob < 1.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "mix_prob must be in (0, 1)");
    if (!(lr >= 0.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "learning rate must be >= 0");
    if (train_pool > (1u << 24)) return fail(TR_ERR_INVALID_ARGUMENT, "train_pool too large");
    x->guide = g;
    x->guide_mix = mix_prob;
    x->guide_lr = lr;
    x->guide_pool = train_pool;     // ensure_guided reallocates the pool when its size changes
    x->pool_pending = 0;            // samples collected for another guide are not trained on
    return TR_OK;
}

extern "C" tr_status tr_set_guide_scope(tr_ctx* x, uint32_t depths, float min_roughness) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if (!(min_roughness >= 0.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "min_roughness must be >= 0");
    x->guide_depth = depths;
    x->guide_min_alpha = min_roughness;
    return TR_OK;
}

extern "C" {

tr_status tr_set_stream(tr_ctx* x, void* stream) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    try {
        TR_CUDA(cudaSetDevice(x->device));
        TR_CUDA(cudaStreamSynchronize(x->s()));
    } catch (const CudaError& e) {
        return fail(TR_ERR_CUDA, e.what());
    }
    x->user_stream = static_cast<cudaStream_t>(stream);
    return TR_OK;
}

tr_status tr_set_profiling(tr_ctx* x, int on) {
    if (!x) return fail(TR_ERR_INVALID_ARGUMENT, "null context");
    if (on < 0 || on > 2) return fail(TR_ERR_INVALID_ARGUMENT, "profiling must be 0, 1 or 2");
    x->profiling = on;
    x->prof_marks.clear();          // launches timed under another setting are dropped
    x->prof_next = 0;
    for (double& v : x->prof_sum) v = 0.0;
    x->prof_dirty = false;
    return TR_OK;
}

tr_status tr_destroy(tr_ctx* x) {
    if (!x) return TR_OK;
    cudaSetDevice(x->device);
    cudaStreamSynchronize(x->s());
    if (x->stream) cudaStreamSynchronize(x->stream);
    x->release();
    delete x;
    return TR_OK;
}

}  // extern "C"
