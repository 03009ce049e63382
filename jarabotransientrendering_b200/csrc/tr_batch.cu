// tr_batch.cu - multi-scene rendering (no counterpart in the reference renderer): the scenes of
// several contexts rendered in shared wavefront batches, each batch one replay of a captured
// CUDA graph, plus the autotuner that picks the batch's launch shape.
//
// Planning (host): every scene's work (pixels x camera-sample chunks) is cut into segments and
// packed into batches of at most `capacity` path slots and kMaxSegments segments; a segment is
// one scene's contiguous pixel range for one sample chunk, so a small scene shares a batch with
// others and a large one spans several.  The plan goes to device memory as BatchDesc records;
// the multi-scene kernels find a slot's segment by binary search over the current descriptor
// (*cur), so the launch sequence of a batch does not depend on the batch and is captured once:
//   memset(counters) -> raygen -> depth x (extend, shade, [guide], shadow) -> [train gather]
//   -> splat -> advance(*cur)
// for each of four wave lanes (own wave buffers, cursor and stream pair; lane k renders batches
// k, k + 4, ...) as parallel branches of one graph, replayed once per group of four batches.
#include "tr_internal.h"

#include <chrono>
#include <cstring>

using namespace tri;

struct tr_batch {
    int device = 0;
    cudaStream_t stream = nullptr;          // lane 0's stream (every call forks from and joins it)
    cudaStream_t shadow_stream = nullptr;   // shadow launches beside the next depth's extend
    // lanes 1..kLanes-1: batch k runs on lane k mod kLanes, each with its own wave and streams
    static constexpr int kLanes = 4;
    cudaStream_t lane_stream[kLanes - 1] = {}, lane_shadow[kLanes - 1] = {};
    cudaEvent_t dep[8] = {};                // ordering events between the streams, used in turn
    uint32_t next_dep = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<tr_ctx*> ctx;
    std::vector<void*> allocs;
    size_t bytes = 0;

    trk::SceneSlot* d_scenes = nullptr;
    trk::BatchDesc* d_batches = nullptr;
    uint32_t batches_cap = 0;
    uint32_t* d_cur = nullptr;              // [lane]: index of the batch the lane is on
    trk::Wave wave{};
    trk::Wave lane_wave[kLanes - 1]{};      // the other lanes' (share wave.stats)
    uint32_t max_bounces = 1, bvh_depth = 0;
    int trace_grid = 0;
    tr_batch_config cfg{1u << 21, 256, 1, 1};

    // learned proposal
    tr_guide* guide = nullptr;
    float mix = 0.5f, lr = 1e-3f;
    uint32_t pool = 0;
    trk::GuideWave gw{};
    uint4* lane_vrec[kLanes - 1] = {};      // the other lanes' guided-vertex records
    uint32_t gw_capacity = 0;
    uint32_t* pool_state = nullptr;

    // captured graph and the launch shape it replays
    struct Shape {
        uint32_t capacity = 0, shade_block = 0, max_blocks = 0, guided = 0, pool = 0;
        float mix = 0.f, keep = 0.f;
        bool operator==(const Shape& o) const {
            return capacity == o.capacity && shade_block == o.shade_block && max_blocks == o.max_blocks &&
                   guided == o.guided && pool == o.pool && mix == o.mix && keep == o.keep;
        }
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    Shape shape{};

    tr_stats stats{};

    template <class T>
    T* alloc(size_t n) {
        T* p = tri::dalloc<T>(n, bytes);
        allocs.push_back(p);
        return p;
    }
    void drop(void* p) {
        if (!p) return;
        cudaFree(p);
        allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
};

namespace {

struct Plan {
    std::vector<trk::BatchDesc> batches;
    uint32_t max_blocks = 0;
    uint64_t slots = 0;
    std::vector<uint64_t> scene_slots;      // per scene
};

// pixels per splat block of a segment: the automatic width (whole pixels filling one block)
// divided by the configuration's splat_div
uint32_t splat_width(const tr_batch* b, uint32_t per_pix) {
    return std::max<uint32_t>(1u, trk::splat_pixels_per_block(per_pix) / std::max<uint32_t>(1u, b->cfg.splat_div));
}

Plan make_plan(const tr_batch* b, const uint64_t* s_begin, const uint32_t* s_count) {
    Plan pl;
    pl.scene_slots.assign(b->ctx.size(), 0);
    const uint32_t cap = b->cfg.capacity;
    trk::BatchDesc bd{};
    uint32_t used = 0;
    auto flush = [&]() {
        if (bd.nseg == 0) return;
        pl.max_blocks = std::max(pl.max_blocks, bd.n_blocks);
        pl.batches.push_back(bd);
        bd = trk::BatchDesc{};
        used = 0;
    };
    for (uint32_t i = 0; i < b->ctx.size(); ++i) {
        const uint32_t count = s_count[i];
        if (!count) continue;
        const tr_ctx* x = b->ctx[i];
        const uint32_t ninc = x->integ.incoming_samples;
        const uint32_t W = x->film.width, H = x->film.height;
        const uint32_t npix_total = W * H;
        const uint32_t ns_chunk = std::max<uint32_t>(1u, std::min<uint32_t>(count, cap / ninc));
        for (uint32_t sb = 0; sb < count; sb += ns_chunk) {
            const uint32_t ns = std::min(ns_chunk, count - sb);
            const uint32_t per_pix = ns * ninc;
            const uint32_t G = splat_width(b, per_pix);
            uint32_t pix = 0;
            while (pix < npix_total) {
                const uint32_t free = cap - used;
                if (free < per_pix || bd.nseg == (uint32_t)trk::kMaxSegments) {
                    flush();
                    continue;
                }
                const uint32_t take = std::min(npix_total - pix, free / per_pix);
                trk::Batch& sg = bd.seg[bd.nseg++];
                sg = trk::Batch{};
                sg.win_x0 = 0; sg.win_y0 = 0; sg.win_w = W;
                sg.pix_begin = pix; sg.npix = take;
                sg.s0 = s_begin[i] + sb; sg.ns = ns; sg.ninc = ninc;
                sg.n_slots = take * per_pix;
                sg.slot_begin = used;
                sg.scene = i;
                sg.blk_begin = bd.n_blocks;
                sg.splat_g = G;
                bd.n_blocks += (take + G - 1) / G;
                bd.n_slots += sg.n_slots;
                bd.max_depth = std::max(bd.max_depth, x->integ.max_bounces);
                used += sg.n_slots;
                pix += take;
                pl.slots += sg.n_slots;
                pl.scene_slots[i] += sg.n_slots;
            }
        }
    }
    flush();
    return pl;
}

void ensure_lane(tr_batch* b, trk::Wave& w, uint32_t capacity, unsigned long long* stats);

void ensure_batch_wave(tr_batch* b, uint32_t capacity) {
    bool same = b->wave.capacity == capacity;
    for (const trk::Wave& w : b->lane_wave) same = same && w.capacity == capacity;
    if (same) return;
    b->drop_graph();
    ensure_lane(b, b->wave, capacity, nullptr);
    for (trk::Wave& w : b->lane_wave) ensure_lane(b, w, capacity, b->wave.stats);
}

// one lane's wave buffers; `stats` null: allocate the statistics counters, else share them
void ensure_lane(tr_batch* b, trk::Wave& w, uint32_t capacity, unsigned long long* stats) {
    b->drop(w.ray_o); b->drop(w.ray_d); b->drop(w.thr); b->drop(w.rng); b->drop(w.hit); b->drop(w.q[0]);
    b->drop(w.q[1]); b->drop(w.sh_o); b->drop(w.sh_d); b->drop(w.sh_L); b->drop(w.rec); b->drop(w.rec_n);
    w.ray_o = b->alloc<float4>(capacity);
    w.ray_d = b->alloc<float4>(capacity);
    w.thr = b->alloc<float4>(capacity);
    w.rng = b->alloc<unsigned long long>(capacity);
    w.hit = b->alloc<float4>(capacity);
    w.q[0] = b->alloc<uint32_t>(capacity);
    w.q[1] = b->alloc<uint32_t>(capacity);
    w.sh_o = b->alloc<float4>(capacity);
    w.sh_d = b->alloc<float4>(capacity);
    w.sh_L = b->alloc<float4>(capacity);
    w.rec = b->alloc<float4>((size_t)capacity * std::max<uint32_t>(1u, b->max_bounces));
    w.rec_n = b->alloc<uint8_t>(capacity);
    b->drop(w.cam_dist);
    w.cam_dist = b->alloc<float>(capacity);
    b->drop(w.target);
    bool tsm = false;
    for (tr_ctx* x : b->ctx) tsm = tsm || (x->integ.flags & TR_FLAG_TIME_SAMPLING) != 0;
    w.target = tsm ? b->alloc<float4>(capacity) : nullptr;
    if (!w.counters) w.counters = b->alloc<uint32_t>(trk::kCounters);
    if (stats) {
        w.stats = stats;
    } else if (!w.stats) {
        w.stats = b->alloc<unsigned long long>(8);
        TR_CUDA(cudaMemsetAsync(w.stats, 0, 8 * sizeof(unsigned long long), b->stream));
    }
    w.capacity = capacity;
}

void ensure_batch_guided(tr_batch* b, uint32_t capacity) {
    if (b->gw_capacity == capacity && b->gw.pool_cap == b->pool && b->pool_state) return;
    b->drop_graph();
    trk::GuideWave& g = b->gw;
    b->drop(g.vrec); b->drop(g.pool_feat); b->drop(g.pool_dir); b->drop(g.pool_w); b->drop(g.pool_meta);
    g.vrec = b->alloc<uint4>((size_t)capacity * 5);
    for (uint4*& v : b->lane_vrec) {
        b->drop(v);
        v = b->alloc<uint4>((size_t)capacity * 5);
    }
    const uint32_t pc = std::max<uint32_t>(1u, b->pool);
    g.pool_feat = b->alloc<uint4>((size_t)pc * 8);
    g.pool_dir = b->alloc<float>((size_t)pc * 3);
    g.pool_w = b->alloc<float>(pc);
    g.pool_meta = b->alloc<uint4>(pc);
    g.pool_cap = b->pool;
    if (!b->pool_state) b->pool_state = b->alloc<uint32_t>(2);
    b->gw_capacity = capacity;
}

trk::Params batch_params(const tr_batch* b, const Plan& pl, int lane) {
    trk::Params p{};
    p.wave = lane ? b->lane_wave[lane - 1] : b->wave;
    p.bvh_depth = b->bvh_depth;
    p.max_bounces = b->max_bounces;
    p.multi.scenes = b->d_scenes;
    p.multi.batches = b->d_batches;
    p.multi.cur = b->d_cur + lane;
    p.multi.nscenes = (uint32_t)b->ctx.size();
    p.multi.max_splat_blocks = std::max<uint32_t>(1u, pl.max_blocks);
    p.multi.shade_block = b->cfg.shade_block;
    if (b->guide) {
        p.guide = b->gw;
        p.guide.net = guide_dev(b->guide);
        p.guide.err = guide_err(b->guide);
        if (lane) p.guide.vrec = b->lane_vrec[lane - 1];
        p.guide.tag = 1u;       // the lanes fill the pool at once: entries tagged by batch index
        p.guide.min_alpha = kGuideMinAlpha;
    }
    return p;
}

// `to` waits for the work enqueued on `from` so far (inside a capture: a graph dependency)
void order(tr_batch* b, cudaStream_t from, cudaStream_t to) {
    cudaEvent_t e = b->dep[b->next_dep++ % 8u];
    TR_CUDA(cudaEventRecord(e, from));
    TR_CUDA(cudaStreamWaitEvent(to, e, 0));
}

// the launches of one batch; `count` is incremented by the number of kernels.  The shadow
// launch of depth d runs on the second stream beside the closest-hit launch of depth d + 1
// (both only read what shade(d) wrote); shade(d + 1) refills the shadow queue and waits for it.
void enqueue_batch(tr_batch* b, const trk::Params& p, cudaStream_t s, cudaStream_t sh, uint64_t& count) {
    const bool guided = b->guide != nullptr;
    TR_CUDA(cudaMemsetAsync(p.wave.counters, 0, trk::kCounters * sizeof(uint32_t), s));
    TR_CUDA(trk::launch_raygen(p, s));
    for (uint32_t d = 0; d < b->max_bounces; ++d) {
        TR_CUDA(trk::launch_extend(p, (int)d, b->trace_grid, s));
        if (d > 0) order(b, sh, s);
        TR_CUDA(trk::launch_shade(p, (int)d, s));
        if (guided) { TR_CUDA(trk::launch_guide(p, (int)d, b->pool_state, s)); ++count; }
        order(b, s, sh);
        TR_CUDA(trk::launch_shadow(p, (int)d, b->trace_grid, sh));
        count += 3;
    }
    if (b->max_bounces) order(b, sh, s);
    if (guided && b->pool) { TR_CUDA(trk::launch_train_gather(p, b->pool_state, s)); count += 2; }
    TR_CUDA(trk::launch_splat(p, s));
    TR_CUDA(trk::launch_advance(p.multi.cur, (uint32_t)tr_batch::kLanes, s));   // this lane's next batch
    count += 3;
}

// kLanes batches, one per lane: the other lanes fork from lane 0's stream and join it again, so
// a capture of the group holds all of them as parallel branches.
void enqueue_group(tr_batch* b, const trk::Params* p, uint64_t& count) {
    for (int k = 0; k + 1 < tr_batch::kLanes; ++k) order(b, b->stream, b->lane_stream[k]);
    enqueue_batch(b, p[0], b->stream, b->shadow_stream, count);
    for (int k = 0; k + 1 < tr_batch::kLanes; ++k) enqueue_batch(b, p[k + 1], b->lane_stream[k], b->lane_shadow[k], count);
    for (int k = 0; k + 1 < tr_batch::kLanes; ++k) order(b, b->lane_stream[k], b->stream);
}

tr_status batch_render(tr_batch* b, const uint64_t* s_begin, const uint32_t* s_count) {
    for (uint32_t i = 0; i < b->ctx.size(); ++i)
        if (s_count[i] && s_begin[i] + s_count[i] > (1ull << 32))
            return fail(TR_ERR_INVALID_ARGUMENT, "camera sample index must stay below 2^32");
    TR_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = b->stream;
    Plan pl = make_plan(b, s_begin, s_count);
    b->stats.kernel_launches = 0;
    b->stats.train_steps = 0;
    b->stats.render_ms = 0.0;
    if (pl.batches.empty()) return TR_OK;
    // batches run in groups of kLanes, one per lane; a count that is not a multiple ends with
    // empty batches (no slots, no splat blocks: their kernels find no work)
    while (pl.batches.size() % (size_t)tr_batch::kLanes) pl.batches.push_back(trk::BatchDesc{});
    ensure_batch_wave(b, b->cfg.capacity);
    const bool guided = b->guide != nullptr;
    if (guided) {
        ensure_batch_guided(b, b->cfg.capacity);
        b->gw.keep_prob = b->pool ? std::min(1.0f, (float)b->pool / (1.5f * (float)pl.slots)) : 0.0f;
        b->gw.mix_prob = b->mix;
        TR_CUDA(cudaMemsetAsync(b->pool_state, 0, 2 * sizeof(uint32_t), s));
        // entries are tagged by batch index: no tag of an earlier render may remain
        if (b->pool) TR_CUDA(cudaMemsetAsync(b->gw.pool_meta, 0, (size_t)b->pool * sizeof(uint4), s));
    }
    if (pl.batches.size() > b->batches_cap) {
        b->drop_graph();
        b->drop(b->d_batches);
        b->batches_cap = (uint32_t)pl.batches.size() * 2;
        b->d_batches = b->alloc<trk::BatchDesc>(b->batches_cap);
    }
    TR_CUDA(cudaMemcpyAsync(b->d_batches, pl.batches.data(), pl.batches.size() * sizeof(trk::BatchDesc),
                            cudaMemcpyHostToDevice, s));
    // lane k starts at batch k
    TR_CUDA(cudaMemsetAsync(b->d_cur, 0, tr_batch::kLanes * sizeof(uint32_t), s));
    for (int k = 1; k < tr_batch::kLanes; ++k) TR_CUDA(trk::launch_advance(b->d_cur + k, (uint32_t)k, s));
    trk::Params pv[tr_batch::kLanes];
    for (int k = 0; k < tr_batch::kLanes; ++k) pv[k] = batch_params(b, pl, k);
    const trk::Params& p0 = pv[0];

    tr_batch::Shape shape;
    shape.capacity = b->cfg.capacity;
    shape.shade_block = b->cfg.shade_block;
    shape.max_blocks = p0.multi.max_splat_blocks;
    shape.guided = guided ? 1u : 0u;
    shape.pool = b->pool;
    shape.mix = guided ? b->gw.mix_prob : 0.f;
    shape.keep = guided ? b->gw.keep_prob : 0.f;

    uint64_t launches = 0;
    TR_CUDA(cudaEventRecord(b->ev0, s));
    const size_t groups = pl.batches.size() / (size_t)tr_batch::kLanes;    // groups of kLanes batches
    size_t done = 0;
    if (b->cfg.use_graph) {
        if (!(b->exec && shape == b->shape)) {
            // new launch shape: the first group runs directly (which also performs the kernels'
            // one-time attribute calls outside any capture), then one group is captured for the
            // remaining groups and later calls with the same shape
            enqueue_group(b, pv, launches);
            done = 1;
            b->drop_graph();
            if (done < groups) {
                uint64_t n_capt = 0;
                TR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                try {
                    enqueue_group(b, pv, n_capt);
                } catch (...) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(s, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                TR_CUDA(cudaStreamEndCapture(s, &b->graph));
                TR_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
                b->shape = shape;
            }
        }
        // kernels per replay (kLanes batches of enqueue_batch)
        const uint64_t per = (uint64_t)tr_batch::kLanes *
                             (3 + 3ull * b->max_bounces + (guided ? b->max_bounces + (b->pool ? 2 : 0) : 0));
        for (; done < groups; ++done) {
            TR_CUDA(cudaGraphLaunch(b->exec, s));
            launches += per;
        }
    } else {
        for (; done < groups; ++done) enqueue_group(b, pv, launches);
    }
    TR_CUDA(cudaEventRecord(b->ev1, s));
    TR_CUDA(cudaEventSynchronize(b->ev1));
    float ms = 0.f;
    TR_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    unsigned long long st[8];
    TR_CUDA(cudaMemcpy(st, b->wave.stats, sizeof(st), cudaMemcpyDeviceToHost));
    b->stats.closest_rays = st[0];
    b->stats.shadow_rays = st[1];
    b->stats.splats = st[2];
    b->stats.paths += pl.slots;
    b->stats.render_ms = ms;
    b->stats.kernel_launches = launches;
    for (uint32_t i = 0; i < b->ctx.size(); ++i) {
        tr_ctx* x = b->ctx[i];
        const uint64_t cs = (uint64_t)x->film.width * x->film.height * s_count[i];
        b->stats.camera_samples += cs;
        x->stats.camera_samples += cs;
        x->stats.paths += pl.scene_slots[i];
    }
    if (guided) return train_on_pool(b->guide, b->gw, b->pool_state, b->pool, b->lr, s, b->stats);
    return TR_OK;
}

}  // namespace

extern "C" {

tr_status tr_batch_create(tr_ctx* const* contexts, uint32_t n, tr_batch** out) {
    if (!out) return fail(TR_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    if (!contexts || n == 0) return fail(TR_ERR_INVALID_ARGUMENT, "no contexts");
    if (n > (uint32_t)trk::kMaxSegments)
        return fail(TR_ERR_INVALID_ARGUMENT, "a batch holds at most " + std::to_string(trk::kMaxSegments) + " scenes");
    for (uint32_t i = 0; i < n; ++i) {
        if (!contexts[i]) return fail(TR_ERR_INVALID_ARGUMENT, "context " + std::to_string(i) + " is null");
        if (contexts[i]->device != contexts[0]->device)
            return fail(TR_ERR_INVALID_ARGUMENT, "all contexts of a batch must be on one device");
        if (contexts[i]->film.bounce_films)
            return fail(TR_ERR_NOT_SUPPORTED, "contexts with bounce films render through tr_render, not in a batch");
        if (contexts[i]->integ.flags & TR_FLAG_BIDIRECTIONAL)
            return fail(TR_ERR_NOT_SUPPORTED, "contexts with light subpaths render through tr_render, not in a batch");
    }
    tr_batch* b = new (std::nothrow) tr_batch();
    if (!b) return fail(TR_ERR_OUT_OF_MEMORY, "host allocation");
    try {
        b->device = contexts[0]->device;
        TR_CUDA(cudaSetDevice(b->device));
        TR_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        TR_CUDA(cudaStreamCreateWithFlags(&b->shadow_stream, cudaStreamNonBlocking));
        for (int k = 0; k + 1 < tr_batch::kLanes; ++k) {
            TR_CUDA(cudaStreamCreateWithFlags(&b->lane_stream[k], cudaStreamNonBlocking));
            TR_CUDA(cudaStreamCreateWithFlags(&b->lane_shadow[k], cudaStreamNonBlocking));
        }
        for (cudaEvent_t& e : b->dep) TR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        TR_CUDA(cudaEventCreate(&b->ev0));
        TR_CUDA(cudaEventCreate(&b->ev1));
        std::vector<trk::SceneSlot> slots(n);
        for (uint32_t i = 0; i < n; ++i) {
            tr_ctx* x = contexts[i];
            b->ctx.push_back(x);
            const trk::Params px = make_params(x);
            trk::SceneSlot& S = slots[i];
            S.scene = px.scene;
            S.cam = px.cam;
            S.film = px.film;
            S.seed = px.seed;
            S.max_bounces = px.max_bounces;
            S.sqrt_spp = px.sqrt_spp;
            S.flags = px.flags;
            b->max_bounces = std::max(b->max_bounces, x->integ.max_bounces);
            b->bvh_depth = std::max(b->bvh_depth, x->bvh_depth);
        }
        b->d_scenes = b->alloc<trk::SceneSlot>(n);
        // ordered on the batch's stream (a plain cudaMemcpy from pageable memory may return
        // before the data lands, on a stream that does not order with this one)
        TR_CUDA(cudaMemcpyAsync(b->d_scenes, slots.data(), n * sizeof(trk::SceneSlot), cudaMemcpyHostToDevice, b->stream));
        TR_CUDA(cudaStreamSynchronize(b->stream));
        b->d_cur = b->alloc<uint32_t>(tr_batch::kLanes);
        b->trace_grid = trk::trace_grid_size(b->device, b->bvh_depth, true);
        b->stats.device_bytes = b->bytes;
    } catch (const CudaError& e) {
        for (void* p : b->allocs) cudaFree(p);
        for (cudaEvent_t e : b->dep)
            if (e) cudaEventDestroy(e);
        if (b->shadow_stream) cudaStreamDestroy(b->shadow_stream);
        for (int k = 0; k + 1 < tr_batch::kLanes; ++k) {
            if (b->lane_stream[k]) cudaStreamDestroy(b->lane_stream[k]);
            if (b->lane_shadow[k]) cudaStreamDestroy(b->lane_shadow[k]);
        }
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
    *out = b;
    return TR_OK;
}

tr_status tr_batch_set_config(tr_batch* b, const tr_batch_config* cfg) {
    if (!b || !cfg) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    if (cfg->capacity < (1u << 16) || cfg->capacity > (1u << 23))
        return fail(TR_ERR_INVALID_ARGUMENT, "capacity must be in [65536, 8388608]");
    if (cfg->shade_block != 128 && cfg->shade_block != 256)
        return fail(TR_ERR_INVALID_ARGUMENT, "shade_block must be 128 or 256");
    if (cfg->splat_div == 0 || cfg->splat_div > 16) return fail(TR_ERR_INVALID_ARGUMENT, "splat_div must be in [1, 16]");
    for (tr_ctx* x : b->ctx)
        if ((uint64_t)x->integ.incoming_samples > cfg->capacity)
            return fail(TR_ERR_INVALID_ARGUMENT, "capacity below a scene's paths per camera sample");
    b->cfg = *cfg;
    b->cfg.use_graph = cfg->use_graph ? 1u : 0u;
    return TR_OK;
}

tr_status tr_batch_get_config(tr_batch* b, tr_batch_config* cfg) {
    if (!b || !cfg) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    *cfg = b->cfg;
    return TR_OK;
}

tr_status tr_batch_render(tr_batch* b, const uint64_t* sample_begin, const uint32_t* sample_count) {
    if (!b || !sample_begin || !sample_count) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    for (tr_ctx* x : b->ctx) x->film_clean = false;
    try {
        return batch_render(b, sample_begin, sample_count);
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? TR_ERR_OUT_OF_MEMORY : TR_ERR_CUDA, e.what());
    }
}

tr_status tr_batch_autotune(tr_batch* b, const uint64_t* sample_begin, const uint32_t* trial_samples,
                            tr_batch_config* best, uint32_t* trials_run) {
    if (!b || !sample_begin || !trial_samples) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    const size_t n = b->ctx.size();
    std::vector<uint64_t> begin(sample_begin, sample_begin + n);
    uint32_t trials = 0;
    const tr_batch_config start = b->cfg;
    // one timed trial of configuration c (device time of the batches)
    auto trial = [&](const tr_batch_config& c, double& ms) -> tr_status {
        tr_status st = tr_batch_set_config(b, &c);
        if (st != TR_OK) return st;
        st = tr_batch_render(b, begin.data(), trial_samples);
        if (st != TR_OK) return st;
        for (size_t i = 0; i < n; ++i) begin[i] += trial_samples[i];
        ++trials;
        ms = b->stats.render_ms;
        return TR_OK;
    };
    // coordinate descent: queue capacity, then shade block, then film tile width; each candidate
    // is run twice and its faster time kept (the first run of a new shape includes its capture)
    tr_batch_config cur = start;
    double cur_ms = 0.0;
    auto best_of = [&](const tr_batch_config& c, double& ms) -> tr_status {
        double a = 0.0, bb = 0.0;
        tr_status st = trial(c, a);
        if (st == TR_OK) st = trial(c, bb);
        ms = std::min(a, bb);
        return st;
    };
    tr_status st = best_of(cur, cur_ms);
    if (st != TR_OK) return st;
    const uint32_t caps[] = {1u << 19, 1u << 20, 1u << 21, 1u << 22};
    for (uint32_t cap : caps) {
        if (cap == cur.capacity) continue;
        tr_batch_config c = cur;
        c.capacity = cap;
        double ms = 0.0;
        if (best_of(c, ms) != TR_OK) continue;       // e.g. out of memory: skip the candidate
        if (ms < cur_ms) { cur = c; cur_ms = ms; }
    }
    for (uint32_t blk : {128u, 256u}) {
        if (blk == cur.shade_block) continue;
        tr_batch_config c = cur;
        c.shade_block = blk;
        double ms = 0.0;
        if (best_of(c, ms) != TR_OK) continue;
        if (ms < cur_ms) { cur = c; cur_ms = ms; }
    }
    for (uint32_t dv : {1u, 2u, 4u}) {
        if (dv == cur.splat_div) continue;
        tr_batch_config c = cur;
        c.splat_div = dv;
        double ms = 0.0;
        if (best_of(c, ms) != TR_OK) continue;
        if (ms < cur_ms) { cur = c; cur_ms = ms; }
    }
    st = tr_batch_set_config(b, &cur);
    if (best) *best = cur;
    if (trials_run) *trials_run = trials;
    return st;
}

tr_status tr_batch_set_guide(tr_batch* b, tr_guide* g, float mix_prob, float lr, uint32_t train_pool) {
    if (!b) return fail(TR_ERR_INVALID_ARGUMENT, "null batch");
    if (!g) { b->guide = nullptr; b->drop_graph(); return TR_OK; }
    for (tr_ctx* x : b->ctx)
        if (!(x->integ.flags & TR_FLAG_ORTHONORMAL_FRAME))
            return fail(TR_ERR_INVALID_ARGUMENT, "guided rendering needs TR_FLAG_ORTHONORMAL_FRAME on every context");
    if (g->device != b->device) return fail(TR_ERR_INVALID_ARGUMENT, "guide and batch are on different devices");
    if (!(mix_prob > 0.0f && mix_prob < 1.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "mix_prob must be in (0, 1)");
    if (!(lr >= 0.0f)) return fail(TR_ERR_INVALID_ARGUMENT, "learning rate must be >= 0");
    if (train_pool > (1u << 24)) return fail(TR_ERR_INVALID_ARGUMENT, "train_pool too large");
    b->guide = g;
    b->mix = mix_prob;
    b->lr = lr;
    b->pool = train_pool;
    b->drop_graph();
    return TR_OK;
}

tr_status tr_batch_stats(tr_batch* b, tr_stats* out) {
    if (!b || !out) return fail(TR_ERR_INVALID_ARGUMENT, "null argument");
    b->stats.device_bytes = b->bytes;
    b->stats.bvh_depth = b->bvh_depth;
    *out = b->stats;
    return TR_OK;
}

tr_status tr_batch_destroy(tr_batch* b) {
    if (!b) return TR_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->drop_graph();
    for (void* p : b->allocs) cudaFree(p);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    for (cudaEvent_t e : b->dep)
        if (e) cudaEventDestroy(e);
    if (b->shadow_stream) cudaStreamDestroy(b->shadow_stream);
    for (int k = 0; k + 1 < tr_batch::kLanes; ++k) {
        if (b->lane_stream[k]) cudaStreamDestroy(b->lane_stream[k]);
        if (b->lane_shadow[k]) cudaStreamDestroy(b->lane_shadow[k]);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return TR_OK;
}

}  // extern "C"
