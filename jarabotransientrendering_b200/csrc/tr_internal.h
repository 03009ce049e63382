// tr_internal.h - host-side internals shared by the C ABI translation units (tr_api.cu: one
// scene per context; tr_batch.cu: many contexts rendered in shared wavefront batches).
#pragma once
#include "transient_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <functional>
#include <vector>

#include "tr_guide.cuh"
#include "tr_kernels.cuh"

namespace tri {

// records msg as the thread's last error (tr_last_error) and returns s
tr_status fail(tr_status s, const std::string& msg);

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const char* what) : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)), code(c) {}
};

#define TR_CUDA(call)                                           \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) throw CudaError(e_, #call);      \
    } while (0)

// Device memory of contexts, guides and batches comes from one stream-ordered pool per device
// that keeps freed memory for the next allocations (release threshold unlimited), so creating
// and destroying contexts does not map and unmap gigabytes each time; memory goes back to the
// driver only through tr_release_cached_memory or at exit.  Frees stay cudaFree (which waits
// for the device and returns the block to its pool).
cudaMemPool_t device_pool(int device);
// pool memory of `device` reserved but not in use (free for the next allocations)
size_t pool_idle_bytes(int device);

template <class T>
T* dalloc(size_t count, size_t& total) {
    if (count == 0) count = 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    void* p = nullptr;
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&p, count * sizeof(T), device_pool(dev), 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);     // usable from every stream
    if (e != cudaSuccess) throw CudaError(e, "device allocation");
    total += count * sizeof(T);
    return static_cast<T*>(p);
}

constexpr uint32_t kMaxBounces = 63;            // counters hold 64 depths
constexpr uint32_t kDefaultCapacity = 1u << 21; // path slots per wavefront batch
#ifndef TR_WAVE_LANES
#define TR_WAVE_LANES 4
#endif
constexpr int kWaveLanes = TR_WAVE_LANES;        // wave buffer sets batches alternate between
// default roughness below which GGX vertices sample their BSDF instead of the learned proposal
constexpr float kGuideMinAlpha = 0.5f;

}  // namespace tri

using tri::dalloc;

struct tr_guide {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    size_t bytes = 0;
    float* params = nullptr;   // FP32 master copy
    float* grads = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    uint8_t* w_fwd = nullptr;  // packed BF16 tiles
    uint8_t* w_bwd = nullptr;
    int* err = nullptr;
    float* scalars = nullptr;  // [0] weight sum, [1] loss
    uint32_t cap = 0;
    uint4* act = nullptr;
    float* out = nullptr;
    uint4* dy_bf = nullptr;
    uint4* dh = nullptr;       // BF16 hidden-layer gradients [3][n][64]
    uint32_t step = 0;
    uint32_t spin = trg::kWaitPolls;   // mbarrier polls before a tensor-core wait times out
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
    trg::GuideDev dev() const {
        return trg::GuideDev{reinterpret_cast<const uint4*>(w_fwd), reinterpret_cast<const uint4*>(w_bwd),
                             params + 4 * 4096, spin};
    }
    void ensure(uint32_t n) {
        if (cap >= n) return;
        drop(act); drop(out); drop(dy_bf); drop(dh);
        act = alloc<uint4>((size_t)3 * n * 8);
        out = alloc<float>((size_t)n * trg::kOut);
        dy_bf = alloc<uint4>((size_t)n * 8);
        dh = alloc<uint4>((size_t)3 * n * 8);
        cap = n;
    }
};

struct tr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    size_t bytes = 0;
    std::vector<void*> allocs;

    // scene
    float4* d_nodes = nullptr;
    float4* d_tris = nullptr;
    float4* d_tri_ng = nullptr;
    float4* d_mats = nullptr;
    float4* d_mats2 = nullptr;
    float4* d_lights = nullptr;
    trk::SceneDev scene{};
    uint32_t nt = 0, bvh_nodes = 0, bvh_depth = 0, bvh_levels = 0;   // bvh_depth: stack entries - 1
    double bvh_ms = 0.0;

    tr_camera cam{};
    tr_film film{};
    tr_integrator integ{};

    // film
    double* d_streak = nullptr;
    double* d_steady = nullptr;
    double* d_weight = nullptr;
    double* d_bstreak = nullptr;            // per-bounce films (tr_film.bounce_films > 0)
    double* d_bsteady = nullptr;
    double* d_bweight = nullptr;
    double* d_cdepth = nullptr;             // film components (tr_film.components)
    double* d_cpos = nullptr;
    double* d_cnorm = nullptr;

    // wavefront state
    trk::Wave wave{};
    trk::Wave lane_wave[tri::kWaveLanes - 1]{};  // further lanes of batches (share wave.stats)
    uint4* lane_vrec[tri::kWaveLanes - 1]{};      // their guided-vertex records (learned proposal)
    uint32_t lane_vrec_cap[tri::kWaveLanes - 1]{};
    uint32_t guide_tag = 0;                       // last training-pool batch tag handed out
    trk::Wave lwave{};                      // light subpaths (TR_FLAG_BIDIRECTIONAL)
    trk::BidirWave bd{};
    uint32_t* d_lcounters = nullptr;
    // film streaming (tr_render_film)
    cudaStream_t copy_stream = nullptr;
    // shadow rays of one depth beside the closest-hit rays of the next (tr_render_region)
    cudaStream_t shadow_stream = nullptr;
    cudaStream_t lane_stream[tri::kWaveLanes - 1]{}, lane_shadow_stream[tri::kWaveLanes - 1]{};
    cudaStream_t light_stream = nullptr;    // light subpaths beside the eye walks (bidirectional)
    std::vector<cudaEvent_t> dep_events;    // ordering events (no timing), reused in turn
    size_t next_dep = 0;
    float* d_stage = nullptr;               // FP32 staging of one pixel batch's rows
    size_t stage_floats = 0;
    uchar4* d_rgbe = nullptr;               // RGBE film images: [H][W][T] streak cells, then [H][W] steady
    size_t rgbe_cells = 0;
    bool film_clean = true;                 // no samples added since the film was zeroed
    int trace_grid = 0;

    // ray-batch scratch
    float* d_rays = nullptr;
    void* d_hits = nullptr;
    uint32_t ray_cap = 0;
    uint32_t* d_cursor = nullptr;

    tr_stats stats{};
    // learned proposal (tr_set_guide)
    tr_guide* guide = nullptr;
    float guide_mix = 0.5f, guide_lr = 1e-3f;
    uint32_t guide_pool = 0;
    trk::GuideWave gw{};
    uint32_t gw_capacity = 0;
    uint32_t* pool_state = nullptr;       // [0] pool fill, [1] entries with targets
    // Training pools are double-buffered: a render fills the pool in gw while the samples of the
    // previous render (pool_alt, pool_pending entries) train the proposal beside it, on the
    // guide's stream.  The render samples with a snapshot of the network (w_snap, bias_snap)
    // taken when it starts, so the training it overlaps never changes the proposal mid-render.
    struct PoolBuf { uint4* feat = nullptr; float* dir = nullptr; float* w = nullptr; uint4* meta = nullptr;
                     uint32_t* state = nullptr; };
    PoolBuf pool_alt{};
    uint32_t pool_pending = 0;
    uint4* w_snap = nullptr;              // packed forward tiles of the render's network (32 KB)
    float* bias_snap = nullptr;           // and its biases [4][64]
    cudaEvent_t ev_snap = nullptr, ev_train = nullptr;
    uint32_t guide_depth = 0xffffffffu;   // path depths whose surface vertices use the proposal
    float guide_min_alpha = tri::kGuideMinAlpha;   // GGX vertices smoother than this sample their BSDF
    float last_train_loss = 0.0f;
    uint32_t train_steps = 0;
    cudaStream_t user_stream = nullptr;   // caller's stream (tr_set_stream) or null
    int profiling = 0;                    // 0 off, 1 read out per render, 2 read out at tr_stats_get
    std::vector<cudaEvent_t> prof_events; // pool of timing events
    struct ProfMark { int kind; size_t ev; };
    std::vector<ProfMark> prof_marks;     // launches timed and not read out yet
    size_t prof_next = 0;                 // events of prof_events in use
    // read-out kernel times not yet handed to tr_stats_get: raygen, extend, shade, shadow,
    // splat, guide, then the union of the traversal intervals (milliseconds)
    double prof_sum[7] = {0, 0, 0, 0, 0, 0, 0};
    bool prof_dirty = false;              // prof_sum holds read-outs not yet published
    cudaStream_t s() const { return user_stream ? user_stream : stream; }

    template <class T>
    T* alloc(size_t n) {
        T* p = tri::dalloc<T>(n, bytes);
        allocs.push_back(p);
        return p;
    }
    void release() {
        if (ev_snap) { cudaEventDestroy(ev_snap); ev_snap = nullptr; }
        if (ev_train) { cudaEventDestroy(ev_train); ev_train = nullptr; }
        for (cudaEvent_t e : prof_events) cudaEventDestroy(e);
        prof_events.clear();
        for (cudaEvent_t e : dep_events) cudaEventDestroy(e);
        dep_events.clear();
        if (shadow_stream) cudaStreamDestroy(shadow_stream);
        for (int k = 0; k < tri::kWaveLanes - 1; ++k) {
            if (lane_stream[k]) cudaStreamDestroy(lane_stream[k]);
            if (lane_shadow_stream[k]) cudaStreamDestroy(lane_shadow_stream[k]);
            lane_stream[k] = lane_shadow_stream[k] = nullptr;
        }
        if (light_stream) cudaStreamDestroy(light_stream);
        shadow_stream = light_stream = nullptr;
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        copy_stream = nullptr;
        if (stream) cudaStreamDestroy(stream);
        ev0 = ev1 = nullptr;
        stream = nullptr;
    }
};

namespace tri {

void ensure_wave(tr_ctx* x, uint32_t capacity);
void ensure_lane_wave(tr_ctx* x, int k);
void ensure_lane_guided(tr_ctx* x, int k);
void ensure_guided(tr_ctx* x, uint32_t capacity);
trk::Params make_params(tr_ctx* x);
trg::GuideDev guide_dev(tr_guide* g);
int* guide_err(tr_guide* g);
tr_status guide_check_err(tr_guide* g, cudaStream_t s);
// enqueues one training step of the proposal on stream s (no host synchronisation)
void train_enqueue(tr_guide* g, const uint4* x, const float* d_dirs, const float* d_weights, uint32_t n, float lr,
                   cudaStream_t s);
// trains the proposal on the pool a guided render collected (`fill` = pool_state on the device)
tr_status train_on_pool(tr_guide* g, const trk::GuideWave& gw, const uint32_t* pool_state, uint32_t pool,
                        float lr, cudaStream_t s, tr_stats& stats);

}  // namespace tri

namespace trh {
struct GpuNode;
// Figures of a device build (its nodes and leaf order stay on the device).
struct DeviceBvh {
    uint32_t nodes = 0;          // four-child nodes
    uint32_t depth = 0;          // four-child levels on the deepest path
    uint32_t stack = 0;          // traversal stack entries a ray can need
    uint32_t binary_depth = 0;
    uint32_t leaves = 0;
    double build_ms = 0.0;
};
// Binned-SAH build on the device (bvh_gpu.cu) from device-resident vertices [nv][3] and
// triangles [nt][3], collapsed to four-child nodes as build_bvh does: the nodes go to
// alloc_nodes(count), the triangle ids in leaf order to d_order [nt].  False on invalid input or
// a one-leaf scene (the host builder then builds, or reports which index or vertex is wrong).
bool build_bvh_device(const float* d_vertices, uint32_t nv, const uint32_t* d_triangles, uint32_t nt,
                      uint32_t max_leaf, cudaStream_t s, const std::function<GpuNode*(size_t)>& alloc_nodes,
                      uint32_t* d_order, DeviceBvh& out);
}  // namespace trh
