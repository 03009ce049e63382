// tr_kernels.cuh - parameters shared by the host scheduler and the wavefront kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "tr_guide.cuh"

namespace trk {

constexpr int kStack = 96;          // max traversal stack entries per thread (3 per four-child level + 1)
constexpr int kTraceBlock = 128;    // threads per traversal block
constexpr int kTraceMinBlocks = 8;  // register budget: 8 traversal blocks per SM
constexpr int kSplatBlock = 512;    // threads per splat block
constexpr int kMaxLights = 64;
constexpr int kMaxMaterials = 256;

// Scene as the kernels see it (device pointers).
struct SceneDev {
    const float4* nodes;      // 4 float4 per two-child node
    const float4* tris;       // 3 float4 per triangle, leaf order (v0.w = triangle id)
    const float4* tri_ng;     // per triangle id: geometric normal xyz, material index (bits)
    const float4* mats;       // per material: kd.rgb, kind (bits)
    const float4* mats2;      // per material: alpha, 0, 0, 0
    const float4* lights;     // 5 float4 per light: (pos, kind) (I, area) (left,0) (up,0) (normal,0)
    uint32_t num_lights;
    uint32_t medium;          // 0/1
    float sig_s[3], sig_t[3];
    float lambda;             // free-flight rate: mean extinction avg(sigma_t), or 4 / (film
                              // duration) in time-sampling mode
    float g;
    uint32_t bvh_depth;       // traversal stack entries - 1 (3 per four-child level)
    float bmin[3], binv[3];   // scene box (feature normalisation of the learned proposal)
};

constexpr uint32_t kFlagOrthoFrame = 1u;   // TR_FLAG_ORTHONORMAL_FRAME
constexpr uint32_t kFlagTimeSampling = 2u; // TR_FLAG_TIME_SAMPLING
constexpr uint32_t kFlagBidirectional = 4u; // TR_FLAG_BIDIRECTIONAL
constexpr uint32_t kBidirMaxBounces = 16u;

// Bidirectional connections (light subpaths; all null unless TR_FLAG_BIDIRECTIONAL).  Subpath
// vertices are [vertex][4][capacity] float4 records, slot-minor so a warp's loads coalesce:
// (position, delay) (geometric normal, vertex pdf) (Lambertian albedo, 0) (vertex value, 0).
struct BidirWave {
    float4* lvert;            // light subpath vertices
    float4* evert;            // eye subpath vertices
    uint8_t* nl;              // light vertices per slot
    uint8_t* ne;              // eye vertices per slot
    float4* L0;               // light subpath value (emitted intensity, times cos for a rectangle)
    uint32_t nvert;           // vertices kept per subpath: max_bounces - 1
    // connection rays of one eye depth (a shadow queue, up to nvert per slot): origin + tfar,
    // direction + (bin | bounce << 24 | kConnRay | kConnNoRecord), contribution + (slot | record << 24)
    float4* co_o;
    float4* co_d;
    float4* co_L;
    uint8_t* valid;           // [record][slot]: 1 when the connection's record was written
    uint32_t ncand;           // connection records a slot can have: max_bounces (max_bounces - 1) / 2
};
// flags in a shadow-queue entry's bin word: a connection ray (record when the segment is
// blocked, at the record index carried with the slot), and one whose sample has no record
constexpr uint32_t kConnRay = 1u << 31;
constexpr uint32_t kConnNoRecord = 1u << 30;
// state of the light subpath stream (another PCG32 state and increment than the eye walk's)
constexpr unsigned long long kLightStateSalt = 0xD1B54A32D192ED03ULL;
constexpr unsigned long long kLightSeqSalt = 0x3C6EF372FE94F82AULL;

// Guided mode state (all null when rendering without the learned proposal).
struct GuideWave {
    // [capacity][5] guided-vertex records, one per vertex whose direction waits for the
    // proposal, in queue order: (pos, time) (incoming dir, RR albedo) (throughput, material)
    // (geometric normal, slot) (RNG state, RNG increment)
    uint4* vrec;
    trg::GuideDev net;        // network weights (canonical tiles) and biases
    int* err;                 // set to 1 when a tensor-core wait times out
    float mix_prob;           // probability of sampling the proposal (else the BSDF)
    // training pool
    uint4* pool_feat;         // [pool_cap][64] bf16
    float* pool_dir;          // [pool_cap][3]
    float* pool_w;            // [pool_cap] target weight (filled by k_train_gather)
    uint4* pool_meta;         // [pool_cap] slot, depth, throughput luminance (bits), unused
    uint32_t pool_cap;
    float keep_prob;          // probability that a guided vertex becomes a training sample
    // batch tag written into pool_meta[k].w (0: untagged; the batch's entries are then the
    // pool range filled since the previous gather)
    uint32_t tag;
    // GGX vertices smoother than this roughness sample their BSDF in the shading kernel instead of
    // the proposal (glossy lobes are already sampled close to the product by the BSDF sampler)
    float min_alpha;
};

struct CameraDev {
    float pos[3], nv[3], uv[3], vv[3], fd;
};

// One contiguous slot range of one scene within a wavefront batch: pixels [0, npix) of a
// pixel list (window rows, row-major) times camera samples [s0, s0+ns) times incoming samples
// [0, ninc); slot = slot_begin + ((pixel_local * ns) + s_local) * ninc + j.
struct Batch {
    uint32_t win_x0, win_y0, win_w;     // pixel list = window rows, row-major
    uint32_t pix_begin;                 // first window-local pixel index of this segment
    uint32_t npix;
    unsigned long long s0;
    uint32_t ns, ninc;
    uint32_t n_slots;                   // slots of this segment (= of the batch in single-scene mode)
    uint32_t slot_begin;                // first slot (0 in single-scene mode)
    uint32_t scene;                     // index into MultiDev::scenes (0 in single-scene mode)
    uint32_t blk_begin;                 // first splat block of this segment
    uint32_t splat_g;                   // pixels per splat block
};

// Multi-scene rendering (tr_batch): per-scene data and the batch descriptors live in device
// memory; the kernels of one batch read descriptor *cur, so one captured CUDA graph replays
// every batch (its last node advances *cur).
constexpr int kMaxSegments = 16;
struct BatchDesc {
    uint32_t nseg, n_slots, n_blocks, max_depth;
    Batch seg[kMaxSegments];
};
struct Wave {
    float4* ray_o;            // o.xyz, tfar (sampled free-flight distance or +inf)
    float4* ray_d;            // d.xyz, accumulated time
    float4* thr;              // throughput rgb, pending pdf factor (RR prob * direction pdf)
    unsigned long long* rng;  // PCG32 state (increment derived from the camera sample)
    float4* hit;              // t, triangle id (bits), u, v
    uint32_t* q[2];           // extend queues (ping-pong)
    float4* sh_o;             // shadow: origin, tfar
    float4* sh_d;             // shadow: direction, time bin (bits)
    float4* sh_L;             // shadow: contribution rgb, slot (bits)
    float4* rec;              // splat records [bounce][capacity]: rgb, bin | depth << 24 (bits)
    float* cam_dist;          // camera-to-first-surface distance per slot (camera unwarp)
    float4* target;           // light point drawn for the path (time-sampling mode)
    uint8_t* rec_n;           // records per slot
    uint32_t* counters;       // see counter_* helpers below
    unsigned long long* stats;// closest, shadow, splats, paths (accumulated)
    uint32_t capacity;
};

struct FilmDev {
    double* streak;           // [H][W][T][3]
    double* steady;           // [H][W][3]
    double* weight;           // [H][W]
    uint32_t W, H, T;
    float exposure, offset;
    uint32_t unwarp;          // bin by path time minus the camera-to-first-surface distance
    uint32_t nbounce;         // per-bounce films (0 = none)
    double* bstreak;          // [nbounce][H][W][T][3]
    double* bsteady;          // [nbounce][H][W][3]
    double* bweight;          // [nbounce][H][W]
    uint32_t comps;           // film components (TR_COMP_* bits)
    double* cdepth;           // [H][W] camera-ray record sums
    double* cpos;             // [H][W][3]
    double* cnorm;            // [H][W][3]
    // set on the splat launch of a batch whose pixels are final (last sample chunk) when the film
    // is delivered as RGBE images: each splat block encodes its pixels once it has added them
    uchar4* rgbe_streak = nullptr;   // [H][W][T]
    uchar4* rgbe_steady = nullptr;   // [H][W]
    // the film held no samples before this render, which has one sample chunk: a splat block's
    // pixels hold only its own additions, so cells it did not add to are zero
    uint32_t rgbe_fresh = 0;
};

// bin of a radiance sample outside the time window: kept (with bounce films only) because the
// sample still counts for its bounce film's weight and for the base steady image
constexpr uint32_t kBinOutside = 0xffffffu;

struct SceneSlot {            // one scene of a multi-scene batch
    SceneDev scene;
    CameraDev cam;
    FilmDev film;
    unsigned long long seed;
    uint32_t max_bounces, sqrt_spp, flags, pad;
};

struct MultiDev {
    const SceneSlot* scenes;
    const BatchDesc* batches;
    uint32_t* cur;               // index of the batch being rendered
    uint32_t nscenes;
    // launch shapes (host side): grids cover the largest batch of the plan
    uint32_t max_splat_blocks;
    uint32_t shade_block;        // threads per shade block (128 or 256)
};

struct Params {
    SceneDev scene;
    CameraDev cam;
    FilmDev film;
    Wave wave;
    Batch batch;
    unsigned long long seed;
    uint32_t max_bounces;
    uint32_t sqrt_spp;
    uint32_t bvh_depth;
    uint32_t flags;
    GuideWave guide;
    MultiDev multi;              // used by the kMulti kernel variants only
    BidirWave bd;                // light subpaths and vertex connections
};

// ---- per-slot view (device) ------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ const BatchDesc& cur_batch(const Params& p) { return p.multi.batches[*p.multi.cur]; }

// segment holding `slot` (segments are contiguous and ordered by slot_begin)
__device__ __forceinline__ const Batch& seg_of_slot(const BatchDesc& B, uint32_t slot) {
    uint32_t lo = 0, hi = B.nseg;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (B.seg[mid].slot_begin <= slot) lo = mid; else hi = mid;
    }
    return B.seg[lo];
}
// segment owning splat block `blk`
__device__ __forceinline__ const Batch& seg_of_block(const BatchDesc& B, uint32_t blk) {
    uint32_t lo = 0, hi = B.nseg;
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (B.seg[mid].blk_begin <= blk) lo = mid; else hi = mid;
    }
    return B.seg[lo];
}
#endif

// counters layout (uint32): [0, 64) extend counts per depth, [64, 128) shadow counts per
// depth, [128, 192) extend fetch cursors, [192, 256) shadow fetch cursors, [256, 320)
// guided-vertex counts per depth; training-pool fill lives in its own counter.
constexpr int kCounters = 320;
__host__ __device__ constexpr int cnt_ext(int d) { return d; }
__host__ __device__ constexpr int cnt_sh(int d) { return 64 + d; }
__host__ __device__ constexpr int cur_ext(int d) { return 128 + d; }
__host__ __device__ constexpr int cur_sh(int d) { return 192 + d; }
__host__ __device__ constexpr int cnt_guide(int d) { return 256 + d; }

// host launchers (tr_kernels.cu)
cudaError_t launch_raygen(const Params& p, cudaStream_t s);
cudaError_t launch_extend(const Params& p, int depth, int grid, cudaStream_t s);
cudaError_t launch_shade(const Params& p, int depth, cudaStream_t s);
cudaError_t launch_shadow(const Params& p, int depth, int grid, cudaStream_t s);
// bsel < 0: the film itself; bsel = b: per-bounce film b (records of bounce min(depth, N-1) == b)
// pixels per splat block: automatic (whole pixels filling one block) in single-scene mode,
// each segment's splat_g in multi-scene mode
cudaError_t launch_splat(const Params& p, cudaStream_t s, int bsel = -1);
// per-bounce film weights: +1 per camera sample with a record of that bounce film
cudaError_t launch_bounce_weights(const Params& p, cudaStream_t s);
// bidirectional connections: light subpath generation on the light wave `pl` (its own rays,
// queues and counters; target, stats and vertex arrays shared), then the connections
cudaError_t launch_light_raygen(const Params& pl, cudaStream_t s);
cudaError_t launch_light_shade(const Params& pl, int depth, cudaStream_t s);
// connection rays of eye depth ie into the connection queue (counter cnt_sh(max_bounces + ie)),
// then, after k_shadow has traced them, the slot's connection records compacted in order
cudaError_t launch_connect_gen(const Params& p, int ie, cudaStream_t s);
cudaError_t launch_connect_compact(const Params& p, cudaStream_t s);
// Scene set-up on the device: the leaf-ordered triangle records (v0 + id, v1, v2) from the
// builder's order, and per triangle id the reference geometric normal
// normalize(cross(p2 - p0, p1 - p0)) (World.h:449) with the material index.
cudaError_t launch_build_tris(const float* vertices, const uint32_t* triangles, const uint32_t* material,
                              const uint32_t* order, uint32_t nt, float4* tris, float4* tri_ng, cudaStream_t s);
// FP64 film sums -> FP32 (film streaming)
cudaError_t launch_to_f32(const double* src, float* dst, size_t n, cudaStream_t s);

cudaError_t launch_advance(uint32_t* cur, uint32_t step, cudaStream_t s);
cudaError_t launch_trace_user(const SceneDev& sc, const float* rays, uint32_t n, int any_hit,
                              void* out_hits, uint32_t* cursor, int grid, cudaStream_t s);
// fused proposal inference + one-sample MIS direction sampling of the guided vertices of `depth`
cudaError_t launch_guide(const Params& p, int depth, uint32_t* pool_state, cudaStream_t s);
cudaError_t launch_train_gather(const Params& p, uint32_t* pool_state, cudaStream_t s);
int trace_grid_size(int device, uint32_t bvh_depth, bool multi = false);
size_t trace_smem_bytes(uint32_t bvh_depth);
uint32_t splat_pixels_per_block(uint32_t slots_per_pixel);

}  // namespace trk
