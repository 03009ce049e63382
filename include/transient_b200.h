/*
 * transient_b200.h - C ABI of the B200 transient path tracer.
 *
 * The GPU path replaces the reference renderer's CPU render call
 *   RenderEngine<D,Radiance,RadAtt>::render(name, World&, Integrator*, const Camera&,
 *                                           Film*, Sampler*)              (src/Renderer/RenderEngine.h:67-68)
 * as overridden by TransientRenderer::render                             (src/Renderer/TransientRenderer.h:76-201),
 * together with the scene set-up it depends on (World::add_triangle_mesh / add_light /
 * set_medium / freeze, src/RayTracing/World.h:209-550,695-707) and the film read-out
 * (StreakCameraFilm::write, src/Film/StreakCameraFilm.h:233-242).
 *
 * Everything is plain C: flat arrays, explicit sizes, integer status codes.  No C++
 * exception crosses this boundary; the reference's exceptions (bad mesh, missing
 * integrator) come back as TR_ERR_INVALID_ARGUMENT with a message in tr_last_error().
 * Calls on one context must be serialised by the caller (the reference renderer is
 * single-threaded and not re-entrant either: src/Utils/RandomNumbers.h:227).
 */
#ifndef TRANSIENT_B200_H
#define TRANSIENT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TR_ABI_VERSION 2

typedef enum tr_status {
    TR_OK = 0,
    TR_ERR_INVALID_ARGUMENT = 1, /* bad sizes / indices / NaN geometry / unknown kinds        */
    TR_ERR_CUDA = 2,             /* a CUDA runtime call failed (message in tr_last_error)      */
    TR_ERR_OUT_OF_MEMORY = 3,    /* film or path state does not fit in device memory           */
    TR_ERR_NOT_SUPPORTED = 4,    /* feature not available in this build                        */
    TR_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up                         */
    TR_ERR_NO_DEVICE = 6,        /* no CUDA device / wrong architecture                        */
    TR_ERR_IO = 7                /* file could not be read or written                          */
} tr_status;

/* ---- scene description (mirrors what World owns after parse_args) ---------------------- */

enum { TR_MAT_LAMBERTIAN = 0, TR_MAT_GGX = 1 };

/* Lambertian: UberMaterial holding one Lambertian(Kd)      (bunnykiller.cpp:328-337,
 *             src/Material/Reflectance/Lambertian.h:68-122)
 * GGX:        microfacet reflector, Kd = Schlick F0, alpha = GGX roughness (no reference
 *             counterpart; Walter et al. 2007 evaluation, Heitz 2018 visible-normal sampling). */
typedef struct tr_material {
    uint32_t kind;
    float kd[3];
    float alpha;
    float reserved[3];
} tr_material;

enum { TR_LIGHT_POINT = 0, TR_LIGHT_RECT = 1 };

/* Point light:  position, intensity                       (src/LightSource/PointLightSource.h:141-171)
 * Rect light:   position = corner, left/up = edge vectors already scaled by the size,
 *               normal, area; as RectangularAreaLightSource::setup builds them
 *               (src/LightSource/RectangularAreaLightSource.h:66-80,221-248). */
typedef struct tr_light {
    uint32_t kind;
    float position[3];
    float intensity[3];
    float left[3];
    float up[3];
    float normal[3];
    float area;
} tr_light;

/* Homogeneous world medium with a Henyey-Greenstein phase function
 * (src/Media/HomogeneousMedium.h:32-199, HenyeyGreensteinPhaseFunction.h:218-276). */
typedef struct tr_medium {
    uint32_t enabled;
    float sigma_a[3];
    float sigma_s[3];
    float g;
} tr_medium;

typedef struct tr_scene {
    const float* vertices;            /* [num_vertices][3]                                     */
    uint32_t num_vertices;
    const uint32_t* triangles;        /* [num_triangles][3], 0-based                           */
    uint32_t num_triangles;           /* triangle id = index here (OBJ face order per mesh)    */
    const uint32_t* triangle_material;/* [num_triangles]                                       */
    const tr_material* materials;
    uint32_t num_materials;
    const tr_light* lights;
    uint32_t num_lights;
    tr_medium medium;
} tr_scene;

/* Pinhole camera basis as PinholeCamera builds it (src/Camera/PinholeCamera.h:56-91):
 * direction(px,py) = normalize(nv*focal_distance + 2*uv*px - 2*vv*py). */
typedef struct tr_camera {
    float position[3];
    float nv[3];
    float uv[3];
    float vv[3];
    float focal_distance;
} tr_camera;

/* Streak film (src/Film/StreakCameraFilm.h:91-121): width x height pixels, time_bins bins of
 * `exposure` path-length units starting at `offset`; time_bins < 16777215 (24-bit bin field).
 * camera_unwarp ("-camera-unwarp"): bin every sample by its path time minus the distance from
 *   the camera to the first surface along its camera ray (StreakCameraFilm.h:167, World.h:749-766).
 * bounce_films ("-multibounce-streak N"): N > 0 adds N per-bounce streak films as
 *   MultibounceStreakFilm does (src/Film/MultibounceStreakCameraFilm.h:151-171): a sample of
 *   bounce b goes to film min(b, N-1); film b's weight counts the camera samples with at least
 *   one sample of that film (inside the time window or not); the context's steady image is
 *   then the base Film's, the sum of all samples (Film.h:263-284).  N <= 32.              */
typedef struct tr_film {
    uint32_t width;
    uint32_t height;
    uint32_t time_bins;
    float exposure;
    float offset;
    uint32_t camera_unwarp;
    uint32_t bounce_films;
    uint32_t components;       /* TR_COMP_* bits ("-film-depth", "-film-positions", "-film-normals") */
} tr_film;

/* Film components (FilmComponents.h; Film::add_components, Film.h:127-145): per pixel, the
 * sum over camera samples of World::Li's camera-ray record (World.h:749-766) -- the distance
 * to the closest surface at any distance (FLT_MAX when there is none), and that point's
 * position and normal (zero when none).  tr_write_film writes them averaged as
 * "<name>_depth.hdr", "<name>_positions.raw" and "<name>_normals.raw" (Film.h:357-471).    */
#define TR_COMP_DEPTH 2u
#define TR_COMP_POSITIONS 8u
#define TR_COMP_NORMALS 16u

/* Unidirectional path tracing with next-event estimation, the only mode the reference CLI runs
 * (src/Integrator/BidirectionalPathTracing.h:122-137,1099-1140; ProgramParams.h:162-164).
 * sqrt_spp strata per axis (StratifiedSampler.h:47-89), incoming_samples paths per camera
 * sample ("-bidirectional-path-tracing N"), max_bounces = "-max-nb-bounces". */
typedef struct tr_integrator {
    uint32_t max_bounces;
    uint32_t sqrt_spp;
    uint32_t incoming_samples;
    uint32_t flags;             /* TR_FLAG_* */
    uint64_t seed;
} tr_integrator;

/* Lambertian directions in an orthonormal frame around the normal.  Without the flag the
 * frame of Intersection::set_coordinate_system (src/RayTracing/Intersection.h:167-178) is
 * reproduced exactly, including its non-orthogonal branch, so results match the reference;
 * that frame's true sampling density is not cos/pi, so guided rendering (which combines
 * densities by MIS) requires this flag, as does the plain render it is compared against. */
#define TR_FLAG_ORTHONORMAL_FRAME 1u

/* Time sampling ("-time-sampling": TransientRenderer(f_log, true) ->
 * BidirectionalPathTracing::set_mode(SamplingMode::Transient),
 * src/Integrator/BidirectionalPathTracing.h:189-206).  Each path draws one light point; free
 * flights in the medium have the rate 4 / (time_bins * exposure) instead of the mean extinction;
 * walks end when their time passes the film's (no Russian roulette); medium directions come
 * from the time-angular sampler towards the light point (SamplingTechniques.h TimeAngular,
 * BidirectionalPathTracing.h:342-431), falling back to the phase function.  The reference's
 * sampler density and weights are reproduced as they are, including its rare huge weights
 * (inverted time bounds), so films match the reference's distribution, heavy tail included. */
#define TR_FLAG_TIME_SAMPLING 2u

/* Bidirectional connections: light subpaths and eye-light vertex connections
 * (BidirectionalPathTracing::set_path_tracing_only(false), reachable through the reference's
 * API; src/Integrator/BidirectionalPathTracing.h:1099-1140, :975-1045, :697-897,
 * src/Integrator/PathMIS.h:63-111).  Defined as the reference defines it: with
 * TR_FLAG_TIME_SAMPLING, in scenes without a medium, Lambertian materials, max_bounces <= 16
 * (other combinations return TR_ERR_NOT_SUPPORTED: outside time-sampling mode the reference's
 * light subpath starts from an uninitialised light sample, and in a medium its time-sampled
 * connections dereference a null medium).  Each path draws one light point, emits a light
 * subpath from it and connects every eye vertex ie with every light vertex il for
 * ie + il + 2 <= max_bounces, with the reference's MIS quantity (accumulated by addition,
 * divided by) and its visibility convention (a pair counts when the segment between the
 * vertices is blocked: World::intersects returns true on a hit and the reference connects on
 * true).  Not with the learned proposal, multi-scene batches or tr_render_region_noalloc. */
#define TR_FLAG_BIDIRECTIONAL 4u
#define TR_BIDIR_MAX_BOUNCES 16u

/* ---- ray-batch interface (correctness batch of World::first_intersection / intersects) --- */

/* One ray = 8 floats: origin xyz, tnear, direction xyz, tfar.                               */
typedef struct tr_hit {
    float t;            /* hit distance (tfar of the closest hit)                            */
    uint32_t prim_id;   /* triangle id, 0xffffffff = miss                                    */
    float u, v;         /* barycentrics: p = (1-u-v) p0 + u p1 + v p2                        */
} tr_hit;

#define TR_INVALID_ID 0xffffffffu

typedef struct tr_stats {
    uint64_t paths;            /* paths traced (camera samples x incoming samples)          */
    uint64_t camera_samples;   /* camera samples accumulated into the film                  */
    uint64_t closest_rays;     /* closest-hit queries                                        */
    uint64_t shadow_rays;      /* any-hit (shadow) queries                                   */
    uint64_t splats;           /* radiance samples landing inside the film window            */
    double   render_ms;        /* device time of the last tr_render call                     */
    double   bvh_build_ms;     /* host time of the BVH build                                 */
    uint32_t bvh_nodes;
    uint32_t bvh_depth;
    uint64_t device_bytes;     /* device memory held by the context                          */
    uint64_t kernel_launches;  /* kernels launched by the last tr_render call                */
    /* per-kernel device time of the last tr_render call (tr_set_profiling(ctx,1)) or of the
     * renders since the previous tr_stats_get (tr_set_profiling(ctx,2)),
     * measured with CUDA events around each launch on the stream it runs on.  Shadow launches
     * run on a second stream beside the next depth's closest-hit launch, so extend_ms and
     * shadow_ms overlap; trace_ms below is the time either of them was running.              */
    double   raygen_ms, extend_ms, shade_ms, shadow_ms, splat_ms;
    uint64_t extend_launches, shadow_launches;
    double   guide_ms;         /* proposal inference + guided sampling (profiling on)        */
    uint64_t train_steps;      /* proposal training steps run by the last tr_render call     */
    float    train_loss;       /* loss of the last training step                             */
    double   trace_ms;         /* union of the extend and shadow launch intervals (profiling on) */
} tr_stats;

/* ---- lifetime ----------------------------------------------------------------------------- */

typedef struct tr_ctx tr_ctx;

/* Uploads the scene, builds the BVH and allocates the streak film on `device`.
 * Replaces World::add_triangle_mesh + World::freeze and the film allocation.               */
tr_status tr_create(const tr_scene* scene, const tr_camera* camera, const tr_film* film,
                    const tr_integrator* integrator, int device, tr_ctx** out);

/* Device memory that destroyed contexts, guides and batches freed is kept by the library (one
 * memory pool per device) and reused by later ones, so creating and destroying contexts in a
 * loop does not map and unmap the film each time.  This returns the kept memory of `device`
 * to the driver (after waiting for the device); no counterpart in the reference.            */
tr_status tr_release_cached_memory(int device);

/* Renders camera samples [sample_begin, sample_begin + sample_count) of every pixel and adds
 * them to the film (the while-loop of TransientRenderer::render).  Additive: calling it for
 * [0,a) then [a,b) equals one call for [0,b).  Camera sample s uses stratum s mod sqrt_spp^2. */
tr_status tr_render(tr_ctx* ctx, uint64_t sample_begin, uint32_t sample_count);

/* As tr_render but only for the pixel window [x0,x1) x [y0,y1) (the reference's
 * -film-scanline / -film-single-pixel partial renders, bunnykiller.cpp:1770-1791).          */
tr_status tr_render_region(tr_ctx* ctx, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                           uint64_t sample_begin, uint32_t sample_count);

/* Zeroes film, steady image and weights. */
tr_status tr_clear_film(tr_ctx* ctx);

/* Copies the accumulated (not yet averaged) film to host memory; any pointer may be NULL.
 *   streak: [height][width][time_bins][3] sums of radiance per time bin
 *   steady: [height][width][3]            sums of in-window radiance (Film::m_image)
 *   weight: [height][width]               number of camera samples (Film::m_weight)
 * Dividing streak/steady by weight gives what StreakCameraFilm::average_and_save_slice writes. */
tr_status tr_get_film(tr_ctx* ctx, double* streak, double* steady, double* weight);

/* Renders like tr_render and delivers the film's accumulated sums (all samples rendered so
 * far, same layout as tr_get_film) into host memory, copying each group of pixel rows as soon
 * as its last samples are splatted, so the device-to-host transfer overlaps the rendering of
 * the remaining rows -- as the reference saves each scanline once it is done
 * (StreakCameraFilm::average_and_save_slice, StreakCameraFilm.h:356-437).  type TR_FILM_F64
 * delivers double sums; TR_FILM_F32 delivers float sums (rounded on the device; the
 * reference's film itself accumulates in float), half the bytes.  streak/steady/weight point
 * to arrays of that type (any may be NULL).  The copies overlap the rendering only when the
 * host arrays are page-locked (cudaHostAlloc / cudaHostRegister); with pageable memory the call
 * is still correct but serialises them.  Returns when the film is in host memory.
 * type TR_FILM_RGBE delivers what tr_write_film writes instead of sums: each film cell averaged
 * (sum / weight, in double, rounded to float, NaN -> 0) and RGBE-encoded on the device exactly
 * as the .hdr writer encodes it (ImageIO.h:146-193), 4 bytes per cell.  streak is
 * [height][width][time_bins][4] bytes -- for each scanline y, the pixel data of its streak
 * file "<name>_%04d.hdr" when time_bins >= 8 (that file stores rows x, columns t; with fewer
 * bins the file holds the transpose) -- and steady is [height][width][4], the pixel data of
 * "<name>.hdr"; weight must be NULL.  A third of the FP32 bytes (a twelfth of FP64).          */
enum { TR_FILM_F64 = 0, TR_FILM_F32 = 1, TR_FILM_RGBE = 2 };
tr_status tr_render_film(tr_ctx* ctx, uint64_t sample_begin, uint32_t sample_count, int type, void* streak,
                         void* steady, void* weight);

/* Same as tr_get_film but into device memory owned by the caller (no host copy).  Both copy on
 * the context's stream after its pending renders and return when the copy is complete; the
 * caller's own pending work on the destination must be finished first.                      */
tr_status tr_get_film_device(tr_ctx* ctx, double* d_streak, double* d_steady, double* d_weight);

/* Component sums (any may be NULL; the film must have the component): depth [H][W],
 * positions [H][W][3], normals [H][W][3] (double, divide by weight to average).               */
tr_status tr_get_film_components(tr_ctx* ctx, double* depth, double* positions, double* normals);

/* Per-bounce film `bounce` (< bounce_films) of the context, layouts as tr_get_film.           */
tr_status tr_get_film_bounce(tr_ctx* ctx, uint32_t bounce, double* streak, double* steady, double* weight);

/* Writes the averaged film the way the reference does: one RGBE .hdr streak image per
 * scanline "<name>_%04d.hdr" (time_bins x width) and the steady image "<name>.hdr"
 * (StreakCameraFilm.h:356-437, Film.h:357-471, ImageIO.h:146-193).  With bounce films, the
 * per-scanline streak images of film b are "<name>_b%02d_%04d.hdr" (b + 1, as
 * MultibounceStreakFilm names them) and "<name>.hdr" is the base steady image.             */
tr_status tr_write_film(tr_ctx* ctx, const char* name);

/* Closest-hit (any_hit = 0) or occlusion (any_hit = 1) queries for n host rays.
 * Closest hit: smallest t in (tnear, tfar], ties broken by the lower triangle id.
 * Occlusion: prim_id is any triangle with t in (tnear, tfar], or TR_INVALID_ID.             */
tr_status tr_trace_rays(tr_ctx* ctx, const float* rays, uint32_t n, int any_hit, tr_hit* out);

/* Same with device pointers on the caller's CUDA stream (cudaStream_t passed as void*). */
tr_status tr_trace_rays_device(tr_ctx* ctx, const float* d_rays, uint32_t n, int any_hit,
                               tr_hit* d_out, void* stream);

/* Render without allocating.  No counterpart in the reference renderer: it exists for callers
 * that cannot allocate GPU memory once their set-up is done -- for example engines whose own
 * memory pool owns the whole device and forbids foreign cudaMalloc calls, or frame loops that
 * cannot afford cudaMalloc's implicit device-wide synchronisation in the middle of a frame.
 * tr_render may grow its path buffers with cudaMalloc; this entry
 * point instead keeps the per-path state of the wavefront in one fixed array compiled into
 * the library (25.3 MiB per GPU that loads the library, held until the process exits).
 * It adds camera samples [sample_begin, sample_begin + sample_count) of the pixel window
 * [x0,x1) x [y0,y1) to the context's film, exactly as tr_render_region does, asynchronously
 * on `stream` (cudaStream_t as void*, NULL = the context's stream).
 * Limits: (x1-x0)*(y1-y0)*sample_count*incoming_samples <= TR_NOALLOC_MAX_PATHS paths per
 * call and max_bounces <= TR_NOALLOC_MAX_BOUNCES; larger requests return
 * TR_ERR_INVALID_ARGUMENT -- split the window or the sample range over several calls.
 * The array is shared by every call in the process on that GPU: calls that can overlap on
 * the GPU (different streams, or different contexts on one device) race and corrupt each
 * other's paths, so issue them on one stream.  tr_create looks the array's device address up
 * on its device (cudaGetSymbolAddress, which also loads the array there), so the calls only
 * read a cached address; should that set-up look-up have failed, the first call retries it,
 * so make the first call before any stream capture begins.  The paths, rays and splats of
 * these calls count in tr_stats_get like tr_render's (read after the call's stream has
 * finished). */
#define TR_NOALLOC_MAX_PATHS 65536u
#define TR_NOALLOC_MAX_BOUNCES 16u
tr_status tr_render_region_noalloc(tr_ctx* ctx, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                                   uint64_t sample_begin, uint32_t sample_count, void* stream);

/* ---- learned directional proposal (no counterpart in the reference renderer) -------------
 * An MLP maps a surface vertex's features (64 BF16 values: sin/cos encoded position, position,
 * normal, outgoing direction, normalised path length, zero padding) through three hidden
 * layers of 64 ReLU units to 8 von Mises-Fisher lobes (per lobe: weight logit, unnormalised
 * mean xyz, raw concentration r with kappa = 0.05 + 2000 sigmoid(r - 8)).  Forward and hidden-layer backward run as BF16
 * tcgen05 tensor-core kernels with FP32 accumulation; training minimises
 * -sum_i w_i log q(dir_i | x_i) / sum_i w_i with Adam.
 * Parameters (TR_GUIDE_PARAMS floats): weights [4][64 in][64 out], then biases [4][64]. */
#define TR_GUIDE_PARAMS 16640
#define TR_GUIDE_OUTPUTS 40
typedef struct tr_guide tr_guide;
tr_status tr_guide_create(int device, uint64_t seed, tr_guide** out);
tr_status tr_guide_set_params(tr_guide* g, const float* params);
tr_status tr_guide_get_params(tr_guide* g, float* params);
/* d_features: device [n][64] bf16 (uint16 bits); d_out: device [n][40] float. */
tr_status tr_guide_forward(tr_guide* g, const uint16_t* d_features, uint32_t n, float* d_out, void* stream);
/* One training step on device batch (features [n][64] bf16, dirs [n][3], weights [n]):
 * gradients into the guide (tr_guide_get_grads), then Adam with step size lr when lr > 0.
 * *loss (may be NULL) receives the batch loss before the update. */
tr_status tr_guide_train_step(tr_guide* g, const uint16_t* d_features, const float* d_dirs, const float* d_weights,
                              uint32_t n, float lr, float* loss, void* stream);
tr_status tr_guide_get_grads(tr_guide* g, float* grads);
/* Wait limit of the guide's tensor-core kernels: how many times a kernel polls the mbarrier of
 * its own MMAs before the wait counts as timed out (default 2^24; 0 = every wait times out at
 * once).  A timed-out kernel records the error, waits (with the full bound) for the MMAs it
 * issued, frees its tensor memory and returns; the call that launched it then returns
 * TR_ERR_TIMEOUT and the guide stays usable.  For tests and diagnostics of that path. */
tr_status tr_guide_set_wait_limit(tr_guide* g, uint32_t polls);
tr_status tr_guide_destroy(tr_guide* g);

/* Renders the context with the learned proposal: surface directions are drawn from the
 * mixture with probability mix_prob and from the BSDF otherwise, combined by one-sample MIS
 * (balance heuristic) so the film converges to the same image as without a guide.  When
 * train_pool > 0, every tr_render call collects up to train_pool (vertex, direction, weight)
 * samples from its own paths and then trains the guide on them (Adam, learning_rate, batches
 * of 65,536).  Needs TR_FLAG_ORTHONORMAL_FRAME.  guide = NULL detaches.  The guide must live
 * on the context's device and outlive its use. */
tr_status tr_set_guide(tr_ctx* ctx, tr_guide* guide, float mix_prob, float learning_rate, uint32_t train_pool);
/* Which surface vertices sample with the proposal (one-sample MIS with the BSDF): those at path
 * depth < depths on Lambertian materials and on GGX materials with roughness alpha >=
 * min_roughness; the others sample their BSDF only.  Default: every depth, min_roughness 0.5 --
 * a glossy lobe is already sampled close to the BSDF x incident-light product by the BSDF
 * sampler, so guiding it costs inference and gains little (measured on the guided workload's
 * alpha 0.2 floor: 3 ms more per 64-spp pass for 2 % less variance).  Either way the estimator is
 * unbiased. */
tr_status tr_set_guide_scope(tr_ctx* ctx, uint32_t depths, float min_roughness);

/* Counters of the context (tr_stats).  Waits for the context's stream, then reads the device
 * ray and splat counters, which every render entry point adds to. */
tr_status tr_stats_get(tr_ctx* ctx, tr_stats* out);

/* ---- multi-scene batches (no counterpart in the reference renderer) -------------------------
 * The scenes of n contexts (each keeps its own BVH, materials, lights, medium, camera,
 * integrator settings and film) are rendered together: a wavefront batch holds the path slots
 * of up to 16 scenes, and the launches of one batch (ray generation, the per-depth extend /
 * shade / [guide] / shadow kernels, splat) are captured once as a CUDA graph that is replayed
 * for every batch; the kernels read the batch being rendered from device memory.  Each scene's
 * film receives exactly the samples it would receive from tr_render on its own context (same
 * per-path random streams).  The contexts must live on one device, outlive the batch, and not
 * be rendered through their own calls while a batch call runs; contexts with bounce films
 * are rendered with tr_render (TR_ERR_NOT_SUPPORTED here). */
typedef struct tr_batch tr_batch;

typedef struct tr_batch_config {
    uint32_t capacity;       /* path slots per wavefront batch (queue size), 65,536 .. 8,388,608 */
    uint32_t shade_block;    /* threads per shade block: 128 or 256 */
    uint32_t splat_div;      /* pixels per splat block = the automatic count (whole pixels filling
                              * one 512-thread block) / splat_div (1, 2, 4, ...)                  */
    uint32_t use_graph;      /* 1: replay the batch launches from a captured CUDA graph; 0: launch directly */
} tr_batch_config;

tr_status tr_batch_create(tr_ctx* const* contexts, uint32_t n, tr_batch** out);
tr_status tr_batch_set_config(tr_batch* b, const tr_batch_config* cfg);
tr_status tr_batch_get_config(tr_batch* b, tr_batch_config* cfg);
/* Adds camera samples [sample_begin[i], sample_begin[i] + sample_count[i]) of every pixel of
 * scene i to context i's film (a count of 0 skips the scene).                               */
tr_status tr_batch_render(tr_batch* b, const uint64_t* sample_begin, const uint32_t* sample_count);
/* Project autotuner: times candidate configurations (queue capacity, shade block, pixels per
 * splat block), trial k rendering samples [sample_begin[i] + k*trial_samples[i], +trial_samples[i])
 * of scene i, keeps the fastest configuration and returns it in best.  The trial renders add
 * to the films like any render; *trials_run = number of trials.                              */
tr_status tr_batch_autotune(tr_batch* b, const uint64_t* sample_begin, const uint32_t* trial_samples,
                            tr_batch_config* best, uint32_t* trials_run);
/* As tr_set_guide, for all scenes of the batch: one network serves every scene (its features
 * carry the scene index).  Every context needs TR_FLAG_ORTHONORMAL_FRAME.                     */
tr_status tr_batch_set_guide(tr_batch* b, tr_guide* guide, float mix_prob, float learning_rate, uint32_t train_pool);
/* Counters of the batch (paths, rays, splats accumulated; render_ms, kernel_launches,
 * train_steps of the last tr_batch_render call).                                             */
tr_status tr_batch_stats(tr_batch* b, tr_stats* out);
tr_status tr_batch_destroy(tr_batch* b);

/* Runs all later work of the context on the caller's CUDA stream (cudaStream_t as void*;
 * NULL restores the context's own stream).  The stream must belong to the context's device. */
tr_status tr_set_stream(tr_ctx* ctx, void* stream);

/* Per-kernel CUDA-event timing inside tr_render: 0 off; 1 on, the times of each render read out
 * when it ends (tr_stats: the last render's); 2 on, read out at the next tr_stats_get (tr_stats:
 * the sums over the renders since the previous read, or the previous sums again when no render
 * ran since), which keeps the read-out, about 1.5 us of
 * host time per timed launch, out of the renders.                                          */
tr_status tr_set_profiling(tr_ctx* ctx, int on);
tr_status tr_destroy(tr_ctx* ctx);

const char* tr_status_string(tr_status s);
/* Thread-local message of the last failing call on this thread. */
const char* tr_last_error(void);
int tr_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* TRANSIENT_B200_H */
