/*
 * tr_oracle.h - CPU oracle for the transient path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference renderer's
 * algorithm (LeksiDor/JaraboTransientRendering, "BunnyKiller") used to check the CUDA
 * implementation.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs may load it; the product never links or calls it.
 *
 * Parity status: pinned.  The restatement is checked against the reference's own
 * integrator, sampler, camera, lights, media and streak film compiled from the reference
 * sources (oracle/ref_harness.cpp -> oracle/_ref/ref_render; statistical agreement per time
 * bin and in total energy), and its ray casting against a restatement of the reference's
 * Embree Moeller-Trumbore intersector and against the reference's own triangle test.
 *
 * The path sampling follows, step by step:
 *   camera sample        src/Sampling/StratifiedSampler.h:47-89, src/Film/Film.h:222-225,
 *                        src/Camera/PinholeCamera.h:82-91
 *   random walk          src/Integrator/BidirectionalPathTracing.h:240-307 (free flight),
 *                        :336-431 (outgoing direction), :447-481 (termination), :485-644
 *   next-event estimate  BidirectionalPathTracing.h:649-692 and :975-1045,
 *                        src/Integrator/Path.h:183-256 (scattering / attenuation),
 *                        src/LightSource/PointLightSource.h:141-171,
 *                        src/LightSource/RectangularAreaLightSource.h:221-248
 *   materials / phase    src/Material/Reflectance/Lambertian.h:68-122,
 *                        src/RayTracing/Intersection.h:167-178 (shading frame),
 *                        src/Media/PhaseFunction/HenyeyGreensteinPhaseFunction.h:218-276,
 *                        src/Media/HomogeneousMedium.h:77-80
 *   streak splat         src/Film/StreakCameraFilm.h:139-192,279-315
 *   RNG                  src/Utils/RandomNumbers.h:59-228 (PCG32)
 * with one deliberate difference: every path owns its own PCG32 stream (the reference
 * draws from one global stream), in the same draw order as the CUDA kernels, so that a
 * GPU path and an oracle path with the same id are the same random walk.
 */
#ifndef TR_ORACLE_H
#define TR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field layout as the product's C ABI structs (include/transient_b200.h), declared
 * independently so that the oracle builds without the product. */
typedef struct orc_material { uint32_t kind; float kd[3]; float alpha; float reserved[3]; } orc_material;
typedef struct orc_light {
    uint32_t kind; float position[3]; float intensity[3]; float left[3]; float up[3];
    float normal[3]; float area;
} orc_light;
typedef struct orc_medium { uint32_t enabled; float sigma_a[3]; float sigma_s[3]; float g; } orc_medium;
typedef struct orc_scene {
    const float* vertices; uint32_t num_vertices;
    const uint32_t* triangles; uint32_t num_triangles;
    const uint32_t* triangle_material;
    const orc_material* materials; uint32_t num_materials;
    const orc_light* lights; uint32_t num_lights;
    orc_medium medium;
} orc_scene;
typedef struct orc_camera { float position[3]; float nv[3]; float uv[3]; float vv[3]; float focal_distance; } orc_camera;
typedef struct orc_film {
    uint32_t width, height, time_bins; float exposure; float offset;
    uint32_t camera_unwarp;   /* bin by path time minus the camera-to-first-surface distance */
    uint32_t bounce_films;    /* N > 0: per-bounce streak films (MultibounceStreakFilm)       */
    uint32_t components;      /* FilmComponents bits: 2 depth, 8 positions, 16 normals        */
} orc_film;
typedef struct orc_integrator { uint32_t max_bounces, sqrt_spp, incoming_samples, flags; uint64_t seed; } orc_integrator;
#define ORC_FLAG_ORTHONORMAL_FRAME 1u
#define ORC_FLAG_TIME_SAMPLING 2u      /* "-time-sampling": BidirectionalPathTracing SamplingMode::Transient */
#define ORC_FLAG_BIDIRECTIONAL 4u      /* light subpaths + vertex connections (set_path_tracing_only(false));
                                          with ORC_FLAG_TIME_SAMPLING, scenes without a medium */
#define ORC_BIDIR_MAX_BOUNCES 16u
typedef struct orc_hit { float t; uint32_t prim_id; float u, v; } orc_hit;

typedef struct orc_ctx orc_ctx;

int  orc_create(const orc_scene* s, const orc_camera* c, const orc_film* f, const orc_integrator* it,
                orc_ctx** out);
void orc_destroy(orc_ctx* ctx);

/* Canonical binary SAH BVH statistics (16 bins, <= 4 triangles per leaf). */
void orc_bvh_info(const orc_ctx* ctx, uint32_t* nodes, uint32_t* leaves, uint32_t* depth);

/* Watertight closest-hit / occlusion queries (rays: 8 floats each, o tnear d tfar).
 * node_visits / tri_tests (may be NULL) receive per-ray counts on the canonical BVH. */
void orc_trace(const orc_ctx* ctx, const float* rays, uint32_t n, int any_hit, orc_hit* out,
               uint32_t* node_visits, uint32_t* tri_tests);

/* Closest hit with the reference's Embree Moeller-Trumbore test restated
 * (kernels/geometry/triangle_intersector_moeller.h:66-104, t = T * rcp(absDen) with one
 * Newton step as in common/simd/vfloat8_avx.h:242-254). */
void orc_trace_moller(const orc_ctx* ctx, const float* rays, uint32_t n, orc_hit* out);
/* Embree's Moeller terms (T, |den|, U, V) of ray i against triangle ids[i]. */
void orc_moller_terms(const orc_ctx* ctx, const float* rays, const uint32_t* ids, uint32_t n,
                      float* T, float* absden, float* U, float* V);

/* Renders camera samples [sample_begin, sample_begin+sample_count) of the pixel window and
 * ADDS them into full-frame buffers (any may be NULL):
 *   streak [H][W][T][3], steady [H][W][3], weight [H][W]  (double).
 * stats (may be NULL, else 8 values) receives {paths, closest_rays, shadow_rays, splats,
 * closest node visits, closest triangle tests, shadow node visits, shadow triangle tests}
 * where visits/tests count the work of each query on the canonical binary SAH BVH.      */
int orc_render(const orc_ctx* ctx, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
               uint64_t sample_begin, uint32_t sample_count, int nthreads,
               double* streak, double* steady, double* weight, uint64_t* stats);

/* As orc_render, plus the per-bounce films of a film with bounce_films = N > 0 (any may be
 * NULL): bstreak [N][H][W][T][3], bsteady [N][H][W][3], bweight [N][H][W], following
 * MultibounceStreakFilm::add_samples (src/Film/MultibounceStreakCameraFilm.h:151-171): a
 * radiance sample of bounce b goes to film min(b, N-1); bounce film b's weight counts the camera
 * samples with at least one sample of that film (inside the time window or not).  With N > 0
 * the main steady image is the base Film's (Film.h:263-284): every sample, also those outside
 * the time window.                                                                              */
int orc_render_bounces(const orc_ctx* ctx, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                       uint64_t sample_begin, uint32_t sample_count, int nthreads,
                       double* streak, double* steady, double* weight,
                       double* bstreak, double* bsteady, double* bweight, uint64_t* stats);

/* As orc_render_bounces, plus the film components of Film::add_components (Film.h:127-145)
 * summed per camera sample (any may be NULL): depth [H][W] = distance to the closest surface
 * along the camera ray (FLT_MAX when none), positions [H][W][3] and normals [H][W][3] of that
 * surface point (zero when none) -- World::Li's record (World.h:749-766).                     */
int orc_render_ex(const orc_ctx* ctx, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                  uint64_t sample_begin, uint32_t sample_count, int nthreads,
                  double* streak, double* steady, double* weight,
                  double* bstreak, double* bsteady, double* bweight,
                  double* depth, double* positions, double* normals, uint64_t* stats);

/* One path's splat records, for per-path comparisons: returns the number of records
 * (<= cap) of path (pixel x, y, camera sample s, incoming sample j). */
int orc_path_records(const orc_ctx* ctx, uint32_t x, uint32_t y, uint64_t s, uint32_t j,
                     uint32_t* bins, float* rgb, int cap);

/* GGX material kernels (unit tests): one visible-normal sample (weight = f cos / pdf per
 * channel) and the evaluation f(wo, wi) * max(0, n.wi).  Return 0 when no direction results. */
int  orc_ggx_sample(const float* kd, float alpha, const float* n, const float* wo, float x1, float x2,
                    float* wi, float* weight, float* pdf);
void orc_ggx_eval_cos(const float* kd, float alpha, const float* n, const float* wo, const float* wi, float* out);

/* The math kernels shared by the oracle and the CUDA path, exposed for unit tests. */
/* Henyey-Greenstein phase function (unit tests): density of a cosine, and the cosine the
 * inverse-CDF sampler returns for a uniform number x. */
float orc_hg_eval(float g, float cs);
float orc_hg_sample_cos(float g, float x);

float orc_log(float x);
float orc_exp(float x);
void  orc_sincos2pi(float xi, float* s, float* c);
uint32_t orc_pcg32_first(uint64_t state, uint64_t seq, uint32_t k);   /* k-th output */

#ifdef __cplusplus
}
#endif
#endif
