/*
 * tr_oracle.c - CPU oracle (test infrastructure) for the transient path-tracing hot path.
 * See tr_oracle.h for what it restates and why.  Build: oracle/Makefile, with
 * -ffp-contract=off so that every a*b+c rounds twice exactly like the CUDA kernels, which
 * are compiled with -fmad=false and use explicit fmaf where a fused operation is meant.
 */
#include "tr_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

#define SIGMA_VIS 1e-5f            /* _SIGMA_VISIBILITY_, src/bunnykiller.h:76-78 */
#define INV_PI_F 0.318309873f
#define INV_2PI_F 0.159154943f
#define INV_4PI_F 0.0795774683f
#define LIGHT_STATE_SALT 0xD1B54A32D192ED03ULL
#define LIGHT_SEQ_SALT 0x3C6EF372FE94F82AULL
#define MAX_STACK 128

typedef struct { float x, y, z; } v3;
static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 muls(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 mulv(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 divs(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
static inline float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 normalize(v3 a) { return divs(a, sqrtf(dot(a, a))); }
static inline float avg3(v3 a) { return ((a.x + a.y) + a.z) / 3.0f; }
static inline float comp(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
static inline v3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

/* ------------------------------------------------------------------------------------------
 * Math kernels.  Written from the mathematics so that the CPU and the GPU evaluate the very
 * same sequence of correctly rounded operations:
 *   log: Cody-Waite split of ln 2, mantissa reduced to [sqrt(1/2), sqrt(2)), then
 *        log m = 2 atanh s, s = (m-1)/(m+1), atanh series to s^11;
 *   exp: Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, Taylor series to r^7, 2^k by
 *        exponent construction;
 *   sincos(2 pi xi): exact quadrant reduction on xi (xi*4 - rint(xi*4)), Taylor series of
 *        sin to a^9 and cos to a^10 on |a| <= pi/4.
 * ---------------------------------------------------------------------------------------- */
#define LN2_HI 0.693145751953125f
#define LN2_LO 1.42860677e-06f
#define INV_LN2 1.44269502f
#define PI_2_F 1.57079637f

static inline float as_f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t as_u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

float orc_log(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    int e = 0;
    uint32_t b = as_u(x);
    if ((b >> 23) == 0) { x = x * 8388608.0f; b = as_u(x); e = -23; }
    e += (int)((b >> 23) & 0xffu) - 127;
    float m = as_f((b & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float p = fmaf(z, 0.0909090936f, 0.111111112f);
    p = fmaf(z, p, 0.142857149f);
    p = fmaf(z, p, 0.200000003f);
    p = fmaf(z, p, 0.333333343f);
    float s2 = s + s;
    float r = fmaf(s2 * z, p, s2);
    float fe = (float)e;
    return fmaf(fe, LN2_HI, fmaf(fe, LN2_LO, r));
}

float orc_exp(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return INFINITY;
    if (x < -103.972076f) return 0.0f;
    float k = rintf(x * INV_LN2);
    float r = fmaf(-k, LN2_HI, x);
    r = fmaf(-k, LN2_LO, r);
    float p = fmaf(r, 0.000198412701f, 0.00138888892f);
    p = fmaf(r, p, 0.00833333377f);
    p = fmaf(r, p, 0.0416666679f);
    p = fmaf(r, p, 0.166666672f);
    p = fmaf(r, p, 0.5f);
    p = fmaf(r, p, 1.0f);
    p = fmaf(r, p, 1.0f);
    int ki = (int)k;
    if (ki > 127) return (p * as_f(254u << 23)) * as_f((uint32_t)(ki - 127 + 127) << 23);
    if (ki < -126) return (p * as_f((uint32_t)(ki + 100 + 127) << 23)) * as_f((uint32_t)(-100 + 127) << 23);
    return p * as_f((uint32_t)(ki + 127) << 23);
}

void orc_sincos2pi(float xi, float* s, float* c) {
    float u = xi * 4.0f;
    float q = rintf(u);
    float r = u - q;
    float a = r * PI_2_F;
    float z = a * a;
    float ps = fmaf(z, 2.75573188e-06f, -0.000198412701f);
    ps = fmaf(z, ps, 0.00833333377f);
    ps = fmaf(z, ps, -0.166666672f);
    float sa = fmaf(a * z, ps, a);
    float pc = fmaf(z, -2.75573200e-07f, 2.48015876e-05f);
    pc = fmaf(z, pc, -0.00138888892f);
    pc = fmaf(z, pc, 0.0416666679f);
    pc = fmaf(z, pc, -0.5f);
    float ca = fmaf(z, pc, 1.0f);
    switch (((int)q) & 3) {
        case 0: *s = sa; *c = ca; break;
        case 1: *s = ca; *c = -sa; break;
        case 2: *s = -sa; *c = -ca; break;
        default: *s = -ca; *c = sa; break;
    }
}

/* ------------------------------------------------------------------------------------------
 * PCG32 (src/Utils/RandomNumbers.h:119-128 next_int, :83-98 next_float, :167-174 seed).
 * ---------------------------------------------------------------------------------------- */
typedef struct { uint64_t state, inc; } pcg;
static inline uint32_t pcg_next(pcg* r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}
static inline void pcg_seed(pcg* r, uint64_t state, uint64_t seq) {
    r->state = 0u;
    r->inc = (seq << 1u) | 1u;
    pcg_next(r);
    r->state += state;
    pcg_next(r);
}
static inline float pcg_float(pcg* r) { return as_f((pcg_next(r) >> 9) | 0x3f800000u) - 1.0f; }

uint32_t orc_pcg32_first(uint64_t state, uint64_t seq, uint32_t k) {
    pcg r;
    pcg_seed(&r, state, seq);
    uint32_t v = 0;
    for (uint32_t i = 0; i <= k; ++i) v = pcg_next(&r);
    return v;
}

/* Stream assignment shared with the CUDA kernels: camera sample c = (pixel << 32) | s. */
#define GOLDEN64 0x9E3779B97F4A7C15ULL
static inline uint64_t cam_id(uint32_t pixel, uint64_t s) { return ((uint64_t)pixel << 32) | (s & 0xffffffffULL); }

/* ------------------------------------------------------------------------------------------
 * Canonical binary SAH BVH: 16 centroid bins, split until <= 4 triangles per leaf.
 * ---------------------------------------------------------------------------------------- */
typedef struct { float lo[3], hi[3]; } aabb;
typedef struct { aabb box; int32_t left, right; uint32_t first, count; } bnode;

struct orc_ctx {
    uint32_t nt, nm, nl;
    v3* p0; v3* p1; v3* p2;     /* triangle vertices by triangle id */
    v3* ng;                     /* reference geometric normal */
    uint32_t* mat;
    orc_material* mats;
    orc_light* lights;
    orc_medium med;
    orc_camera cam;
    orc_film film;
    orc_integrator integ;
    bnode* nodes; uint32_t nnodes, nleaves, depth;
    uint32_t* order;            /* triangle ids in leaf order */
};

static inline void box_empty(aabb* b) {
    for (int k = 0; k < 3; ++k) { b->lo[k] = FLT_MAX; b->hi[k] = -FLT_MAX; }
}
static inline void box_grow(aabb* b, const aabb* o) {
    for (int k = 0; k < 3; ++k) {
        if (o->lo[k] < b->lo[k]) b->lo[k] = o->lo[k];
        if (o->hi[k] > b->hi[k]) b->hi[k] = o->hi[k];
    }
}
static inline float box_area(const aabb* b) {
    float dx = b->hi[0] - b->lo[0], dy = b->hi[1] - b->lo[1], dz = b->hi[2] - b->lo[2];
    if (dx < 0) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

typedef struct { aabb* tb; float* cen; uint32_t* idx; bnode* nodes; uint32_t n; } bld;

static uint32_t build_rec(bld* B, uint32_t first, uint32_t count, uint32_t depth, uint32_t* maxd) {
    uint32_t me = B->n++;
    bnode* nd = &B->nodes[me];
    box_empty(&nd->box);
    aabb cb; box_empty(&cb);
    for (uint32_t i = first; i < first + count; ++i) {
        uint32_t t = B->idx[i];
        box_grow(&nd->box, &B->tb[t]);
        aabb c = {{B->cen[3 * t], B->cen[3 * t + 1], B->cen[3 * t + 2]},
                  {B->cen[3 * t], B->cen[3 * t + 1], B->cen[3 * t + 2]}};
        box_grow(&cb, &c);
    }
    if (depth > *maxd) *maxd = depth;
    if (count <= 4) {
        nd->left = nd->right = -1; nd->first = first; nd->count = count;
        return me;
    }
    float best = FLT_MAX; int bax = -1, bsplit = -1;
    for (int ax = 0; ax < 3; ++ax) {
        float ext = cb.hi[ax] - cb.lo[ax];
        if (!(ext > 0.0f)) continue;
        aabb bb[16]; uint32_t bc[16];
        for (int b = 0; b < 16; ++b) { box_empty(&bb[b]); bc[b] = 0; }
        for (uint32_t i = first; i < first + count; ++i) {
            uint32_t t = B->idx[i];
            int b = (int)((B->cen[3 * t + ax] - cb.lo[ax]) / ext * 16.0f);
            if (b > 15) b = 15;
            if (b < 0) b = 0;
            box_grow(&bb[b], &B->tb[t]); bc[b]++;
        }
        float ra[16]; uint32_t rc[16]; aabb acc; box_empty(&acc); uint32_t n = 0;
        for (int b = 15; b > 0; --b) { box_grow(&acc, &bb[b]); n += bc[b]; ra[b] = box_area(&acc); rc[b] = n; }
        box_empty(&acc); n = 0;
        for (int b = 0; b < 15; ++b) {
            box_grow(&acc, &bb[b]); n += bc[b];
            if (n == 0 || rc[b + 1] == 0) continue;
            float cost = box_area(&acc) * (float)n + ra[b + 1] * (float)rc[b + 1];
            if (cost < best) { best = cost; bax = ax; bsplit = b; }
        }
    }
    uint32_t mid;
    if (bax < 0) {
        mid = first + count / 2;
    } else {
        float ext = cb.hi[bax] - cb.lo[bax];
        uint32_t i = first, j = first + count;
        while (i < j) {
            uint32_t t = B->idx[i];
            int b = (int)((B->cen[3 * t + bax] - cb.lo[bax]) / ext * 16.0f);
            if (b > 15) b = 15;
            if (b < 0) b = 0;
            if (b <= bsplit) { ++i; } else { --j; uint32_t tmp = B->idx[i]; B->idx[i] = B->idx[j]; B->idx[j] = tmp; }
        }
        mid = i;
        if (mid == first || mid == first + count) mid = first + count / 2;
    }
    int32_t l = (int32_t)build_rec(B, first, mid - first, depth + 1, maxd);
    int32_t r = (int32_t)build_rec(B, mid, first + count - mid, depth + 1, maxd);
    nd = &B->nodes[me];
    nd->left = l; nd->right = r; nd->first = 0; nd->count = 0;
    return me;
}

int orc_create(const orc_scene* s, const orc_camera* c, const orc_film* f, const orc_integrator* it,
               orc_ctx** out) {
    if (!s || !c || !f || !it || !out || s->num_triangles == 0 || s->num_lights == 0) return 1;
    if (it->flags & ORC_FLAG_BIDIRECTIONAL) {
        /* the well-defined part of the reference: time-sampling mode, no medium, Lambertian
         * surfaces, at most 16 bounces (see bidirectional connections below) */
        if (!(it->flags & ORC_FLAG_TIME_SAMPLING) || s->medium.enabled || it->max_bounces > ORC_BIDIR_MAX_BOUNCES)
            return 1;
        for (uint32_t m = 0; m < s->num_materials; ++m)
            if (s->materials[m].kind != 0) return 1;
    }
    orc_ctx* x = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    uint32_t nt = s->num_triangles;
    x->nt = nt; x->nm = s->num_materials; x->nl = s->num_lights;
    x->p0 = (v3*)malloc(sizeof(v3) * nt); x->p1 = (v3*)malloc(sizeof(v3) * nt);
    x->p2 = (v3*)malloc(sizeof(v3) * nt); x->ng = (v3*)malloc(sizeof(v3) * nt);
    x->mat = (uint32_t*)malloc(sizeof(uint32_t) * nt);
    x->mats = (orc_material*)malloc(sizeof(orc_material) * (s->num_materials ? s->num_materials : 1));
    x->lights = (orc_light*)malloc(sizeof(orc_light) * s->num_lights);
    memcpy(x->mats, s->materials, sizeof(orc_material) * s->num_materials);
    memcpy(x->lights, s->lights, sizeof(orc_light) * s->num_lights);
    x->med = s->medium; x->cam = *c; x->film = *f; x->integ = *it;
    aabb* tb = (aabb*)malloc(sizeof(aabb) * nt);
    float* cen = (float*)malloc(sizeof(float) * 3 * nt);
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t* tri = &s->triangles[3 * t];
        v3 a = ld3(&s->vertices[3 * tri[0]]), b = ld3(&s->vertices[3 * tri[1]]), cc = ld3(&s->vertices[3 * tri[2]]);
        x->p0[t] = a; x->p1[t] = b; x->p2[t] = cc;
        /* World.h:449: ng = cross(p2 - p0, p1 - p0).normalized() */
        x->ng[t] = normalize(cross(sub(cc, a), sub(b, a)));
        x->mat[t] = s->triangle_material[t];
        for (int k = 0; k < 3; ++k) {
            float va = comp(a, k), vb = comp(b, k), vc = comp(cc, k);
            tb[t].lo[k] = fminf(va, fminf(vb, vc));
            tb[t].hi[k] = fmaxf(va, fmaxf(vb, vc));
            cen[3 * t + k] = 0.5f * (tb[t].lo[k] + tb[t].hi[k]);
        }
    }
    bld B;
    B.tb = tb; B.cen = cen; B.idx = (uint32_t*)malloc(sizeof(uint32_t) * nt);
    for (uint32_t t = 0; t < nt; ++t) B.idx[t] = t;
    B.nodes = (bnode*)malloc(sizeof(bnode) * (2 * nt + 1)); B.n = 0;
    uint32_t maxd = 0;
    build_rec(&B, 0, nt, 0, &maxd);
    /* one ulp outward so that a ray lying in a face plane (zero direction component, origin
       on the face) still sees a non-empty slab interval */
    for (uint32_t i = 0; i < B.n; ++i)
        for (int k = 0; k < 3; ++k) {
            B.nodes[i].box.lo[k] = nextafterf(B.nodes[i].box.lo[k], -INFINITY);
            B.nodes[i].box.hi[k] = nextafterf(B.nodes[i].box.hi[k], INFINITY);
        }
    x->nodes = B.nodes; x->nnodes = B.n; x->order = B.idx; x->depth = maxd;
    x->nleaves = 0;
    for (uint32_t i = 0; i < B.n; ++i) if (B.nodes[i].left < 0) x->nleaves++;
    free(tb); free(cen);
    *out = x;
    return 0;
}

void orc_destroy(orc_ctx* x) {
    if (!x) return;
    free(x->p0); free(x->p1); free(x->p2); free(x->ng); free(x->mat); free(x->mats);
    free(x->lights); free(x->nodes); free(x->order); free(x);
}

void orc_bvh_info(const orc_ctx* x, uint32_t* nodes, uint32_t* leaves, uint32_t* depth) {
    if (nodes) *nodes = x->nnodes - x->nleaves;   /* interior nodes = 64-byte two-child records */
    if (leaves) *leaves = x->nleaves;
    if (depth) *depth = x->depth;
}

/* ------------------------------------------------------------------------------------------
 * Watertight ray/triangle test (Woop, Benthin, Wald, "Watertight Ray/Triangle
 * Intersection", JCGT 2(1), 2013) with a fixed operation order shared with the CUDA kernel.
 * ---------------------------------------------------------------------------------------- */
typedef struct {
    v3 o, d; float tnear, tfar;
    int kx, ky, kz; float Sx, Sy, Sz;
    v3 inv;   /* conservative box-test reciprocals */
} wray;

static inline void wray_setup(wray* r, v3 o, v3 d, float tnear, float tfar) {
    r->o = o; r->d = d; r->tnear = tnear; r->tfar = tfar;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0; float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) { kz = 2; }
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (comp(d, kz) < 0.0f) { int t = kx; kx = ky; ky = t; }
    r->kx = kx; r->ky = ky; r->kz = kz;
    float dz = comp(d, kz);
    r->Sx = comp(d, kx) / dz; r->Sy = comp(d, ky) / dz; r->Sz = 1.0f / dz;
    float e = 1e-30f;
    r->inv = mk(1.0f / (fabsf(d.x) > e ? d.x : copysignf(e, d.x)),
                1.0f / (fabsf(d.y) > e ? d.y : copysignf(e, d.y)),
                1.0f / (fabsf(d.z) > e ? d.z : copysignf(e, d.z)));
}

/* returns 1 and fills t,u,v when the triangle is hit with t in (tnear, tfar] */
static inline int wt_hit(const wray* r, v3 p0, v3 p1, v3 p2, float tfar, float* t, float* u, float* v) {
    v3 A = sub(p0, r->o), B = sub(p1, r->o), C = sub(p2, r->o);
    float Akz = comp(A, r->kz), Bkz = comp(B, r->kz), Ckz = comp(C, r->kz);
    float Ax = fmaf(-r->Sx, Akz, comp(A, r->kx)), Ay = fmaf(-r->Sy, Akz, comp(A, r->ky));
    float Bx = fmaf(-r->Sx, Bkz, comp(B, r->kx)), By = fmaf(-r->Sy, Bkz, comp(B, r->ky));
    float Cx = fmaf(-r->Sx, Ckz, comp(C, r->kx)), Cy = fmaf(-r->Sy, Ckz, comp(C, r->ky));
    float U = fmaf(Cx, By, -(Cy * Bx));
    float V = fmaf(Ax, Cy, -(Ay * Cx));
    float W = fmaf(Bx, Ay, -(By * Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
    float det = (U + V) + W;
    if (det == 0.0f) return 0;
    /* distance from the plane equation with Embree's fused dot/cross
       (common/math/vec3.h:193-198): Ng = e1 x e2, e1 = p0 - p1, e2 = p2 - p0 */
    v3 e1 = sub(p0, p1), e2 = sub(p2, p0);
    v3 Ng = mk(fmaf(e1.y, e2.z, -(e1.z * e2.y)), fmaf(e1.z, e2.x, -(e1.x * e2.z)), fmaf(e1.x, e2.y, -(e1.y * e2.x)));
    float den = fmaf(Ng.x, r->d.x, fmaf(Ng.y, r->d.y, Ng.z * r->d.z));
    float T = fmaf(Ng.x, A.x, fmaf(Ng.y, A.y, Ng.z * A.z));
    float tt = T / den;
    if (!(tt > r->tnear && tt <= tfar)) return 0;
    *t = tt; *u = V / det; *v = W / det;
    return 1;
}

/* Conservative slab test (Ize, "Robust BVH Ray Traversal", JCGT 2(2), 2013: tmax*(1+2*gamma3)). */
static inline int box_hit(const wray* r, const aabb* b, float tfar, float* tent) {
    float t0x = (b->lo[0] - r->o.x) * r->inv.x, t1x = (b->hi[0] - r->o.x) * r->inv.x;
    float t0y = (b->lo[1] - r->o.y) * r->inv.y, t1y = (b->hi[1] - r->o.y) * r->inv.y;
    float t0z = (b->lo[2] - r->o.z) * r->inv.z, t1z = (b->hi[2] - r->o.z) * r->inv.z;
    float tmin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), r->tnear));
    float tmax = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), tfar));
    tmax *= 1.00000036f;
    *tent = tmin;
    return tmin <= tmax;
}

/* closest hit: smallest t, ties -> lower triangle id; any_hit: first found */
static int trace1(const orc_ctx* x, const wray* r, int any_hit, orc_hit* h, uint32_t* nv, uint32_t* nt) {
    float best = r->tfar; uint32_t bid = 0xffffffffu; float bu = 0, bv = 0;
    uint32_t stack[MAX_STACK]; int sp = 0;
    uint32_t visits = 0, tests = 0;
    uint32_t cur = 0;
    float te;
    if (!box_hit(r, &x->nodes[0].box, best, &te)) goto done;
    for (;;) {
        const bnode* nd = &x->nodes[cur];
        if (nd->left < 0) {
            for (uint32_t i = nd->first; i < nd->first + nd->count; ++i) {
                uint32_t id = x->order[i];
                float t, u, v;
                ++tests;
                if (wt_hit(r, x->p0[id], x->p1[id], x->p2[id], best, &t, &u, &v)) {
                    if (t < best || bid == 0xffffffffu || (t == best && id < bid)) {
                        best = t; bid = id; bu = u; bv = v;
                        if (any_hit) goto done;
                    }
                }
            }
        } else {
            ++visits;
            float tl, tr;
            int hl = box_hit(r, &x->nodes[nd->left].box, best, &tl);
            int hr = box_hit(r, &x->nodes[nd->right].box, best, &tr);
            if (hl && hr) {
                uint32_t nearc = (uint32_t)(tl <= tr ? nd->left : nd->right);
                uint32_t farc = (uint32_t)(tl <= tr ? nd->right : nd->left);
                if (sp < MAX_STACK) stack[sp++] = farc;
                cur = nearc;
                continue;
            } else if (hl) { cur = (uint32_t)nd->left; continue; }
            else if (hr) { cur = (uint32_t)nd->right; continue; }
        }
        if (sp == 0) break;
        cur = stack[--sp];
    }
done:
    h->t = best; h->prim_id = bid; h->u = bu; h->v = bv;
    if (bid == 0xffffffffu) h->t = r->tfar;
    if (nv) *nv = visits;
    if (nt) *nt = tests;
    return bid != 0xffffffffu;
}

void orc_trace(const orc_ctx* x, const float* rays, uint32_t n, int any_hit, orc_hit* out,
               uint32_t* node_visits, uint32_t* tri_tests) {
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = &rays[8 * i];
        wray r;
        wray_setup(&r, mk(q[0], q[1], q[2]), mk(q[4], q[5], q[6]), q[3], q[7]);
        trace1(x, &r, any_hit, &out[i], node_visits ? &node_visits[i] : NULL, tri_tests ? &tri_tests[i] : NULL);
    }
}

/* ---- Embree Moeller-Trumbore restated (kernels/geometry/triangle_intersector_moeller.h) --- */
/* Embree's fused vector ops (common/math/vec3.h:193,198; madd/msub = fused multiply-add/sub) */
static inline float fdot(v3 a, v3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
static inline v3 fcross(v3 a, v3 b) {
    return mk(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}
static inline float rcp_nr(float a) {
#if defined(__x86_64__)
    float r = _mm_cvtss_f32(_mm_rcp_ss(_mm_set_ss(a)));
    return r * fmaf(-r, a, 2.0f);           /* AVX2 path: r * fnmadd(r, a, 2) */
#else
    return 1.0f / a;
#endif
}

void orc_trace_moller(const orc_ctx* x, const float* rays, uint32_t n, orc_hit* out) {
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = &rays[8 * i];
        wray r;
        wray_setup(&r, mk(q[0], q[1], q[2]), mk(q[4], q[5], q[6]), q[3], q[7]);
        float best = q[7]; uint32_t bid = 0xffffffffu; float bu = 0, bv = 0;
        uint32_t stack[MAX_STACK]; int sp = 0; uint32_t cur = 0; float te;
        if (box_hit(&r, &x->nodes[0].box, 3.4e38f, &te)) for (;;) {
            const bnode* nd = &x->nodes[cur];
            if (nd->left < 0) {
                for (uint32_t k = nd->first; k < nd->first + nd->count; ++k) {
                    uint32_t id = x->order[k];
                    /* Triangle4: v0, e1 = v0 - v1, e2 = v2 - v0, Ng = cross(e1, e2) (triangle.h:52,162-163) */
                    v3 v0 = x->p0[id];
                    v3 e1 = sub(v0, x->p1[id]), e2 = sub(x->p2[id], v0);
                    v3 Ng = fcross(e1, e2);
                    v3 C = sub(v0, r.o);
                    v3 R = fcross(r.d, C);
                    float den = fdot(Ng, r.d);
                    float absDen = fabsf(den);
                    uint32_t sgn = as_u(den) & 0x80000000u;
                    float U = as_f(as_u(fdot(R, e2)) ^ sgn);
                    float V = as_f(as_u(fdot(R, e1)) ^ sgn);
                    if (!(den != 0.0f && U >= 0.0f && V >= 0.0f && U + V <= absDen)) continue;
                    float T = as_f(as_u(fdot(Ng, C)) ^ sgn);
                    if (!(absDen * r.tnear < T && T <= absDen * best)) continue;
                    float rc = rcp_nr(absDen);
                    float t = T * rc;
                    if (t < best || (t == best && id < bid)) { best = t; bid = id; bu = U * rc; bv = V * rc; }
                }
            } else {
                float tl, tr;
                int hl = box_hit(&r, &x->nodes[nd->left].box, best, &tl);
                int hr = box_hit(&r, &x->nodes[nd->right].box, best, &tr);
                if (hl && hr) {
                    if (sp < MAX_STACK) stack[sp++] = (uint32_t)(tl <= tr ? nd->right : nd->left);
                    cur = (uint32_t)(tl <= tr ? nd->left : nd->right); continue;
                } else if (hl) { cur = (uint32_t)nd->left; continue; }
                else if (hr) { cur = (uint32_t)nd->right; continue; }
            }
            if (sp == 0) break;
            cur = stack[--sp];
        }
        out[i].t = bid == 0xffffffffu ? q[7] : best; out[i].prim_id = bid; out[i].u = bu; out[i].v = bv;
    }
}

/* Embree's Moeller-Trumbore terms for ray i against triangle ids[i] (same operations as the
 * leaf loop above, triangle_intersector_moeller.h:66-104): the unnormalised distance T, |den|
 * and the edge terms U, V, so that a caller can form the exact quotients T/|den| etc. and
 * bound the reference's Newton-refined reciprocal against them.  ids[i] = ~0u gives zeros. */
void orc_moller_terms(const orc_ctx* x, const float* rays, const uint32_t* ids, uint32_t n,
                      float* T_out, float* absden_out, float* U_out, float* V_out) {
    for (uint32_t i = 0; i < n; ++i) {
        const float* q = &rays[8 * i];
        const uint32_t id = ids[i];
        T_out[i] = absden_out[i] = U_out[i] = V_out[i] = 0.0f;
        if (id >= x->nt) continue;
        v3 o = mk(q[0], q[1], q[2]), d = mk(q[4], q[5], q[6]);
        v3 v0 = x->p0[id];
        v3 e1 = sub(v0, x->p1[id]), e2 = sub(x->p2[id], v0);
        v3 Ng = fcross(e1, e2);
        v3 C = sub(v0, o);
        v3 R = fcross(d, C);
        float den = fdot(Ng, d);
        uint32_t sgn = as_u(den) & 0x80000000u;
        T_out[i] = as_f(as_u(fdot(Ng, C)) ^ sgn);
        absden_out[i] = fabsf(den);
        U_out[i] = as_f(as_u(fdot(R, e2)) ^ sgn);
        V_out[i] = as_f(as_u(fdot(R, e1)) ^ sgn);
    }
}

/* ------------------------------------------------------------------------------------------
 * The transient path tracer.
 * ---------------------------------------------------------------------------------------- */
/* bin = BIN_OUTSIDE for a sample outside the time window (kept only for bounce films) */
#define BIN_OUTSIDE 0xffffffu
typedef struct { uint32_t bin; uint32_t depth; float L[3]; } srec;

typedef struct {
    uint64_t closest, shadow, splats;
    uint64_t c_nodes, c_tris, s_nodes, s_tris;   /* canonical-BVH work of the queries */
} pstats;

static inline float hg_eval(float g, float cs) {
    /* (1 - g^2) / (4 pi (1 + g^2 - 2 g cos)^1.5), HenyeyGreensteinPhaseFunction.h:254-276 */
    float gg = g * g;
    float b = (1.0f + gg) - (2.0f * g) * cs;
    return ((1.0f - gg) * INV_4PI_F) / (b * sqrtf(b));
}

/* cosine to the propagation direction of an HG sample by the inverse CDF
 * (HenyeyGreensteinPhaseFunction.h:218-240); uniform for |g| < 1e-4 */
static inline float hg_sample_cos(float g, float x2) {
    float ct;
    if (fabsf(g) < 1e-4f) {
        ct = 1.0f - 2.0f * x2;
    } else {
        float gg = g * g;
        float a = (1.0f - gg) / ((1.0f - g) + (2.0f * g) * x2);
        ct = ((1.0f + gg) - a * a) / (2.0f * g);
        if (ct < -1.0f) ct = -1.0f;
        if (ct > 1.0f) ct = 1.0f;
    }
    return ct;
}

float orc_hg_eval(float g, float cs) { return hg_eval(g, cs); }
float orc_hg_sample_cos(float g, float x) { return hg_sample_cos(g, x); }

static inline int is_finite3(const float* L) {
    return isfinite(L[0]) && isfinite(L[1]) && isfinite(L[2]);
}

/* ------------------------------------------------------------------------------------------
 * GGX microfacet reflection (no counterpart in the reference; restated from the published
 * methods): D, Smith height-correlated G2 and Schlick F of Walter et al. 2007 ("Microfacet
 * models for refraction through rough surfaces", EGSR), visible-normal sampling of Heitz 2018
 * ("Sampling the GGX distribution of visible normals", JCGT 7(4)).  Local frame around the
 * geometric normal: Duff et al. 2017.  Reflection only; the back side absorbs.
 * ---------------------------------------------------------------------------------------- */
#define PI_F 3.14159274f
typedef struct { v3 t1, t2, n; } frame3;
static inline frame3 make_frame(v3 n) {
    float sg = copysignf(1.0f, n.z);
    float a = -1.0f / (sg + n.z);
    float b = n.x * n.y * a;
    frame3 F;
    F.t1 = mk(1.0f + sg * n.x * n.x * a, sg * b, -sg * n.x);
    F.t2 = mk(b, sg + n.y * n.y * a, -n.y);
    F.n = n;
    return F;
}
static inline v3 to_local(const frame3* F, v3 w) { return mk(dot(w, F->t1), dot(w, F->t2), dot(w, F->n)); }
static inline v3 to_world(const frame3* F, v3 l) {
    return add(add(muls(F->t1, l.x), muls(F->t2, l.y)), muls(F->n, l.z));
}
static inline float ggx_D(float a2, float hz) {
    float c = hz * hz;
    float d = c * (a2 - 1.0f) + 1.0f;
    return a2 / ((PI_F * d) * d);
}
static inline float ggx_lambda(float a2, v3 w) {
    float t2 = (w.x * w.x + w.y * w.y) / (w.z * w.z);
    return (-1.0f + sqrtf(1.0f + a2 * t2)) * 0.5f;
}
static inline float schlick(float f0, float c) {
    float m = 1.0f - c;
    float m2 = m * m;
    return f0 + (1.0f - f0) * ((m2 * m2) * m);
}
/* f(wo, wi) * max(0, n.wi); wo = towards the previous vertex, wi = towards the light */
static v3 ggx_eval_cos(v3 kd, float alpha, v3 n, v3 wo_w, v3 wi_w) {
    frame3 F = make_frame(n);
    v3 wo = to_local(&F, wo_w), wi = to_local(&F, wi_w);
    if (!(wo.z > 0.0f) || !(wi.z > 0.0f)) return mk(0.0f, 0.0f, 0.0f);
    v3 h = normalize(add(wo, wi));
    float a2 = alpha * alpha;
    float D = ggx_D(a2, h.z);
    float G2 = 1.0f / ((1.0f + ggx_lambda(a2, wo)) + ggx_lambda(a2, wi));
    float c = dot(wo, h);
    if (c < 0.0f) c = 0.0f;
    float common = (D * G2) / (4.0f * wo.z);
    return mk(schlick(kd.x, c) * common, schlick(kd.y, c) * common, schlick(kd.z, c) * common);
}
/* visible-normal sample; returns 0 when the reflected direction leaves below the surface */
static int ggx_sample(v3 kd, float alpha, v3 n, v3 wo_w, float sp, float cp, float x2, v3* wi_w, v3* fa, float* pa) {
    frame3 F = make_frame(n);
    v3 wo = to_local(&F, wo_w);
    if (!(wo.z > 0.0f)) return 0;
    v3 Vh = normalize(mk(alpha * wo.x, alpha * wo.y, wo.z));
    float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    v3 T1 = lensq > 0.0f ? divs(mk(-Vh.y, Vh.x, 0.0f), sqrtf(lensq)) : mk(1.0f, 0.0f, 0.0f);
    v3 T2 = cross(Vh, T1);
    float r = sqrtf(x2);
    float t1 = r * cp, t2 = r * sp;
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    float tz2 = (1.0f - t1 * t1) - t2 * t2;
    float tz = sqrtf(tz2 > 0.0f ? tz2 : 0.0f);
    v3 Nh = add(add(muls(T1, t1), muls(T2, t2)), muls(Vh, tz));
    v3 h = normalize(mk(alpha * Nh.x, alpha * Nh.y, Nh.z > 0.0f ? Nh.z : 0.0f));
    float c = dot(wo, h);
    v3 wi = sub(muls(h, 2.0f * c), wo);
    if (!(wi.z > 0.0f)) return 0;
    float a2 = alpha * alpha;
    float Lo = ggx_lambda(a2, wo), Li = ggx_lambda(a2, wi);
    float G1 = 1.0f / (1.0f + Lo);
    float G2 = 1.0f / ((1.0f + Lo) + Li);
    float pdf = (G1 * ggx_D(a2, h.z)) / (4.0f * wo.z);
    float w = G2 / G1;
    if (c < 0.0f) c = 0.0f;
    *fa = mk((schlick(kd.x, c) * w) * pdf, (schlick(kd.y, c) * w) * pdf, (schlick(kd.z, c) * w) * pdf);
    *pa = pdf;
    *wi_w = normalize(to_world(&F, wi));
    return 1;
}

/* exposed for unit tests: weight (f cos / pdf) and pdf of one sample, and eval */
int orc_ggx_sample(const float* kd, float alpha, const float* n, const float* wo, float x1, float x2,
                   float* wi, float* weight, float* pdf) {
    float sp, cp;
    orc_sincos2pi(x1, &sp, &cp);
    v3 w, fa; float pa;
    if (!ggx_sample(ld3(kd), alpha, ld3(n), ld3(wo), sp, cp, x2, &w, &fa, &pa)) return 0;
    wi[0] = w.x; wi[1] = w.y; wi[2] = w.z;
    weight[0] = fa.x / pa; weight[1] = fa.y / pa; weight[2] = fa.z / pa;
    *pdf = pa;
    return 1;
}
void orc_ggx_eval_cos(const float* kd, float alpha, const float* n, const float* wo, const float* wi, float* out) {
    v3 r = ggx_eval_cos(ld3(kd), alpha, ld3(n), ld3(wo), ld3(wi));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

/* The vector-to-vector matrix of Moeller & Hughes ("Efficiently building a matrix to rotate
 * one vector to another", JGT 4(4), 1999) from +y to `to`, applied to d and normalised -- the
 * reference's transform_matrix_to (VectorN.h:427-521).  The time-angular sampler passes the
 * unnormalised target offset as `to` (BidirectionalPathTracing.h:392), for which the matrix is
 * not a rotation; the same construction is used here so the sampled directions match. */
static v3 mh_from_y(v3 to, v3 d) {
    const v3 fr = mk(0.0f, 1.0f, 0.0f);
    v3 v = mk(fr.y * to.z - fr.z * to.y, fr.z * to.x - fr.x * to.z, fr.x * to.y - fr.y * to.x);
    float e = (fr.x * to.x + fr.y * to.y) + fr.z * to.z;
    float m[3][3];
    if (fabsf(e) > 1.0f - 1e-4f) {
        /* near-parallel: reflections through the coordinate axis least aligned with +y (z) */
        v3 xa = mk(0.0f, 0.0f, 1.0f);
        v3 u = sub(xa, fr);
        v3 w = sub(xa, to);
        float c1 = 2.0f / dot(u, u), c2 = 2.0f / dot(w, w);
        float c3 = (c1 * c2) * dot(u, w);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                m[i][j] = ((-c1 * comp(u, i)) * comp(u, j) - (c2 * comp(w, i)) * comp(w, j)) + (c3 * comp(w, i)) * comp(u, j);
                if (i == j) m[i][j] += 1.0f;
            }
    } else {
        float h = 1.0f / (1.0f + e);
        float hvx = h * v.x, hvz = h * v.z, hvxy = hvx * v.y, hvxz = hvx * v.z, hvyz = hvz * v.y;
        m[0][0] = e + hvx * v.x; m[0][1] = hvxy - v.z;           m[0][2] = hvxz + v.y;
        m[1][0] = hvxy + v.z;    m[1][1] = e + (h * v.y) * v.y;   m[1][2] = hvyz - v.x;
        m[2][0] = hvxz - v.y;    m[2][1] = hvyz + v.x;           m[2][2] = e + hvz * v.z;
    }
    v3 r = mk((m[0][0] * d.x + m[0][1] * d.y) + m[0][2] * d.z, (m[1][0] * d.x + m[1][1] * d.y) + m[1][2] * d.z,
              (m[2][0] * d.x + m[2][1] * d.y) + m[2][2] * d.z);
    return normalize(r);
}

/* World::Li's record of a camera ray: closest surface distance (FLT_MAX when none), position
 * and normal of that point (zero when none). */
typedef struct { float t; v3 pos, n; } camrec;

/* ---- bidirectional connections (set_path_tracing_only(false)) ----
 * Defined here as in the reference for time-sampling mode in scenes without a medium.  (Outside
 * time-sampling mode the reference draws no light sample before its light subpath,
 * BidirectionalPathTracing.h:1108-1113, so the subpath starts from an uninitialised LightSample
 * with pdf 0 and every connection is non-finite and dropped; with a medium its time-sampled
 * connections build a medium vertex from a ray without a medium, :766-790, and dereference a null
 * medium.)  Light subpaths start in vacuum as in the reference (Ray(pos, dir, false) carries no
 * medium, :1121-1124).
 *
 * A subpath vertex (Path::Vertex, Path.h:36-140): position, delay, geometric normal, vertex pdf
 * (m_pi), Lambertian albedo, vertex value (m_f, throughput over pdfs). */
typedef struct { v3 pos; float time; v3 n; float pdf; v3 kd; v3 f; } bvert;

/* PathMIS::connection_probability (PathMIS.h:49-60): the density with which path0[i0] samples
 * the direction towards path1[i1]; Lambertian::p = max(0, cos) / pi (Lambertian.h:82-93). */
static float conn_prob(const bvert* from, const bvert* to) {
    v3 d = normalize(sub(to->pos, from->pos));
    float c = dot(d, from->n);
    return (c > 0.0f ? c : 0.0f) * INV_PI_F;
}

/* PathMIS::compute_weight with beta = 1 (MIS_Balance, BidirectionalPathTracing.h:902-924,
 * PathMIS.h:63-111), restated as it is: the ratios are accumulated by addition along each
 * subpath, and the caller divides by the result. */
static float mis_weight(const bvert* ev, const bvert* lv, int t, int s) {
    float iw = 1.0f;
    if (s > 1) {
        float p_s_1 = conn_prob(&ev[t], &lv[s]) / lv[s].pdf;
        iw = iw + p_s_1;
        float p_i_0 = p_s_1;
        for (int i = s - 1; i > 0; --i) {
            float p_i = conn_prob(&lv[i + 1], &lv[i]);
            p_i = p_i_0 + p_i / lv[i].pdf;
            iw = iw + p_i;
            p_i_0 = p_i;
        }
    }
    if (t > 1) {
        float p_t_1 = conn_prob(&lv[s], &ev[t]) / ev[t].pdf;
        iw = iw + p_t_1;
        float p_i_0 = p_t_1;
        for (int i = t - 1; i > 0; --i) {
            float p_i = conn_prob(&ev[i + 1], &ev[i]);
            p_i = p_i_0 + p_i / ev[i].pdf;
            iw = iw + p_i;
            p_i_0 = p_i;
        }
    }
    return (float)(1.0 / (double)iw);
}

/* Lambertian direction sampling at a surface vertex, in the frame the eye path uses (the
 * orthonormal frame with ORC_FLAG_ORTHONORMAL_FRAME, else Intersection::set_coordinate_system's). */
static void lambert_sample(const orc_ctx* x, v3 n, v3 kd, float x1, float x2, v3* nd, v3* fa, float* pa) {
    float sp, cp;
    orc_sincos2pi(x1, &sp, &cp);
    float ct = sqrtf(x2);
    float stt = sqrtf(1.0f - ct * ct);
    if (x->integ.flags & ORC_FLAG_ORTHONORMAL_FRAME) {
        frame3 Fr = make_frame(n);
        *nd = to_world(&Fr, mk(cp * stt, sp * stt, ct));
        *fa = mk((kd.x * INV_PI_F) * ct, (kd.y * INV_PI_F) * ct, (kd.z * INV_PI_F) * ct);
    } else {
        v3 aux = fabsf(n.x) > fabsf(n.z) ? mk(-n.y, n.x, n.z) : mk(0.0f, -n.z, n.y);
        v3 tv = normalize(aux);
        v3 tu = cross(n, tv);
        v3 w = add(add(muls(tu, cp * stt), muls(n, ct)), muls(tv, sp * stt));
        *nd = normalize(w);
        float ca = fabsf(dot(n, *nd));
        *fa = mk((kd.x * INV_PI_F) * ca, (kd.y * INV_PI_F) * ca, (kd.z * INV_PI_F) * ca);
    }
    *pa = ct * INV_PI_F;
}

/* The light subpath (generate_path FROM_LIGHT, BidirectionalPathTracing.h:486-644, started at
 * :1121-1124): emission from the path's light point in a direction drawn from the light stream
 * rl (PointLightSource::sample: uniform sphere, PointLightSource.h:174-183, Sampling.h:80-94;
 * RectangularAreaLightSource::sample: cosine lobe about the normal, RectangularAreaLightSource.h:
 * 252-276, Sampling.h:131-143), initial pdf p0 = (1 / lights) * emission pdf, value L0 = the
 * emitted intensity (times cos for the rectangle).  Vertices are stored while the subpath's
 * time stays within the film (TotalTime termination, no Russian roulette); at most maxv. */
static int light_subpath(const orc_ctx* x, pcg* rl, const orc_light* L, v3 lpos, int maxv, float total_time,
                         bvert* lv, v3* L0, pstats* st) {
    float e1 = pcg_float(rl), e2 = pcg_float(rl);
    float sp, cp;
    orc_sincos2pi(e1, &sp, &cp);
    v3 dir;
    float pdf_dir;
    if (L->kind == 1) {
        float ct = sqrtf(e2);
        float stt = sqrtf(1.0f - ct * ct);
        v3 ln = ld3(L->normal);
        dir = mh_from_y(ln, mk(cp * stt, ct, sp * stt));
        pdf_dir = ct * INV_PI_F;
        float dl = dot(dir, ln);
        *L0 = mk(L->intensity[0] * dl, L->intensity[1] * dl, L->intensity[2] * dl);
        pdf_dir = (1.0f / L->area) * pdf_dir;
    } else {
        float ct = (float)(1.0 - 2.0 * (double)e2);
        float stt = sqrtf(1.0f - ct * ct);
        dir = mk(cp * stt, ct, sp * stt);
        pdf_dir = INV_4PI_F;
        *L0 = ld3(L->intensity);
    }
    float pi = (1.0f / (float)x->nl) * pdf_dir;
    v3 org = lpos, f = mk(1.0f, 1.0f, 1.0f);
    float time = 0.0f;
    int n = 0;
    while (n < maxv) {
        wray r;
        wray_setup(&r, org, dir, SIGMA_VIS, INFINITY);
        orc_hit h;
        st->closest++;
        uint32_t cv = 0, ct2 = 0;
        int hit = trace1(x, &r, 0, &h, &cv, &ct2);
        st->c_nodes += cv; st->c_tris += ct2;
        if (!hit) break;
        float dist = h.t;
        f = mk(f.x / pi, f.y / pi, f.z / pi);
        time = time + dist;
        if (time > total_time) break;
        v3 pos = add(org, muls(dir, dist));
        v3 nrm = x->ng[h.prim_id];
        v3 kd = ld3(x->mats[x->mat[h.prim_id]].kd);
        lv[n].pos = pos; lv[n].time = time; lv[n].n = nrm; lv[n].pdf = pi; lv[n].kd = kd; lv[n].f = f;
        ++n;
        if (n >= maxv) break;
        float x1 = pcg_float(rl), x2 = pcg_float(rl);
        v3 nd, fa;
        float pa;
        lambert_sample(x, nrm, kd, x1, x2, &nd, &fa, &pa);
        f = mulv(f, fa);
        pi = 1.0f * pa;
        org = pos; dir = nd;
    }
    return n;
}

/* One random walk; appends its splat records (at most max_bounces) to rec; fills cr (if not
 * NULL) with the camera ray's record. */
static int trace_path(const orc_ctx* x, v3 org, v3 dir, pcg* rng, pcg* rl, float inv_inc, srec* rec, pstats* st,
                      camrec* cr) {
    const orc_film* F = &x->film;
    const int medium = x->med.enabled != 0;
    v3 sig_s = ld3(x->med.sigma_s), sig_t = add(ld3(x->med.sigma_a), ld3(x->med.sigma_s));
    float lambda = medium ? avg3(sig_t) : 0.0f;
    float g = x->med.g;
    float total_time = (float)F->time_bins * F->exposure + F->offset;
    uint32_t maxb = x->integ.max_bounces;
    const int unwarp = F->camera_unwarp != 0;
    const int need_cam = unwarp || F->components != 0;   /* camera ray traced to any distance */
    const int bounce_films = F->bounce_films != 0;
    /* World::Li's camera-ray record distance (World.h:749-766): the closest surface along the
     * camera ray, FLT_MAX when there is none (Ray.h:74-84) */
    float cam_dist = FLT_MAX;
    int nrec = 0;

    v3 f = mk(1.0f, 1.0f, 1.0f);
    float pi = 1.0f, time = 0.0f;
    /* time-sampling mode (set_mode(Transient), BidirectionalPathTracing.h:189-206): free flight
     * at rate m_avg_nb_vertices_path (4) / film length (:240-307), medium directions aimed at a
     * light point drawn for the path (:1107-1113, :385-431), total-time termination (:447-481) */
    const int tsm = (x->integ.flags & ORC_FLAG_TIME_SAMPLING) != 0;
    v3 target = mk(0.0f, 0.0f, 0.0f);
    const int bidir = rl != NULL && (x->integ.flags & ORC_FLAG_BIDIRECTIONAL) != 0;
    bvert lv[ORC_BIDIR_MAX_BOUNCES], ev[ORC_BIDIR_MAX_BOUNCES];
    int nlv = 0;
    v3 L0 = mk(0.0f, 0.0f, 0.0f);
    if (tsm) {
        /* World::sample_light + LightSource::sample(light_sample, pdf): the emission point
         * (PointLightSource.h:174-183, RectangularAreaLightSource.h:252-276) */
        float xl = pcg_float(rng);
        uint32_t li = (uint32_t)(xl * (float)x->nl);
        if (li >= x->nl) li = x->nl - 1;
        const orc_light* L = &x->lights[li];
        target = ld3(L->position);
        if (L->kind == 1) {
            float xu = pcg_float(rng), xv = pcg_float(rng);
            target = add(add(target, muls(ld3(L->left), xu)), muls(ld3(L->up), xv));
        }
        if (medium) lambda = 4.0f / ((float)F->time_bins * F->exposure);
        /* the light subpath from the same light point (its own random stream) */
        if (bidir && maxb >= 2) nlv = light_subpath(x, rl, L, target, (int)maxb - 1, total_time, lv, &L0, st);
    }
    float dsamp = INFINITY;
    if (medium) dsamp = -orc_log(pcg_float(rng)) / lambda;

    for (uint32_t depth = 0; depth < maxb; ++depth) {
        wray r;
        /* with camera unwarp the camera ray is traced to infinity (its surface distance is the
         * unwarp offset); surface vs medium below is decided by h.t < dsamp either way */
        wray_setup(&r, org, dir, SIGMA_VIS, (medium && !(need_cam && depth == 0)) ? dsamp : INFINITY);
        orc_hit h;
        st->closest++;
        uint32_t cv = 0, ct = 0;
        int hit = trace1(x, &r, 0, &h, &cv, &ct);
        st->c_nodes += cv; st->c_tris += ct;
        if (depth == 0 && hit) cam_dist = h.t;
        if (depth == 0 && cr) {
            cr->t = hit ? h.t : FLT_MAX;
            cr->pos = hit ? add(org, muls(dir, h.t)) : mk(0.0f, 0.0f, 0.0f);
            cr->n = hit ? x->ng[h.prim_id] : mk(0.0f, 0.0f, 0.0f);
        }
        int surface = hit && (!medium || h.t < dsamp);
        if (!medium && !hit) break;
        float dist, pd;
        if (surface) { dist = h.t; pd = medium ? orc_exp(-(dist * lambda)) : 1.0f; }
        else { dist = dsamp; pd = orc_exp(-(dist * lambda)) * lambda; }
        float ptot = pi * pd;
        if (medium) {
            f = mk((f.x * orc_exp(-(dist * sig_t.x))) / ptot, (f.y * orc_exp(-(dist * sig_t.y))) / ptot,
                   (f.z * orc_exp(-(dist * sig_t.z))) / ptot);
        } else {
            f = mk(f.x / ptot, f.y / ptot, f.z / ptot);
        }
        time = time + dist;
        v3 pos = add(org, muls(dir, dist));
        if (time > total_time) break;

        v3 n = mk(0, 0, 0), kd = mk(0, 0, 0);
        int ggx = 0;
        float alpha = 0.0f;
        if (surface) {
            n = x->ng[h.prim_id];
            const orc_material* m = &x->mats[x->mat[h.prim_id]];
            kd = ld3(m->kd);
            ggx = m->kind == 1;
            alpha = m->alpha;
        }
        v3 wo = mk(-dir.x, -dir.y, -dir.z);

        /* ---- next-event estimation (connect_vertex_with_light + transient connect_paths) ---- */
        {
            float xl = pcg_float(rng);
            uint32_t li = (uint32_t)(xl * (float)x->nl);
            if (li >= x->nl) li = x->nl - 1;
            const orc_light* L = &x->lights[li];
            float pl = 1.0f / (float)x->nl;
            v3 lp = ld3(L->position);
            int ok = 1;
            v3 irr;
            if (L->kind == 1) {
                float xu = pcg_float(rng), xv = pcg_float(rng);
                lp = add(add(lp, muls(ld3(L->left), xu)), muls(ld3(L->up), xv));
                pl = pl * (1.0f / L->area);
            }
            v3 ld = sub(pos, lp);
            float d2 = dot(ld, ld);
            float dl = sqrtf(d2);
            ld = divs(ld, dl);
            if (L->kind == 1) {
                float dot_l = dot(ld, ld3(L->normal));
                if (!(dot_l > 0.0f)) ok = 0;
                float a = dot_l / (dl * dl);
                irr = mk(L->intensity[0] * a, L->intensity[1] * a, L->intensity[2] * a);
            } else {
                irr = mk(L->intensity[0] / d2, L->intensity[1] / d2, L->intensity[2] / d2);
            }
            if (ok) {
                v3 wl = mk(-ld.x, -ld.y, -ld.z);
                v3 fe;
                if (surface && ggx) {
                    fe = ggx_eval_cos(kd, alpha, n, wo, wl);
                } else if (surface) {
                    float cs = dot(wl, n);
                    float cl = cs > 0.0f ? cs : 0.0f;
                    fe = mk((kd.x * INV_PI_F) * cl, (kd.y * INV_PI_F) * cl, (kd.z * INV_PI_F) * cl);
                } else {
                    float ph = hg_eval(g, dot(dir, wl));
                    fe = mk(ph * sig_s.x, ph * sig_s.y, ph * sig_s.z);
                }
                v3 att = mk(1.0f, 1.0f, 1.0f);
                if (medium) att = mk(orc_exp(-(sig_t.x * dl)), orc_exp(-(sig_t.y * dl)), orc_exp(-(sig_t.z * dl)));
                float scale = inv_inc / pl;
                float Lc[3] = {(f.x * (fe.x * (irr.x * att.x))) * scale,
                               (f.y * (fe.y * (irr.y * att.y))) * scale,
                               (f.z * (fe.z * (irr.z * att.z))) * scale};
                float tt = time + dl;
                float tc = unwarp ? tt - cam_dist : tt;          /* StreakCameraFilm.h:167 */
                float ps = (tc - F->offset) / F->exposure;
                int inside = ps < (float)F->time_bins && ps >= 0.0f;
                int finite = is_finite3(Lc);
                int useful = inside && finite && (Lc[0] != 0.0f || Lc[1] != 0.0f || Lc[2] != 0.0f);
                /* bounce films count every visible light connection (the sample exists in the
                 * reference whatever its time or radiance; non-finite radiance becomes 0,
                 * TransientRenderer.h:165-169); otherwise only useful samples are traced */
                if (useful || bounce_films) {
                    wray sr;
                    wray_setup(&sr, lp, ld, SIGMA_VIS, dl - SIGMA_VIS);
                    orc_hit sh;
                    st->shadow++;
                    uint32_t sv = 0, stt2 = 0;
                    int occluded = trace1(x, &sr, 1, &sh, &sv, &stt2);
                    st->s_nodes += sv; st->s_tris += stt2;
                    if (!occluded) {
                        rec[nrec].bin = inside ? (uint32_t)floorf(ps) : BIN_OUTSIDE;
                        rec[nrec].depth = depth;
                        for (int c = 0; c < 3; ++c) rec[nrec].L[c] = finite ? Lc[c] : 0.0f;
                        nrec++;
                        st->splats++;
                    }
                }
            }
        }

        /* ---- connections of this eye vertex with the light subpath's vertices (transient
         * connect_paths, BidirectionalPathTracing.h:1018-1041; connect_vertices' shadow
         * connection, :840-871): only pairs with ie + il + 2 <= max_bounces and delays within
         * the film; the connection counts when World::intersects reports a blocker between the
         * two vertices (that query returns true on a hit, World.h:617-639 / 693-697, and the
         * reference connects on true); value fe * (fv * (f_l * L0)) / (1 * w) with w the
         * MIS quantity above, time = distance + both delays, bounce ie + il + 1 ---- */
        if (bidir && surface && depth + 2 <= maxb) {
            bvert* E = &ev[depth];
            E->pos = pos; E->time = time; E->n = n; E->pdf = ptot; E->kd = kd; E->f = f;
            for (int il = 0; il < nlv; ++il) {
                if (depth + (uint32_t)il + 2 > maxb) break;
                if (time + lv[il].time > total_time) break;
                const bvert* Lv = &lv[il];
                v3 l2e = sub(pos, Lv->pos);
                float dd = sqrtf(dot(l2e, l2e));
                l2e = divs(l2e, dd);
                if ((dd + time) + Lv->time > total_time) continue;
                wray sr;
                wray_setup(&sr, Lv->pos, l2e, SIGMA_VIS, dd - SIGMA_VIS);
                orc_hit sh;
                st->shadow++;
                uint32_t sv = 0, stt2 = 0;
                int blocked = trace1(x, &sr, 1, &sh, &sv, &stt2);
                st->s_nodes += sv; st->s_tris += stt2;
                if (!blocked) continue;
                float ce = -dot(l2e, n), cl = dot(l2e, Lv->n);
                ce = ce > 0.0f ? ce : 0.0f;
                cl = cl > 0.0f ? cl : 0.0f;
                v3 fe = mk((kd.x * INV_PI_F) * ce, (kd.y * INV_PI_F) * ce, (kd.z * INV_PI_F) * ce);
                v3 fl = mk((Lv->kd.x * INV_PI_F) * cl, (Lv->kd.y * INV_PI_F) * cl, (Lv->kd.z * INV_PI_F) * cl);
                float att = 1.0f / (dd * dd);
                v3 fv = mk((fe.x * fl.x) * att, (fe.y * fl.y) * att, (fe.z * fl.z) * att);
                float w = mis_weight(ev, lv, (int)depth, il);
                float Lc[3] = {((f.x * (fv.x * (Lv->f.x * L0.x))) / w) * inv_inc,
                               ((f.y * (fv.y * (Lv->f.y * L0.y))) / w) * inv_inc,
                               ((f.z * (fv.z * (Lv->f.z * L0.z))) / w) * inv_inc};
                float tt = dd + (time + Lv->time);
                float tc = unwarp ? tt - cam_dist : tt;
                float ps = (tc - F->offset) / F->exposure;
                int inside = ps < (float)F->time_bins && ps >= 0.0f;
                int finite = is_finite3(Lc);
                rec[nrec].bin = inside ? (uint32_t)floorf(ps) : BIN_OUTSIDE;
                rec[nrec].depth = depth + (uint32_t)il + 1u;
                for (int c = 0; c < 3; ++c) rec[nrec].L[c] = finite ? Lc[c] : 0.0f;
                if (inside || bounce_films) { nrec++; st->splats++; }
            }
        }

        if (depth + 1 >= maxb) break;

        /* ---- termination (sample_termination): Russian roulette, or none with total-time
         * termination (the film-time test above ends the walk) ---- */
        float albedo = surface ? avg3(kd) : avg3(mk(sig_s.x / sig_t.x, sig_s.y / sig_t.y, sig_s.z / sig_t.z));
        float prr = 1.0f;
        if (!tsm) {
            if (pcg_float(rng) > albedo) break;
            prr = albedo;
        }

        /* ---- outgoing direction (sample_outgoing_ray) ---- */
        v3 fa; float pa; v3 nd;
        float nds_first = 0.0f;
        int angular_done = 0;
        if (tsm && !surface) {
            /* the next free-flight distance r is drawn first (generate_path, :530-545) and the
             * direction from the time-angular sampler towards the target (SamplingTechniques.h
             * TimeAngular) with probability p_ts = 1, else the phase function (:371-431) */
            nds_first = -orc_log(pcg_float(rng)) / lambda;
            const float r = nds_first;
            v3 l = sub(target, pos);
            float mod = sqrtf(dot(l, l));
            float ta = mod + time;
            float tb = (float)F->time_bins * F->exposure + F->offset;
            float t_a = ta, t_b = tb;
            if (r > mod) t_a = fmaxf(t_a, 2.0f * r - mod); else t_a = fmaxf(t_a, mod);
            t_b = fminf(t_b, 2.0f * r + mod);
            int use_ts = !((tb - (ta + r)) < F->exposure);
            (void)pcg_float(rng);                          /* the technique choice xi < p_ts */
            if (use_ts) {
                float e = pcg_float(rng), e2 = pcg_float(rng);
                float t = e * (t_b - t_a) + t_a;
                /* TimeAngular::theta_t (SamplingTechniques.h:186-191): the cosine is evaluated in
                 * double (its constants are double) and stored as a float, then clamped */
                float ct = (float)((((double)(mod * mod) + ((2.0 * (double)t) * (double)r)) - (double)(t * t)) /
                                   ((2.0 * (double)r) * (double)mod));
                ct = ct < -1.0f ? -1.0f : (ct > 1.0f ? 1.0f : ct);
                /* theta = acos(ct) is a float.  At ct = -1 it is the float nearest pi, which lies
                 * above pi, so sin(theta) is the small negative number pi - (float)pi: this is
                 * what the reference gets whenever the bounds are inverted (t_a > t_b, the current
                 * delay exceeding 2r), and its density dtdtheta / (t_b - t_a) is then a small
                 * positive number that can pass the 1e-5 test.  Elsewhere sin(acos(ct)) agrees
                 * with sqrt(1 - ct^2) to rounding. */
                float st = ct == -1.0f ? (float)(3.14159265358979323846 - (double)3.14159265358979323846f)
                                       : (float)sqrt(1.0 - (double)ct * (double)ct);
                float sp2, cp2;
                orc_sincos2pi(e2, &sp2, &cp2);
                nd = mh_from_y(l, mk(cp2 * st, ct, sp2 * st));
                float ph = hg_eval(g, dot(dir, nd));
                fa = mk(ph * sig_s.x, ph * sig_s.y, ph * sig_s.z);
                /* the reference's density: TimeAngular::pdf(theta) / (2 pi) (:233-236, and
                 * BidirectionalPathTracing.h:400-402 with p_ts = 1), a density in theta used as
                 * a solid-angle density (no 1 / sin(theta)); restated as is, with its operand
                 * types (float products and sums, double where a double constant enters) */
                float dtdth = (float)((double)((mod * r) * st) /
                                      sqrt((double)(r * r + mod * mod) - ((2.0 * (double)r) * (double)mod) * (double)ct));
                float pdf_theta = dtdth / (t_b - t_a);
                pa = (float)((double)pdf_theta / (2.0 * 3.14159265358979323846));
                angular_done = pa >= 1e-5f;                /* else phase-function sampling */
            }
        }
        if (!angular_done) {
        float x1 = pcg_float(rng), x2 = pcg_float(rng);
        float sp, cp;
        orc_sincos2pi(x1, &sp, &cp);
        if (surface && ggx) {
            if (!ggx_sample(kd, alpha, n, wo, sp, cp, x2, &nd, &fa, &pa)) break;
        } else if (surface && (x->integ.flags & ORC_FLAG_ORTHONORMAL_FRAME)) {
            /* cosine sampling in an orthonormal frame (Duff et al. 2017) */
            float ct = sqrtf(x2);
            float stt = sqrtf(1.0f - ct * ct);
            frame3 Fr = make_frame(n);
            nd = to_world(&Fr, mk(cp * stt, sp * stt, ct));
            fa = mk((kd.x * INV_PI_F) * ct, (kd.y * INV_PI_F) * ct, (kd.z * INV_PI_F) * ct);
            pa = ct * INV_PI_F;
        } else if (surface) {
            /* Lambertian cosine sampling in the frame of Intersection::set_coordinate_system */
            float ct = sqrtf(x2);
            float stt = sqrtf(1.0f - ct * ct);
            v3 aux = fabsf(n.x) > fabsf(n.z) ? mk(-n.y, n.x, n.z) : mk(0.0f, -n.z, n.y);
            v3 tv = normalize(aux);
            v3 tu = cross(n, tv);
            v3 w = add(add(muls(tu, cp * stt), muls(n, ct)), muls(tv, sp * stt));
            nd = normalize(w);
            float ca = fabsf(dot(n, nd));
            fa = mk((kd.x * INV_PI_F) * ca, (kd.y * INV_PI_F) * ca, (kd.z * INV_PI_F) * ca);
            pa = ct * INV_PI_F;
        } else {
            float ct = hg_sample_cos(g, x2);
            float stt = sqrtf(1.0f - ct * ct);
            /* orthonormal frame around the propagation direction (Duff et al., JCGT 6(1), 2017) */
            float sg = copysignf(1.0f, dir.z);
            float aa = -1.0f / (sg + dir.z);
            float bb = dir.x * dir.y * aa;
            v3 t1 = mk(1.0f + sg * dir.x * dir.x * aa, sg * bb, -sg * dir.x);
            v3 t2 = mk(bb, sg + dir.y * dir.y * aa, -dir.y);
            nd = add(add(muls(t1, cp * stt), muls(t2, sp * stt)), muls(dir, ct));
            float ph = hg_eval(g, ct);
            fa = mk(ph * sig_s.x, ph * sig_s.y, ph * sig_s.z);
            pa = ph;
        }
        }
        f = mulv(f, fa);
        pi = prr * pa;
        org = pos; dir = nd;
        if (medium) dsamp = (tsm && !surface) ? nds_first : -orc_log(pcg_float(rng)) / lambda;
    }
    return nrec;
}

static void camera_ray(const orc_ctx* x, uint32_t px, uint32_t py, uint64_t s, v3* o, v3* d) {
    const orc_film* F = &x->film;
    uint32_t strata = x->integ.sqrt_spp;
    uint32_t spp = strata * strata;
    uint32_t st = (uint32_t)(s % spp);
    uint32_t subx = st % strata, suby = st / strata;
    pcg r;
    pcg_seed(&r, x->integ.seed, cam_id(py * F->width + px, s));
    float inv = 1.0f / (float)strata;
    float shx = ((float)subx + pcg_float(&r)) * inv;
    float shy = ((float)suby + pcg_float(&r)) * inv;
    float posx = fminf((float)px + shx, nextafterf((float)(px + 1), 0.0f));
    float posy = fminf((float)py + shy, nextafterf((float)(py + 1), 0.0f));
    float W = (float)F->width, H = (float)F->height;
    float ratio = W / H;
    float ix = (posx - W / 2.0f) / W;
    float iy = ((posy - H / 2.0f) / H) / ratio;
    const orc_camera* c = &x->cam;
    v3 nv = ld3(c->nv), uv = ld3(c->uv), vv = ld3(c->vv);
    v3 dd = sub(add(muls(nv, c->focal_distance), muls(muls(uv, 2.0f), ix)), muls(muls(vv, 2.0f), iy));
    *d = normalize(dd);
    *o = ld3(c->position);
}

static inline void path_rng(const orc_ctx* x, pcg* r, uint32_t pixel, uint64_t s, uint32_t j) {
    pcg_seed(r, x->integ.seed + (uint64_t)(j + 1) * GOLDEN64, cam_id(pixel, s));
}

/* The light subpath's stream (bidirectional connections): another state and increment, so the
 * eye walk draws exactly what it draws without light subpaths. */
static inline void light_rng(const orc_ctx* x, pcg* r, uint32_t pixel, uint64_t s, uint32_t j) {
    pcg_seed(r, x->integ.seed + (uint64_t)(j + 1) * GOLDEN64 + LIGHT_STATE_SALT, cam_id(pixel, s) ^ LIGHT_SEQ_SALT);
}

int orc_path_records(const orc_ctx* x, uint32_t px, uint32_t py, uint64_t s, uint32_t j,
                     uint32_t* bins, float* rgb, int cap) {
    v3 o, d;
    camera_ray(x, px, py, s, &o, &d);
    pcg r;
    path_rng(x, &r, py * x->film.width + px, s, j);
    srec rec[256];
    pstats st;
    memset(&st, 0, sizeof(st));
    pcg rl;
    light_rng(x, &rl, py * x->film.width + px, s, j);
    int n = trace_path(x, o, d, &r, &rl, 1.0f / (float)x->integ.incoming_samples, rec, &st, NULL);
    if (n > cap) n = cap;
    for (int i = 0; i < n; ++i) {
        bins[i] = rec[i].bin;
        rgb[3 * i] = rec[i].L[0]; rgb[3 * i + 1] = rec[i].L[1]; rgb[3 * i + 2] = rec[i].L[2];
    }
    return n;
}

typedef struct {
    const orc_ctx* x; uint32_t x0, x1, y0, y1; uint64_t s0; uint32_t ns;
    double *streak, *steady, *weight;
    double *bstreak, *bsteady, *bweight;
    double *cdepth, *cpos, *cnorm;
    uint32_t row_begin, row_step;
    uint64_t paths; pstats st;
} job;

static void* render_rows(void* arg) {
    job* J = (job*)arg;
    const orc_ctx* x = J->x;
    const orc_film* F = &x->film;
    uint32_t T = F->time_bins, W = F->width;
    const uint32_t NB = F->bounce_films;
    const size_t npix = (size_t)F->width * F->height;
    uint32_t ninc = x->integ.incoming_samples;
    float inv_inc = 1.0f / (float)ninc;
    srec rec[256];
    for (uint32_t y = J->y0 + J->row_begin; y < J->y1; y += J->row_step) {
        for (uint32_t px = J->x0; px < J->x1; ++px) {
            uint32_t pixel = y * W + px;
            for (uint64_t s = J->s0; s < J->s0 + J->ns; ++s) {
                v3 o, d;
                camera_ray(x, px, y, s, &o, &d);
                if (J->weight) J->weight[pixel] += 1.0;
                uint64_t present = 0;          /* bounce films with a sample of this camera sample */
                for (uint32_t j = 0; j < ninc; ++j) {
                    pcg r, rl;
                    path_rng(x, &r, pixel, s, j);
                    light_rng(x, &rl, pixel, s, j);
                    camrec cr;
                    int n = trace_path(x, o, d, &r, &rl, inv_inc, rec, &J->st, j == 0 ? &cr : NULL);
                    J->paths++;
                    if (j == 0) {
                        if (J->cdepth) J->cdepth[pixel] += (double)cr.t;
                        for (int c = 0; c < 3; ++c) {
                            if (J->cpos) J->cpos[(size_t)pixel * 3 + c] += (double)comp(cr.pos, c);
                            if (J->cnorm) J->cnorm[(size_t)pixel * 3 + c] += (double)comp(cr.n, c);
                        }
                    }
                    for (int i = 0; i < n; ++i) {
                        const int inside = rec[i].bin != BIN_OUTSIDE;
                        for (int c = 0; c < 3; ++c) {
                            if (J->streak && inside) J->streak[((size_t)pixel * T + rec[i].bin) * 3 + c] += (double)rec[i].L[c];
                            if (J->steady && (inside || NB)) J->steady[(size_t)pixel * 3 + c] += (double)rec[i].L[c];
                        }
                        if (NB) {
                            const uint32_t b = rec[i].depth < NB ? rec[i].depth : NB - 1;
                            present |= 1ull << b;
                            for (int c = 0; c < 3 && inside; ++c) {
                                if (J->bstreak)
                                    J->bstreak[(((size_t)b * npix + pixel) * T + rec[i].bin) * 3 + c] += (double)rec[i].L[c];
                                if (J->bsteady) J->bsteady[((size_t)b * npix + pixel) * 3 + c] += (double)rec[i].L[c];
                            }
                        }
                    }
                }
                for (uint32_t b = 0; b < NB && J->bweight; ++b)
                    if (present >> b & 1ull) J->bweight[(size_t)b * npix + pixel] += 1.0;
            }
        }
    }
    return NULL;
}

int orc_render(const orc_ctx* x, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
               uint64_t sample_begin, uint32_t sample_count, int nthreads,
               double* streak, double* steady, double* weight, uint64_t* stats) {
    return orc_render_bounces(x, x0, y0, x1, y1, sample_begin, sample_count, nthreads, streak, steady, weight,
                              NULL, NULL, NULL, stats);
}

int orc_render_bounces(const orc_ctx* x, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                       uint64_t sample_begin, uint32_t sample_count, int nthreads,
                       double* streak, double* steady, double* weight,
                       double* bstreak, double* bsteady, double* bweight, uint64_t* stats) {
    return orc_render_ex(x, x0, y0, x1, y1, sample_begin, sample_count, nthreads, streak, steady, weight,
                         bstreak, bsteady, bweight, NULL, NULL, NULL, stats);
}

int orc_render_ex(const orc_ctx* x, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                  uint64_t sample_begin, uint32_t sample_count, int nthreads,
                  double* streak, double* steady, double* weight,
                  double* bstreak, double* bsteady, double* bweight,
                  double* cdepth, double* cpos, double* cnorm, uint64_t* stats) {
    if (x->film.bounce_films > 64) return 1;
    if (x1 > x->film.width || y1 > x->film.height || x0 > x1 || y0 > y1) return 1;
    if (x->integ.max_bounces > 255) return 1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    job J[256];
    pthread_t th[256];
    for (int i = 0; i < nthreads; ++i) {
        J[i].x = x; J[i].x0 = x0; J[i].x1 = x1; J[i].y0 = y0; J[i].y1 = y1;
        J[i].s0 = sample_begin; J[i].ns = sample_count;
        J[i].streak = streak; J[i].steady = steady; J[i].weight = weight;
        J[i].bstreak = bstreak; J[i].bsteady = bsteady; J[i].bweight = bweight;
        J[i].cdepth = cdepth; J[i].cpos = cpos; J[i].cnorm = cnorm;
        J[i].row_begin = (uint32_t)i; J[i].row_step = (uint32_t)nthreads;
        J[i].paths = 0; memset(&J[i].st, 0, sizeof(pstats));
    }
    if (nthreads == 1) {
        render_rows(&J[0]);
    } else {
        for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, render_rows, &J[i]);
        for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
    }
    if (stats) {
        memset(stats, 0, 8 * sizeof(uint64_t));
        for (int i = 0; i < nthreads; ++i) {
            stats[0] += J[i].paths; stats[1] += J[i].st.closest; stats[2] += J[i].st.shadow;
            stats[3] += J[i].st.splats; stats[4] += J[i].st.c_nodes; stats[5] += J[i].st.c_tris;
            stats[6] += J[i].st.s_nodes; stats[7] += J[i].st.s_tris;
        }
    }
    return 0;
}
