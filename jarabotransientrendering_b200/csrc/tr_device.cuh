// tr_device.cuh - device-side building blocks of the transient path tracer (sm_100a).
//
// Compiled with -fmad=false: a*b+c is two correctly rounded operations unless written as
// fmaf(), so every kernel evaluates the same IEEE operation sequence as a plain C compiler
// with -ffp-contract=off.  That makes a path traced here bit-identical to the same path
// traced by a CPU restatement that uses the same formulas.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace trd {

constexpr float kSigmaVis = 1e-5f;          // _SIGMA_VISIBILITY_ (src/bunnykiller.h:76-78)
constexpr float kInvPi = 0.318309873f;
constexpr float kInv4Pi = 0.0795774683f;
constexpr unsigned long long kGolden64 = 0x9E3779B97F4A7C15ULL;
constexpr uint32_t kInvalid = 0xffffffffu;

struct f3 { float x, y, z; };
__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ f3 mulv(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ f3 divs(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ f3 normalize(f3 a) { return divs(a, sqrtf(dot(a, a))); }
__host__ __device__ __forceinline__ float avg3(f3 a) { return ((a.x + a.y) + a.z) / 3.0f; }
__host__ __device__ __forceinline__ float comp(f3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
__device__ __forceinline__ f3 f3of(float4 v) { return mk(v.x, v.y, v.z); }

// ---------------------------------------------------------------------------------------
// Math kernels written from the mathematics (same formulas as the CPU restatement):
//   log  - Cody-Waite split of ln 2, mantissa in [sqrt(1/2), sqrt(2)), 2*atanh(s) series;
//   exp  - Cody-Waite reduction, Taylor series to r^7, 2^k by exponent construction;
//   sincos(2*pi*xi) - exact quadrant reduction on xi, Taylor series on |a| <= pi/4.
// ---------------------------------------------------------------------------------------
constexpr float kLn2Hi = 0.693145751953125f;
constexpr float kLn2Lo = 1.42860677e-06f;
constexpr float kInvLn2 = 1.44269502f;
constexpr float kPi2 = 1.57079637f;

__device__ __forceinline__ float tr_log(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -__int_as_float(0x7f800000) : __int_as_float(0x7fffffff);
    if (x == __int_as_float(0x7f800000)) return x;
    int e = 0;
    uint32_t b = __float_as_uint(x);
    if ((b >> 23) == 0) { x = x * 8388608.0f; b = __float_as_uint(x); e = -23; }
    e += (int)((b >> 23) & 0xffu) - 127;
    float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
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
    return fmaf(fe, kLn2Hi, fmaf(fe, kLn2Lo, r));
}

__device__ __forceinline__ float tr_exp(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return __int_as_float(0x7f800000);
    if (x < -103.972076f) return 0.0f;
    float k = rintf(x * kInvLn2);
    float r = fmaf(-k, kLn2Hi, x);
    r = fmaf(-k, kLn2Lo, r);
    float p = fmaf(r, 0.000198412701f, 0.00138888892f);
    p = fmaf(r, p, 0.00833333377f);
    p = fmaf(r, p, 0.0416666679f);
    p = fmaf(r, p, 0.166666672f);
    p = fmaf(r, p, 0.5f);
    p = fmaf(r, p, 1.0f);
    p = fmaf(r, p, 1.0f);
    int ki = (int)k;
    if (ki > 127) return (p * __uint_as_float(254u << 23)) * __uint_as_float((uint32_t)(ki) << 23);
    if (ki < -126) return (p * __uint_as_float((uint32_t)(ki + 227) << 23)) * __uint_as_float(27u << 23);
    return p * __uint_as_float((uint32_t)(ki + 127) << 23);
}

__device__ __forceinline__ void tr_sincos2pi(float xi, float* s, float* c) {
    float u = xi * 4.0f;
    float q = rintf(u);
    float r = u - q;
    float a = r * kPi2;
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

// ---------------------------------------------------------------------------------------
// PCG32, the reference's generator (src/Utils/RandomNumbers.h:119-128,83-98,167-174).
// Stream of camera sample c = (pixel << 32) | s; jitter stream seeded with `seed`, path j
// seeded with seed + (j+1)*golden on the same sequence.
// ---------------------------------------------------------------------------------------
struct Pcg { unsigned long long state, inc; };
__device__ __forceinline__ uint32_t pcg_next(Pcg& r) {
    unsigned long long old = r.state;
    r.state = old * 6364136223846793005ULL + r.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((0u - rot) & 31u));
}
__device__ __forceinline__ void pcg_seed(Pcg& r, unsigned long long state, unsigned long long seq) {
    r.state = 0ull;
    r.inc = (seq << 1u) | 1ull;
    pcg_next(r);
    r.state += state;
    pcg_next(r);
}
__device__ __forceinline__ float pcg_float(Pcg& r) {
    return __uint_as_float((pcg_next(r) >> 9) | 0x3f800000u) - 1.0f;
}
__host__ __device__ __forceinline__ unsigned long long cam_id(uint32_t pixel, unsigned long long s) {
    return ((unsigned long long)pixel << 32) | (s & 0xffffffffull);
}

// ---------------------------------------------------------------------------------------
// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2(1), 2013) for the inside/outside
// decision; the hit distance comes from the plane equation.  Operation order fixed: same
// expression tree as the CPU restatement, fused where fmaf is written.
// ---------------------------------------------------------------------------------------
struct WRay {
    f3 o, d;
    float tnear;
    int kx, ky, kz;
    float Sx, Sy;
    f3 inv;       // reciprocal direction for the slab test
};

__device__ __forceinline__ void wray_setup(WRay& r, f3 o, f3 d, float tnear) {
    r.o = o; r.d = d; r.tnear = tnear;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0; float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) { kz = 2; }
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (comp(d, kz) < 0.0f) { int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    float dz = comp(d, kz);
    r.Sx = comp(d, kx) / dz; r.Sy = comp(d, ky) / dz;
    const float e = 1e-30f;
    r.inv = mk(1.0f / (fabsf(d.x) > e ? d.x : copysignf(e, d.x)),
               1.0f / (fabsf(d.y) > e ? d.y : copysignf(e, d.y)),
               1.0f / (fabsf(d.z) > e ? d.z : copysignf(e, d.z)));
}

__device__ __forceinline__ bool wt_hit(const WRay& r, f3 p0, f3 p1, f3 p2, float tfar,
                                       float& t, float& u, float& v) {
    f3 A = p0 - r.o, B = p1 - r.o, C = p2 - r.o;
    float Akz = comp(A, r.kz), Bkz = comp(B, r.kz), Ckz = comp(C, r.kz);
    float Ax = fmaf(-r.Sx, Akz, comp(A, r.kx)), Ay = fmaf(-r.Sy, Akz, comp(A, r.ky));
    float Bx = fmaf(-r.Sx, Bkz, comp(B, r.kx)), By = fmaf(-r.Sy, Bkz, comp(B, r.ky));
    float Cx = fmaf(-r.Sx, Ckz, comp(C, r.kx)), Cy = fmaf(-r.Sy, Ckz, comp(C, r.ky));
    float U = fmaf(Cx, By, -(Cy * Bx));
    float V = fmaf(Ax, Cy, -(Ay * Cx));
    float W = fmaf(Bx, Ay, -(By * Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = (U + V) + W;
    if (det == 0.0f) return false;
    // distance from the plane equation, Embree's fused dot/cross order: Ng = e1 x e2 with
    // e1 = p0 - p1, e2 = p2 - p0; t = dot(Ng, p0 - o) / dot(Ng, d)
    f3 e1 = p0 - p1, e2 = p2 - p0;
    f3 Ng = mk(fmaf(e1.y, e2.z, -(e1.z * e2.y)), fmaf(e1.z, e2.x, -(e1.x * e2.z)), fmaf(e1.x, e2.y, -(e1.y * e2.x)));
    float den = fmaf(Ng.x, r.d.x, fmaf(Ng.y, r.d.y, Ng.z * r.d.z));
    float T = fmaf(Ng.x, A.x, fmaf(Ng.y, A.y, Ng.z * A.z));
    float tt = T / den;
    if (!(tt > r.tnear && tt <= tfar)) return false;
    t = tt; u = V / det; v = W / det;
    return true;
}

}  // namespace trd
