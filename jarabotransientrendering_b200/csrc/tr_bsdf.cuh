// tr_bsdf.cuh - device helpers shared by the shading kernel (tr_kernels.cu) and the guided
// sampling kernel (tr_guided.cu): warp lane masks, local frames, GGX microfacet reflection.
#pragma once
#include "tr_device.cuh"

namespace trk {
using namespace trd;

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// GGX microfacet reflection (no reference counterpart): D, height-correlated Smith G2 and
// Schlick F of Walter et al. 2007; visible-normal sampling of Heitz 2018 (JCGT 7(4)); local
// frame around the geometric normal by Duff et al. 2017.  Reflection only; the back side absorbs.
struct Frame3 { f3 t1, t2, n; };
__device__ __forceinline__ Frame3 make_frame(f3 n) {
    const float sg = copysignf(1.0f, n.z);
    const float a = -1.0f / (sg + n.z);
    const float b = n.x * n.y * a;
    return Frame3{mk(1.0f + sg * n.x * n.x * a, sg * b, -sg * n.x), mk(b, sg + n.y * n.y * a, -n.y), n};
}
__device__ __forceinline__ f3 to_local(const Frame3& F, f3 w) { return mk(dot(w, F.t1), dot(w, F.t2), dot(w, F.n)); }
__device__ __forceinline__ f3 to_world(const Frame3& F, f3 l) { return ((F.t1 * l.x) + (F.t2 * l.y)) + (F.n * l.z); }
__device__ __forceinline__ float ggx_D(float a2, float hz) {
    const float c = hz * hz;
    const float d = c * (a2 - 1.0f) + 1.0f;
    return a2 / ((3.14159274f * d) * d);
}
__device__ __forceinline__ float ggx_lambda(float a2, f3 w) {
    const float t2 = (w.x * w.x + w.y * w.y) / (w.z * w.z);
    return (-1.0f + sqrtf(1.0f + a2 * t2)) * 0.5f;
}
__device__ __forceinline__ float schlick(float f0, float c) {
    const float m = 1.0f - c;
    const float m2 = m * m;
    return f0 + (1.0f - f0) * ((m2 * m2) * m);
}
// f(wo, wi) * max(0, n.wi)
__device__ __forceinline__ f3 ggx_eval_cos(f3 kd, float alpha, f3 n, f3 wo_w, f3 wi_w) {
    const Frame3 F = make_frame(n);
    const f3 wo = to_local(F, wo_w), wi = to_local(F, wi_w);
    if (!(wo.z > 0.0f) || !(wi.z > 0.0f)) return mk(0.0f, 0.0f, 0.0f);
    const f3 h = normalize(wo + wi);
    const float a2 = alpha * alpha;
    const float D = ggx_D(a2, h.z);
    const float G2 = 1.0f / ((1.0f + ggx_lambda(a2, wo)) + ggx_lambda(a2, wi));
    float c = dot(wo, h);
    if (c < 0.0f) c = 0.0f;
    const float common = (D * G2) / (4.0f * wo.z);
    return mk(schlick(kd.x, c) * common, schlick(kd.y, c) * common, schlick(kd.z, c) * common);
}
__device__ __forceinline__ bool ggx_sample(f3 kd, float alpha, f3 n, f3 wo_w, float sp, float cp, float x2,
                                           f3& wi_w, f3& fa, float& pa) {
    const Frame3 F = make_frame(n);
    const f3 wo = to_local(F, wo_w);
    if (!(wo.z > 0.0f)) return false;
    const f3 Vh = normalize(mk(alpha * wo.x, alpha * wo.y, wo.z));
    const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    const f3 T1 = lensq > 0.0f ? divs(mk(-Vh.y, Vh.x, 0.0f), sqrtf(lensq)) : mk(1.0f, 0.0f, 0.0f);
    const f3 T2 = cross(Vh, T1);
    const float r = sqrtf(x2);
    const float t1 = r * cp;
    float t2 = r * sp;
    const float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    const float tz2 = (1.0f - t1 * t1) - t2 * t2;
    const float tz = sqrtf(tz2 > 0.0f ? tz2 : 0.0f);
    const f3 Nh = ((T1 * t1) + (T2 * t2)) + (Vh * tz);
    const f3 h = normalize(mk(alpha * Nh.x, alpha * Nh.y, Nh.z > 0.0f ? Nh.z : 0.0f));
    float c = dot(wo, h);
    const f3 wi = (h * (2.0f * c)) - wo;
    if (!(wi.z > 0.0f)) return false;
    const float a2 = alpha * alpha;
    const float Lo = ggx_lambda(a2, wo), Li = ggx_lambda(a2, wi);
    const float G1 = 1.0f / (1.0f + Lo);
    const float G2 = 1.0f / ((1.0f + Lo) + Li);
    const float pdf = (G1 * ggx_D(a2, h.z)) / (4.0f * wo.z);
    const float w = G2 / G1;
    if (c < 0.0f) c = 0.0f;
    fa = mk((schlick(kd.x, c) * w) * pdf, (schlick(kd.y, c) * w) * pdf, (schlick(kd.z, c) * w) * pdf);
    pa = pdf;
    wi_w = normalize(to_world(F, wi));
    return true;
}

__device__ __forceinline__ bool finite3(float a, float b, float c) {
    return isfinite(a) && isfinite(b) && isfinite(c);
}

// density of ggx_sample's direction (visible-normal sampling) at wi_w
__device__ __forceinline__ float ggx_pdf(float alpha, f3 n, f3 wo_w, f3 wi_w) {
    const Frame3 F = make_frame(n);
    const f3 wo = to_local(F, wo_w), wi = to_local(F, wi_w);
    if (!(wo.z > 0.0f) || !(wi.z > 0.0f)) return 0.0f;
    const f3 h = normalize(wo + wi);
    const float a2 = alpha * alpha;
    const float G1 = 1.0f / (1.0f + ggx_lambda(a2, wo));
    return (G1 * ggx_D(a2, h.z)) / (4.0f * wo.z);
}

}  // namespace trk
