// tr_guide_math.cuh - von Mises-Fisher mixture of the learned proposal (decode, density,
// sampling); shared by the training kernels and the guided path-sampling kernel.
#pragma once
#include <cstdint>
#include "tr_guide.cuh"

namespace trg {

// vMF mixture decoding shared by sampling and training
struct Lobe { float pi, mx, my, mz, kappa, mnorm, sig; };     // sig = d kappa / d raw

__device__ __forceinline__ void decode_mixture(const float* o, Lobe* L) {
    float amax = -3.4e38f;
#pragma unroll
    for (int j = 0; j < kLobes; ++j) amax = fmaxf(amax, o[5 * j]);
    float sum = 0.0f;
#pragma unroll
    for (int j = 0; j < kLobes; ++j) { L[j].pi = expf(o[5 * j] - amax); sum += L[j].pi; }
#pragma unroll
    for (int j = 0; j < kLobes; ++j) {
        L[j].pi /= sum;
        const float x = o[5 * j + 1], y = o[5 * j + 2], z = o[5 * j + 3];
        float n = sqrtf(x * x + y * y + z * z);
        if (!(n > 1e-6f)) { L[j].mx = 0.0f; L[j].my = 0.0f; L[j].mz = 1.0f; n = 1e-6f; }
        else { L[j].mx = x / n; L[j].my = y / n; L[j].mz = z / n; }
        L[j].mnorm = n;
        const float sg = 1.0f / (1.0f + expf(kKappaShift - o[5 * j + 4]));
        L[j].kappa = kKappaMin + kKappaMax * sg;
        L[j].sig = kKappaMax * sg * (1.0f - sg);
    }
}
// log of the normalised vMF density, stable for small and large kappa
__device__ __forceinline__ float log_vmf(float kappa, float cosang) {
    return logf(kappa) - 1.83787706f /* log 2pi */ - log1pf(-expf(-2.0f * kappa)) + kappa * (cosang - 1.0f);
}


// density of the mixture at unit direction (dx, dy, dz)
__device__ __forceinline__ float mixture_pdf(const Lobe* L, float dx, float dy, float dz) {
    float q = 0.0f;
#pragma unroll
    for (int j = 0; j < kLobes; ++j) {
        const float c = L[j].mx * dx + L[j].my * dy + L[j].mz * dz;
        q += L[j].pi * expf(log_vmf(L[j].kappa, c));
    }
    return q;
}

// Draws a direction: lobe by its weight (u0), then the vMF sampler of Jakob 2012 ("Numerically
// stable sampling of the von Mises Fisher distribution on S^2"): w = 1 + log(u1 + (1-u1)
// exp(-2 kappa)) / kappa, azimuth 2 pi u2 in an orthonormal frame around the mean.
__device__ __forceinline__ void mixture_sample(const Lobe* L, float u0, float u1, float u2, float* d) {
    // lobe j is the first whose cumulative weight exceeds u0 (the last if rounding leaves none);
    // unrolled selects keep the lobes in registers
    float kap = L[kLobes - 1].kappa, mx = L[kLobes - 1].mx, my = L[kLobes - 1].my, mz = L[kLobes - 1].mz;
    float cum = 0.0f;
    bool found = false;
#pragma unroll
    for (int j = 0; j < kLobes - 1; ++j) {
        cum += L[j].pi;
        const bool take = !found && u0 < cum;
        kap = take ? L[j].kappa : kap;
        mx = take ? L[j].mx : mx;
        my = take ? L[j].my : my;
        mz = take ? L[j].mz : mz;
        found = found || take;
    }
    float w = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * kap)) / kap;
    w = fminf(fmaxf(w, -1.0f), 1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    const float sg = copysignf(1.0f, mz);
    const float a = -1.0f / (sg + mz);
    const float b = mx * my * a;
    float sp, cp;
    sincospif(2.0f * u2, &sp, &cp);
    const float t1x = 1.0f + sg * mx * mx * a, t1y = sg * b, t1z = -sg * mx;
    const float t2x = b, t2y = sg + my * my * a, t2z = -my;
    d[0] = w * mx + s * (cp * t1x + sp * t2x);
    d[1] = w * my + s * (cp * t1y + sp * t2y);
    d[2] = w * mz + s * (cp * t1z + sp * t2z);
}

// ---------------------------------------------------------------------------------------------
// Renderer-side mixture: decoded once per vertex into what sampling and density evaluation
// need, with the fast hardware approximations of exp/log/rsqrt/division.  The sampler and the
// density read the same decoded values, so the density used in the MIS weight is the one of
// the sampling procedure up to float rounding (relative ~1e-6).
//   e_j    = exp(a_j - max a)                     (unnormalised lobe weight)
//   coef_j = pi_j * kappa_j / (2 pi (1 - exp(-2 kappa_j)))
//   pdf(w) = sum_j coef_j exp(kappa_j (mu_j . w - 1))
// ---------------------------------------------------------------------------------------------
struct SampLobe { float e, mx, my, mz, kappa, coef; };

// returns sum_j e_j
__device__ __forceinline__ float decode_sampling(const float* o, SampLobe* L) {
    float amax = o[0];
#pragma unroll
    for (int j = 1; j < kLobes; ++j) amax = fmaxf(amax, o[5 * j]);
    float sum = 0.0f;
#pragma unroll
    for (int j = 0; j < kLobes; ++j) {
        L[j].e = __expf(o[5 * j] - amax);
        sum += L[j].e;
        const float x = o[5 * j + 1], y = o[5 * j + 2], z = o[5 * j + 3];
        const float n2 = fmaf(x, x, fmaf(y, y, z * z));
        if (n2 > 1e-12f) {
            const float r = rsqrtf(n2);
            L[j].mx = x * r; L[j].my = y * r; L[j].mz = z * r;
        } else {
            L[j].mx = 0.0f; L[j].my = 0.0f; L[j].mz = 1.0f;
        }
        L[j].kappa = kKappaMin + kKappaMax * __frcp_rn(1.0f + __expf(kKappaShift - o[5 * j + 4]));
    }
    const float inv_sum = __frcp_rn(sum);
#pragma unroll
    for (int j = 0; j < kLobes; ++j) {
        const float k = L[j].kappa;
        L[j].coef = __fdividef(L[j].e * inv_sum * k * 0.159154943f /* 1/(2 pi) */, 1.0f - __expf(-2.0f * k));
    }
    return sum;
}

__device__ __forceinline__ float sampling_pdf(const SampLobe* L, float dx, float dy, float dz) {
    float q = 0.0f;
#pragma unroll
    for (int j = 0; j < kLobes; ++j) {
        const float c = fmaf(L[j].mx, dx, fmaf(L[j].my, dy, L[j].mz * dz));
        q = fmaf(L[j].coef, __expf(L[j].kappa * (c - 1.0f)), q);
    }
    return q;
}

// lobe by u0 * sum of e_j, then Jakob 2012 within the lobe (see mixture_sample)
__device__ __forceinline__ void sampling_draw(const SampLobe* L, float sum, float u0, float u1, float u2, float* d) {
    float kap = L[kLobes - 1].kappa, mx = L[kLobes - 1].mx, my = L[kLobes - 1].my, mz = L[kLobes - 1].mz;
    const float t = u0 * sum;
    float cum = 0.0f;
    bool found = false;
#pragma unroll
    for (int j = 0; j < kLobes - 1; ++j) {
        cum += L[j].e;
        const bool take = !found && t < cum;
        kap = take ? L[j].kappa : kap;
        mx = take ? L[j].mx : mx;
        my = take ? L[j].my : my;
        mz = take ? L[j].mz : mz;
        found = found || take;
    }
    float w = 1.0f + __fdividef(__logf(u1 + (1.0f - u1) * __expf(-2.0f * kap)), kap);
    w = fminf(fmaxf(w, -1.0f), 1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - w * w));
    const float sg = copysignf(1.0f, mz);
    const float a = -__frcp_rn(sg + mz);
    const float b = mx * my * a;
    float sp, cp;
    __sincosf(6.283185307f * u2, &sp, &cp);
    const float t1x = 1.0f + sg * mx * mx * a, t1y = sg * b, t1z = -sg * mx;
    const float t2x = b, t2y = sg + my * my * a, t2z = -my;
    d[0] = fmaf(w, mx, s * fmaf(cp, t1x, sp * t2x));
    d[1] = fmaf(w, my, s * fmaf(cp, t1y, sp * t2y));
    d[2] = fmaf(w, mz, s * fmaf(cp, t1z, sp * t2z));
}

}  // namespace trg
