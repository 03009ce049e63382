// tr_guide_math.cuh - von Mises-Fisher mixture of the learned proposal (decode, density,
// sampling); shared by the training kernels and the guided path-sampling kernel.
#pragma once
#include <cstdint>
#include "tr_guide.cuh"

namespace trg {

// vMF mixture decoding shared by sampling and training
struct Lobe { float pi, mx, my, mz, kappa, mnorm, sig; };

__device__ __forceinline__ float softplusf(float x) { return x > 20.0f ? x : log1pf(expf(x)); }

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
        const float kr = o[5 * j + 4];
        L[j].kappa = fminf(softplusf(kr) + kKappaMin, kKappaMax);
        L[j].sig = (softplusf(kr) + kKappaMin < kKappaMax) ? 1.0f / (1.0f + expf(-kr)) : 0.0f;
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

}  // namespace trg
