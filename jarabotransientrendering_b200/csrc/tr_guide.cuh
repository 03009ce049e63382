// tr_guide.cuh - learned directional proposal: MLP (64 -> 3x64 ReLU -> 40) predicting a mixture
// of 8 von Mises-Fisher lobes, trained online on the renderer's own radiance samples.
// No counterpart in the reference renderer.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace trg {

constexpr int kIn = 64;          // padded feature width
constexpr int kHidden = 64;
constexpr int kLobes = 8;
constexpr int kOut = 5 * kLobes; // per lobe: weight logit, mean xyz (unnormalised), concentration
constexpr int kLayers = 4;
constexpr int kParams = kLayers * 64 * 64 + kLayers * 64;   // weights [l][in][out] then biases [l][out]
constexpr int kTile = 128;       // rows per tcgen05 tile (MMA M)
// default number of mbarrier polls before a wait for a CTA's own tensor-core work times out
constexpr uint32_t kWaitPolls = 1u << 24;
// concentration kappa = kKappaMin + kKappaMax * sigmoid(raw - kKappaShift): about exp(raw - 0.4)
// for small kappa (scale-free Adam steps), smoothly saturating at kKappaMax
constexpr float kKappaMin = 0.05f, kKappaMax = 2000.0f, kKappaShift = 8.0f;

// Features of a surface vertex (46 used of 64, rest zero):
//   [0,36)  sin/cos(2^k pi p_d), k = 0..5, d = x,y,z      (p normalised to the scene box)
//   [36,39) p normalised, [39,42) geometric normal, [42,45) outgoing direction (towards the
//   previous vertex), [45] path length / film time length
constexpr int kFeatUsed = 46;

struct GuideDev {
    const uint4* w_fwd;    // 4 canonical K-major B tiles (Wt: [out][in]) bf16, 8 KB each
    const uint4* w_bwd;    // 4 canonical K-major B tiles (W: [in][out]) bf16
    const float* bias;     // [4][64]
    uint32_t spin;         // polls of an mbarrier before a tensor-core wait counts as timed out
};

// m_dev (optional): the row count in device memory, at most m (rows beyond it are skipped)
cudaError_t mlp_forward(const GuideDev& g, const uint4* x, uint32_t m, float* out, uint4* act, int* err,
                        cudaStream_t s, const uint32_t* m_dev = nullptr);
cudaError_t mlp_backward(const GuideDev& g, const uint4* dy, const uint4* act, uint32_t m, uint4* dh, int* err,
                         cudaStream_t s);
int mlp_grid(int device);
// CTAs of `kernel` that fit on the device at once (SMs x CTAs per SM, from the kernel's
// registers, shared memory and `tmem_cols` tensor-memory columns per CTA), for persistent loops
int resident_grid(int device, const void* kernel, int threads, size_t dyn_smem, int tmem_cols = 64);
cudaError_t pack_weights(const float* params, uint8_t* w_fwd, uint8_t* w_bwd, cudaStream_t s);
cudaError_t mix_grad(const float* out, const float* dirs, const float* w, uint32_t m, float* wsum, uint4* dy_bf,
                     float* loss, cudaStream_t s);
// weight-gradient operands of the four layers: gw[l] += prev[l]^T grad[l], gb[l] += column sums
struct DwLayers {
    const uint4* prev[4];      // [m][64] bf16 layer inputs (features, H1, H2, H3)
    const uint4* grad_bf[4];   // [m][64] bf16 gradients w.r.t. the layer outputs
    float* gw[4];
    float* gb[4];
};
// tensor-core weight gradients; `spin` bounds each mbarrier wait (timeout: *err = 1)
cudaError_t weight_grad(const DwLayers& L, uint32_t m, uint32_t spin, int* err, cudaStream_t s);
cudaError_t adam(float* params, const float* grads, float* m1, float* m2, uint32_t n, float lr, uint32_t step,
                 cudaStream_t s);

}  // namespace trg
