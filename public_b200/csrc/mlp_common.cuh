// Pieces of the closure MLP shared by its own kernels (closure_mlp.cu) and by the direct pass that
// evaluates it in place (fused.cu): sizes and parameter offsets, the input / output scaling, the GELU
// with its erf approximation, and the staging of BF16 operands in the canonical K-major layout of
// tcgen05.mma (tcgen05.cuh).  No counterpart in the reference: CRUNA has no learned component.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "../../include/cruna_b200.h"
#include "tcgen05.cuh"

namespace cruna {
namespace mlp {

constexpr int IN = 12, HID = 64, OUT = 6;
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID, OW3 = OB2 + HID,
              OB3 = OW3 + OUT * HID, NPARAMS = OB3 + OUT;
static_assert(NPARAMS == CRUNA_MLP_NPARAMS, "parameter count");
constexpr long long kWaitLimit = 1LL << 22;  // mbarrier polls before a kernel gives up (error flag)

struct Scaling {
  float in_mean[IN];
  float in_inv[IN];   // 1 / in_scale
  float out_scale[OUT];
};

// erf by the rational approximation of Abramowitz & Stegun, Handbook of Mathematical Functions, 7.1.26
// (|error| <= 1.5e-7, far below the BF16 rounding of the activations), with fast reciprocal and
// exponential; e2 returns exp(-x^2) for the GELU derivative.  The activations cost most of the
// forward kernel's instructions, so this replaces erff.
__device__ __forceinline__ float erf_as(float x, float &e2) {
  const float ax = fabsf(x);
  const float t = __fdividef(1.0f, fmaf(0.3275911f, ax, 1.0f));
  float p = fmaf(1.061405429f, t, -1.453152027f);
  p = fmaf(p, t, 1.421413741f);
  p = fmaf(p, t, -0.284496736f);
  p = fmaf(p, t, 0.254829592f);
  e2 = __expf(-ax * ax);
  return copysignf(1.0f - p * t * e2, x);
}

// GELU (erf form) 0.5 z (1 + erf(z / sqrt 2)) and its derivative Phi(z) + z phi(z)
__device__ __forceinline__ float gelu(float z) {
  float e2;
  return 0.5f * z * (1.0f + erf_as(z * 0.70710678118654752f, e2));
}
__device__ __forceinline__ float gelu_and_grad(float z, float &grad) {
  float e2;  // exp(-z^2 / 2)
  const float cdf = 0.5f * (1.0f + erf_as(z * 0.70710678118654752f, e2));
  grad = cdf + z * e2 * 0.39894228040143268f;
  return z * cdf;
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // .x = a (low half), .y = b
  return *reinterpret_cast<uint32_t *>(&h);
}

// 8 consecutive row elements (k0 .. k0+7, k0 % 8 == 0) of row r of an R x K tile
__device__ __forceinline__ void put8(__nv_bfloat16 *tile, int r, int k0, int K, const float *v) {
  uint4 u;
  u.x = pack2(v[0], v[1]);
  u.y = pack2(v[2], v[3]);
  u.z = pack2(v[4], v[5]);
  u.w = pack2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(tile + tc::kmaj(r, k0, K)) = u;
}

// stage weights as B operands ([N][K], K-major); transposed copies for the backward products
__device__ inline void stage_weights(const float *__restrict__ P, __nv_bfloat16 *W1, __nv_bfloat16 *W2, __nv_bfloat16 *W3,
                              __nv_bfloat16 *W3T, __nv_bfloat16 *W2T) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < HID * 16; i += nt) {
    const int r = i >> 4, k = i & 15;
    W1[tc::kmaj(r, k, 16)] = __float2bfloat16_rn(k < IN ? P[OW1 + r * IN + k] : 0.0f);
  }
  for (int i = tid; i < HID * HID; i += nt) {
    const int r = i >> 6, k = i & 63;
    W2[tc::kmaj(r, k, 64)] = __float2bfloat16_rn(P[OW2 + r * HID + k]);
    if (W2T) W2T[tc::kmaj(k, r, 64)] = __float2bfloat16_rn(P[OW2 + r * HID + k]);
  }
  for (int i = tid; i < 16 * HID; i += nt) {
    const int r = i >> 6, k = i & 63;
    const float w = r < OUT ? P[OW3 + r * HID + k] : 0.0f;
    W3[tc::kmaj(r, k, 64)] = __float2bfloat16_rn(w);
    if (W3T) W3T[tc::kmaj(k, r, 16)] = __float2bfloat16_rn(w);  // [64][16]: (j, o) = W3[o][j]
  }
}

}  // namespace mlp

// device parameters, scaling and error flag of a network (closure_mlp.cu), for kernels that evaluate
// it in place
void mlp_device_view(struct cruna_mlp *h, const float **P, mlp::Scaling *sc, int **flag);

}  // namespace cruna
