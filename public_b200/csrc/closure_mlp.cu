// Subgrid-closure MLP on the 5th-generation tensor cores (tcgen05, BF16 operands in shared memory,
// FP32 accumulators in TMEM).  No counterpart in the reference: CRUNA has no learned component.
//
// Network: 12 normalised features -> 64 -> 64 (GELU, erf form) -> 6 subgrid-stress components.
// Parameters are FP32 masters (5382 values: W1[64][12], b1, W2[64][64], b2, W3[6][64], b3); every
// kernel rounds them to BF16 as it stages them in shared memory.  One CTA of 128 threads processes
// tiles of 128 samples (the MMA's M): thread t owns sample t of the tile and TMEM lane t.
//   forward  (k_mlp_forward): x -> [MMA K=16, N=64] -> GELU -> [MMA K=64, N=64] -> GELU ->
//            [MMA K=64, N=16] -> y; inference for the coarse solver and the training loss.
//   gradient (k_mlp_grad):    forward, then dy -> dH2 = dy W3, dZ2 = dH2 * GELU'(z2) ->
//            dH1 = dZ2 W2, dZ1 = dH1 * GELU'(z1), and the weight gradients as tensor-core products
//            over the samples (K = 128 per tile, accumulated in TMEM across the CTA's tiles); a row of
//            ones appended to one operand yields each bias gradient in the same product.
// Per-CTA partial gradients are summed in a fixed order (deterministic); Adam updates the masters.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cruna_b200.h"
#include "cruna_internal.cuh"
#include "mlp_common.cuh"
#include "tcgen05.cuh"

namespace cruna {
namespace mlp {

__device__ __forceinline__ void load_features(const float *__restrict__ X, long long row, bool valid,
                                              const Scaling &sc, float *x) {
#pragma unroll
  for (int f = 0; f < 16; ++f) x[f] = 0.0f;
  if (valid) {
#pragma unroll
    for (int f = 0; f < IN; ++f) x[f] = (X[row * IN + f] - sc.in_mean[f]) * sc.in_inv[f];
  }
}

// ------------------------------------------------------------------------------------------------
// forward
// ------------------------------------------------------------------------------------------------
struct FwdSmem {
  __nv_bfloat16 W1[HID * 16];
  __nv_bfloat16 W2[HID * HID];
  __nv_bfloat16 W3[16 * HID];
  __nv_bfloat16 X[128 * 16];
  __nv_bfloat16 H1[128 * HID];
  __nv_bfloat16 H2[128 * HID];
  float b1[HID], b2[HID], b3[16];
  uint64_t mbar;
  uint32_t tmem;
};

__global__ void __launch_bounds__(128) k_mlp_forward(const float *__restrict__ P, const __grid_constant__ Scaling sc,
                                                     const float *__restrict__ X, float *__restrict__ Y, long long n,
                                                     int *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  FwdSmem &S = *reinterpret_cast<FwdSmem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  stage_weights(P, S.W1, S.W2, S.W3, nullptr, nullptr);
  if (tid < HID) {
    S.b1[tid] = P[OB1 + tid];
    S.b2[tid] = P[OB2 + tid];
  }
  if (tid < 16) S.b3[tid] = tid < OUT ? P[OB3 + tid] : 0.0f;
  if (tid == 0) tc::mbar_init(&S.mbar, 1);
  if (warp == 0) tc::tmem_alloc(&S.tmem, 128);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tb = S.tmem, lane = (uint32_t)(warp * 32) << 16;
  const uint32_t aX = tc::smem_addr(S.X), aH1 = tc::smem_addr(S.H1), aH2 = tc::smem_addr(S.H2);
  const uint32_t aW1 = tc::smem_addr(S.W1), aW2 = tc::smem_addr(S.W2), aW3 = tc::smem_addr(S.W3);
  uint32_t phase = 0;
  int ok = 1;
  const long long ntiles = (n + 127) / 128;
  // raw features of the block's next tile, loaded one tile ahead so their latency overlaps the
  // current tile's three products
  float raw[IN];
  auto fetch = [&](long long t) {
    const long long r = t * 128 + tid;
    const bool ld = t < ntiles && r < n;
#pragma unroll
    for (int f = 0; f < IN; ++f) raw[f] = ld ? X[r * IN + f] : 0.0f;
  };
  fetch(blockIdx.x);
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long row = tile * 128 + tid;
    const bool valid = row < n;
    float v[16];
#pragma unroll
    for (int f = 0; f < 16; ++f) v[f] = 0.0f;
    if (valid) {  // load_features' transform
#pragma unroll
      for (int f = 0; f < IN; ++f) v[f] = (raw[f] - sc.in_mean[f]) * sc.in_inv[f];
    }
    put8(S.X, tid, 0, 16, v);
    put8(S.X, tid, 8, 16, v + 8);
    fetch(tile + gridDim.x);
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      tc::gemm_bf16(tb + 0, aX, aW1, 16, 64, false);
      tc::commit(&S.mbar);
    }
    ok = __syncthreads_and(tc::mbar_wait(&S.mbar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    tc::fence_after();
    for (int c = 0; c < 4; ++c) {
      tc::tmem_ld16(tb + lane + c * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + S.b1[c * 16 + i]);
      put8(S.H1, tid, c * 16, 64, v);
      put8(S.H1, tid, c * 16 + 8, 64, v + 8);
    }
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      tc::gemm_bf16(tb + 64, aH1, aW2, 64, 64, false);
      tc::commit(&S.mbar);
    }
    ok = __syncthreads_and(tc::mbar_wait(&S.mbar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    tc::fence_after();
    for (int c = 0; c < 4; ++c) {
      tc::tmem_ld16(tb + lane + 64 + c * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + S.b2[c * 16 + i]);
      put8(S.H2, tid, c * 16, 64, v);
      put8(S.H2, tid, c * 16 + 8, 64, v + 8);
    }
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      tc::gemm_bf16(tb + 0, aH2, aW3, 64, 16, false);
      tc::commit(&S.mbar);
    }
    ok = __syncthreads_and(tc::mbar_wait(&S.mbar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    tc::fence_after();
    tc::tmem_ld16(tb + lane + 0, v);
    if (valid) {
#pragma unroll
      for (int o = 0; o < OUT; ++o) Y[row * OUT + o] = (v[o] + S.b3[o]) * sc.out_scale[o];
    }
    tc::fence_before();
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    tc::mbar_wait(&S.mbar, phase, kWaitLimit);  // let an MMA still in flight finish before the free
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0) tc::tmem_free(tb, 128);
}

// ------------------------------------------------------------------------------------------------
// gradient of the mean squared error over a batch (samples gathered through idx)
// ------------------------------------------------------------------------------------------------
// TMEM columns (256 allocated): per tile A = D1 / dH2, B = D2 / dH1, C = D3; accumulated over the
// CTA's tiles: P2 = dW2 | db2 (80 columns), P3 = dW3^T | db3 row, P1 = dW1 | db1.
constexpr uint32_t C_A = 0, C_B = 64, C_P2 = 128, C_C = 208, C_P3 = 224, C_P1 = 240;

struct GradSmem {
  __nv_bfloat16 W1[HID * 16];     // B [64][16]
  __nv_bfloat16 W2[HID * HID];    // B [64][64]
  __nv_bfloat16 W3[16 * HID];     // B [16][64]
  __nv_bfloat16 W3T[HID * 16];    // B [64][16]
  __nv_bfloat16 W2T[HID * HID];   // B [64][64]
  __nv_bfloat16 X[128 * 16];      // A [128][16]
  __nv_bfloat16 XT[16 * 128];     // B [16][128]: rows 0..11 features, row 12 ones
  __nv_bfloat16 H1T[80 * 128];    // B [80][128]: rows 0..63 h1, row 64 ones
  __nv_bfloat16 dY[128 * 16];     // A [128][16]
  __nv_bfloat16 dYT[16 * 128];    // B [16][128]: rows 0..5 dy
  // A operands with fewer than 128 meaningful rows: rows past the end read the next array (results of
  // those rows are discarded), so these four stay in this order
  __nv_bfloat16 H2T[80 * 128];    // A: rows 0..63 h2, row 64 ones
  __nv_bfloat16 dZ2T[64 * 128];   // A
  __nv_bfloat16 dZ1T[64 * 128];   // A
  __nv_bfloat16 H2[128 * HID];    // A [128][64]
  __nv_bfloat16 H1[128 * HID];    // A [128][64], then dZ2 in the backward pass
  float g1[HID * 128];            // GELU'(z1), [j][sample]
  float g2[HID * 128];            // GELU'(z2)
  float b1[HID], b2[HID], b3[16];
  float loss[4];
  uint64_t mbar;
  uint32_t tmem;
};

__device__ __forceinline__ bool step_wait(GradSmem &S, uint32_t &phase, int &ok) {
  ok = __syncthreads_and(tc::mbar_wait(&S.mbar, phase, kWaitLimit));
  phase ^= 1;
  return ok;
}

__global__ void __launch_bounds__(128, 1) k_mlp_grad(const float *__restrict__ P, const __grid_constant__ Scaling sc,
                                                     const float *__restrict__ X, const float *__restrict__ Yt,
                                                     const int *__restrict__ idx, int batch,
                                                     float *__restrict__ partial, int *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  stage_weights(P, S.W1, S.W2, S.W3, S.W3T, S.W2T);
  if (tid < HID) {
    S.b1[tid] = P[OB1 + tid];
    S.b2[tid] = P[OB2 + tid];
  }
  if (tid < 16) S.b3[tid] = tid < OUT ? P[OB3 + tid] : 0.0f;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f), one = __float2bfloat16_rn(1.0f);
  for (int s = tid; s < 128; s += 128) {  // constant rows: ones and zero padding
    for (int r = 12; r < 16; ++r) S.XT[tc::kmaj(r, s, 128)] = r == 12 ? one : zero;
    for (int r = 64; r < 80; ++r) {
      S.H1T[tc::kmaj(r, s, 128)] = r == 64 ? one : zero;
      S.H2T[tc::kmaj(r, s, 128)] = r == 64 ? one : zero;
    }
    for (int r = OUT; r < 16; ++r) S.dYT[tc::kmaj(r, s, 128)] = zero;
  }
  if (tid == 0) tc::mbar_init(&S.mbar, 1);
  if (warp == 0) tc::tmem_alloc(&S.tmem, 256);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tb = S.tmem, lane = (uint32_t)(warp * 32) << 16;
  const uint32_t aX = tc::smem_addr(S.X), aXT = tc::smem_addr(S.XT), aH1 = tc::smem_addr(S.H1),
                 aH1T = tc::smem_addr(S.H1T), aH2 = tc::smem_addr(S.H2), aH2T = tc::smem_addr(S.H2T),
                 adY = tc::smem_addr(S.dY), adYT = tc::smem_addr(S.dYT), adZ2T = tc::smem_addr(S.dZ2T),
                 adZ1T = tc::smem_addr(S.dZ1T);
  const uint32_t aW1 = tc::smem_addr(S.W1), aW2 = tc::smem_addr(S.W2), aW3 = tc::smem_addr(S.W3),
                 aW3T = tc::smem_addr(S.W3T), aW2T = tc::smem_addr(S.W2T);
  const float dscale = 2.0f / ((float)batch * (float)OUT);
  uint32_t phase = 0;
  int ok = 1;
  float lsum = 0.0f;
  const int ntiles = batch / 128;
  bool first = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long long row = idx[tile * 128 + tid];
    float v[16], t[OUT];
    load_features(X, row, true, sc, v);
#pragma unroll
    for (int o = 0; o < OUT; ++o) t[o] = Yt[row * OUT + o] / sc.out_scale[o];
    put8(S.X, tid, 0, 16, v);
    put8(S.X, tid, 8, 16, v + 8);
#pragma unroll
    for (int f = 0; f < IN; ++f) S.XT[tc::kmaj(f, tid, 128)] = __float2bfloat16_rn(v[f]);
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {  // z1 = x W1^T
      tc::fence_after();
      tc::gemm_bf16(tb + C_A, aX, aW1, 16, 64, false);
      tc::commit(&S.mbar);
    }
    if (!step_wait(S, phase, ok)) break;
    tc::fence_after();
    for (int c = 0; c < 4; ++c) {
      tc::tmem_ld16(tb + lane + C_A + c * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = c * 16 + i;
        const float z = v[i] + S.b1[j];
        float gz;
        v[i] = gelu_and_grad(z, gz);
        S.g1[j * 128 + tid] = gz;
        S.H1T[tc::kmaj(j, tid, 128)] = __float2bfloat16_rn(v[i]);
      }
      put8(S.H1, tid, c * 16, 64, v);
      put8(S.H1, tid, c * 16 + 8, 64, v + 8);
    }
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {  // z2 = h1 W2^T
      tc::fence_after();
      tc::gemm_bf16(tb + C_B, aH1, aW2, 64, 64, false);
      tc::commit(&S.mbar);
    }
    if (!step_wait(S, phase, ok)) break;
    tc::fence_after();
    for (int c = 0; c < 4; ++c) {
      tc::tmem_ld16(tb + lane + C_B + c * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = c * 16 + i;
        const float z = v[i] + S.b2[j];
        float gz;
        v[i] = gelu_and_grad(z, gz);
        S.g2[j * 128 + tid] = gz;
        S.H2T[tc::kmaj(j, tid, 128)] = __float2bfloat16_rn(v[i]);
      }
      put8(S.H2, tid, c * 16, 64, v);
      put8(S.H2, tid, c * 16 + 8, 64, v + 8);
    }
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {  // y = h2 W3^T
      tc::fence_after();
      tc::gemm_bf16(tb + C_C, aH2, aW3, 64, 16, false);
      tc::commit(&S.mbar);
    }
    if (!step_wait(S, phase, ok)) break;
    tc::fence_after();
    tc::tmem_ld16(tb + lane + C_C, v);
    float dy[16];
#pragma unroll
    for (int o = 0; o < 16; ++o) dy[o] = 0.0f;
#pragma unroll
    for (int o = 0; o < OUT; ++o) {
      const float e = v[o] + S.b3[o] - t[o];
      lsum += e * e;
      dy[o] = dscale * e;
      S.dYT[tc::kmaj(o, tid, 128)] = __float2bfloat16_rn(dy[o]);
    }
    put8(S.dY, tid, 0, 16, dy);
    put8(S.dY, tid, 8, 16, dy + 8);
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {  // dH2 = dy W3; [dW3^T | db3] += [h2 | 1]^T dy
      tc::fence_after();
      tc::gemm_bf16(tb + C_A, adY, aW3T, 16, 64, false);
      tc::gemm_bf16(tb + C_P3, aH2T, adYT, 128, 16, !first);
      tc::commit(&S.mbar);
    }
    if (!step_wait(S, phase, ok)) break;
    tc::fence_after();
    for (int c = 0; c < 4; ++c) {  // dZ2 = dH2 * GELU'(z2), into the H1 array (h1 is done as an A operand)
      tc::tmem_ld16(tb + lane + C_A + c * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = c * 16 + i;
        v[i] = v[i] * S.g2[j * 128 + tid];
        S.dZ2T[tc::kmaj(j, tid, 128)] = __float2bfloat16_rn(v[i]);
      }
      put8(S.H1, tid, c * 16, 64, v);
      put8(S.H1, tid, c * 16 + 8, 64, v + 8);
    }
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {  // dH1 = dZ2 W2; [dW2 | db2] += dZ2^T [h1 | 1]
      tc::fence_after();
      tc::gemm_bf16(tb + C_B, aH1, aW2T, 64, 64, false);
      tc::gemm_bf16(tb + C_P2, adZ2T, aH1T, 128, 80, !first);
      tc::commit(&S.mbar);
    }
    if (!step_wait(S, phase, ok)) break;
    tc::fence_after();
    for (int c = 0; c < 4; ++c) {  // dZ1 = dH1 * GELU'(z1)
      tc::tmem_ld16(tb + lane + C_B + c * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = c * 16 + i;
        S.dZ1T[tc::kmaj(j, tid, 128)] = __float2bfloat16_rn(v[i] * S.g1[j * 128 + tid]);
      }
    }
    tc::fence_before();
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {  // [dW1 | db1] += dZ1^T [x | 1]
      tc::fence_after();
      tc::gemm_bf16(tb + C_P1, adZ1T, aXT, 128, 16, !first);
      tc::commit(&S.mbar);
    }
    if (!step_wait(S, phase, ok)) break;
    tc::fence_after();
    first = false;
  }
  // per-CTA partial gradients: lanes 0..63 hold the rows j / i; lane 64 holds db3
  float *out = partial + (long long)blockIdx.x * (NPARAMS + 1);
  if (ok && !first) {
    float v[16];
    if (warp < 2) {
      const int j = tid;
      for (int c = 0; c < 5; ++c) {
        tc::tmem_ld16(tb + lane + C_P2 + c * 16, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = c * 16 + i;
          if (col < HID) out[OW2 + j * HID + col] = v[i];
          else if (col == HID) out[OB2 + j] = v[i];
        }
      }
      tc::tmem_ld16(tb + lane + C_P1, v);
#pragma unroll
      for (int f = 0; f < IN; ++f) out[OW1 + j * IN + f] = v[f];
      out[OB1 + j] = v[IN];
      tc::tmem_ld16(tb + lane + C_P3, v);
#pragma unroll
      for (int o = 0; o < OUT; ++o) out[OW3 + o * HID + j] = v[o];
    } else if (warp == 2) {
      tc::tmem_ld16(tb + lane + C_P3, v);
      if (tid == 64) {
#pragma unroll
        for (int o = 0; o < OUT; ++o) out[OB3 + o] = v[o];
      }
    }
  } else if (ok) {  // a CTA without tiles contributes zeros
    for (int p = tid; p < NPARAMS; p += 128) out[p] = 0.0f;
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((tid & 31) == 0) S.loss[warp] = lsum;
  __syncthreads();
  if (tid == 0) out[NPARAMS] = ((S.loss[0] + S.loss[1]) + S.loss[2]) + S.loss[3];
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    tc::mbar_wait(&S.mbar, phase, kWaitLimit);
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0) tc::tmem_free(tb, 256);
}

// fixed-order sum of the per-CTA partials: grad[p] = sum_b partial[b][p]; grad[NPARAMS] = loss sum
__global__ void k_reduce(const float *__restrict__ partial, int nblk, float *__restrict__ grad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= NPARAMS; p += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int b = 0; b < nblk; ++b) s += partial[(long long)b * (NPARAMS + 1) + p];
    grad[p] = s;
  }
}

// Adam (Kingma & Ba) with bias correction, eps added to sqrt(v_hat)
__global__ void k_adam(float *__restrict__ P, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NPARAMS; p += gridDim.x * blockDim.x) {
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp;
    const float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    P[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
  }
}

__global__ void k_loss_store(const float *__restrict__ grad, float inv_count, float *__restrict__ hist, int step) {
  if (threadIdx.x == 0 && blockIdx.x == 0) hist[step] = grad[NPARAMS] * inv_count;
}

}  // namespace mlp
}  // namespace cruna

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
using namespace cruna::mlp;

struct cruna_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  Scaling sc{};
  float *P = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *partial = nullptr, *hist = nullptr;
  int *flag = nullptr, *idx = nullptr;
  long long idx_cap = 0;
  int hist_cap = 0;
  long long adam_t = 0;
  bool attrs = false;
};

namespace {

struct MlpError {
  int code;
  std::string msg;
};

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw MlpError{CRUNA_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

template <class F>
int mlp_guard(cruna_mlp *h, F &&f) {
  if (!h) return CRUNA_ERR_ARG;
  try {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    return f();
  } catch (const MlpError &e) {
    h->err = e.msg;
    return e.code;
  } catch (const std::exception &e) {
    h->err = e.what();
    return CRUNA_ERR_CUDA;
  }
}

void set_attrs(cruna_mlp *h) {
  if (h->attrs) return;
  ck(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FwdSmem)),
     "forward smem attribute");
  ck(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem)),
     "gradient smem attribute");
  h->attrs = true;
}

int sm_count(int device) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n > 0 ? n : 148;
}

void check_flag(cruna_mlp *h) {
  int f = 0;
  ck(cudaMemcpyAsync(&f, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "flag copy");
  ck(cudaStreamSynchronize(h->stream), "stream synchronize");
  if (f) {
    ck(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream), "flag reset");
    throw MlpError{CRUNA_ERR_CUDA, "tensor-core MLP kernel timed out waiting for its MMA"};
  }
}

void ensure_idx(cruna_mlp *h, long long n) {
  if (n <= h->idx_cap) return;
  if (h->idx) cudaFree(h->idx);
  h->idx = nullptr;
  ck(cudaMalloc(&h->idx, sizeof(int) * n), "index buffer");
  h->idx_cap = n;
}

// one gradient evaluation of the batch idx[0 .. batch): grad (+ loss sum at NPARAMS)
void run_grad(cruna_mlp *h, const float *X, const float *Y, const int *idx, int batch) {
  set_attrs(h);
  const int tiles = batch / 128;
  const int nblk = std::min(tiles, sm_count(h->device));
  k_mlp_grad<<<nblk, 128, sizeof(GradSmem), h->stream>>>(h->P, h->sc, X, Y, idx, batch, h->partial, h->flag);
  ck(cudaGetLastError(), "k_mlp_grad launch");
  k_reduce<<<(NPARAMS + 256) / 256, 256, 0, h->stream>>>(h->partial, nblk, h->grad);
  ck(cudaGetLastError(), "k_reduce launch");
}

}  // namespace

namespace cruna {
void mlp_device_view(cruna_mlp *h, const float **P, mlp::Scaling *sc, int **flag) {
  *P = h->P;
  *sc = h->sc;
  *flag = h->flag;
}

// forward pass enqueued on a caller's stream (the coarse solver's), no host synchronisation; a wait that
// timed out inside the kernel raises the MLP's error flag, reported by its next checked call
void mlp_forward_stream(cruna_mlp *h, const float *X, float *Y, long long n, cudaStream_t stream) {
  try {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (n <= 0) return;
    set_attrs(h);
    const long long tiles = (n + 127) / 128;
    const int nblk = (int)std::min<long long>(tiles, 4LL * sm_count(h->device));
    k_mlp_forward<<<nblk, 128, sizeof(FwdSmem), stream>>>(h->P, h->sc, X, Y, n, h->flag);
    ck(cudaGetLastError(), "k_mlp_forward launch");
  } catch (const MlpError &e) {
    throw ApiError{e.code, e.msg};
  }
}
}  // namespace cruna

extern "C" {

int cruna_mlp_create(int device, uint64_t seed, cruna_mlp **out) {
  if (!out) return CRUNA_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return CRUNA_ERR_NODEVICE;
  }
  cruna_mlp *h = new cruna_mlp();
  h->device = device;
  int rc = mlp_guard(h, [&]() -> int {
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    const int nblk = 1024;
    ck(cudaMalloc(&h->P, sizeof(float) * NPARAMS), "params");
    ck(cudaMalloc(&h->m, sizeof(float) * NPARAMS), "adam m");
    ck(cudaMalloc(&h->v, sizeof(float) * NPARAMS), "adam v");
    ck(cudaMalloc(&h->grad, sizeof(float) * (NPARAMS + 1)), "grad");
    ck(cudaMalloc(&h->partial, sizeof(float) * (NPARAMS + 1) * nblk), "partials");
    ck(cudaMalloc(&h->flag, sizeof(int)), "flag");
    ck(cudaMemset(h->flag, 0, sizeof(int)), "flag");
    ck(cudaMemset(h->m, 0, sizeof(float) * NPARAMS), "adam m");
    ck(cudaMemset(h->v, 0, sizeof(float) * NPARAMS), "adam v");
    // uniform +-1/sqrt(fan_in) initialisation from a seeded 64-bit Mersenne twister
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<float> p(NPARAMS);
    for (int i = 0; i < NPARAMS; ++i) {
      const double fan = i < OB1 ? IN : (i < OW2 ? IN : (i < OW3 ? HID : HID));
      p[i] = (float)(U(gen) / std::sqrt(fan));
    }
    ck(cudaMemcpy(h->P, p.data(), sizeof(float) * NPARAMS, cudaMemcpyHostToDevice), "params upload");
    for (int f = 0; f < IN; ++f) {
      h->sc.in_mean[f] = 0.0f;
      h->sc.in_inv[f] = 1.0f;
    }
    for (int o = 0; o < OUT; ++o) h->sc.out_scale[o] = 1.0f;
    return CRUNA_OK;
  });
  if (rc != CRUNA_OK) {
    cruna_mlp_free(h);
    return rc;
  }
  *out = h;
  return CRUNA_OK;
}

void cruna_mlp_free(cruna_mlp *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (void *p : {(void *)h->P, (void *)h->m, (void *)h->v, (void *)h->grad, (void *)h->partial, (void *)h->hist,
                  (void *)h->flag, (void *)h->idx})
    if (p) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

const char *cruna_mlp_last_error(const cruna_mlp *h) { return h ? h->err.c_str() : "null handle"; }

int cruna_mlp_set_params(cruna_mlp *h, const float *params) {
  return mlp_guard(h, [&]() -> int {
    if (!params) throw MlpError{CRUNA_ERR_ARG, "null params"};
    ck(cudaMemcpyAsync(h->P, params, sizeof(float) * NPARAMS, cudaMemcpyHostToDevice, h->stream), "params");
    ck(cudaMemsetAsync(h->m, 0, sizeof(float) * NPARAMS, h->stream), "adam m");
    ck(cudaMemsetAsync(h->v, 0, sizeof(float) * NPARAMS, h->stream), "adam v");
    ck(cudaStreamSynchronize(h->stream), "sync");
    h->adam_t = 0;
    return CRUNA_OK;
  });
}

int cruna_mlp_get_params(cruna_mlp *h, float *params) {
  return mlp_guard(h, [&]() -> int {
    if (!params) throw MlpError{CRUNA_ERR_ARG, "null params"};
    ck(cudaMemcpyAsync(params, h->P, sizeof(float) * NPARAMS, cudaMemcpyDeviceToHost, h->stream), "params");
    ck(cudaStreamSynchronize(h->stream), "sync");
    return CRUNA_OK;
  });
}

int cruna_mlp_set_scaling(cruna_mlp *h, const float *in_mean, const float *in_scale, const float *out_scale) {
  return mlp_guard(h, [&]() -> int {
    if (!in_mean || !in_scale || !out_scale) throw MlpError{CRUNA_ERR_ARG, "null scaling"};
    for (int f = 0; f < IN; ++f) {
      if (!(in_scale[f] > 0.0f)) throw MlpError{CRUNA_ERR_ARG, "input scales must be positive"};
      h->sc.in_mean[f] = in_mean[f];
      h->sc.in_inv[f] = 1.0f / in_scale[f];
    }
    for (int o = 0; o < OUT; ++o) {
      if (!(out_scale[o] > 0.0f)) throw MlpError{CRUNA_ERR_ARG, "output scales must be positive"};
      h->sc.out_scale[o] = out_scale[o];
    }
    return CRUNA_OK;
  });
}

int cruna_mlp_forward_dev(cruna_mlp *h, const float *X, float *Y, long long n) {
  return mlp_guard(h, [&]() -> int {
    if (n < 0 || (n > 0 && (!X || !Y))) throw MlpError{CRUNA_ERR_ARG, "bad forward arguments"};
    if (n == 0) return CRUNA_OK;
    set_attrs(h);
    const long long tiles = (n + 127) / 128;
    const int nblk = (int)std::min<long long>(tiles, 4LL * sm_count(h->device));
    k_mlp_forward<<<nblk, 128, sizeof(FwdSmem), h->stream>>>(h->P, h->sc, X, Y, n, h->flag);
    ck(cudaGetLastError(), "k_mlp_forward launch");
    check_flag(h);
    return CRUNA_OK;
  });
}

int cruna_mlp_grad_dev(cruna_mlp *h, const float *X, const float *Y, int n, float *grad_host, float *loss) {
  return mlp_guard(h, [&]() -> int {
    if (n <= 0 || n % 128 != 0 || !X || !Y) throw MlpError{CRUNA_ERR_ARG, "n must be a positive multiple of 128"};
    ensure_idx(h, n);
    std::vector<int> id(n);
    for (int i = 0; i < n; ++i) id[i] = i;
    ck(cudaMemcpyAsync(h->idx, id.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->stream), "indices");
    run_grad(h, X, Y, h->idx, n);
    std::vector<float> g(NPARAMS + 1);
    ck(cudaMemcpyAsync(g.data(), h->grad, sizeof(float) * (NPARAMS + 1), cudaMemcpyDeviceToHost, h->stream), "grad");
    check_flag(h);
    if (grad_host) std::memcpy(grad_host, g.data(), sizeof(float) * NPARAMS);
    if (loss) *loss = g[NPARAMS] / ((float)n * OUT);
    return CRUNA_OK;
  });
}

int cruna_mlp_train_dev(cruna_mlp *h, const float *X, const float *Y, long long n, int batch, int steps, float lr,
                        uint64_t seed, float *loss_hist) {
  return mlp_guard(h, [&]() -> int {
    if (batch <= 0 || batch % 128 != 0 || n < batch || steps < 0 || !X || !Y)
      throw MlpError{CRUNA_ERR_ARG, "need batch a positive multiple of 128, n >= batch, steps >= 0"};
    if (steps > h->hist_cap) {
      if (h->hist) cudaFree(h->hist);
      h->hist = nullptr;
      ck(cudaMalloc(&h->hist, sizeof(float) * std::max(steps, 1)), "loss history");
      h->hist_cap = steps;
    }
    const long long per_epoch = n / batch;
    ensure_idx(h, per_epoch * batch);
    std::mt19937_64 gen(seed);
    std::vector<int> perm(n);
    for (long long i = 0; i < n; ++i) perm[i] = (int)i;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int s = 0; s < steps; ++s) {
      const long long e = s % per_epoch;
      if (e == 0) {  // new epoch: reshuffle, upload the batches of this epoch
        std::shuffle(perm.begin(), perm.end(), gen);
        ck(cudaMemcpyAsync(h->idx, perm.data(), sizeof(int) * per_epoch * batch, cudaMemcpyHostToDevice, h->stream),
           "indices");
        ck(cudaStreamSynchronize(h->stream), "sync");
      }
      run_grad(h, X, Y, h->idx + e * batch, batch);
      ++h->adam_t;
      const float c1 = 1.0f - std::pow(b1, (float)h->adam_t), c2 = 1.0f - std::pow(b2, (float)h->adam_t);
      k_adam<<<(NPARAMS + 255) / 256, 256, 0, h->stream>>>(h->P, h->m, h->v, h->grad, lr, b1, b2, eps, c1, c2);
      ck(cudaGetLastError(), "k_adam launch");
      k_loss_store<<<1, 32, 0, h->stream>>>(h->grad, 1.0f / ((float)batch * OUT), h->hist, s);
      ck(cudaGetLastError(), "k_loss_store launch");
    }
    if (loss_hist && steps > 0)
      ck(cudaMemcpyAsync(loss_hist, h->hist, sizeof(float) * steps, cudaMemcpyDeviceToHost, h->stream), "losses");
    check_flag(h);
    return CRUNA_OK;
  });
}

}  // extern "C"
