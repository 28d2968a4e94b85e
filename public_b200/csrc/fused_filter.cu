// Fused filter_i1 -> filter_i2 -> filter_i3 sequence (src/main/computation_direct.f90:85-95,
// src/filter/filter_i*_mpi_cartesian.f90) for the explicit periodic 10th-order filter (no reference
// counterpart: the interior stencil of filter_pen_core_o10_i_c_o.f90:182-199 at alpha = 0 with
// periodic wrap, blended q <- q - s*(q - F q)).
//
// Two passes apply the three directional filters in the reference's order to all five variables:
// pass 1 filters each plane in x and then y on 32 x 32 tiles with 5-wide halos (corners included,
// so the y filter sees x-filtered halo rows); pass 2 filters in z with a per-thread register queue
// of 11 planes.  Each pass reads and writes the state once.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "cruna_internal.cuh"
#include "fused_common.cuh"
#include "tcgen05.cuh"

namespace cruna {

namespace {

constexpr int FR = 5;    // o10 filter half-width
constexpr int FXT = 32, FYT = 32, FTHR = 256;

struct FilterArgs {
  Grid g;
  int n[3];
  int on[3];             // direction filtered this step
  double c[FR + 1];      // interior coefficients a0..a5
  double blend;          // strength s
  int kc;
  const double *in;
  double *out;
};

__device__ __forceinline__ int wrapi(int g, int n) { return ((g % n) + n) % n; }

// F q with the blend, in the oracle's order: t = a0*q; t += a_m*(q_{+m}+q_{-m}); q - s*(q - t)
__device__ __forceinline__ double filt(const FilterArgs &a, const double *p, int s) {
  double t = a.c[0] * p[0];
#pragma unroll
  for (int m = 1; m <= FR; ++m) t = t + a.c[m] * (p[m * s] + p[-m * s]);
  return p[0] - a.blend * (p[0] - t);
}

// pass 1: x then y filter of one plane, one variable at a time (tile offsets computed once).
// Both directional filters read their taps from per-thread register windows: the x filter takes
// XQ consecutive points of one row from the tile stored transposed (raw[x][y], consecutive threads on
// consecutive rows), the y filter RPT consecutive points of one column; the odd row pitches RTS and XFS
// keep every shared-memory access free of bank conflicts.
__global__ void __launch_bounds__(FTHR, 4) k_filter_xy(const __grid_constant__ FilterArgs a) {
  constexpr int PW = FXT + 2 * FR, PH = FYT + 2 * FR;
  constexpr int NL = (PW * PH + FTHR - 1) / FTHR;
  constexpr int RTS = PH + 1, XFS = FXT + 1;
  __shared__ double raw[PW * RTS];  // raw[lx * RTS + ly], halo coordinates
  __shared__ double xf[PH * XFS];   // xf[ly * XFS + x]
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * FXT, j0 = blockIdx.y * FYT, k = blockIdx.z;
  const long long N = a.g.N, n1 = a.g.n1, n12 = (long long)a.g.n1 * a.g.n2;
  const long long kofs = n12 * k;
  int goff[NL];
#pragma unroll
  for (int m = 0; m < NL; ++m) {
    const int c = tid + m * FTHR;
    goff[m] = -1;
    if (c < PW * PH) {
      const int lx = c % PW - FR, ly = c / PW - FR;
      const int gi = a.on[0] ? wrapi(i0 + lx, a.n[0]) : min(max(i0 + lx, 0), a.n[0] - 1);
      const int gj = a.on[1] ? wrapi(j0 + ly, a.n[1]) : min(max(j0 + ly, 0), a.n[1] - 1);
      goff[m] = gi + (int)n1 * gj;
    }
  }
  double nxt[NL];
#pragma unroll
  for (int m = 0; m < NL; ++m)
    if (goff[m] >= 0) nxt[m] = a.in[goff[m] + kofs];
  for (int v = 0; v < 5; ++v) {
    double *out = a.out + v * N;
#pragma unroll
    for (int m = 0; m < NL; ++m) {
      const int c = tid + m * FTHR;
      if (goff[m] >= 0) raw[(c % PW) * RTS + c / PW] = nxt[m];
    }
    if (v + 1 < 5) {
      const double *in1 = a.in + (v + 1) * N;
#pragma unroll
      for (int m = 0; m < NL; ++m)
        if (goff[m] >= 0) nxt[m] = in1[goff[m] + kofs];
    }
    __syncthreads();
    {  // x filter: each thread takes XQ consecutive points of a row (all PH rows, halo rows included)
      constexpr int XQ = 4, NXW = XQ + 2 * FR;
      for (int t = tid; t < PH * (FXT / XQ); t += FTHR) {
        const int ly = t % PH, x0 = (t / PH) * XQ;
        if (a.on[0]) {
          double w[NXW];
#pragma unroll
          for (int m = 0; m < NXW; ++m) w[m] = raw[(x0 + m) * RTS + ly];
#pragma unroll
          for (int u = 0; u < XQ; ++u) xf[ly * XFS + x0 + u] = filt(a, w + u + FR, 1);
        } else {
#pragma unroll
          for (int u = 0; u < XQ; ++u) xf[ly * XFS + x0 + u] = raw[(x0 + u + FR) * RTS + ly];
        }
      }
    }
    __syncthreads();
    {  // y filter: each thread takes a column and FYT / 8 consecutive rows from a register window
      constexpr int RPT = FYT / (FTHR / FXT), NW = RPT + 2 * FR;
      const int lx = tid % FXT, ly0 = (tid / FXT) * RPT;
      double w[NW];
#pragma unroll
      for (int m = 0; m < NW; ++m) w[m] = xf[(ly0 + m) * XFS + lx];
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const int gi = i0 + lx, gj = j0 + ly0 + r;
        if (gi < a.g.n1 && gj < a.g.n2) out[gi + n1 * gj + kofs] = a.on[1] ? filt(a, w + r + FR, 1) : w[r + FR];
      }
    }
    __syncthreads();
  }
}

// pass 2: z filter, one variable per block (blockIdx.z = chunk * 5 + variable) with a per-thread
// register queue of 2*FR+1 planes, the next plane loaded one step ahead
__global__ void __launch_bounds__(FTHR) k_filter_z(const __grid_constant__ FilterArgs a) {
  constexpr int NQ = 2 * FR + 1;
  const int i = blockIdx.x * 32 + threadIdx.x % 32, j = blockIdx.y * 8 + threadIdx.x / 32;
  if (i >= a.g.n1 || j >= a.g.n2) return;
  const int v = blockIdx.z % 5, chunk = blockIdx.z / 5;
  const int k0 = chunk * a.kc, k1 = min(k0 + a.kc, a.g.n3);
  const long long N = a.g.N, n12 = (long long)a.g.n1 * a.g.n2;
  const long long col = i + (long long)a.g.n1 * j + v * N;
  const int n3 = a.n[2];
  const double *in = a.in + col;
  double *out = a.out + col;
  constexpr int PD = 4;  // planes in flight ahead of the queue
  double q[NQ], nx[PD];
#pragma unroll
  for (int m = 0; m < NQ - 1; ++m) q[m] = in[n12 * wrapi(k0 - FR + m, n3)];
#pragma unroll
  for (int d = 0; d < PD; ++d) nx[d] = (k0 + d < k1) ? in[n12 * wrapi(k0 + FR + d, n3)] : 0.0;
  for (int k = k0; k < k1; ++k) {
    q[NQ - 1] = nx[0];
#pragma unroll
    for (int d = 0; d < PD - 1; ++d) nx[d] = nx[d + 1];
    if (k + PD < k1) nx[PD - 1] = in[n12 * wrapi(k + PD + FR, n3)];
    out[n12 * k] = filt(a, q + FR, 1);
#pragma unroll
    for (int m = 0; m < NQ - 1; ++m) q[m] = q[m + 1];
  }
}

// pass 2 with the loads in shared memory: the block's 32 x 8 tile of one variable streams plane by
// plane into a ring of ZD shared slots by TMA (cp.async.bulk.tensor, issued ZD planes ahead by one
// thread, completion counted on a per-slot mbarrier), so no registers hold loads in flight.  Plane
// coordinates wrap periodically on the host side of each copy.  Every wait is bounded: when one runs
// out the block records it in err, waits (bounded) for its copies in flight and returns.
constexpr int ZD = 8;                          // planes in flight
constexpr long long kTmaWaitLimit = 1LL << 22;

__device__ __forceinline__ void tma_plane(const CUtensorMap *tm, double *dst, uint64_t *bar, int x, int y, int z,
                                          int v) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(bar)), "r"(32 * 8 * 8)
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(tc::smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(v), "r"(tc::smem_addr(bar))
      : "memory");
}

__global__ void __launch_bounds__(FTHR) k_filter_z_tma(const __grid_constant__ CUtensorMap tm,
                                                      const __grid_constant__ FilterArgs a, int *err) {
  constexpr int NQ = 2 * FR + 1;
  __shared__ __align__(128) double ring[ZD][FTHR];
  __shared__ __align__(8) uint64_t full[ZD];
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 8;
  const int i = i0 + tid % 32, j = j0 + tid / 32;
  const int v = blockIdx.z % 5, chunk = blockIdx.z / 5;
  const int k0 = chunk * a.kc, k1 = min(k0 + a.kc, a.g.n3);
  const int n3 = a.n[2];
  const int kfirst = k0 - FR, nplanes = k1 - k0 + 2 * FR;  // planes kfirst .. kfirst + nplanes - 1
  const long long n12 = (long long)a.g.n1 * a.g.n2;
  double *out = a.out + (long long)v * a.g.N + i + (long long)a.g.n1 * j;
  if (tid == 0) {
    for (int s = 0; s < ZD; ++s) tc::mbar_init(&full[s], 1);
    for (int idx = 0; idx < min(ZD, nplanes); ++idx)
      tma_plane(&tm, ring[idx], &full[idx], i0, j0, wrapi(kfirst + idx, n3), v);
  }
  __syncthreads();
  double q[NQ];
  int ok = 1, issued = min(ZD, nplanes);
  for (int idx = 0; idx < nplanes; ++idx) {
    const int s = idx % ZD;
    ok = __syncthreads_and(ok && tc::mbar_wait(&full[s], (uint32_t)((idx / ZD) & 1), kTmaWaitLimit));
    if (!ok) break;
    // every thread is past the read of plane idx - 1: its slot takes plane idx - 1 + ZD
    if (tid == 0 && idx >= 1 && idx - 1 + ZD < nplanes) {
      tc::fence_async_smem();
      const int r = idx - 1 + ZD;
      tma_plane(&tm, ring[r % ZD], &full[r % ZD], i0, j0, wrapi(kfirst + r, n3), v);
      issued = r + 1;
    }
#pragma unroll
    for (int m = 0; m < NQ - 1; ++m) q[m] = q[m + 1];
    q[NQ - 1] = ring[s][tid];
    if (idx >= 2 * FR && i < a.g.n1 && j < a.g.n2) out[n12 * (kfirst + idx - FR)] = filt(a, q + FR, 1);
  }
  if (!ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      // the copies possibly still in flight are the last ZD issued (one per slot, its latest phase)
      for (int r = max(0, issued - ZD); r < issued; ++r)
        tc::mbar_wait(&full[r % ZD], (uint32_t)((r / ZD) & 1), kTmaWaitLimit);
    }
    __syncthreads();
  }
}

// 4-D tensor map (n1, n2, n3, 5) of a Fortran-ordered FP64 state with a 32 x 8 x 1 x 1 box; false
// when the layout does not meet TMA's rules (n1 even, so every row stride is a multiple of 16 bytes)
bool state_tensor_map(const cruna_ctx *c, const double *state, CUtensorMap *tm) {
  if (c->g.n1 % 2 != 0 || (reinterpret_cast<uintptr_t>(state) & 15) != 0) return false;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return false;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[4] = {(cuuint64_t)c->g.n1, (cuuint64_t)c->g.n2, (cuuint64_t)c->g.n3, 5};
  const cuuint64_t strides[3] = {(cuuint64_t)c->g.n1 * 8, (cuuint64_t)c->g.n1 * c->g.n2 * 8,
                                 (cuuint64_t)c->g.N * 8};
  const cuuint32_t box[4] = {32, 8, 1, 1}, elem[4] = {1, 1, 1, 1};
  return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double *>(state), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

namespace fz {
bool tma_field_map(const double *base, int n1, int n2, int n3, int nf, long long fstride, int bx, int by, int bf,
                   CUtensorMap *tm) {
  if (n1 % 2 != 0 || fstride % 2 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  if (bx < 1 || bx > 256 || by < 1 || by > 256 || bf < 1 || bf > 256 || (bx * 8) % 16 != 0) return false;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return false;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[4] = {(cuuint64_t)n1, (cuuint64_t)n2, (cuuint64_t)n3, (cuuint64_t)nf};
  const cuuint64_t strides[3] = {(cuuint64_t)n1 * 8, (cuuint64_t)n1 * n2 * 8, (cuuint64_t)fstride * 8};
  const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)bf}, elem[4] = {1, 1, 1, 1};
  return encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double *>(base), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace fz

// filters usable by the fused passes: the explicit periodic o10 filter or none, in every direction
bool filter_fused_supported(const cruna_ctx *c) {
  double ref[FR + 1] = {0};
  bool have = false;
  for (int d = 0; d < 3; ++d) {
    const LineOp &op = c->fop[d];
    if (op.kind == OP_COPY) continue;
    if (!(op.periodic && !op.solve && op.r == FR && op.blend > 0.0)) return false;
    if (have) {
      for (int m = 0; m <= FR; ++m)
        if (op.c[m] != ref[m] || op.blend != c->fop[0].blend) return false;
    } else {
      for (int m = 0; m <= FR; ++m) ref[m] = op.c[m];
      have = true;
    }
  }
  return true;
}

// out = filter_i3(filter_i2(filter_i1(in))) restricted to the directions with on[d] != 0; in != out.
// Uses the stage buffer st[2] (free after a time step) as the intermediate between the two passes.
void filter3_fused(cruna_ctx *c, const double *in, double *out, const int on_in[3]) {
  FilterArgs a;
  a.g = c->g;
  bool any = false;
  for (int d = 0; d < 3; ++d) {
    a.n[d] = c->cfg.n[d];
    a.on[d] = on_in[d] && c->fop[d].kind != OP_COPY;
    any = any || a.on[d];
  }
  if (!any) {
    copy_state(c, out, in, 5);
    return;
  }
  for (int d = 0; d < 3; ++d)
    if (a.on[d]) {
      for (int m = 0; m <= FR; ++m) a.c[m] = c->fop[d].c[m];
      a.blend = c->fop[d].blend;
    }
  double *tmp = c->st[2];
  const double *src = in;
  a.kc = 1;
  if (a.on[0] || a.on[1]) {
    a.in = src;
    a.out = a.on[2] ? tmp : out;
    const int bx = (c->g.n1 + FXT - 1) / FXT, by = (c->g.n2 + FYT - 1) / FYT;
    ProfScope ps(c, "filter_xy");
    k_filter_xy<<<dim3(bx, by, c->g.n3), FTHR, 0, c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
    src = tmp;
  }
  if (a.on[2]) {
    a.in = src;
    a.out = out;
    const int zx = (c->g.n1 + 31) / 32, zy = (c->g.n2 + 7) / 8;
    const int n3 = c->g.n3;
    int nz = std::max(1, std::min(std::max(1, n3 / 32), (16 * 148 + 5 * zx * zy - 1) / (5 * zx * zy)));
    a.kc = (n3 + nz - 1) / nz;
    nz = (n3 + a.kc - 1) / a.kc;
    ProfScope ps(c, "filter_z");
    CUtensorMap tm;
    if (state_tensor_map(c, src, &tm))
      k_filter_z_tma<<<dim3(zx, zy, 5 * nz), FTHR, 0, c->stream>>>(tm, a, c->flag + 1);
    else
      k_filter_z<<<dim3(zx, zy, 5 * nz), FTHR, 0, c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
  }
}

}  // namespace cruna
