// Shared pieces of the fused z-marching kernels: the explicit line operator in compact form and
// the derivative evaluators on shared-memory rows (x, y) and register columns (z).
#pragma once

#include <cuda.h>

#include <cmath>

#include "cruna_internal.cuh"
#include "mlp_common.cuh"
#include "tcgen05.cuh"

namespace cruna {
namespace fz {

constexpr int TX = 32;
constexpr int TY = 4;
constexpr int NG = 15;   // pass-G outputs per point

// compact description of an explicit line operator for the fused kernels
struct DirOpF {
  int n = 1, kind = 0, periodic = 0, r = 0, nb = 0, bw = 0;
  double c[5] = {0};
  double brow[2][5] = {{0}};
  double scale = 0.0;    // 1/(dx*div)
  double scale_h = 0.0;  // heat-flux derivatives: 1/div (reference, h absent) or 1/(dx*div)
};

struct FusedArgs {
  Grid g;
  DirOpF op[3];
  int kc;                       // z-chunk length of one block
  // material (ns_rho_rhou_p_trafos.f90)
  double WoR, mu0, T0, cp_over_pr, gamma;
  double p_ref, T_ref;          // FP32 path offsets (0 in the FP64 path)
  // pass G
  const double *q;
  void *gbuf;                   // NG fields of T
  // pass D
  double *rhs;
  const double *force;
  int stage;                    // 0: write rhs; 1..4: RK4 stage update
  double dt;
  const double *q0;
  double *acc;
  double *qnext;
  // learned closure evaluated inside pass G (its CL instantiation): network parameters and scaling,
  // filter width, scale-free features / outputs, the network's error flag
  const float *cl_P = nullptr;
  mlp::Scaling cl_sc;
  double cl_delta = 0.0;
  int cl_norm = 0;
  int *cl_err = nullptr;
};

__host__ __device__ constexpr int ring_slots(int R) { return 2 * R + 1; }

// z-chunk length of one block of a z-marching kernel on a (bx, by) grid of plane tiles: enough chunks
// that the grid covers at least 4 blocks per SM of the 148, each chunk at least 4R planes long (the
// ring start-up reads 2R planes).  nz receives the number of chunks.
inline int z_chunk(int n3, int bx, int by, int R, int &nz) {
  nz = n3 < 1 ? 1 : (4 * 148 + bx * by - 1) / (bx * by);
  if (nz > n3) nz = n3;
  if (nz < 1) nz = 1;
  int kc = (n3 + nz - 1) / nz;
  const int kmin = n3 < 4 * R ? n3 : 4 * R;
  if (kc < kmin) kc = kmin;
  nz = (n3 + kc - 1) / kc;
  return kc;
}

// z-chunking balanced against the launch waves: `tiles` plane tiles, `resident` blocks of the kernel per
// SM and `sms` SMs.  Among the chunk counts whose chunks stay at least 4R planes long it picks the one
// that maximises the filled fraction of the last wave times kc / (kc + R/2) (each chunk first reads 2R
// planes, about a quarter of a marching step each).  Returns kc; nz receives the number of chunks.
inline int z_chunk_balanced(int n3, int tiles, int resident, int sms, int R, int &nz) {
  if (resident < 1 || sms < 1 || tiles < 1) return z_chunk(n3, 1, tiles, R, nz);
  const int kmin = n3 < 4 * R ? n3 : 4 * R;
  double best = -1.0;
  int best_kc = n3;
  nz = 1;
  for (int z = 1; z <= n3 && z <= 256; ++z) {
    const int kc = (n3 + z - 1) / z;
    if (kc < kmin) break;
    const int nzr = (n3 + kc - 1) / kc;
    const double waves = (double)tiles * nzr / ((double)resident * sms);
    const double eff = waves / std::ceil(waves) * (double)kc / (kc + 0.5 * R);
    if (eff > best + 1e-9) {
      best = eff;
      best_kc = kc;
      nz = nzr;
    }
  }
  return best_kc;
}

// SM count of the current device (cached per device ordinal)
inline int device_sms() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return 148;
  }
  if (!cache[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1) {
      cudaGetLastError();
      v = 148;
    }
    cache[dev] = v;
  }
  return cache[dev];
}

// resident blocks per SM of a kernel at a launch shape (0 when the query fails)
template <typename K>
int resident_blocks(K kernel, int threads, size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

template <typename T, int R>
__device__ __forceinline__ T dsm(const DirOpF &op, const T *p, int s, int i) {
  // derivative (unscaled) at line position i; p points at the point, neighbours at p[m*s]
  if (op.kind == 0) return T(0);
  if (op.periodic || (i >= op.nb && i < op.n - op.nb)) {
    T t = T(op.c[1]) * (p[s] - p[-s]);
#pragma unroll
    for (int m = 2; m <= R; ++m)
      if (m <= op.r) t = t + T(op.c[m]) * (p[m * s] - p[-m * s]);
    return t;
  }
  const bool start = i < op.nb;
  const int row = start ? i : op.n - 1 - i;
  T t = T(0);
  for (int m = 0; m < op.bw; ++m) {
    const int j = start ? m : op.n - 1 - m;
    const T v = p[(j - i) * s];
    t = (m == 0) ? T(op.brow[row][0]) * v : t + T(op.brow[row][m]) * v;
  }
  return start ? t : -t;
}

// derivative of a product a*b
template <typename T, int R>
__device__ __forceinline__ T dsm2(const DirOpF &op, const T *a, const T *b, int s, int i) {
  if (op.kind == 0) return T(0);
  if (op.periodic || (i >= op.nb && i < op.n - op.nb)) {
    T t = T(op.c[1]) * (a[s] * b[s] - a[-s] * b[-s]);
#pragma unroll
    for (int m = 2; m <= R; ++m)
      if (m <= op.r) t = t + T(op.c[m]) * (a[m * s] * b[m * s] - a[-m * s] * b[-m * s]);
    return t;
  }
  const bool start = i < op.nb;
  const int row = start ? i : op.n - 1 - i;
  T t = T(0);
  for (int m = 0; m < op.bw; ++m) {
    const int j = start ? m : op.n - 1 - m;
    const T v = a[(j - i) * s] * b[(j - i) * s];
    t = (m == 0) ? T(op.brow[row][0]) * v : t + T(op.brow[row][m]) * v;
  }
  return start ? t : -t;
}

// z-derivatives from a register column v[0..2R] centred at v[R]: the closure rows are evaluated with
// compile-time offsets only, so the column stays in registers
template <typename T, int R>
__device__ __forceinline__ T dsz(const DirOpF &op, const T *v, int k) {
  if (op.kind == 0) return T(0);
  if (op.periodic || (k >= op.nb && k < op.n - op.nb)) {
    T t = T(op.c[1]) * (v[R + 1] - v[R - 1]);
#pragma unroll
    for (int m = 2; m <= R; ++m)
      if (m <= op.r) t = t + T(op.c[m]) * (v[R + m] - v[R - m]);
    return t;
  }
  const bool start = k < op.nb;
  const int row = start ? k : op.n - 1 - k;
  T t = T(0);
  bool first = true;
  if (start) {
#pragma unroll
    for (int o = -R; o <= R; ++o) {
      const int j = k + o;
      if (j >= 0 && j < op.bw) {
        const T c = T(op.brow[row][j]);
        t = first ? c * v[R + o] : t + c * v[R + o];
        first = false;
      }
    }
    return t;
  }
#pragma unroll
  for (int o = R; o >= -R; --o) {
    const int m = op.n - 1 - (k + o);
    if (m >= 0 && m < op.bw) {
      const T c = T(op.brow[row][m]);
      t = first ? c * v[R + o] : t + c * v[R + o];
      first = false;
    }
  }
  return -t;
}

template <typename T, int R>
__device__ __forceinline__ T dsz2(const DirOpF &op, const T *a, const T *b, int k) {
  if (op.kind == 0) return T(0);
  if (op.periodic || (k >= op.nb && k < op.n - op.nb)) {
    T t = T(op.c[1]) * (a[R + 1] * b[R + 1] - a[R - 1] * b[R - 1]);
#pragma unroll
    for (int m = 2; m <= R; ++m)
      if (m <= op.r) t = t + T(op.c[m]) * (a[R + m] * b[R + m] - a[R - m] * b[R - m]);
    return t;
  }
  const bool start = k < op.nb;
  const int row = start ? k : op.n - 1 - k;
  T t = T(0);
  bool first = true;
  if (start) {
#pragma unroll
    for (int o = -R; o <= R; ++o) {
      const int j = k + o;
      if (j >= 0 && j < op.bw) {
        const T c = T(op.brow[row][j]);
        const T v = a[R + o] * b[R + o];
        t = first ? c * v : t + c * v;
        first = false;
      }
    }
    return t;
  }
#pragma unroll
  for (int o = R; o >= -R; --o) {
    const int m = op.n - 1 - (k + o);
    if (m >= 0 && m < op.bw) {
      const T c = T(op.brow[row][m]);
      const T v = a[R + o] * b[R + o];
      t = first ? c * v : t + c * v;
      first = false;
    }
  }
  return -t;
}

// global index along a direction for a cell offset; -1 when outside an open line
__device__ __forceinline__ int gidx(const DirOpF &op, int g) {
  if (g >= 0 && g < op.n) return g;
  if (op.periodic) return ((g % op.n) + op.n) % op.n;
  return -1;
}



// ---- compile-time specialised evaluators -------------------------------------------------------
// PER = true: every direction is periodic with half-width exactly R, so the stencil needs no
// boundary logic and no predicates; PER = false falls back to the run-time operator (closures,
// empty directions, smaller half-widths).
template <typename T, int R>
__device__ __forceinline__ T dper(const DirOpF &op, const T *p, int s) {
  T t = T(op.c[1]) * (p[s] - p[-s]);
#pragma unroll
  for (int m = 2; m <= R; ++m) t = t + T(op.c[m]) * (p[m * s] - p[-m * s]);
  return t;
}
template <typename T, int R>
__device__ __forceinline__ T dper2(const DirOpF &op, const T *a, const T *b, int s) {
  T t = T(op.c[1]) * (a[s] * b[s] - a[-s] * b[-s]);
#pragma unroll
  for (int m = 2; m <= R; ++m) t = t + T(op.c[m]) * (a[m * s] * b[m * s] - a[-m * s] * b[-m * s]);
  return t;
}
template <typename T, int R, bool PER>
__device__ __forceinline__ T D1(const DirOpF &op, const T *p, int s, int i) {
  if constexpr (PER) return dper<T, R>(op, p, s);
  else return dsm<T, R>(op, p, s, i);
}
template <typename T, int R, bool PER>
__device__ __forceinline__ T D2(const DirOpF &op, const T *a, const T *b, int s, int i) {
  if constexpr (PER) return dper2<T, R>(op, a, b, s);
  else return dsm2<T, R>(op, a, b, s, i);
}
// z versions on register columns v[0..2R] centred at v[R]
template <typename T, int R, bool PER>
__device__ __forceinline__ T Dz1(const DirOpF &op, const T *v, int k) {
  if constexpr (PER) return dper<T, R>(op, v + R, 1);
  else return dsz<T, R>(op, v, k);
}
template <typename T, int R, bool PER>
__device__ __forceinline__ T Dz2(const DirOpF &op, const T *a, const T *b, int k) {
  if constexpr (PER) return dper2<T, R>(op, a + R, b + R, 1);
  else return dsz2<T, R>(op, a, b, k);
}

// halo strip cell h (no corners) of a TX x TY tile with R-wide halos -> local (lx, ly)
template <int R>
__device__ __forceinline__ void halo_cell(int h, int &lx, int &ly) {
  if (h < 2 * R * TY) {
    const int side = h / (R * TY), e = h % (R * TY);
    ly = e / R;
    lx = side == 0 ? -R + e % R : TX + e % R;
  } else {
    const int e2 = h - 2 * R * TY;
    const int side = e2 / (R * TX), e = e2 % (R * TX);
    lx = e % TX;
    ly = side == 0 ? -R + e / TX : TY + e / TX;
  }
}

// per-thread halo cells: smem cell offset and in-plane global offset (-1: outside an open line)
template <int R>
struct HaloSet {
  static constexpr int NH = 2 * R * (TX + TY);
  static constexpr int PER_THREAD = (NH + TX * TY - 1) / (TX * TY);
  int cell[PER_THREAD];
  int goff[PER_THREAD];
  __device__ __forceinline__ void init(const DirOpF &ox, const DirOpF &oy, int i0, int j0, int tid, int n1) {
    constexpr int PW = TX + 2 * R;
#pragma unroll
    for (int c = 0; c < PER_THREAD; ++c) {
      const int h = tid + c * TX * TY;
      cell[c] = -1;
      goff[c] = -1;
      if (h < NH) {
        int lx, ly;
        halo_cell<R>(h, lx, ly);
        const int hi = gidx(ox, i0 + lx), hj = gidx(oy, j0 + ly);
        cell[c] = (ly + R) * PW + (lx + R);
        if (hi >= 0 && hj >= 0) goff[c] = hi + n1 * hj;
      }
    }
  }
};

DirOpF to_dir(const LineOp &op, double dx, bool heat_dx);
int halo_of(const LineOp &op);

// ---- TMA plumbing of the fused passes ------------------------------------------------------------
// Bounded spin of an mbarrier wait (iterations of try_wait); a block whose wait runs out records it in
// the context's error flag, waits (again bounded) for its copies in flight and returns.
constexpr long long kTmaSpinLimit = 1LL << 22;

// 4-D tensor map (x, y, z, field) over nf Fortran-ordered fields of n1 x n2 x n3 doubles, fields
// fstride elements apart, with a (bx, by, 1, bf) box; false when the layout does not meet TMA's rules
// (16-byte aligned base, row / plane / field strides multiples of 16 bytes, i.e. n1 even).
bool tma_field_map(const double *base, int n1, int n2, int n3, int nf, long long fstride, int bx, int by, int bf,
                   CUtensorMap *tm);

// this thread's arrival on `bar` announcing `bytes` of TMA writes
__device__ __forceinline__ void tma_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(bar)), "r"(bytes)
               : "memory");
}
// plain arrival (a phase without copies)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_addr(bar)) : "memory");
}
// box at (x, y, z, f) of the map into dst (this CTA's shared memory), completion counted on bar
__device__ __forceinline__ void tma_load4(const CUtensorMap *tm, void *dst, uint64_t *bar, int x, int y, int z,
                                          int f) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(tc::smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(f), "r"(tc::smem_addr(bar))
      : "memory");
}

}  // namespace fz
}  // namespace cruna
