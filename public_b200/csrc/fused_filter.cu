// Fused filter_i1 -> filter_i2 -> filter_i3 sequence (src/main/computation_direct.f90:85-95,
// src/filter/filter_i*_mpi_cartesian.f90) for the explicit periodic 10th-order filter (no reference
// counterpart: the interior stencil of filter_pen_core_o10_i_c_o.f90:182-199 at alpha = 0 with
// periodic wrap, blended q <- q - s*(q - F q)).
//
// One z-marching pass applies the three directional filters in the reference's order to all five
// variables: each plane is loaded once with an R = 5 halo (corners included), x-filtered on the
// halo rows, y-filtered into a per-thread z column of 2R+1 planes, and z-filtered from that column.
// The output goes to a second buffer (the filter reads neighbours), so the state is read and written
// once per step instead of twice per direction.
#include "cruna_internal.cuh"
#include "fused_common.cuh"

namespace cruna {

using namespace fz;

namespace {

constexpr int FR = 5;    // o10 filter half-width

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

__global__ void __launch_bounds__(TX *TY, 2) k_filter3(const __grid_constant__ FilterArgs a) {
  constexpr int PW = TX + 2 * FR, PH = TY + 2 * FR, PS = PW * PH;
  constexpr int XS = TX * PH;           // x-filtered rows (all y incl. halo) per variable
  constexpr int NS = 2 * FR + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *raw = reinterpret_cast<double *>(smem_raw);   // [5][PH][PW]
  double *xf = raw + 5 * PS;                            // [5][PH][TX]
  double *ring = xf + 5 * XS;                           // [NS][5][TY*TX]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const long long N = a.g.N, n1 = a.g.n1, n12 = (long long)a.g.n1 * a.g.n2;
  const bool inside = (i0 + tx) < a.g.n1 && (j0 + ty) < a.g.n2;

  // filters plane kk of the input in x then y into ring slot kk (this thread's column)
  auto xy_plane = [&](int kk) {
    const int gk = a.on[2] ? wrapi(kk, a.n[2]) : kk;
    const bool valid = gk >= 0 && gk < a.n[2];
    __syncthreads();
    if (valid) {
      for (int cidx = tid; cidx < PW * PH; cidx += TX * TY) {
        const int lx = cidx % PW - FR, ly = cidx / PW - FR;
        const int gi = a.on[0] ? wrapi(i0 + lx, a.n[0]) : min(max(i0 + lx, 0), a.n[0] - 1);
        const int gj = a.on[1] ? wrapi(j0 + ly, a.n[1]) : min(max(j0 + ly, 0), a.n[1] - 1);
        const long long pt = gi + n1 * gj + n12 * gk;
#pragma unroll
        for (int v = 0; v < 5; ++v) raw[v * PS + cidx] = a.in[pt + v * N];
      }
    }
    __syncthreads();
    if (valid) {
      for (int cidx = tid; cidx < TX * PH; cidx += TX * TY) {
        const int lx = cidx % TX, ly = cidx / TX;          // ly in [0, PH)
        const double *p = raw + ly * PW + (lx + FR);
#pragma unroll
        for (int v = 0; v < 5; ++v) xf[v * XS + cidx] = a.on[0] ? filt(a, p + v * PS, 1) : p[v * PS];
      }
    }
    __syncthreads();
    if (valid) {
      const int sl = ((kk % NS) + NS) % NS;
      const double *p = xf + (ty + FR) * TX + tx;
#pragma unroll
      for (int v = 0; v < 5; ++v)
        ring[(sl * 5 + v) * (TX * TY) + tid] = a.on[1] ? filt(a, p + v * XS, TX) : p[v * XS];
    }
  };
  for (int kk = k0 - FR; kk < k0 + FR; ++kk) xy_plane(kk);
  for (int k = k0; k < k1; ++k) {
    xy_plane(k + FR);
    if (inside) {
      const int slot = k % NS;
      const long long pt = (i0 + tx) + n1 * (j0 + ty) + n12 * k;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        double col[NS];
#pragma unroll
        for (int m = -FR; m <= FR; ++m) col[m + FR] = ring[(((slot + m + NS) % NS) * 5 + v) * (TX * TY) + tid];
        a.out[pt + v * N] = a.on[2] ? filt(a, col + FR, 1) : col[FR];
      }
    }
  }
}

size_t smem_filter3() {
  return sizeof(double) *
         (5 * (TX + 2 * FR) * (TY + 2 * FR) + 5 * TX * (TY + 2 * FR) + (2 * FR + 1) * 5 * TX * TY);
}

}  // namespace

// filters usable by the fused pass: the explicit periodic o10 filter or none, in every direction
bool filter_fused_supported(const cruna_ctx *c) {
  double ref[FR + 1] = {0};
  bool have = false;
  for (int d = 0; d < 3; ++d) {
    const LineOp &op = c->fop[d];
    if (op.kind == OP_COPY) continue;
    if (!(op.periodic && !op.solve && op.r == FR && op.blend > 0.0)) return false;
    if (have) {
      for (int m = 0; m <= FR; ++m)
        if (op.c[m] != ref[m]) return false;
    } else {
      for (int m = 0; m <= FR; ++m) ref[m] = op.c[m];
      have = true;
    }
  }
  return true;
}

// out = filter_i3(filter_i2(filter_i1(in))) restricted to the directions with on[d] != 0
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
  a.in = in;
  a.out = out;
  static bool configured = false;
  if (!configured) {
    CRUNA_CUDA_CHECK(
        cudaFuncSetAttribute(k_filter3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_filter3()));
    configured = true;
  }
  const int bx = (c->g.n1 + TX - 1) / TX, by = (c->g.n2 + TY - 1) / TY;
  const int n3 = c->g.n3;
  int nz = std::max(1, std::min(n3, (4 * 148 + bx * by - 1) / (bx * by)));
  int kc = (n3 + nz - 1) / nz;
  kc = std::max(kc, std::min(n3, 4 * FR));
  nz = (n3 + kc - 1) / kc;
  a.kc = kc;
  ProfScope ps(c, "filter3");
  k_filter3<<<dim3(bx, by, nz), dim3(TX, TY), smem_filter3(), c->stream>>>(a);
  CRUNA_LAUNCH_CHECK(c);
}

}  // namespace cruna
