// Forward-mode dual numbers with K derivative slots: exact Jacobians of small point-wise maps (the
// characteristic boundary treatments) for the discrete adjoint.  All operators are hidden friends,
// so unqualified sqrt / arithmetic on plain doubles keeps resolving to the usual functions.
#pragma once
#include <cmath>

namespace cruna {

template <int K>
struct Dual {
  double v;
  double d[K];
  __host__ __device__ Dual() : v(0.0) {
    for (int i = 0; i < K; ++i) d[i] = 0.0;
  }
  __host__ __device__ Dual(double x) : v(x) {  // NOLINT: implicit on purpose (constants)
    for (int i = 0; i < K; ++i) d[i] = 0.0;
  }
  __host__ __device__ static Dual seed(double x, int slot) {
    Dual r(x);
    r.d[slot] = 1.0;
    return r;
  }
  friend __host__ __device__ Dual operator+(const Dual &a, const Dual &b) {
    Dual r(a.v + b.v);
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
  }
  friend __host__ __device__ Dual operator-(const Dual &a, const Dual &b) {
    Dual r(a.v - b.v);
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
  }
  friend __host__ __device__ Dual operator-(const Dual &a) {
    Dual r(-a.v);
    for (int i = 0; i < K; ++i) r.d[i] = -a.d[i];
    return r;
  }
  friend __host__ __device__ Dual operator*(const Dual &a, const Dual &b) {
    Dual r(a.v * b.v);
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
  }
  friend __host__ __device__ Dual operator/(const Dual &a, const Dual &b) {
    const double inv = 1.0 / b.v;
    Dual r(a.v / b.v);
    for (int i = 0; i < K; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
  }
  friend __host__ __device__ Dual operator+(const Dual &a, double b) { return a + Dual(b); }
  friend __host__ __device__ Dual operator+(double a, const Dual &b) { return Dual(a) + b; }
  friend __host__ __device__ Dual operator-(const Dual &a, double b) { return a - Dual(b); }
  friend __host__ __device__ Dual operator-(double a, const Dual &b) { return Dual(a) - b; }
  friend __host__ __device__ Dual operator*(const Dual &a, double b) {
    Dual r(a.v * b);
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * b;
    return r;
  }
  friend __host__ __device__ Dual operator*(double a, const Dual &b) { return b * a; }
  friend __host__ __device__ Dual operator/(const Dual &a, double b) { return a / Dual(b); }
  friend __host__ __device__ Dual operator/(double a, const Dual &b) { return Dual(a) / b; }
  friend __host__ __device__ bool operator<(const Dual &a, double b) { return a.v < b; }
  friend __host__ __device__ Dual sqrt(const Dual &a) {
    const double s = ::sqrt(a.v);
    Dual r(s);
    const double h = 0.5 / s;
    for (int i = 0; i < K; ++i) r.d[i] = a.d[i] * h;
    return r;
  }
};

}  // namespace cruna
