// common.cuh -- error plumbing, device buffers and small numeric helpers shared
// by the MQCT B200 kernels and the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mqct_b200.h"

namespace mqct {

constexpr double kPi = 3.14159265358979323846;
// Unit constants of the reference (MQCT_SOURCE_CODES/iotest.f:19-25).
constexpr double kAuToEv = 27.21113845;
constexpr double kEvToWn = 8065.5448;
constexpr double kAmuToAu = 1822.8885;
constexpr double kCmToHartree = 1.0 / kEvToWn / kAuToEv;

void set_error(const char* fmt, ...);
// Device -> pageable host copy of a result after the work queued on `after`: large ones
// through pinned staging slots and host threads (hostcopy.cu), small ones as one copy on
// `after`; complete on return either way.  Returns an MQCT_ code.
int copy_d2h_host(void* dst, const void* src, size_t bytes, cudaStream_t after);

#define MQCT_CUDA_TRY(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::mqct::set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr,                 \
                        cudaGetErrorString(_e));                                   \
      return MQCT_E_CUDA;                                                          \
    }                                                                              \
  } while (0)

#define MQCT_ARG_CHECK(cond, ...)                                                  \
  do {                                                                             \
    if (!(cond)) {                                                                 \
      ::mqct::set_error(__VA_ARGS__);                                              \
      return MQCT_E_ARG;                                                           \
    }                                                                              \
  } while (0)

// Owning device allocation; freed on destruction.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    return cudaMalloc((void**)&p, count * sizeof(T));
  }
  cudaError_t upload(const T* host, size_t count, cudaStream_t s = 0) {
    cudaError_t e = alloc(count);
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  cudaError_t upload(const std::vector<T>& v, cudaStream_t s = 0) {
    return upload(v.data(), v.size(), s);
  }
};

// ---------------------------------------------------------------- host helpers
// Gauss-Legendre nodes/weights on [-1,1] by Newton iteration on P_n
// (the quadrature of MQCT_SOURCE_CODES/suppl_routines.f:157-204).
void gauss_legendre(int n, double* x, double* w);

struct Axis {
  std::vector<double> x, w;
  double half = 0.0;  // half-length of the interval (xbl, xgl, ...)
};
Axis axis_gl(int n, double lo, double hi);
Axis axis_mid(int n, double lo, double hi);

int asym_top_level(double A, double B, double C, int j, int ka, int kc, double* energy,
                   double* vec);

}  // namespace mqct

// ---------------------------------------------------------------- device helpers
namespace mqct_dev {

// Wigner small-d in the Jacobi-polynomial form with the case selection of
// MQCT_SOURCE_CODES/pot_comp.f:256-309 (Djkm); returns d for (j, k, m, beta).
__host__ __device__ inline double wigner_d(int j, int k, int m, double beta,
                                           const double* logfact) {
  int n = j + k;
  if (j - k < n) n = j - k;
  if (j + m < n) n = j + m;
  if (j - m < n) n = j - m;
  int a = 0, lam = 0;
  if (n == j + m) { a = k - m; lam = 0; }
  if (n == j - m) { a = m - k; lam = k - m; }
  if (n == j + k) { a = m - k; lam = k - m; }
  if (n == j - k) { a = k - m; lam = 0; }
  int b = 2 * j - 2 * n - a;
  double x = cos(beta);
  // Jacobi P_n^(a,b)(x) by the three-term recurrence
  // (MQCT_SOURCE_CODES/suppl_routines.f:116-145).
  double pm2 = 1.0, pm1 = 0.0, p = 1.0;
  if (n >= 1) {
    pm1 = (1.0 + 0.5 * (a + b)) * x + 0.5 * (a - b);
    p = pm1;
    for (int i = 2; i <= n; ++i) {
      double r = (double)i;
      double c1 = 2.0 * r * (r + a + b) * (2.0 * r - 2.0 + a + b);
      double c2 = (2.0 * r - 1.0 + a + b) * (2.0 * r + a + b) * (2.0 * r - 2.0 + a + b);
      double c3 = (2.0 * r - 1.0 + a + b) * (a + b) * (double)(a - b);
      double c4 = -2.0 * (r - 1.0 + a) * (r - 1.0 + b) * (2.0 * r + a + b);
      p = ((c3 + c2 * x) * pm1 + c4 * pm2) / c1;
      pm2 = pm1;
      pm1 = p;
    }
  }
  // sqrt(C(2j-n, n+a)) / sqrt(C(n+b, b)) from log factorials
  double l1 = logfact[2 * j - n] - logfact[2 * j - n - (n + a)] - logfact[n + a];
  double l2 = logfact[n + b] - logfact[n] - logfact[b];
  double coef = sqrt(exp(l1)) / sqrt(exp(l2));
  double sb = sin(0.5 * beta), cb = cos(0.5 * beta);
  double pa = 1.0, pb = 1.0;
  for (int i = 0; i < a; ++i) pa *= sb;
  for (int i = 0; i < b; ++i) pb *= cb;
  double sgn = (lam % 2 == 0) ? 1.0 : -1.0;
  return p * sgn * coef * pa * pb;
}

// Associated Legendre with Condon-Shortley phase
// (MQCT_SOURCE_CODES/suppl_routines.f:207-243).
__host__ __device__ inline double plgndr(int l, int m, double x) {
  double pmm = 1.0;
  if (m > 0) {
    double somx2 = sqrt((1.0 - x) * (1.0 + x));
    double fact = 1.0;
    for (int i = 1; i <= m; ++i) {
      pmm = -pmm * fact * somx2;
      fact += 2.0;
    }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2 * m + 1) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0.0;
  for (int ll = m + 2; ll <= l; ++ll) {
    pll = (x * (2 * ll - 1) * pmmp1 - (ll + m - 1) * pmm) / (ll - m);
    pmm = pmmp1;
    pmmp1 = pll;
  }
  return pll;
}

// <j1 m1 j2 m2 | J M> by Racah's closed form from log factorials lf[n] = ln n!
// (the coefficient of CG, MQCT_SOURCE_CODES/suppl_routines.f:246-252).
__host__ __device__ inline double clebsch_gordan(int j1, int m1, int j2, int m2, int J, int M,
                                                 const double* lf) {
  if (m1 + m2 != M || J < abs(j1 - j2) || J > j1 + j2 || abs(m1) > j1 || abs(m2) > j2 ||
      abs(M) > J)
    return 0.0;
  const double pre = 0.5 * (log(2.0 * J + 1.0) + lf[J + j1 - j2] + lf[J - j1 + j2] +
                            lf[j1 + j2 - J] - lf[j1 + j2 + J + 1] + lf[J + M] + lf[J - M] +
                            lf[j1 - m1] + lf[j1 + m1] + lf[j2 - m2] + lf[j2 + m2]);
  double sum = 0.0;
  for (int k = 0; k <= j1 + j2 - J; ++k) {
    const int a = j1 - m1 - k, b = j2 + m2 - k, c = J - j2 + m1 + k, d = J - j1 - m2 + k;
    if (a < 0 || b < 0 || c < 0 || d < 0) continue;
    const double t = exp(pre - lf[k] - lf[j1 + j2 - J - k] - lf[a] - lf[b] - lf[c] - lf[d]);
    sum += (k & 1) ? -t : t;
  }
  return sum;
}

}  // namespace mqct_dev
