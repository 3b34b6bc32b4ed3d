// surrogate.cu -- learned surrogate of the potential energy surface.
//
// A multilayer perceptron V(R, angles) with SiLU hidden layers stands in for the
// many-term PES evaluation of the matrix build (the USER_DEFINED_PES plugin,
// called through MQCT_SOURCE_CODES/pes_sys_type.f for every grid point and R).
// Everything runs on the GPU with the kernels of this file: seeded sampling of
// training points from the product's own PES routine, a tiled FP32 GEMM with
// fused bias and activation, the backward pass, and Adam.  The matrix plan uses
// the trained network for the PES table and checks it: at every radial point a
// sample of grid points is evaluated exactly, and a radial point whose residual
// exceeds the bound is re-evaluated exactly on the whole grid.
//
// Features (11): (R - c)/s and cos, sin of the five angles (beta1, gamma1,
// alpha2, beta2, gamma2; unused angles are 0).  Target: asinh(V / 100 cm^-1) / 4,
// which compresses the repulsive wall.  Parameters are FP32 (W_l row-major
// [in][out], b_l [out]); accumulation is FP32.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <vector>

#include "common.cuh"
#include "pes.cuh"

using namespace mqct;

namespace mqct {

constexpr int SG_IN = 11;
constexpr double SG_VSCALE = 100.0;  // cm^-1
constexpr double SG_YSCALE = 4.0;

// ---------------------------------------------------------------- sampling
__device__ inline uint64_t sg_mix(uint64_t x) {  // splitmix64 finaliser
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
__device__ inline double sg_uniform(uint64_t seed, uint64_t i, int d) {
  return (double)(sg_mix(seed ^ sg_mix(i * 8 + (uint64_t)d)) >> 11) * (1.0 / 9007199254740992.0);
}

__device__ inline void sg_features(double R, const double* ang, double r_c, double r_s, float* f) {
  f[0] = (float)((R - r_c) / r_s);
  for (int a = 0; a < 5; ++a) {
    double s, c;
    sincos(ang[a], &s, &c);
    f[1 + 2 * a] = (float)c;
    f[2 + 2 * a] = (float)s;
  }
}

__device__ inline double sg_target(double v) { return asinh(v / SG_VSCALE) / SG_YSCALE; }
__device__ inline double sg_value(double y) { return SG_VSCALE * sinh(y * SG_YSCALE); }

// n seeded points: R ~ U(r_lo, r_hi); beta angles ~ U(0, pi), the others ~ U(0, 2 pi)
// (the grid's domain); the angles a system type does not use stay 0.
__global__ void sg_sample_kernel(int64_t n, uint64_t seed, int sys_type, PesDev pes, double r_lo,
                                 double r_hi, double r_c, double r_s, float* __restrict__ X,
                                 float* __restrict__ Y, double* __restrict__ V) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double R = r_lo + (r_hi - r_lo) * sg_uniform(seed, (uint64_t)i, 0);
  double ang[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  ang[0] = kPi * sg_uniform(seed, (uint64_t)i, 1);
  if (sys_type != 1) ang[1] = 2.0 * kPi * sg_uniform(seed, (uint64_t)i, 2);
  if (sys_type == 0) {
    ang[2] = 2.0 * kPi * sg_uniform(seed, (uint64_t)i, 3);
    ang[3] = kPi * sg_uniform(seed, (uint64_t)i, 4);
    ang[4] = 2.0 * kPi * sg_uniform(seed, (uint64_t)i, 5);
  }
  sg_features(R, ang, r_c, r_s, X + (size_t)i * SG_IN);
  const double v = pes_at(sys_type, pes, R, ang);
  Y[i] = (float)sg_target(v);
  if (V) V[i] = v;
}

// Features of caller-given points (R, beta1, gamma1, alpha2, beta2, gamma2).
__global__ void sg_features_kernel(int64_t n, const double* __restrict__ args, double r_c,
                                   double r_s, float* __restrict__ X) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* a = args + 6 * i;
  sg_features(a[0], a + 1, r_c, r_s, X + (size_t)i * SG_IN);
}

// ---------------------------------------------------------------- GEMM
// C[M x N] = op(A)[M x K] op(B)[K x N] (+ bias[N]); op = transpose when TA/TB.
// Storage row-major: A is M x K (K x M when TA), B is K x N (N x K when TB).
// With Z != nullptr the pre-activation is stored in Z and C = silu(Z).
// 64 x 64 tiles, K steps of 16, 256 threads with 4 x 4 outputs each.
constexpr int SG_BM = 64, SG_BN = 64, SG_BK = 16;
template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
sg_gemm_kernel(int M, int N, int K, const float* __restrict__ A, const float* __restrict__ B,
               const float* __restrict__ bias, float* __restrict__ Z, float* __restrict__ C) {
  __shared__ float As[SG_BK][SG_BM + 4];
  __shared__ float Bs[SG_BK][SG_BN + 4];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int m0 = blockIdx.y * SG_BM, n0 = blockIdx.x * SG_BN;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += SG_BK) {
    for (int q = tid; q < SG_BM * SG_BK; q += 256) {
      const int mm = q / SG_BK, kk = q % SG_BK;
      const int m = m0 + mm, k = k0 + kk;
      float v = 0.f;
      if (m < M && k < K) v = TA ? A[(size_t)k * M + m] : A[(size_t)m * K + k];
      As[kk][mm] = v;
    }
    for (int q = tid; q < SG_BN * SG_BK; q += 256) {
      const int kk = q / SG_BN, nn = q % SG_BN;
      const int n = n0 + nn, k = k0 + kk;
      float v = 0.f;
      if (n < N && k < K) v = TB ? B[(size_t)n * K + k] : B[(size_t)k * N + n];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < SG_BK; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j] + (bias ? bias[n] : 0.f);
      if (Z) {
        Z[(size_t)m * N + n] = v;
        v = v / (1.f + __expf(-v));
      }
      C[(size_t)m * N + n] = v;
    }
  }
}

// dZ = dH * silu'(Z), silu'(z) = s (1 + z (1 - s)), s = 1/(1+e^-z); dZ may alias dH
__global__ void sg_silu_back_kernel(int64_t n, const float* __restrict__ Z, const float* dH,
                                    float* dZ) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = Z[i], s = 1.f / (1.f + __expf(-z));
  dZ[i] = dH[i] * s * (1.f + z * (1.f - s));
}

// Mean squared error over the batch and its gradient d(loss)/d(pred).
__global__ void sg_loss_kernel(int n, const float* __restrict__ pred, const float* __restrict__ y,
                               float* __restrict__ dpred, double* __restrict__ loss) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = pred[i] - y[i];
    dpred[i] = 2.f * d / (float)n;
    acc += (double)d * d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    *loss = s / n;
  }
}

// db[j] = sum_i dZ[i, j]  (one thread per column, fixed order)
__global__ void sg_colsum_kernel(int rows, int cols, const float* __restrict__ dZ,
                                 float* __restrict__ db) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float s = 0.f;
  for (int i = 0; i < rows; ++i) s += dZ[(size_t)i * cols + j];
  db[j] = s;
}

__global__ void sg_adam_kernel(int64_t n, float* __restrict__ p, const float* __restrict__ g,
                               float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                               float b2, float eps, float c1, float c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void sg_gather_kernel(int n, const int* __restrict__ idx, const float* __restrict__ X,
                                 const float* __restrict__ Y, float* __restrict__ Xb,
                                 float* __restrict__ Yb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = idx[i];
#pragma unroll
  for (int d = 0; d < SG_IN; ++d) Xb[(size_t)i * SG_IN + d] = X[(size_t)s * SG_IN + d];
  Yb[i] = Y[s];
}

__global__ void sg_to_value_kernel(int64_t n, const float* __restrict__ y, double* __restrict__ v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = sg_value((double)y[i]);
}

// ---------------------------------------------------------------- the network
struct Surrogate {
  int sys_type = 0, hidden = 256, n_hidden = 4;
  double r_lo = 4.0, r_hi = 25.0, r_c = 14.5, r_s = 10.5;
  uint64_t seed = 1;
  std::vector<int> dims;               // SG_IN, hidden x n_hidden, 1
  std::vector<size_t> w_off, b_off;    // offsets into the flat parameter vector
  size_t n_par = 0;
  DevBuf<float> par, grad, adam_m, adam_v;
  int64_t adam_t = 0;
  // PES copy
  int pes_kind = 0, pes_n_terms = 0, pes_n1 = 0, pes_n2 = 0;
  DevBuf<double> pes_p, pes_s1, pes_s2;
  // workspace for a batch of up to cap rows: Z_l, H_l per layer, gradients
  int cap = 0;
  std::vector<DevBuf<float>> Zs, Hs;
  DevBuf<float> dA, dB, dpred, xb, yb;
  DevBuf<double> d_loss;
  cudaStream_t stream = nullptr;  // own stream (training, predict)
  cudaStream_t cur = nullptr;     // stream of the call in progress

  PesDev pes_dev() const {
    return PesDev{pes_kind, pes_n_terms, pes_n1, pes_n2, pes_p.p, pes_s1.p, pes_s2.p, nullptr};
  }
  int n_layers() const { return (int)dims.size() - 1; }

  int ensure_workspace(int rows) {
    if (rows <= cap) return MQCT_OK;
    cap = rows;
    const int L = n_layers();
    Zs.resize(L);
    Hs.resize(L);
    for (int l = 0; l < L; ++l) {
      MQCT_CUDA_TRY(Zs[l].alloc((size_t)rows * dims[l + 1]));
      MQCT_CUDA_TRY(Hs[l].alloc((size_t)rows * dims[l + 1]));
    }
    MQCT_CUDA_TRY(dA.alloc((size_t)rows * hidden));
    MQCT_CUDA_TRY(dB.alloc((size_t)rows * hidden));
    MQCT_CUDA_TRY(dpred.alloc((size_t)rows));
    MQCT_CUDA_TRY(xb.alloc((size_t)rows * SG_IN));
    MQCT_CUDA_TRY(yb.alloc((size_t)rows));
    return MQCT_OK;
  }

  template <bool TA, bool TB>
  int gemm(int M, int N, int K, const float* A, const float* B, const float* bias, float* Z,
           float* C) {
    dim3 g((N + SG_BN - 1) / SG_BN, (M + SG_BM - 1) / SG_BM);
    sg_gemm_kernel<TA, TB><<<g, 256, 0, cur>>>(M, N, K, A, B, bias, Z, C);
    MQCT_CUDA_TRY(cudaGetLastError());
    return MQCT_OK;
  }

  // Forward pass of `rows` feature rows; the output (target units) ends in Hs[L-1].
  int forward(const float* X, int rows) {
    const int L = n_layers();
    const float* h = X;
    for (int l = 0; l < L; ++l) {
      const bool last = l == L - 1;
      int rc = gemm<false, false>(rows, dims[l + 1], dims[l], h, par.p + w_off[l], par.p + b_off[l],
                                  last ? nullptr : Zs[l].p, Hs[l].p);
      if (rc) return rc;
      h = Hs[l].p;
    }
    return MQCT_OK;
  }

  // Loss and parameter gradients (into grad) of one batch.
  int loss_grad(const float* X, const float* y, int rows, double* loss_host) {
    int rc = ensure_workspace(rows);
    if (rc) return rc;
    rc = forward(X, rows);
    if (rc) return rc;
    const int L = n_layers();
    sg_loss_kernel<<<1, 1024, 0, cur>>>(rows, Hs[L - 1].p, y, dpred.p, d_loss.p);
    MQCT_CUDA_TRY(cudaGetLastError());
    float* dZ = dpred.p;  // gradient w.r.t. the pre-activation of layer l
    for (int l = L - 1; l >= 0; --l) {
      const float* h_in = l == 0 ? X : Hs[l - 1].p;
      // dW_l = h_in^T dZ, db_l = colsum(dZ)
      rc = gemm<true, false>(dims[l], dims[l + 1], rows, h_in, dZ, nullptr, nullptr,
                             grad.p + w_off[l]);
      if (rc) return rc;
      sg_colsum_kernel<<<(dims[l + 1] + 127) / 128, 128, 0, cur>>>(rows, dims[l + 1], dZ,
                                                                     grad.p + b_off[l]);
      MQCT_CUDA_TRY(cudaGetLastError());
      if (l == 0) break;
      // dH_{l-1} = dZ W_l^T, then through the activation
      float* dH = (dZ == dA.p) ? dB.p : dA.p;
      rc = gemm<false, true>(rows, dims[l], dims[l + 1], dZ, par.p + w_off[l], nullptr, nullptr, dH);
      if (rc) return rc;
      const int64_t n = (int64_t)rows * dims[l];
      sg_silu_back_kernel<<<(unsigned)((n + 255) / 256), 256, 0, cur>>>(n, Zs[l - 1].p, dH, dH);
      MQCT_CUDA_TRY(cudaGetLastError());
      dZ = dH;
    }
    if (loss_host) {
      MQCT_CUDA_TRY(cudaMemcpyAsync(loss_host, d_loss.p, sizeof(double), cudaMemcpyDeviceToHost,
                                    cur));
      MQCT_CUDA_TRY(cudaStreamSynchronize(cur));
    }
    return MQCT_OK;
  }

  int adam_step(float lr) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)adam_t), c2 = 1.f - powf(b2, (float)adam_t);
    sg_adam_kernel<<<(unsigned)((n_par + 255) / 256), 256, 0, cur>>>(
        (int64_t)n_par, par.p, grad.p, adam_m.p, adam_v.p, lr, b1, b2, 1e-8f, c1, c2);
    MQCT_CUDA_TRY(cudaGetLastError());
    return MQCT_OK;
  }

  // Predicted V (cm^-1) at n feature rows, in batches.
  int predict_features(const float* X, int64_t n, double* v_out) {
    const int B = 65536;
    int rc = ensure_workspace((int)std::min<int64_t>(n, B));
    if (rc) return rc;
    const int L = n_layers();
    for (int64_t s = 0; s < n; s += B) {
      const int rows = (int)std::min<int64_t>(B, n - s);
      rc = forward(X + s * SG_IN, rows);
      if (rc) return rc;
      sg_to_value_kernel<<<(rows + 255) / 256, 256, 0, cur>>>(rows, Hs[L - 1].p, v_out + s);
      MQCT_CUDA_TRY(cudaGetLastError());
    }
    return MQCT_OK;
  }

  int init(int32_t st, const mqct_pes_t* pes, int32_t hid, int32_t nh, uint64_t sd, double rlo,
           double rhi) {
    MQCT_ARG_CHECK(st == 1 || st == 4 || st == 0, "surrogate supports SYS_TYPE 1, 4 and 0");
    MQCT_ARG_CHECK(pes && pes->params && pes->n_terms > 0, "surrogate needs an analytic PES");
    MQCT_ARG_CHECK((st == 0 && pes->kind == MQCT_PES_SITES2) ||
                       (st != 0 && (pes->kind == MQCT_PES_LEGENDRE || pes->kind == MQCT_PES_SITES1)),
                   "PES kind %d not usable for SYS_TYPE %d", pes->kind, st);
    MQCT_ARG_CHECK(hid >= 8 && hid <= 1024 && nh >= 1 && nh <= 8, "bad network shape");
    MQCT_ARG_CHECK(rhi > rlo && rlo > 0, "bad R range");
    sys_type = st;
    hidden = hid;
    n_hidden = nh;
    seed = sd;
    r_lo = rlo;
    r_hi = rhi;
    r_c = 0.5 * (rlo + rhi);
    r_s = 0.5 * (rhi - rlo);
    MQCT_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    cur = stream;
    dims.assign(1, SG_IN);
    for (int i = 0; i < nh; ++i) dims.push_back(hid);
    dims.push_back(1);
    n_par = 0;
    for (int l = 0; l + 1 < (int)dims.size(); ++l) {
      w_off.push_back(n_par);
      n_par += (size_t)dims[l] * dims[l + 1];
      b_off.push_back(n_par);
      n_par += dims[l + 1];
    }
    // He-style initialisation from the seed (host RNG; deterministic)
    std::vector<float> h(n_par, 0.f);
    std::mt19937_64 rng(sd);
    for (int l = 0; l + 1 < (int)dims.size(); ++l) {
      std::normal_distribution<double> nd(0.0, std::sqrt(2.0 / dims[l]));
      for (size_t q = 0; q < (size_t)dims[l] * dims[l + 1]; ++q) h[w_off[l] + q] = (float)nd(rng);
    }
    MQCT_CUDA_TRY(par.upload(h, stream));
    MQCT_CUDA_TRY(grad.alloc(n_par));
    MQCT_CUDA_TRY(adam_m.alloc(n_par));
    MQCT_CUDA_TRY(adam_v.alloc(n_par));
    MQCT_CUDA_TRY(cudaMemsetAsync(adam_m.p, 0, n_par * sizeof(float), stream));
    MQCT_CUDA_TRY(cudaMemsetAsync(adam_v.p, 0, n_par * sizeof(float), stream));
    MQCT_CUDA_TRY(d_loss.alloc(1));
    pes_kind = pes->kind;
    pes_n_terms = pes->n_terms;
    const size_t per = pes->kind == MQCT_PES_LEGENDRE ? 3 : (pes->kind == MQCT_PES_SITES1 ? 6 : 7);
    MQCT_CUDA_TRY(pes_p.upload(pes->params, per * (size_t)pes->n_terms, stream));
    if (pes->kind == MQCT_PES_SITES1 || pes->kind == MQCT_PES_SITES2) {
      MQCT_ARG_CHECK(pes->sites1 && pes->n_sites1 > 0, "PES without sites");
      pes_n1 = pes->n_sites1;
      MQCT_CUDA_TRY(pes_s1.upload(pes->sites1, 3 * (size_t)pes_n1, stream));
      for (int t = 0; t < pes->n_terms; ++t)
        MQCT_ARG_CHECK((int)pes->params[per * t] >= 0 && (int)pes->params[per * t] < pes_n1,
                       "PES term %d references a missing site", t);
    }
    if (pes->kind == MQCT_PES_SITES2) {
      MQCT_ARG_CHECK(pes->sites2 && pes->n_sites2 > 0, "PES without rotor-2 sites");
      pes_n2 = pes->n_sites2;
      MQCT_CUDA_TRY(pes_s2.upload(pes->sites2, 3 * (size_t)pes_n2, stream));
      for (int t = 0; t < pes->n_terms; ++t)
        MQCT_ARG_CHECK((int)pes->params[7 * t + 1] >= 0 && (int)pes->params[7 * t + 1] < pes_n2,
                       "PES term %d references a missing rotor-2 site", t);
    }
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  int train(int64_t n_samples, int epochs, int batch, double lr0, double* loss_epoch,
            double* val_rmse) {
    MQCT_ARG_CHECK(n_samples >= batch && batch >= 16 && batch <= (1 << 20) && epochs >= 1,
                   "bad training sizes");
    MQCT_ARG_CHECK(n_samples < (int64_t)1 << 31, "too many samples");
    cur = stream;
    DevBuf<float> X, Y, Xv, Yv;
    DevBuf<int> perm;
    const int64_t n_val = std::min<int64_t>(65536, std::max<int64_t>(batch, n_samples / 16));
    MQCT_CUDA_TRY(X.alloc((size_t)n_samples * SG_IN));
    MQCT_CUDA_TRY(Y.alloc((size_t)n_samples));
    MQCT_CUDA_TRY(Xv.alloc((size_t)n_val * SG_IN));
    MQCT_CUDA_TRY(Yv.alloc((size_t)n_val));
    const PesDev pd = pes_dev();
    sg_sample_kernel<<<(unsigned)((n_samples + 255) / 256), 256, 0, stream>>>(
        n_samples, seed * 2 + 1, sys_type, pd, r_lo, r_hi, r_c, r_s, X.p, Y.p, nullptr);
    MQCT_CUDA_TRY(cudaGetLastError());
    sg_sample_kernel<<<(unsigned)((n_val + 255) / 256), 256, 0, stream>>>(
        n_val, seed * 2 + 2, sys_type, pd, r_lo, r_hi, r_c, r_s, Xv.p, Yv.p, nullptr);
    MQCT_CUDA_TRY(cudaGetLastError());
    int rc = ensure_workspace(std::max<int>(batch, (int)std::min<int64_t>(n_val, 65536)));
    if (rc) return rc;
    std::vector<int> order(n_samples);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed + 7);
    const int64_t steps_per_epoch = n_samples / batch;
    const int64_t total = steps_per_epoch * epochs;
    int64_t step = 0;
    for (int e = 0; e < epochs; ++e) {
      std::shuffle(order.begin(), order.end(), rng);
      MQCT_CUDA_TRY(perm.upload(order, stream));
      double acc = 0.0;
      for (int64_t b = 0; b < steps_per_epoch; ++b, ++step) {
        sg_gather_kernel<<<(batch + 255) / 256, 256, 0, cur>>>(batch, perm.p + b * batch, X.p,
                                                                 Y.p, xb.p, yb.p);
        MQCT_CUDA_TRY(cudaGetLastError());
        const bool want = b + 1 == steps_per_epoch;
        double l = 0.0;
        rc = loss_grad(xb.p, yb.p, batch, want ? &l : nullptr);
        if (rc) return rc;
        acc = l;
        // cosine decay of the learning rate to 1% of lr0
        const double fr = (double)step / (double)std::max<int64_t>(1, total - 1);
        const double lr = lr0 * (0.01 + 0.99 * 0.5 * (1.0 + std::cos(kPi * fr)));
        rc = adam_step((float)lr);
        if (rc) return rc;
      }
      if (loss_epoch) loss_epoch[e] = acc;
    }
    if (val_rmse) {
      double se = 0.0;
      for (int64_t s = 0; s < n_val; s += 65536) {
        const int rows = (int)std::min<int64_t>(65536, n_val - s);
        rc = forward(Xv.p + s * SG_IN, rows);
        if (rc) return rc;
        sg_loss_kernel<<<1, 1024, 0, stream>>>(rows, Hs[n_layers() - 1].p, Yv.p + s, dpred.p,
                                              d_loss.p);
        MQCT_CUDA_TRY(cudaGetLastError());
        double l = 0.0;
        MQCT_CUDA_TRY(cudaMemcpyAsync(&l, d_loss.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
        MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
        se += l * rows;
      }
      *val_rmse = std::sqrt(se / n_val);
    }
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  ~Surrogate() {
    if (stream) cudaStreamDestroy(stream);
  }
};

// Bridge for the matrix plan (the plan owns no surrogate state).
int surrogate_predict_on(void* sur, const float* X, int64_t n, double* v_out, cudaStream_t st) {
  Surrogate* s = reinterpret_cast<Surrogate*>(sur);
  s->cur = st;
  const int rc = s->predict_features(X, n, v_out);
  s->cur = s->stream;
  return rc;
}
void surrogate_feature_map(const void* sur, int* sys_type, double* r_c, double* r_s) {
  const Surrogate* s = reinterpret_cast<const Surrogate*>(sur);
  *sys_type = s->sys_type;
  *r_c = s->r_c;
  *r_s = s->r_s;
}

}  // namespace mqct

extern "C" {

int mqct_surrogate_create(int32_t sys_type, const mqct_pes_t* pes, int32_t hidden,
                          int32_t n_hidden_layers, uint64_t seed, double r_min, double r_max,
                          mqct_surrogate** out) {
  MQCT_ARG_CHECK(out, "null output pointer");
  *out = nullptr;
  if (mqct_device_count() <= 0) {
    set_error("no CUDA device available");
    return MQCT_E_NODEV;
  }
  auto* s = new Surrogate();
  int rc = s->init(sys_type, pes, hidden, n_hidden_layers, seed, r_min, r_max);
  if (rc) {
    delete s;
    return rc;
  }
  *out = reinterpret_cast<mqct_surrogate*>(s);
  return MQCT_OK;
}

int mqct_surrogate_train(mqct_surrogate* sur, int64_t n_samples, int32_t epochs, int32_t batch,
                         double lr, double* loss_per_epoch, double* val_rmse) {
  MQCT_ARG_CHECK(sur, "null surrogate");
  return reinterpret_cast<Surrogate*>(sur)->train(n_samples, epochs, batch, lr, loss_per_epoch,
                                                  val_rmse);
}

int mqct_surrogate_predict(mqct_surrogate* sur, const double* args, int64_t n, double* v_out) {
  MQCT_ARG_CHECK(sur && args && v_out && n > 0, "null argument");
  Surrogate* s = reinterpret_cast<Surrogate*>(sur);
  DevBuf<double> da, dv;
  DevBuf<float> X;
  MQCT_CUDA_TRY(da.upload(args, (size_t)n * 6, s->stream));
  MQCT_CUDA_TRY(dv.alloc((size_t)n));
  MQCT_CUDA_TRY(X.alloc((size_t)n * SG_IN));
  sg_features_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(n, da.p, s->r_c, s->r_s,
                                                                          X.p);
  MQCT_CUDA_TRY(cudaGetLastError());
  s->cur = s->stream;
  int rc = s->predict_features(X.p, n, dv.p);
  if (rc) return rc;
  MQCT_CUDA_TRY(cudaMemcpyAsync(v_out, dv.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  MQCT_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return MQCT_OK;
}

int64_t mqct_surrogate_n_params(const mqct_surrogate* sur) {
  return sur ? (int64_t)reinterpret_cast<const Surrogate*>(sur)->n_par : 0;
}

int mqct_surrogate_get_params(mqct_surrogate* sur, float* out) {
  MQCT_ARG_CHECK(sur && out, "null argument");
  Surrogate* s = reinterpret_cast<Surrogate*>(sur);
  MQCT_CUDA_TRY(cudaMemcpyAsync(out, s->par.p, s->n_par * sizeof(float), cudaMemcpyDeviceToHost,
                                s->stream));
  MQCT_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return MQCT_OK;
}

int mqct_surrogate_loss_grad(mqct_surrogate* sur, const float* X, const float* y, int32_t n,
                             double* loss, float* grad_out) {
  MQCT_ARG_CHECK(sur && X && y && loss && grad_out && n > 0, "null argument");
  Surrogate* s = reinterpret_cast<Surrogate*>(sur);
  DevBuf<float> dx, dy;
  MQCT_CUDA_TRY(dx.upload(X, (size_t)n * SG_IN, s->stream));
  MQCT_CUDA_TRY(dy.upload(y, (size_t)n, s->stream));
  s->cur = s->stream;
  int rc = s->loss_grad(dx.p, dy.p, n, loss);
  if (rc) return rc;
  MQCT_CUDA_TRY(cudaMemcpyAsync(grad_out, s->grad.p, s->n_par * sizeof(float),
                                cudaMemcpyDeviceToHost, s->stream));
  MQCT_CUDA_TRY(cudaStreamSynchronize(s->stream));
  return MQCT_OK;
}

void mqct_surrogate_destroy(mqct_surrogate* sur) { delete reinterpret_cast<Surrogate*>(sur); }

}  // extern "C"
