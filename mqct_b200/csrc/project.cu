// CALC_EXPANSION_TERMS on the GPU (MQCT_SOURCE_CODES/pot_comp.f:4695-6274): the
// quadrature projection of a PES tabulated on the angular grid onto the expansion
// terms, for SYS_TYPE 7, 8 (rigid top + diatom) and 0 (two rigid tops).
//
// The reference evaluates EXPANSION_TERM (pot_comp.f:3739-3896) at every grid point for
// every term and R point.  A term's angular function factorises,
//   Y_t(g) = sum_m K_t c_tm a_tm(beta1) b_tm(beta2) e^{i(nju1 gamma1 + nju2 gamma2)} e^{-i m alpha2},
// with c_tm = <l1 m l2 -m|l 0>, a = d^{l1}_{nju1 m} and b = the diatom's normalised
// Legendre function of order -m (types 7, 8) or d^{l2}_{nju2,-m} (type 0), so the sum
// over the grid runs as three contractions, one per group of axes:
//   F[R][a2][p][b] = sum_{g1,g2} V[R][a2][b][g1,g2] E_p(g1,g2)       (gamma, per (nju1, nju2) pair p)
//   H[R][p][m][b]  = sum_{a2} F[R][a2][p][b] e^{-i m alpha2} w       (alpha2, per m)
//   S_t(R)         = sum_m sum_b A_tm(b1) B_tm(b2) H[R][p_t][m][b]    (beta1 x beta2 = b)
// with every quadrature weight folded into the tables E, A and B; terms = Re S,
// terms_im = Im S (the reference's intgrlr and intgrli).  The first contraction reads V
// once and carries the bandwidth; the other two run on arrays a few times smaller.
// FP64 throughout; every sum in a fixed order, so results are reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "mqct_b200.h"

namespace mqct {
namespace {

constexpr int kMaxL = 40;          // largest l1, l2, l of a term (log factorials to 127)
constexpr int kThreads = 256;
constexpr int kMBlock = 4;         // m values per thread of the alpha contraction

struct TermDev {
  int pair;     // index of the term's (nju1, nju2) in the pair list
  int m_lo, m_hi;
};

// F[(blk * P + p) * J + j] for row = blk * J + j, blk = R * n_a2 + i_a2,
// j = i_b1 * n_b2 + i_b2: one CTA stages kRows consecutive rows of V (each L = n_g1 * n_g2
// doubles, contiguous in V) in shared memory, threads then run over (p, row).
__global__ void proj_gamma_kernel(const double* __restrict__ V, int64_t n_rows, int L,
                                  int L_pad, int rows_per_cta, int P, int J,
                                  const double2* __restrict__ E, double2* __restrict__ F) {
  extern __shared__ double vs[];
  const int64_t row0 = (int64_t)blockIdx.x * rows_per_cta;
  const int64_t left = n_rows - row0;
  const int nr = left < rows_per_cta ? (int)left : rows_per_cta;
  const double* src = V + row0 * L;
  for (int i = threadIdx.x; i < nr * L; i += blockDim.x) {
    const int r = i / L, k = i - r * L;
    vs[r * L_pad + k] = __ldg(src + i);
  }
  __syncthreads();
  for (int w = threadIdx.x; w < nr * P; w += blockDim.x) {
    const int p = w / nr, r = w - p * nr;
    const double* v = vs + r * L_pad;
    double re = 0.0, im = 0.0;
    for (int k = 0; k < L; ++k) {
      const double2 e = __ldg(E + (size_t)k * P + p);
      re = fma(v[k], e.x, re);
      im = fma(v[k], e.y, im);
    }
    const int64_t row = row0 + r;
    const int64_t blk = row / J;
    const int j = (int)(row - blk * J);
    F[(blk * P + p) * J + j] = make_double2(re, im);
  }
}

// H[((R * P + p) * n_m + mi) * J + j] = sum_{a2} E2[mi][a2] F[R][a2][p][j]; each thread
// forms kMBlock consecutive m values of one (R, p, j).
__global__ void proj_alpha_kernel(const double2* __restrict__ F, int nR, int n_a2, int P, int J,
                                  int n_m, const double2* __restrict__ E2,
                                  double2* __restrict__ H) {
  const int n_mb = (n_m + kMBlock - 1) / kMBlock;
  const int64_t total = (int64_t)nR * P * n_mb * J;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(idx % J);
    int64_t q = idx / J;
    const int mb = (int)(q % n_mb);
    q /= n_mb;
    const int p = (int)(q % P);
    const int R = (int)(q / P);
    const int m0 = mb * kMBlock;
    double2 acc[kMBlock];
#pragma unroll
    for (int u = 0; u < kMBlock; ++u) acc[u] = make_double2(0.0, 0.0);
    for (int a = 0; a < n_a2; ++a) {
      const double2 f = F[(((int64_t)R * n_a2 + a) * P + p) * J + j];
#pragma unroll
      for (int u = 0; u < kMBlock; ++u) {
        if (m0 + u >= n_m) break;
        const double2 e = __ldg(E2 + (size_t)(m0 + u) * n_a2 + a);
        acc[u].x = fma(f.x, e.x, fma(-f.y, e.y, acc[u].x));
        acc[u].y = fma(f.x, e.y, fma(f.y, e.x, acc[u].y));
      }
    }
#pragma unroll
    for (int u = 0; u < kMBlock; ++u) {
      if (m0 + u >= n_m) break;
      H[(((int64_t)R * P + p) * n_m + m0 + u) * J + j] = acc[u];
    }
  }
}

// One warp per (term, R): lanes run over the beta1 x beta2 points, then a fixed
// shuffle tree.  A[t][mi][b1], B[t][mi][b2] hold K_t c_tm a_tm w and b_tm w.
__global__ void proj_terms_kernel(const double2* __restrict__ H, int nR, int r0, int nR_all,
                                  int P, int J, int n_b2, int n_b1, int n_m,
                                  const TermDev* __restrict__ terms, int n_terms,
                                  const double* __restrict__ A, const double* __restrict__ B,
                                  double* __restrict__ out_re, double* __restrict__ out_im) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= (int64_t)n_terms * nR) return;
  const int t = (int)(wid / nR), R = (int)(wid % nR);
  const TermDev td = terms[t];
  double re = 0.0, im = 0.0;
  for (int m = td.m_lo; m <= td.m_hi; ++m) {
    const int mi = m + (n_m - 1) / 2;
    const double2* h = H + (((int64_t)R * P + td.pair) * n_m + mi) * J;
    const double* a = A + ((size_t)t * n_m + mi) * n_b1;
    const double* b = B + ((size_t)t * n_m + mi) * n_b2;
    for (int j = lane; j < J; j += 32) {
      const int i1 = j / n_b2, i2 = j - i1 * n_b2;
      const double w = __ldg(a + i1) * __ldg(b + i2);
      const double2 v = h[j];
      re = fma(w, v.x, re);
      im = fma(w, v.y, im);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  if (lane == 0) {
    out_re[(size_t)t * nR_all + r0 + R] = re;
    if (out_im) out_im[(size_t)t * nR_all + r0 + R] = im;
  }
}

// The reference's checks of a term list before the projection
// (pot_comp.f:5174-5240, 5296-5350, 5557-5690): triangle rule, nju1 >= 0, for SYS_TYPE 0
// nju2 >= 0 when nju1 = 0, and no term twice, a term with (nju1, nju2) -> (-nju1, -nju2)
// counting as the same; for identical partners (type 0) also l1 >= l2, |nju1| >= |nju2|
// when l1 = l2, and the exchange (l1, nju1) <-> (l2, nju2) counting as the same.  Beyond
// the reference: |nju| <= l (the D function is undefined otherwise) and l <= kMaxL.
int check_terms(int sys_type, int n_terms, const int32_t* a_top, int identical) {
  struct Lab {
    int l1, n1, l2, n2, l;
  };
  std::vector<Lab> lab(n_terms);
  for (int t = 0; t < n_terms; ++t) {
    const int32_t* q = a_top + 5 * t;
    Lab& x = lab[t];
    if (sys_type == 0) x = {q[0], q[1], q[2], q[3], q[4]};
    else x = {q[0], q[1], q[2], 0, q[3]};
    MQCT_ARG_CHECK(x.l1 >= 0 && x.l2 >= 0 && x.l >= 0 && x.l1 <= kMaxL && x.l2 <= kMaxL &&
                       x.l <= kMaxL,
                   "term %d: l1, l2, l must be in 0..%d", t + 1, kMaxL);
    MQCT_ARG_CHECK(std::max(std::max(x.l1, x.l2), x.l) * 2 <= x.l1 + x.l2 + x.l,
                   "term %d (%d,%d,%d): TRIANGULAR RULE FAILED", t + 1, x.l1, x.l2, x.l);
    MQCT_ARG_CHECK(x.n1 >= 0, "term %d: the values of M1 should be always positive", t + 1);
    MQCT_ARG_CHECK(!(x.n1 == 0 && x.n2 < 0),
                   "term %d: the values of M2 should be positive only for M1 = 0", t + 1);
    MQCT_ARG_CHECK(x.n1 <= x.l1 && std::abs(x.n2) <= x.l2, "term %d: |nju| exceeds its l",
                   t + 1);
    if (identical) {
      MQCT_ARG_CHECK(x.l1 >= x.l2, "term %d: the values of L2 should be less or equal to L1",
                     t + 1);
      MQCT_ARG_CHECK(!(x.l1 == x.l2 && std::abs(x.n1) < std::abs(x.n2)),
                     "term %d: the values of M1 should be greater or equal to abs(M2) for "
                     "L1 = L2",
                     t + 1);
    }
  }
  for (int t = 0; t < n_terms; ++t)
    for (int u = 0; u < n_terms; ++u) {
      if (u == t) continue;
      const Lab& a = lab[t];
      const Lab& b = lab[u];
      for (int ex = 0; ex < ((identical && sys_type == 0) ? 2 : 1); ++ex) {
        Lab c = ex ? Lab{a.l2, a.n2, a.l1, a.n1, a.l} : a;
        for (int s = 0; s < 2; ++s) {
          if (s == 1) {
            if (c.n1 == 0 && c.n2 == 0) break;
            c.n1 = -c.n1;
            c.n2 = -c.n2;
          }
          MQCT_ARG_CHECK(!(b.l1 == c.l1 && b.n1 == c.n1 && b.l2 == c.l2 && b.n2 == c.n2 &&
                           b.l == c.l),
                         "found two same terms: %d and %d", t + 1, u + 1);
        }
      }
    }
  return MQCT_OK;
}

}  // namespace
}  // namespace mqct

using namespace mqct;

struct mqct_projection_plan {
  int sys_type = 8, n_terms = 0;
  int n_a2 = 0, n_b1 = 0, n_b2 = 0, n_g1 = 0, n_g2 = 1;
  int P = 0, n_m = 0, J = 0, L = 0;
  DevBuf<double2> E, E2;
  DevBuf<double> A, B;
  DevBuf<TermDev> terms;
  DevBuf<double2> F, H;
  int chunk_R = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  float ms[3] = {0.f, 0.f, 0.f};
  bool timed = false;

  ~mqct_projection_plan() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  int init(int sys, int nt, const int32_t* a_top, const mqct_grid_t& g, int identical) {
    MQCT_ARG_CHECK(sys == 7 || sys == 8 || sys == 0,
                   "the projection is built for SYS_TYPE 7, 8 and 0 (got %d)", sys);
    MQCT_ARG_CHECK(nt > 0 && a_top, "no terms");
    MQCT_ARG_CHECK(!identical || sys == 0, "identical partners are SYS_TYPE 0");
    sys_type = sys;
    n_terms = nt;
    n_a2 = g.n_alpha2;
    n_b1 = g.n_beta;
    n_b2 = g.n_beta2;
    n_g1 = g.n_gamma;
    n_g2 = sys == 0 ? g.n_gamma2 : 1;
    MQCT_ARG_CHECK(n_a2 > 0 && n_b1 > 0 && n_b2 > 0 && n_g1 > 0 && n_g2 > 0 && n_a2 <= 4096 &&
                       n_b1 <= 4096 && n_b2 <= 4096 && n_g1 <= 4096 && n_g2 <= 4096,
                   "grid sizes must be in 1..4096 (alpha2 %d, beta1 %d, beta2 %d, gamma1 %d, "
                   "gamma2 %d)",
                   n_a2, n_b1, n_b2, n_g1, n_g2);
    int rc = check_terms(sys, nt, a_top, identical);
    if (rc != MQCT_OK) return rc;
    J = n_b1 * n_b2;
    L = n_g1 * n_g2;
    MQCT_ARG_CHECK((int64_t)L * 8 <= 40 * 1024, "n_gamma1 * n_gamma2 = %d exceeds 5120", L);
    if (mqct_device_count() <= 0) {
      set_error("no CUDA device available");
      return MQCT_E_NODEV;
    }
    // axes as INI_POT_STORAGE sets them (pot_comp.f:1310-1370, 1628-1700)
    const Axis b1 = axis_gl(n_b1, 0.0, kPi), b2 = axis_gl(n_b2, 0.0, kPi);
    auto ang = [&](int n) { return g.eq_gamma ? axis_mid(n, 0.0, 2.0 * kPi) : axis_gl(n, 0.0, 2.0 * kPi); };
    const Axis a2 = ang(n_a2), g1 = ang(n_g1);
    Axis g2 = ang(n_g2);
    if (sys != 0) {  // no second gamma: one point, unit weight
      g2.x.assign(1, 0.0);
      g2.w.assign(1, 1.0);
      g2.half = 1.0;
    }
    const double tail2 = sys == 0 ? 2.0 * kPi : 1.0;  // the alpha1 integral of type 0
    std::vector<double> lf(128);
    lf[0] = 0.0;
    for (int i = 1; i < 128; ++i) lf[i] = lf[i - 1] + std::log((double)i);
    // (nju1, nju2) pairs and the m range
    std::vector<std::pair<int, int>> pairs;
    std::vector<TermDev> td(nt);
    int m_max = 0;
    for (int t = 0; t < nt; ++t) {
      const int32_t* q = a_top + 5 * t;
      const int l1 = q[0], n1 = q[1], l2 = q[2], n2 = sys == 0 ? q[3] : 0;
      const std::pair<int, int> pr(n1, n2);
      auto it = std::find(pairs.begin(), pairs.end(), pr);
      td[t].pair = (int)(it - pairs.begin());
      if (it == pairs.end()) pairs.push_back(pr);
      const int mm = std::min(l1, l2);
      td[t].m_lo = -mm;
      td[t].m_hi = mm;
      m_max = std::max(m_max, mm);
    }
    P = (int)pairs.size();
    n_m = 2 * m_max + 1;
    // E[k][p], k = i_g1 * n_g2 + i_g2
    std::vector<double2> e((size_t)L * P), e2((size_t)n_m * n_a2);
    for (int i5 = 0; i5 < n_g1; ++i5)
      for (int i6 = 0; i6 < n_g2; ++i6)
        for (int p = 0; p < P; ++p) {
          const double ph = pairs[p].first * g1.x[i5] + pairs[p].second * g2.x[i6];
          const double w = g1.w[i5] * g1.half * g2.w[i6] * g2.half * tail2;
          e[((size_t)i5 * n_g2 + i6) * P + p] = make_double2(std::cos(ph) * w, std::sin(ph) * w);
        }
    for (int mi = 0; mi < n_m; ++mi)
      for (int i2 = 0; i2 < n_a2; ++i2) {
        const double ph = -(double)(mi - m_max) * a2.x[i2];
        const double w = a2.w[i2] * a2.half;
        e2[(size_t)mi * n_a2 + i2] = make_double2(std::cos(ph) * w, std::sin(ph) * w);
      }
    // A[t][mi][b1] = K_t c_tm d^{l1}_{nju1 m}(beta1) w, B[t][mi][b2] = b_tm(beta2) w
    std::vector<double> ta((size_t)nt * n_m * n_b1, 0.0), tb((size_t)nt * n_m * n_b2, 0.0);
    for (int t = 0; t < nt; ++t) {
      const int32_t* q = a_top + 5 * t;
      const int l1 = q[0], n1 = q[1], l2 = q[2];
      const int n2 = sys == 0 ? q[3] : 0, l = sys == 0 ? q[4] : q[3];
      const double K = sys == 0 ? std::sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0)) / (8.0 * kPi * kPi)
                                : std::sqrt((2.0 * l1 + 1.0) / 4.0 / kPi);
      for (int m = td[t].m_lo; m <= td[t].m_hi; ++m) {
        const int mi = m + m_max;
        const double c = mqct_dev::clebsch_gordan(l1, m, l2, -m, l, 0, lf.data());
        for (int i = 0; i < n_b1; ++i)
          ta[((size_t)t * n_m + mi) * n_b1 + i] =
              K * c * mqct_dev::wigner_d(l1, n1, m, b1.x[i], lf.data()) * b1.w[i] *
              std::sin(b1.x[i]) * b1.half;
        for (int i = 0; i < n_b2; ++i) {
          double bv;
          if (sys == 0) {
            bv = mqct_dev::wigner_d(l2, n2, -m, b2.x[i], lf.data());
          } else {  // WF_DIAT_TOP(l2, -m, beta2, .) without its phase
            const int am = std::abs(m);
            bv = mqct_dev::plgndr(l2, am, std::cos(b2.x[i])) *
                 std::sqrt((2.0 * l2 + 1.0) / 4.0 / kPi * std::exp(lf[l2 - am] - lf[l2 + am]));
            if (m > 0 && (am & 1)) bv = -bv;
          }
          tb[((size_t)t * n_m + mi) * n_b2 + i] = bv * b2.w[i] * std::sin(b2.x[i]) * b2.half;
        }
      }
    }
    MQCT_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& x : ev) MQCT_CUDA_TRY(cudaEventCreate(&x));
    MQCT_CUDA_TRY(E.upload(e, st));
    MQCT_CUDA_TRY(E2.upload(e2, st));
    MQCT_CUDA_TRY(A.upload(ta, st));
    MQCT_CUDA_TRY(B.upload(tb, st));
    MQCT_CUDA_TRY(terms.upload(td, st));
    MQCT_CUDA_TRY(cudaStreamSynchronize(st));
    return MQCT_OK;
  }

  // R points per pass so that F and H stay within 4 GiB.
  int pass_R(int nR) const {
    const size_t per_R = ((size_t)n_a2 * P * J + (size_t)P * n_m * J) * sizeof(double2);
    const size_t cap = (size_t)4 << 30;
    return (int)std::max<size_t>(1, std::min<size_t>(nR, cap / per_R));
  }

  int execute(const double* d_V, int nR, double* d_terms, double* d_terms_im) {
    MQCT_ARG_CHECK(d_V && d_terms && nR > 0, "null argument or nR <= 0");
    const int rc_R = pass_R(nR);
    if (F.n < (size_t)rc_R * n_a2 * P * J) MQCT_CUDA_TRY(F.alloc((size_t)rc_R * n_a2 * P * J));
    if (H.n < (size_t)rc_R * P * n_m * J) MQCT_CUDA_TRY(H.alloc((size_t)rc_R * P * n_m * J));
    const int L_pad = L | 1;
    const int rows_per_cta = std::max(1, std::min(64, (40 * 1024 / 8) / L_pad));
    const size_t smem = (size_t)rows_per_cta * L_pad * sizeof(double);
    const size_t G = (size_t)n_a2 * J * L;
    bool first = true;
    for (int r0 = 0; r0 < nR; r0 += rc_R) {
      const int nr = std::min(rc_R, nR - r0);
      const int64_t n_rows = (int64_t)nr * n_a2 * J;
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[0], st));
      const int64_t nb = (n_rows + rows_per_cta - 1) / rows_per_cta;
      proj_gamma_kernel<<<(unsigned)nb, kThreads, smem, st>>>(d_V + (size_t)r0 * G, n_rows, L,
                                                              L_pad, rows_per_cta, P, J, E.p, F.p);
      MQCT_CUDA_TRY(cudaGetLastError());
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[1], st));
      const int64_t na = (int64_t)nr * P * ((n_m + kMBlock - 1) / kMBlock) * J;
      const int64_t ba = std::min<int64_t>((na + kThreads - 1) / kThreads, 148 * 64);
      proj_alpha_kernel<<<(unsigned)ba, kThreads, 0, st>>>(F.p, nr, n_a2, P, J, n_m, E2.p, H.p);
      MQCT_CUDA_TRY(cudaGetLastError());
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[2], st));
      const int64_t warps = (int64_t)n_terms * nr;
      proj_terms_kernel<<<(unsigned)((warps * 32 + kThreads - 1) / kThreads), kThreads, 0, st>>>(
          H.p, nr, r0, nR, P, J, n_b2, n_b1, n_m, terms.p, n_terms, A.p, B.p, d_terms,
          d_terms_im);
      MQCT_CUDA_TRY(cudaGetLastError());
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[3], st));
      first = false;
    }
    timed = nR <= rc_R;
    return MQCT_OK;
  }
};

extern "C" int mqct_projection_plan_create(int32_t sys_type, int32_t n_terms,
                                           const int32_t* a_top, const mqct_grid_t* grid,
                                           int32_t identical, mqct_projection_plan** plan) {
  MQCT_ARG_CHECK(grid && plan, "null argument");
  auto* p = new mqct_projection_plan();
  const int rc = p->init(sys_type, n_terms, a_top, *grid, identical);
  if (rc != MQCT_OK) {
    delete p;
    *plan = nullptr;
    return rc;
  }
  *plan = p;
  return MQCT_OK;
}

extern "C" int mqct_projection_plan_execute(mqct_projection_plan* plan, const double* d_V,
                                            int32_t nR, double* d_terms, double* d_terms_im) {
  MQCT_ARG_CHECK(plan, "null plan");
  return plan->execute(d_V, nR, d_terms, d_terms_im);
}

extern "C" int mqct_projection_plan_sync(mqct_projection_plan* plan) {
  MQCT_ARG_CHECK(plan, "null plan");
  MQCT_CUDA_TRY(cudaStreamSynchronize(plan->st));
  return MQCT_OK;
}

extern "C" int mqct_projection_plan_timing(mqct_projection_plan* plan, float* ms_gamma,
                                           float* ms_alpha, float* ms_terms) {
  MQCT_ARG_CHECK(plan && ms_gamma && ms_alpha && ms_terms, "null argument");
  MQCT_ARG_CHECK(plan->timed, "no single-pass execute to time");
  MQCT_CUDA_TRY(cudaEventSynchronize(plan->ev[3]));
  MQCT_CUDA_TRY(cudaEventElapsedTime(ms_gamma, plan->ev[0], plan->ev[1]));
  MQCT_CUDA_TRY(cudaEventElapsedTime(ms_alpha, plan->ev[1], plan->ev[2]));
  MQCT_CUDA_TRY(cudaEventElapsedTime(ms_terms, plan->ev[2], plan->ev[3]));
  return MQCT_OK;
}

extern "C" void mqct_projection_plan_destroy(mqct_projection_plan* plan) { delete plan; }

extern "C" int mqct_project_terms(int32_t sys_type, int32_t n_terms, const int32_t* a_top,
                                  const mqct_grid_t* grid, int32_t identical, int32_t nR,
                                  const double* V, double* terms, double* terms_im) {
  MQCT_ARG_CHECK(V && terms && nR > 0, "null argument or nR <= 0");
  mqct_projection_plan* plan = nullptr;
  int rc = mqct_projection_plan_create(sys_type, n_terms, a_top, grid, identical, &plan);
  if (rc != MQCT_OK) return rc;
  struct Guard {
    mqct_projection_plan* p;
    ~Guard() { delete p; }
  } guard{plan};
  const size_t nV = (size_t)nR * plan->n_a2 * plan->J * plan->L;
  DevBuf<double> dV, dT, dI;
  MQCT_CUDA_TRY(dV.upload(V, nV, plan->st));
  MQCT_CUDA_TRY(dT.alloc((size_t)n_terms * nR));
  if (terms_im) MQCT_CUDA_TRY(dI.alloc((size_t)n_terms * nR));
  rc = plan->execute(dV.p, nR, dT.p, terms_im ? dI.p : nullptr);
  if (rc != MQCT_OK) return rc;
  MQCT_CUDA_TRY(cudaMemcpyAsync(terms, dT.p, sizeof(double) * n_terms * nR,
                                cudaMemcpyDeviceToHost, plan->st));
  if (terms_im)
    MQCT_CUDA_TRY(cudaMemcpyAsync(terms_im, dI.p, sizeof(double) * n_terms * nR,
                                  cudaMemcpyDeviceToHost, plan->st));
  MQCT_CUDA_TRY(cudaStreamSynchronize(plan->st));
  return MQCT_OK;
}
