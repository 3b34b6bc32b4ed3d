// CALC_EXPANSION_TERMS on the GPU (MQCT_SOURCE_CODES/pot_comp.f:4695-6274): the
// quadrature projection of a PES tabulated on the angular grid onto the expansion
// terms, for SYS_TYPE 7, 8 (rigid top + diatom) and 0 (two rigid tops).
//
// The reference evaluates EXPANSION_TERM (pot_comp.f:3739-3896) at every grid point for
// every term and R point.  A term's angular function factorises,
//   Y_t(g) = sum_m K_t c_tm a_tm(beta1) b_tm(beta2) e^{i(nju1 gamma1 + nju2 gamma2)} e^{-i m alpha2},
// with c_tm = <l1 m l2 -m|l 0>, a = d^{l1}_{nju1 m} and b = the diatom's normalised
// Legendre function of order -m (types 7, 8) or d^{l2}_{nju2,-m} (type 0), so the sum
// over the grid runs as four contractions, one per axis group:
//   F[R][a2][p][b]      = sum_{g1,g2} V[R][a2][b][g1,g2] E_p(g1,g2)   (gamma, per pair p = (nju1, nju2))
//   H[R][p][m][b]       = sum_{a2} F[R][a2][p][b] e^{-i m alpha2} w   (alpha2, per m)
//   K[R][p][m][l2][b1]  = sum_{b2} B_{p,l2,m}(b2) H[R][p][m][b1,b2]    (beta2, per l2)
//   S_t(R)              = sum_m sum_{b1} A_tm(b1) K[R][p_t][m][l2_t][b1]   (beta1, per term)
// with every quadrature weight folded into the tables E, A and B; terms = Re S,
// terms_im = Im S (the reference's intgrlr and intgrli).  The first contraction reads V
// once and carries the bandwidth; the others run on arrays 6x to 100x smaller.  The
// gamma and alpha contractions are real GEMMs with a small constant operand, issued as
// FP64 tensor-core MMAs (mma.sync m8n8k4 f64, 256 FMAs per warp instruction) so that the
// kernel stays bound by reading V rather than by instruction issue.  FP64 throughout;
// every sum in a fixed order, so results are reproducible.
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
constexpr int kKSteps = 16;        // k-steps of 4 columns whose V values a lane loads at once

struct TermDev {
  int pair;     // index of the term's (nju1, nju2) in the pair list
  int l2;
  int m_lo, m_hi;
};

// D (8x8) += A (8x4, row) * B (4x8, col) in FP64: lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2 (l%4)], D[l/4][2 (l%4) + 1].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Gamma contraction as the GEMM F(rows x 8 NT) = V(rows x L) Eb(L x 8 NT): V read as the
// row-major matrix of its rows (row = blk * J + j, blk = R * n_a2 + i_a2,
// j = i_b1 * n_b2 + i_b2, L = n_g1 * n_g2 contiguous doubles), Eb the packed table of
// column n = 2 q + part (Re / Im of E for pair 4 tile + q), Lp = L rounded up to 4,
// Eb[(tile * Lp + k) * 8 + n].  A warp takes 8 rows at a time: each lane loads the
// kKSteps values of its (row, column) slots at once (8 rows x 32 bytes per load
// instruction), then the MMAs run over the k-steps for the NT pair tiles.
// F[(blk * P + p) * J + j] (complex).
template <int NT>
__global__ void __launch_bounds__(kThreads)
    proj_gamma_kernel(const double* __restrict__ V, int64_t n_rows, int L, int Lp, int P,
                      int tile0, int J, const double* __restrict__ Eb, double2* __restrict__ F) {
  const int lane = threadIdx.x & 31, kq = lane & 3, rq = lane >> 2;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t tile = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; tile * 8 < n_rows;
       tile += nwarps) {
    const int64_t row = tile * 8 + rq;
    const bool ok = row < n_rows;
    const double* src = V + (ok ? row : 0) * L;
    double c[NT][2];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) c[nt][0] = c[nt][1] = 0.0;
    for (int k0 = 0; k0 < Lp; k0 += 4 * kKSteps) {
      double a[kKSteps];
#pragma unroll
      for (int s = 0; s < kKSteps; ++s) {
        const int k = k0 + 4 * s + kq;
        a[s] = (ok && k < L) ? __ldg(src + k) : 0.0;
      }
#pragma unroll
      for (int s = 0; s < kKSteps; ++s) {
        const int kk = k0 + 4 * s;
        if (kk >= Lp) break;  // the same for the whole warp
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const double b = __ldg(Eb + ((size_t)(tile0 + nt) * Lp + kk + kq) * 8 + rq);
          dmma(c[nt][0], c[nt][1], a[s], b);
        }
      }
    }
    if (ok) {
      const int64_t blk = row / J;
      const int j = (int)(row - blk * J);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int p = 4 * (tile0 + nt) + kq;
        if (p < P) F[(blk * P + p) * J + j] = make_double2(c[nt][0], c[nt][1]);
      }
    }
  }
}

// Alpha contraction, per (R, p): H(m, j) = sum_{a2} E2(m, a2) F(a2, j) in complex numbers,
// as the real GEMM of the rows 2 mi + part_out and the columns 2 a + part_in:
//   Ab[(mt * K2p + k) * 8 + r] = A[8 mt + r][k],  A = [[E2r, -E2i], [E2i, E2r]] interleaved,
// K2p = 2 n_a2 rounded up to 4.  A warp takes (R, p) and 8 consecutive j; MT m-tiles
// starting at mt0.  H[((R * P + p) * n_m + mi) * J + j] (complex).
template <int MT>
__global__ void __launch_bounds__(kThreads)
    proj_alpha_kernel(const double2* __restrict__ F, int nR, int n_a2, int P, int J, int n_m,
                      int K2p, int mt0, const double* __restrict__ Ab, double2* __restrict__ H) {
  const int lane = threadIdx.x & 31, kq = lane & 3, rq = lane >> 2;
  const int n_jt = (J + 7) / 8;
  const int64_t n_tasks = (int64_t)nR * P * n_jt;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const double* Fd = reinterpret_cast<const double*>(F);
  double* Hd = reinterpret_cast<double*>(H);
  for (int64_t task = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; task < n_tasks;
       task += nwarps) {
    const int jt = (int)(task % n_jt);
    const int64_t rp = task / n_jt;  // R * P + p
    const int p = (int)(rp % P);
    const int R = (int)(rp / P);
    const int jb = jt * 8 + rq;  // this lane's column of B
    double c[MT][2];
#pragma unroll
    for (int t = 0; t < MT; ++t) c[t][0] = c[t][1] = 0.0;
    const double* fcol = Fd + (((int64_t)R * n_a2 * P + p) * J + jb) * 2;
    const int64_t fstride = (int64_t)P * J * 2;  // next alpha2
    for (int c0 = 0; c0 < K2p; c0 += 4 * kKSteps) {
      double b[kKSteps];  // this lane's B values of kKSteps k-steps, loaded at once
#pragma unroll
      for (int s = 0; s < kKSteps; ++s) {
        const int k = c0 + 4 * s + kq, a = k >> 1;
        b[s] = (a < n_a2 && jb < J) ? fcol[a * fstride + (k & 1)] : 0.0;
      }
#pragma unroll
      for (int s = 0; s < kKSteps; ++s) {
        const int k0 = c0 + 4 * s;
        if (k0 >= K2p) break;  // the same for the whole warp
#pragma unroll
        for (int t = 0; t < MT; ++t) {
          const double av = __ldg(Ab + ((size_t)(mt0 + t) * K2p + k0 + kq) * 8 + rq);
          dmma(c[t][0], c[t][1], av, b[s]);
        }
      }
    }
    // D[r][n]: row 8 (mt0 + t) + rq = 2 mi + part, column j = 8 jt + 2 kq + i
#pragma unroll
    for (int t = 0; t < MT; ++t) {
      const int row = 8 * (mt0 + t) + rq, mi = row >> 1, part = row & 1;
      if (mi >= n_m) continue;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int j = jt * 8 + 2 * kq + i;
        if (j < J) Hd[((rp * n_m + mi) * J + j) * 2 + part] = c[t][i];
      }
    }
  }
}

// K[((((R * P + p) * n_m + mi) * n_l2 + l2) * n_b1 + i1] = sum_{b2} Bt[p][l2][mi][b2]
// H[R][p][mi][i1 * n_b2 + b2]; zero where |m| > l2.
__global__ void proj_beta2_kernel(const double2* __restrict__ H, int nR, int P, int n_m,
                                  int n_l2, int n_b1, int n_b2, const double* __restrict__ Bt,
                                  double2* __restrict__ K) {
  const int64_t total = (int64_t)nR * P * n_m * n_l2 * n_b1;
  const int m_max = (n_m - 1) / 2;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int i1 = (int)(idx % n_b1);
    int64_t q = idx / n_b1;
    const int l2 = (int)(q % n_l2);
    q /= n_l2;
    const int mi = (int)(q % n_m);
    q /= n_m;
    const int p = (int)(q % P);
    const int R = (int)(q / P);
    double re = 0.0, im = 0.0;
    if (abs(mi - m_max) <= l2) {
      const double* b = Bt + (((size_t)p * n_l2 + l2) * n_m + mi) * n_b2;
      const double2* h = H + ((((int64_t)R * P + p) * n_m + mi) * n_b1 + i1) * n_b2;
      for (int i2 = 0; i2 < n_b2; ++i2) {
        const double w = __ldg(b + i2);
        const double2 v = h[i2];
        re = fma(w, v.x, re);
        im = fma(w, v.y, im);
      }
    }
    K[idx] = make_double2(re, im);
  }
}

// One warp per (term, R): lanes over the (m, beta1) points of the term, then a fixed
// shuffle tree.  S_t(R) = sum_m sum_{b1} A[t][mi][b1] K[R][p_t][mi][l2_t][b1].
__global__ void proj_terms_kernel(const double2* __restrict__ K, int nR, int r0, int nR_all,
                                  int P, int n_m, int n_l2, int n_b1,
                                  const TermDev* __restrict__ terms, int n_terms,
                                  const double* __restrict__ A, double* __restrict__ out_re,
                                  double* __restrict__ out_im) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wid >= (int64_t)n_terms * nR) return;
  const int t = (int)(wid / nR), R = (int)(wid % nR);
  const TermDev td = terms[t];
  const int m_max = (n_m - 1) / 2;
  const int n = (td.m_hi - td.m_lo + 1) * n_b1;
  const double* a = A + ((size_t)t * n_m + td.m_lo + m_max) * n_b1;
  const double2* kb = K + (((int64_t)R * P + td.pair) * n_m + td.m_lo + m_max) * n_l2 * n_b1 +
                      (int64_t)td.l2 * n_b1;
  double re = 0.0, im = 0.0;
  for (int i = lane; i < n; i += 32) {
    const int mo = i / n_b1, i1 = i - mo * n_b1;
    const double w = __ldg(a + i);
    const double2 v = kb[(int64_t)mo * n_l2 * n_b1 + i1];
    re = fma(w, v.x, re);
    im = fma(w, v.y, im);
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
  if (sys_type == 1 || sys_type == 3 || sys_type == 4) {  // (l) or (l, nju): nju >= 0
    for (int t = 0; t < n_terms; ++t) {                    // (pot_comp.f:5005-5010, 5061-5066)
      const int l = a_top[5 * t], nju = sys_type != 1 ? a_top[5 * t + 1] : 0;
      MQCT_ARG_CHECK(l >= 0 && l <= kMaxL, "term %d: l must be in 0..%d", t + 1, kMaxL);
      MQCT_ARG_CHECK(nju >= 0, "term %d: the values of M1 should be always positive", t + 1);
      MQCT_ARG_CHECK(nju <= l, "term %d: |nju| exceeds its l", t + 1);
    }
    return MQCT_OK;
  }
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
  int P = 0, n_m = 0, n_l2 = 0, J = 0, L = 0;
  int Lp = 0, n_pt = 0, K2p = 0, n_mt = 0;  // padded GEMM sizes of the gamma and alpha steps
  DevBuf<double> Eb, Ab;
  DevBuf<double> A, B;
  DevBuf<TermDev> terms;
  DevBuf<double2> F, H, K;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool timed = false;

  ~mqct_projection_plan() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
  }

  int upload_tables(const std::vector<double>& eb, const std::vector<double>& ab,
                    const std::vector<double>& ta, const std::vector<double>& tb,
                    const std::vector<TermDev>& td) {
    MQCT_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& x : ev) MQCT_CUDA_TRY(cudaEventCreate(&x));
    MQCT_CUDA_TRY(Eb.upload(eb, st));
    MQCT_CUDA_TRY(Ab.upload(ab, st));
    MQCT_CUDA_TRY(A.upload(ta, st));
    MQCT_CUDA_TRY(B.upload(tb, st));
    MQCT_CUDA_TRY(terms.upload(td, st));
    MQCT_CUDA_TRY(cudaStreamSynchronize(st));
    return MQCT_OK;
  }

  // SYS_TYPE 1 (diatom + atom, V_2_1(n_beta, n_r)) and 4 (top + atom, V_3_1(n_gamma,
  // n_beta, n_r)), CALC_EXPANSION_TERMS cases 1 and 4 (pot_comp.f:4973-4999, 5054-5104;
  // case 3, the symmetric top, :5000-5053, is case 4):
  //   type 1: terms = sum_beta WF_DIAT_TOP(l, 0; beta) V wb sin(beta) xbl 2 pi
  //   type 4: terms = sum_{beta,gamma} Re((-1)^nju WF_DIAT_TOP(l, nju; beta, gamma)) V wb wg
  //           sin(beta) xbl xgl
  // in the same contractions with the alpha2 and beta2 axes of one point and m = l2 = 0.
  int init_atom(int sys, int nt, const int32_t* a_top, const mqct_grid_t& g) {
    n_b1 = g.n_beta;
    n_g1 = sys == 4 ? g.n_gamma : 1;
    n_a2 = n_b2 = n_g2 = 1;
    MQCT_ARG_CHECK(n_b1 > 0 && n_b1 <= 4096 && n_g1 > 0 && n_g1 <= 4096,
                   "grid sizes must be in 1..4096 (beta %d, gamma %d)", n_b1, n_g1);
    int rc = check_terms(sys, nt, a_top, 0);
    if (rc != MQCT_OK) return rc;
    J = n_b1;
    L = n_g1;
    if (mqct_device_count() <= 0) {
      set_error("no CUDA device available");
      return MQCT_E_NODEV;
    }
    const Axis b1 = axis_gl(n_b1, 0.0, kPi);
    const Axis g1 = g.eq_gamma ? axis_mid(n_g1, 0.0, 2.0 * kPi) : axis_gl(n_g1, 0.0, 2.0 * kPi);
    std::vector<double> lf(128);
    lf[0] = 0.0;
    for (int i = 1; i < 128; ++i) lf[i] = lf[i - 1] + std::log((double)i);
    std::vector<int> nus;
    std::vector<TermDev> td(nt);
    for (int t = 0; t < nt; ++t) {
      const int nju = sys == 4 ? a_top[5 * t + 1] : 0;
      auto it = std::find(nus.begin(), nus.end(), nju);
      td[t].pair = (int)(it - nus.begin());
      if (it == nus.end()) nus.push_back(nju);
      td[t].l2 = 0;
      td[t].m_lo = td[t].m_hi = 0;
    }
    P = (int)nus.size();
    n_m = 1;
    n_l2 = 1;
    Lp = (L + 3) / 4 * 4;
    n_pt = (P + 3) / 4;
    std::vector<double> eb((size_t)(n_pt + 3) / 4 * 4 * Lp * 8, 0.0);
    for (int i = 0; i < n_g1; ++i)
      for (int p = 0; p < P; ++p) {
        const double w = sys == 4 ? g1.w[i] * g1.half : 1.0;
        const double ph = sys == 4 ? nus[p] * g1.x[i] : 0.0;
        double* d = &eb[((size_t)(p / 4) * Lp + i) * 8 + 2 * (p % 4)];
        d[0] = std::cos(ph) * w;
        d[1] = std::sin(ph) * w;
      }
    K2p = 4;  // one alpha2 point of unit weight: H = F
    n_mt = 1;
    std::vector<double> ab((size_t)8 * K2p * 8, 0.0);
    ab[(size_t)0 * 8 + 0] = 1.0;  // row 0 (Re), column 0 (Re)
    ab[(size_t)1 * 8 + 1] = 1.0;  // row 1 (Im), column 1 (Im)
    std::vector<double> ta((size_t)nt * n_b1), tb((size_t)P, 1.0);
    for (int t = 0; t < nt; ++t) {
      const int l = a_top[5 * t], nju = sys == 4 ? a_top[5 * t + 1] : 0;
      const double nrm = std::sqrt((2.0 * l + 1.0) / 4.0 / kPi * std::exp(lf[l - nju] - lf[l + nju]));
      const double sg = (sys == 4 && (nju & 1)) ? -1.0 : 1.0;
      const double tail = sys == 1 ? 2.0 * kPi : 1.0;
      for (int i = 0; i < n_b1; ++i)
        ta[(size_t)t * n_b1 + i] = sg * mqct_dev::plgndr(l, nju, std::cos(b1.x[i])) * nrm *
                                   b1.w[i] * std::sin(b1.x[i]) * b1.half * tail;
    }
    return upload_tables(eb, ab, ta, tb, td);
  }

  int init(int sys, int nt, const int32_t* a_top, const mqct_grid_t& g, int identical) {
    MQCT_ARG_CHECK(sys == 1 || sys == 3 || sys == 4 || sys == 7 || sys == 8 || sys == 9 ||
                       sys == 0,
                   "the projection is built for SYS_TYPE 1, 3, 4, 7, 8, 9 and 0 (got %d)", sys);
    MQCT_ARG_CHECK(!identical || sys == 0, "identical partners are SYS_TYPE 0");
    if (sys == 9) sys = 0;  // case 9 (pot_comp.f:5418-5765) is case 0; EXPANSION_TERM :3859
    MQCT_ARG_CHECK(nt > 0 && a_top, "no terms");
    MQCT_ARG_CHECK(!identical || sys == 0, "identical partners are SYS_TYPE 0");
    sys_type = sys;
    n_terms = nt;
    if (sys == 1 || sys == 3 || sys == 4) return init_atom(sys == 3 ? 4 : sys, nt, a_top, g);
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
    MQCT_ARG_CHECK((int64_t)J <= (1 << 24), "n_beta1 * n_beta2 = %d too large", J);
    if (mqct_device_count() <= 0) {
      set_error("no CUDA device available");
      return MQCT_E_NODEV;
    }
    // axes as INI_POT_STORAGE sets them (pot_comp.f:1310-1370, 1628-1700)
    const Axis b1 = axis_gl(n_b1, 0.0, kPi), b2 = axis_gl(n_b2, 0.0, kPi);
    auto ang = [&](int n) {
      return g.eq_gamma ? axis_mid(n, 0.0, 2.0 * kPi) : axis_gl(n, 0.0, 2.0 * kPi);
    };
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
    // (nju1, nju2) pairs, the m range and the l2 values
    std::vector<std::pair<int, int>> pairs;
    std::vector<TermDev> td(nt);
    int m_max = 0, l2_max = 0;
    for (int t = 0; t < nt; ++t) {
      const int32_t* q = a_top + 5 * t;
      const int l1 = q[0], n1 = q[1], l2 = q[2], n2 = sys == 0 ? q[3] : 0;
      const std::pair<int, int> pr(n1, n2);
      auto it = std::find(pairs.begin(), pairs.end(), pr);
      td[t].pair = (int)(it - pairs.begin());
      if (it == pairs.end()) pairs.push_back(pr);
      td[t].l2 = l2;
      const int mm = std::min(l1, l2);
      td[t].m_lo = -mm;
      td[t].m_hi = mm;
      m_max = std::max(m_max, mm);
      l2_max = std::max(l2_max, l2);
    }
    P = (int)pairs.size();
    n_m = 2 * m_max + 1;
    n_l2 = l2_max + 1;
    // Eb: B operand of the gamma GEMM, Eb[(tile * Lp + k) * 8 + 2 q + part] = Re / Im of
    // e^{i(nju1 gamma1 + nju2 gamma2)} w for pair 4 tile + q at k = i_g1 * n_g2 + i_g2
    Lp = (L + 3) / 4 * 4;
    n_pt = (P + 3) / 4;
    // (tiles padded with zeros to a multiple of 4: a pass covers up to 4 tiles)
    std::vector<double> eb((size_t)(n_pt + 3) / 4 * 4 * Lp * 8, 0.0);
    for (int i5 = 0; i5 < n_g1; ++i5)
      for (int i6 = 0; i6 < n_g2; ++i6)
        for (int p = 0; p < P; ++p) {
          const double ph = pairs[p].first * g1.x[i5] + pairs[p].second * g2.x[i6];
          const double w = g1.w[i5] * g1.half * g2.w[i6] * g2.half * tail2;
          const size_t k = (size_t)i5 * n_g2 + i6;
          double* d = &eb[((size_t)(p / 4) * Lp + k) * 8 + 2 * (p % 4)];
          d[0] = std::cos(ph) * w;
          d[1] = std::sin(ph) * w;
        }
    // Ab: A operand of the alpha GEMM, rows 2 mi + part_out, columns 2 a + part_in of
    // [[E2r, -E2i], [E2i, E2r]], E2 = e^{-i m alpha2} w; Ab[(mt * K2p + k) * 8 + r]
    K2p = (2 * n_a2 + 3) / 4 * 4;
    n_mt = (2 * n_m + 7) / 8;
    // (tiles padded with zeros to a multiple of 8: a pass covers up to 8 tiles)
    std::vector<double> ab((size_t)(n_mt + 7) / 8 * 8 * K2p * 8, 0.0);
    for (int mi = 0; mi < n_m; ++mi)
      for (int i2 = 0; i2 < n_a2; ++i2) {
        const double ph = -(double)(mi - m_max) * a2.x[i2];
        const double w = a2.w[i2] * a2.half;
        const double er = std::cos(ph) * w, ei = std::sin(ph) * w;
        for (int po = 0; po < 2; ++po)
          for (int pi = 0; pi < 2; ++pi) {
            const int row = 2 * mi + po, col = 2 * i2 + pi;
            const double v = po == pi ? er : (po == 0 ? -ei : ei);
            ab[((size_t)(row / 8) * K2p + col) * 8 + row % 8] = v;
          }
      }
    // A[t][mi][b1] = K_t c_tm d^{l1}_{nju1 m}(beta1) w; B[p][l2][mi][b2] = b(beta2) w with
    // b = WF_DIAT_TOP(l2, -m, beta2, .) without its phase (types 7, 8) or
    // d^{l2}_{nju2(p), -m}(beta2) (type 0)
    std::vector<double> ta((size_t)nt * n_m * n_b1, 0.0);
    std::vector<double> tb((size_t)P * n_l2 * n_m * n_b2, 0.0);
    for (int t = 0; t < nt; ++t) {
      const int32_t* q = a_top + 5 * t;
      const int l1 = q[0], n1 = q[1], l2 = q[2];
      const int l = sys == 0 ? q[4] : q[3];
      const double Kt = sys == 0 ? std::sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0)) / (8.0 * kPi * kPi)
                                 : std::sqrt((2.0 * l1 + 1.0) / 4.0 / kPi);
      for (int m = td[t].m_lo; m <= td[t].m_hi; ++m) {
        const int mi = m + m_max;
        const double c = mqct_dev::clebsch_gordan(l1, m, l2, -m, l, 0, lf.data());
        for (int i = 0; i < n_b1; ++i)
          ta[((size_t)t * n_m + mi) * n_b1 + i] =
              Kt * c * mqct_dev::wigner_d(l1, n1, m, b1.x[i], lf.data()) * b1.w[i] *
              std::sin(b1.x[i]) * b1.half;
      }
    }
    for (int p = 0; p < P; ++p)
      for (int l2 = 0; l2 < n_l2; ++l2)
        for (int m = -std::min(l2, m_max); m <= std::min(l2, m_max); ++m) {
          const int mi = m + m_max;
          if (sys == 0 && std::abs(pairs[p].second) > l2) continue;
          for (int i = 0; i < n_b2; ++i) {
            double bv;
            if (sys == 0) {
              bv = mqct_dev::wigner_d(l2, pairs[p].second, -m, b2.x[i], lf.data());
            } else {
              const int am = std::abs(m);
              bv = mqct_dev::plgndr(l2, am, std::cos(b2.x[i])) *
                   std::sqrt((2.0 * l2 + 1.0) / 4.0 / kPi * std::exp(lf[l2 - am] - lf[l2 + am]));
              if (m > 0 && (am & 1)) bv = -bv;
            }
            tb[(((size_t)p * n_l2 + l2) * n_m + mi) * n_b2 + i] =
                bv * b2.w[i] * std::sin(b2.x[i]) * b2.half;
          }
        }
    return upload_tables(eb, ab, ta, tb, td);
  }

  // R points per pass so that F, H and K stay within 4 GiB.
  int pass_R(int nR) const {
    const size_t per_R = ((size_t)n_a2 * P * J + (size_t)P * n_m * J +
                          (size_t)P * n_m * n_l2 * n_b1) *
                         sizeof(double2);
    const size_t cap = (size_t)4 << 30;
    return (int)std::max<size_t>(1, std::min<size_t>(nR, cap / per_R));
  }

  // Warps for n_tasks warp tasks, as whole CTAs, at most 16 CTAs per SM (grid-stride).
  static unsigned ctas(int64_t n_tasks) {
    const int64_t w = kThreads / 32;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_tasks + w - 1) / w, 148 * 16));
  }

  template <int NT>
  int launch_gamma(const double* V, int64_t n_rows, int tile0) {
    proj_gamma_kernel<NT><<<ctas((n_rows + 7) / 8), kThreads, 0, st>>>(V, n_rows, L, Lp, P,
                                                                       tile0, J, Eb.p, F.p);
    MQCT_CUDA_TRY(cudaGetLastError());
    return MQCT_OK;
  }

  template <int MT>
  int launch_alpha(int nr, int mt0) {
    const int64_t tasks = (int64_t)nr * P * ((J + 7) / 8);
    proj_alpha_kernel<MT><<<ctas(tasks), kThreads, 0, st>>>(F.p, nr, n_a2, P, J, n_m, K2p, mt0,
                                                           Ab.p, H.p);
    MQCT_CUDA_TRY(cudaGetLastError());
    return MQCT_OK;
  }

  int execute(const double* d_V, int nR, double* d_terms, double* d_terms_im) {
    MQCT_ARG_CHECK(d_V && d_terms && nR > 0, "null argument or nR <= 0");
    const int rc_R = pass_R(nR);
    if (F.n < (size_t)rc_R * n_a2 * P * J) MQCT_CUDA_TRY(F.alloc((size_t)rc_R * n_a2 * P * J));
    if (H.n < (size_t)rc_R * P * n_m * J) MQCT_CUDA_TRY(H.alloc((size_t)rc_R * P * n_m * J));
    const size_t nK = (size_t)rc_R * P * n_m * n_l2 * n_b1;
    if (K.n < nK) MQCT_CUDA_TRY(K.alloc(nK));
    const size_t G = (size_t)n_a2 * J * L;
    bool first = true;
    for (int r0 = 0; r0 < nR; r0 += rc_R) {
      const int nr = std::min(rc_R, nR - r0);
      const int64_t n_rows = (int64_t)nr * n_a2 * J;
      const double* V = d_V + (size_t)r0 * G;
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[0], st));
      for (int t0 = 0; t0 < n_pt; t0 += 4) {  // up to 4 pair tiles (16 pairs) per pass over V
        const int nt = std::min(4, n_pt - t0);
        const int rc = nt == 1   ? launch_gamma<1>(V, n_rows, t0)
                       : nt == 2 ? launch_gamma<2>(V, n_rows, t0)
                                 : launch_gamma<4>(V, n_rows, t0);
        if (rc != MQCT_OK) return rc;
      }
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[1], st));
      for (int m0 = 0; m0 < n_mt; m0 += 8) {  // up to 8 m tiles (32 m values) per pass
        const int mt = std::min(8, n_mt - m0);
        const int rc = mt == 1   ? launch_alpha<1>(nr, m0)
                       : mt == 2 ? launch_alpha<2>(nr, m0)
                       : mt <= 4 ? launch_alpha<4>(nr, m0)
                                 : launch_alpha<8>(nr, m0);
        if (rc != MQCT_OK) return rc;
      }
      if (first) MQCT_CUDA_TRY(cudaEventRecord(ev[2], st));
      const int64_t nk = (int64_t)nr * P * n_m * n_l2 * n_b1;
      const int64_t bk = std::min<int64_t>((nk + kThreads - 1) / kThreads, 148 * 64);
      proj_beta2_kernel<<<(unsigned)bk, kThreads, 0, st>>>(H.p, nr, P, n_m, n_l2, n_b1, n_b2,
                                                           B.p, K.p);
      MQCT_CUDA_TRY(cudaGetLastError());
      const int64_t nt = (int64_t)n_terms * nr;
      proj_terms_kernel<<<(unsigned)((nt * 32 + kThreads - 1) / kThreads), kThreads, 0, st>>>(
          K.p, nr, r0, nR, P, n_m, n_l2, n_b1, terms.p, n_terms, A.p, d_terms, d_terms_im);
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
