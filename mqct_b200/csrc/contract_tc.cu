// contract_tc.cu -- split-precision tensor-core contraction of the matrix build
// on sm_100a: tcgen05.mma kind::f16 with FP32 accumulators in TMEM.
//
//   M[row, i] = sum_{c, alpha} sum_{g in chunk c} X_alpha[row, g] W[g, i]
//   X = X_hi + X_lo, W = W_hi + W_lo (16-bit parts),
//   D += X_hi W_hi + X_hi W_lo + X_lo W_hi          (FP32 accumulate)
//
// Two 16-bit formats: BF16x3 (8 significant bits per part, ~16 bits kept) and
// F16x3 (11 bits per part, ~22 bits kept; the products of FP16 parts are exact
// in FP32).  FP16's range is narrow, so in F16x3 X is scaled by 2^14 and every
// radial column of W by the power of two that brings its largest entry to
// [2^13, 2^14); the finalize multiplies each column by the exact inverse.
//
// CTA = one 128-row tile of pair rows (one m-block) x all nR radial points.
// Warp roles (320 threads):
//   warp 0      bulk-copy (TMA) producer: per K-chunk the pre-arranged W image
//               (hi and lo planes, K-major core-matrix layout) and the block's
//               rotor-basis slice, one cp.async.bulk each, mbarrier complete_tx;
//   warp 1      TMEM allocator + single-thread MMA issuer;
//   warps 2..9  X producers: X = w_alpha Re(psi_a^* psi_b) in FP32 from the
//               staged basis (the e^{i m alpha} phases of a same-m pair cancel),
//               split to 16-bit hi/lo and written in the core-matrix layout, two
//               threads per tile row (each half of the chunk's K groups), one
//               A stage per alpha point; afterwards the epilogue
//               (tcgen05.ld of the accumulator, FP32 partials to global; the
//               two warps of a TMEM lane quarter take alternate 16-column
//               slices).
// The operand tiles use the K-major SWIZZLE_NONE canonical layout: 8 rows x
// 16 B core matrices, K-adjacent core matrices LBO apart, 8-row groups SBO =
// 128 B apart.  Every mbarrier wait is bounded; on timeout the CTA records an
// error code, drains, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "matrix_plan.cuh"
#include "ptx.cuh"

namespace mqct {

constexpr int TC_M = 128;        // rows per tile
constexpr int TC_KC = 64;        // K elements per chunk (8 core-matrix columns of 8 bf16)
constexpr int TC_PSI_LD = 66;    // float2 per staged basis row (64 + pad)
constexpr int TC_THREADS = 320;
constexpr int TC_PRODUCERS = TC_THREADS - 64;  // X-producer / epilogue threads
constexpr int TC_A_PLANE = TC_M * TC_KC * 2;      // bytes of one bf16 plane of an A stage
constexpr uint32_t TC_SPIN_LIMIT = kSpinLimit;     // bounded mbarrier waits

// Shared-memory matrix descriptor: K-major, SWIZZLE_NONE, version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  return d;                // base offset 0, lbo mode 0, layout SWIZZLE_NONE (0)
}
// Instruction descriptor, kind::f16: BF16 A/B, FP32 D, both K-major.
// a/b format 1 = BF16, 0 = F16 (A and B always of the same type).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t pack_f16(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
// Split of 8 FP32 values into hi and lo 16-bit parts (packed pairs).
template <bool kF16>
__device__ __forceinline__ void split8(const float (&x)[8], uint4& h, uint4& l) {
  float r[8];
  if (kF16) {
    h.x = pack_f16(x[0], x[1]);
    h.y = pack_f16(x[2], x[3]);
    h.z = pack_f16(x[4], x[5]);
    h.w = pack_f16(x[6], x[7]);
    const __half2* hb = reinterpret_cast<const __half2*>(&h);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float2 f = __half22float2(hb[e]);
      r[2 * e] = x[2 * e] - f.x;
      r[2 * e + 1] = x[2 * e + 1] - f.y;
    }
    l.x = pack_f16(r[0], r[1]);
    l.y = pack_f16(r[2], r[3]);
    l.z = pack_f16(r[4], r[5]);
    l.w = pack_f16(r[6], r[7]);
  } else {
    h.x = pack_bf16(x[0], x[1]);
    h.y = pack_bf16(x[2], x[3]);
    h.z = pack_bf16(x[4], x[5]);
    h.w = pack_bf16(x[6], x[7]);
    const __nv_bfloat162* hb = reinterpret_cast<const __nv_bfloat162*>(&h);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float2 f = __bfloat1622float2(hb[e]);
      r[2 * e] = x[2 * e] - f.x;
      r[2 * e + 1] = x[2 * e + 1] - f.y;
    }
    l.x = pack_bf16(r[0], r[1]);
    l.y = pack_bf16(r[2], r[3]);
    l.z = pack_bf16(r[4], r[5]);
    l.w = pack_bf16(r[6], r[7]);
  }
}

// F16x3 column scaling: one CTA per radial column i finds max_g |W[g, i]| and
// writes the exponent s_i with max * 2^s_i in [2^13, 2^14) and the finalize
// factor 2^-(s_i + kXScaleExp).
constexpr int kXScaleExp = 14;
__global__ void tc_wscale_kernel(const double* __restrict__ W, int ldw, int G2,
                                 int* __restrict__ wexp, double* __restrict__ col_scale) {
  __shared__ double red[32];
  const int i = blockIdx.x;
  double m = 0.0;
  for (int g = threadIdx.x; g < G2; g += blockDim.x) m = fmax(m, fabs(W[(size_t)g * ldw + i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
    m = fmax(m, red[0]);
    int e = 0;
    int s = 0;
    if (m > 0.0) {
      frexp(m, &e);  // m = f 2^e, f in [0.5, 1)
      s = 14 - e;
    }
    wexp[i] = s;
    col_scale[i] = ldexp(1.0, -(s + kXScaleExp));
  }
}

// ---------------------------------------------------------------- operand images
// W (FP64, [g][ldw]) -> per chunk c: [plane hi/lo][kg 0..7][ng 0..Npad/8-1][8 rows][8 x 16 bit];
// F16x3 scales column n by 2^wexp[n] first (exact).
template <bool kF16>
__global__ void tc_bimage_kernel(const double* __restrict__ W, int ldw, int G2, int nR, int Npad,
                                 int n_chunks, const int* __restrict__ wexp,
                                 unsigned short* __restrict__ img) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t per_chunk = (int64_t)TC_KC * Npad;
  if (idx >= per_chunk * n_chunks) return;
  int c = (int)(idx / per_chunk);
  int rem = (int)(idx % per_chunk);
  int n = rem / TC_KC, k = rem % TC_KC;
  int g = c * TC_KC + k;
  double w = (g < G2 && n < nR) ? W[(size_t)g * ldw + n] : 0.0;
  unsigned short hi, lo;
  if (kF16) {
    if (n < nR) w = ldexp(w, wexp[n]);
    __half h = __double2half(w);
    __half l = __double2half(w - (double)__half2float(h));
    hi = __half_as_ushort(h);
    lo = __half_as_ushort(l);
  } else {
    __nv_bfloat16 h = __double2bfloat16(w);
    __nv_bfloat16 l = __double2bfloat16(w - (double)__bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
  }
  int kg = k >> 3, e = k & 7, ng = n >> 3, r8 = n & 7;
  size_t plane = (size_t)TC_KC * Npad;
  size_t off = (size_t)c * 2 * plane + (((size_t)kg * (Npad / 8) + ng) * 8 + r8) * 8 + e;
  img[off] = hi;
  img[off + plane] = lo;
}

// psi (FP64, [basis row][G2]) -> per (block, chunk): [local state][TC_PSI_LD] float2.
__global__ void tc_psiimage_kernel(const double2* __restrict__ psi, int G2, int n_chunks,
                                   const int* __restrict__ blk_row0, const int* __restrict__ blk_n,
                                   const int64_t* __restrict__ blk_img_off, int n_blocks,
                                   float2* __restrict__ img, int n_basis_rows) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t per_row = (int64_t)n_chunks * TC_PSI_LD;
  if (idx >= per_row * n_basis_rows) return;
  int row = (int)(idx / per_row);
  int rem = (int)(idx % per_row);
  int c = rem / TC_PSI_LD, k = rem % TC_PSI_LD;
  int b = 0;
  while (b + 1 < n_blocks && blk_row0[b + 1] <= row) ++b;
  int ls = row - blk_row0[b];
  int g = c * TC_KC + k;
  double2 v = (k < TC_KC && g < G2) ? psi[(size_t)row * G2 + g] : make_double2(0.0, 0.0);
  img[blk_img_off[b] + ((int64_t)c * blk_n[b] + ls) * TC_PSI_LD + k] =
      make_float2((float)v.x, (float)v.y);
}

// ---------------------------------------------------------------- main kernel
struct TcArgs {
  int n_units, n_splits, n_chunks, chunks_per_split, n_alpha_it, Npad, N0, N1, nbmax, stages;
  int tmem_cols;
  const int* tile_block;          // per tile
  const int* blk_row0;            // basis row offset per block
  const int* blk_n;
  const int* blk_m;               // m12 of each block
  const int64_t* blk_img_off;     // float2 offset of the block's psi image
  const int* rowa;                // basis row of st1 / st2 per GEMM row
  const int* rowb;
  const float2* psi_img;
  const unsigned short* b_img;    // hi/lo planes of W, BF16 or F16 bits
  const float* alpha;             // alpha nodes (n_alpha_it, or none)
  const float* walpha;            // alpha weights
  float* part;                    // n_splits x n_rows x Npad
  int64_t part_stride;
  int* status;
};

template <bool kF16>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_contract_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // carve shared memory (1024-byte aligned regions)
  uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  unsigned char* sB = reinterpret_cast<unsigned char*>(base);
  const uint32_t b_bytes = 2u * TC_KC * a.Npad * 2u;            // hi + lo planes
  unsigned char* sPsi = sB + ((b_bytes + 1023) & ~1023u);
  const uint32_t psi_bytes_max = (uint32_t)a.nbmax * TC_PSI_LD * 8u;
  unsigned char* sA = sPsi + ((psi_bytes_max + 1023) & ~1023u);
  const uint32_t a_stage = 2u * TC_A_PLANE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sA + a.stages * a_stage);
  // barrier slots: A_full[s], A_empty[s], B_full, B_empty, P_full, P_empty, ACC_full, ACC_empty
  uint64_t* A_full = bars;
  uint64_t* A_empty = bars + 8;
  uint64_t* B_full = bars + 16;
  uint64_t* B_empty = bars + 17;
  uint64_t* P_full = bars + 18;
  uint64_t* P_empty = bars + 19;
  uint64_t* ACC_full = bars + 20;
  uint64_t* ACC_empty = bars + 21;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 24);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 25);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < a.stages; ++s) {
      mbar_init(&A_full[s], TC_PRODUCERS);
      mbar_init(&A_empty[s], 1);
    }
    mbar_init(B_full, 1);
    mbar_init(B_empty, 1);
    mbar_init(P_full, 1);
    mbar_init(P_empty, TC_PRODUCERS);
    mbar_init(ACC_full, 1);
    mbar_init(ACC_empty, TC_PRODUCERS);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- bulk-copy producer
    if (lane == 0) {
      uint32_t pe_phase = 0, be_phase = 0;
      uint32_t bf_last = 0, pf_last = 0, n_issued = 0;  // phase of the last issued copies
      bool first = true;
      for (int u = blockIdx.x; u < a.n_units && !*abort_flag; u += gridDim.x) {
        const int tile = u / a.n_splits, split = u % a.n_splits;
        const int blk = a.tile_block[tile];
        const int nb = a.blk_n[blk];
        const uint32_t psi_bytes = (uint32_t)nb * TC_PSI_LD * 8u;
        const int c0 = split * a.chunks_per_split;
        const int c1 = min(a.n_chunks, c0 + a.chunks_per_split);
        for (int c = c0; c < c1; ++c) {
          if (!first) {
            if (!mbar_wait(B_empty, be_phase, abort_flag, a.status, 11)) break;
            if (!mbar_wait(P_empty, pe_phase, abort_flag, a.status, 12)) break;
            be_phase ^= 1;
            pe_phase ^= 1;
          }
          first = false;
          bf_last = pf_last = n_issued & 1u;
          ++n_issued;
          mbar_expect_tx(B_full, b_bytes);
          bulk_g2s(sB, a.b_img + (size_t)c * 2 * TC_KC * a.Npad, b_bytes, B_full);
          mbar_expect_tx(P_full, psi_bytes);
          bulk_g2s(sPsi, a.psi_img + a.blk_img_off[blk] + (int64_t)c * nb * TC_PSI_LD, psi_bytes,
                   P_full);
        }
      }
      // drain: the last copies must have landed before the CTA exits
      if (!first) {
        if (!*abort_flag) {
          mbar_wait(B_empty, be_phase, abort_flag, a.status, 13);
          mbar_wait(P_empty, pe_phase, abort_flag, a.status, 14);
        } else {
          // on abort: bounded wait for the completion of the copies issued last
          for (uint32_t it = 0; it < TC_SPIN_LIMIT && !mbar_try_wait(B_full, bf_last); ++it) {}
          for (uint32_t it = 0; it < TC_SPIN_LIMIT && !mbar_try_wait(P_full, pf_last); ++it) {}
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      uint32_t bf_phase = 0, ae_phase = 0;
      uint32_t af_phase[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      int stage = 0;
      bool first_unit = true;
      const uint32_t idesc0 = kF16 ? idesc_f16(TC_M, a.N0) : idesc_bf16(TC_M, a.N0);
      const uint32_t idesc1 = a.N1 > 0 ? (kF16 ? idesc_f16(TC_M, a.N1) : idesc_bf16(TC_M, a.N1)) : 0u;
      const uint32_t sA0 = smem_u32(sA), sB0 = smem_u32(sB);
      const uint32_t lbo_a = (TC_M / 8) * 128, lbo_b = (uint32_t)(a.Npad / 8) * 128;
      const uint32_t bplane = (uint32_t)TC_KC * a.Npad * 2;
      for (int u = blockIdx.x; u < a.n_units && !*abort_flag; u += gridDim.x) {
        const int split = u % a.n_splits;
        const int c0 = split * a.chunks_per_split;
        const int c1 = min(a.n_chunks, c0 + a.chunks_per_split);
        if (!first_unit) {  // the epilogue must have drained the accumulator
          if (!mbar_wait(ACC_empty, ae_phase, abort_flag, a.status, 21)) break;
          ae_phase ^= 1;
          tc_fence_after();
        }
        first_unit = false;
        bool acc = false;
        for (int c = c0; c < c1 && !*abort_flag; ++c) {
          if (!mbar_wait(B_full, bf_phase, abort_flag, a.status, 22)) break;
          bf_phase ^= 1;
          for (int al = 0; al < a.n_alpha_it; ++al) {
            if (!mbar_wait(&A_full[stage], af_phase[stage], abort_flag, a.status, 23)) break;
            af_phase[stage] ^= 1;
            tc_fence_after();
            const uint32_t aoff = sA0 + stage * (2 * TC_A_PLANE);
#pragma unroll
            for (int kk = 0; kk < TC_KC / 16; ++kk) {
              // products: (A_hi, B_hi), (A_hi, B_lo), (A_lo, B_hi)
#pragma unroll
              for (int pr = 0; pr < 3; ++pr) {
                const uint32_t ap = (pr == 2) ? 1 : 0, bp = (pr == 1) ? 1 : 0;
                const uint64_t ad = smem_desc(aoff + ap * TC_A_PLANE + kk * 2 * lbo_a, lbo_a, 128);
                const uint32_t boff = sB0 + bp * bplane + kk * 2 * lbo_b;
                const uint32_t accum = acc ? 1u : 0u;
                mma_bf16(tmem, ad, smem_desc(boff, lbo_b, 128), idesc0, accum);
                if (a.N1 > 0)
                  mma_bf16(tmem + (uint32_t)a.N0, ad,
                           smem_desc(boff + (uint32_t)(a.N0 / 8) * 128, lbo_b, 128), idesc1, accum);
                acc = true;
              }
            }
            mma_commit(&A_empty[stage]);  // frees the A stage when these MMAs complete
            stage = (stage + 1) % a.stages;
          }
          mma_commit(B_empty);  // B may be overwritten once this chunk's MMAs complete
        }
        mma_commit(ACC_full);
      }
    }
  } else {
    // ---------------- X producers (warps 2..9) and epilogue
    const int p = (threadIdx.x - 64) & (TC_M - 1);  // tile row generated by this thread
    const int kh = (threadIdx.x - 64) / TC_M;       // half of the chunk's K groups
    uint32_t pf_phase = 0, af_phase = 0;
    uint32_t ae_phase[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool a_used[8] = {false, false, false, false, false, false, false, false};
    int stage = 0;
    const int q = warp & 3;  // TMEM lane quarter accessible to this warp
    for (int u = blockIdx.x; u < a.n_units && !*abort_flag; u += gridDim.x) {
      const int tile = u / a.n_splits, split = u % a.n_splits;
      const int blk = a.tile_block[tile];
      const int row = tile * TC_M + p;
      const int la = a.rowa[row] - a.blk_row0[blk], lb = a.rowb[row] - a.blk_row0[blk];
      const int c0 = split * a.chunks_per_split;
      const int c1 = min(a.n_chunks, c0 + a.chunks_per_split);
      const float2* pa = reinterpret_cast<const float2*>(sPsi) + la * TC_PSI_LD;
      const float2* pb = reinterpret_cast<const float2*>(sPsi) + lb * TC_PSI_LD;
      for (int c = c0; c < c1 && !*abort_flag; ++c) {
        if (!mbar_wait(P_full, pf_phase, abort_flag, a.status, 31)) break;
        pf_phase ^= 1;
        // X_alpha = w_alpha Re((z psi_a)^* (z psi_b)) with z = e^{i m alpha}: both
        // states of a pair have the same m, so |z|^2 = 1 and the integrand at every
        // alpha point equals w_alpha Re(psi_a^* psi_b) exactly.  The product is formed
        // once per chunk and scaled per alpha point; every alpha slice is still
        // contracted by the tensor cores.
        float x0[TC_KC / 16][8];
#pragma unroll
        for (int kq = 0; kq < TC_KC / 16; ++kq) {
          const int kg = kh * (TC_KC / 16) + kq;
#pragma unroll
          for (int e = 0; e < 8; e += 2) {
            const float4 va = *reinterpret_cast<const float4*>(pa + kg * 8 + e);
            const float4 vb = *reinterpret_cast<const float4*>(pb + kg * 8 + e);
            x0[kq][e] = va.x * vb.x + va.y * vb.y;
            x0[kq][e + 1] = va.z * vb.z + va.w * vb.w;
          }
        }
        for (int al = 0; al < a.n_alpha_it; ++al) {
          float wa = a.alpha ? a.walpha[al] : 1.f;
          if (kF16) wa *= (float)(1 << kXScaleExp);  // exact power-of-two scaling
          if (a_used[stage]) {
            const bool ok = mbar_wait(&A_empty[stage], ae_phase[stage], abort_flag, a.status, 32);
            ae_phase[stage] ^= 1;
            if (!ok) break;
          }
          a_used[stage] = true;
          unsigned char* hi = sA + stage * (2 * TC_A_PLANE);
          unsigned char* lo = hi + TC_A_PLANE;
#pragma unroll
          for (int kq = 0; kq < TC_KC / 16; ++kq) {
            const int kg = kh * (TC_KC / 16) + kq;
            float x[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) x[e] = wa * x0[kq][e];
            uint4 h, l;
            split8<kF16>(x, h, l);
            const uint32_t off =
                (uint32_t)(kg * (TC_M / 8) + (p >> 3)) * 128u + (uint32_t)(p & 7) * 16u;
            *reinterpret_cast<uint4*>(hi + off) = h;
            *reinterpret_cast<uint4*>(lo + off) = l;
          }
          fence_proxy_async();
          mbar_arrive(&A_full[stage]);
          stage = (stage + 1) % a.stages;
        }
        mbar_arrive(P_empty);
      }
      // epilogue: accumulator -> FP32 partial sums
      if (!mbar_wait(ACC_full, af_phase, abort_flag, a.status, 33)) break;
      af_phase ^= 1;
      tc_fence_after();
      const int orow = tile * TC_M + q * 32 + lane;
      float* dst = a.part + (int64_t)split * a.part_stride + (int64_t)orow * a.Npad;
      for (int c16 = 16 * ((warp - 2) >> 2); c16 < a.Npad; c16 += 32) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c16, v);
#pragma unroll
        for (int i = 0; i < 16; i += 4)
          *reinterpret_cast<float4*>(dst + c16 + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      }
      tc_fence_before();
      mbar_arrive(ACC_empty);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(a.tmem_cols));
  }
}

// ---------------------------------------------------------------- host side
int MatrixPlan::tc_init() {
  MQCT_ARG_CHECK(nR <= 512, "BF16x3 contraction supports nR <= 512 (got %d)", nR);
  int dev = 0, cc_major = 0, cc_minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&cc_minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (cc_major != 10) {
    set_error("BF16x3 tcgen05 contraction needs an sm_100 device (got sm_%d%d)", cc_major, cc_minor);
    return MQCT_E_NODEV;
  }
  tc = std::make_unique<TcInfo>();
  TcInfo& t = *tc;
  t.npad = (nR + 15) / 16 * 16;
  if (t.npad <= 256) {
    t.n0 = t.npad;
    t.n1 = 0;
  } else {
    t.n0 = std::min(256, (t.npad / 2 + 15) / 16 * 16);
    t.n1 = t.npad - t.n0;
  }
  t.tmem_cols = 32;
  while (t.tmem_cols < t.npad) t.tmem_cols *= 2;
  t.n_chunks = (G2 + TC_KC - 1) / TC_KC;
  // blocks: recover from the GEMM rows (tile_block, basis rows per block)
  std::vector<int> row0, nb, bm;
  {
    // basis rows are block-ordered; recompute block extents from the host copies
    int nblk = 0;
    for (int b : h_tile_block) nblk = std::max(nblk, b + 1);
    row0.assign(nblk, 0);
    nb.assign(nblk, 0);
    bm.assign(nblk, 0);
    for (int i = 0; i < nblk; ++i) {
      row0[i] = h_block_row0[i];
      nb[i] = h_block_n[i];
      bm[i] = h_block_m[i];
    }
  }
  t.n_blocks = (int)row0.size();
  t.nbmax = 0;
  std::vector<int64_t> off(t.n_blocks);
  int64_t acc = 0;
  for (int b = 0; b < t.n_blocks; ++b) {
    off[b] = acc;
    acc += (int64_t)nb[b] * t.n_chunks * TC_PSI_LD;
    t.nbmax = std::max(t.nbmax, nb[b]);
  }
  // shared memory: B image, basis slice, A stages, barriers
  size_t b_bytes = 2ull * TC_KC * t.npad * 2, psi_bytes = (size_t)t.nbmax * TC_PSI_LD * 8;
  auto up = [](size_t x) { return (x + 1023) & ~size_t(1023); };
  int dev_smem = 0;
  cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  t.stages = 4;
  for (; t.stages >= 2; --t.stages) {
    t.smem = 1024 + up(b_bytes) + up(psi_bytes) + (size_t)t.stages * 2 * TC_A_PLANE + 256;
    if (t.smem <= (size_t)dev_smem) break;
  }
  MQCT_ARG_CHECK(t.stages >= 2, "shared memory too small for the tcgen05 tiles (nR=%d, block %d)",
                 nR, t.nbmax);
  // A CTA holding more than half of the SM's 512 TMEM columns must be alone on
  // its SM: request enough shared memory that a second CTA cannot co-reside.
  if (t.tmem_cols > 256) t.smem = std::max(t.smem, (size_t)dev_smem / 2 + 1024);
  MQCT_CUDA_TRY(t.blk_row0.upload(row0, stream));
  MQCT_CUDA_TRY(t.blk_n.upload(nb, stream));
  MQCT_CUDA_TRY(t.blk_m.upload(bm, stream));
  MQCT_CUDA_TRY(t.blk_img_off.upload(off, stream));
  if (n_alpha > 0) {
    std::vector<float> fa(h_alpha.begin(), h_alpha.end()), fw(h_walpha.begin(), h_walpha.end());
    MQCT_CUDA_TRY(t.alpha.upload(fa, stream));
    MQCT_CUDA_TRY(t.walpha.upload(fw, stream));
  }
  // Work split: a unit is one tile over a range of K-chunks, accumulated in
  // TMEM (FP32) and written out as a partial sum that is reduced in FP64.  A
  // unit accumulates at most ~4096 products per output (limits the FP32
  // accumulation error), and there are at least ~6 waves of units.
  cudaDeviceGetAttribute(&t.n_sm, cudaDevAttrMultiProcessorCount, dev);
  const int per_chunk = TC_KC * (n_alpha > 0 ? n_alpha : 1);
  t.chunks_per_split = std::max(1, std::min(t.n_chunks, 4096 / per_chunk));
  int splits = (t.n_chunks + t.chunks_per_split - 1) / t.chunks_per_split;
  while (t.chunks_per_split > 1 && (int64_t)n_tiles * splits < 6LL * t.n_sm) {
    --t.chunks_per_split;
    splits = (t.n_chunks + t.chunks_per_split - 1) / t.chunks_per_split;
  }
  tc_splits = splits;
  tc_ldp = t.npad;
  MQCT_CUDA_TRY(d_part.alloc((size_t)tc_splits * n_rows * tc_ldp));
  MQCT_CUDA_TRY(d_bimg.alloc((size_t)t.n_chunks * 2 * TC_KC * t.npad));
  MQCT_CUDA_TRY(d_psi32.alloc((size_t)acc));
  MQCT_CUDA_TRY(d_status.alloc(1));
  MQCT_CUDA_TRY(cudaMemsetAsync(d_status.p, 0, sizeof(int), stream));
  if (precision == MQCT_PREC_F16X3) {
    MQCT_CUDA_TRY(t.wexp.alloc((size_t)nR));
    MQCT_CUDA_TRY(d_col_scale.alloc((size_t)nR));
    MQCT_CUDA_TRY(cudaFuncSetAttribute(tc_contract_kernel<true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
  } else {
    MQCT_CUDA_TRY(cudaFuncSetAttribute(tc_contract_kernel<false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
  }
  return MQCT_OK;
}

int MatrixPlan::tc_execute() {
  TcInfo& t = *tc;
  const int thr = 256;
  const bool f16 = precision == MQCT_PREC_F16X3;
  int64_t nb_img = (int64_t)t.n_chunks * TC_KC * t.npad;
  const unsigned nbb = (unsigned)((nb_img + thr - 1) / thr);
  if (f16) {
    tc_wscale_kernel<<<(unsigned)nR, 256, 0, stream>>>(d_W.p, ldw, G2, t.wexp.p, d_col_scale.p);
    MQCT_CUDA_TRY(cudaGetLastError());
    tc_bimage_kernel<true><<<nbb, thr, 0, stream>>>(d_W.p, ldw, G2, nR, t.npad, t.n_chunks,
                                                    t.wexp.p, d_bimg.p);
  } else {
    tc_bimage_kernel<false><<<nbb, thr, 0, stream>>>(d_W.p, ldw, G2, nR, t.npad, t.n_chunks,
                                                     nullptr, d_bimg.p);
  }
  MQCT_CUDA_TRY(cudaGetLastError());
  int64_t np_img = (int64_t)n_basis_rows * t.n_chunks * TC_PSI_LD;
  tc_psiimage_kernel<<<(unsigned)((np_img + thr - 1) / thr), thr, 0, stream>>>(
      d_psi.p, G2, t.n_chunks, t.blk_row0.p, t.blk_n.p, t.blk_img_off.p, t.n_blocks, d_psi32.p,
      n_basis_rows);
  MQCT_CUDA_TRY(cudaGetLastError());
  TcArgs a;
  a.n_splits = tc_splits;
  a.n_units = n_tiles * tc_splits;
  a.n_chunks = t.n_chunks;
  a.chunks_per_split = t.chunks_per_split;
  a.n_alpha_it = n_alpha > 0 ? n_alpha : 1;
  a.Npad = t.npad;
  a.N0 = t.n0;
  a.N1 = t.n1;
  a.nbmax = t.nbmax;
  a.stages = t.stages;
  a.tmem_cols = t.tmem_cols;
  a.tile_block = d_tile_block.p;
  a.blk_row0 = t.blk_row0.p;
  a.blk_n = t.blk_n.p;
  a.blk_m = t.blk_m.p;
  a.blk_img_off = t.blk_img_off.p;
  a.rowa = d_rowa.p;
  a.rowb = d_rowb.p;
  a.psi_img = d_psi32.p;
  a.b_img = d_bimg.p;
  a.alpha = n_alpha > 0 ? t.alpha.p : nullptr;
  a.walpha = n_alpha > 0 ? t.walpha.p : nullptr;
  a.part = d_part.p;
  a.part_stride = (int64_t)n_rows * tc_ldp;
  a.status = d_status.p;
  int grid = std::min(a.n_units, t.n_sm);
  if (f16) tc_contract_kernel<true><<<grid, TC_THREADS, t.smem, stream>>>(a);
  else tc_contract_kernel<false><<<grid, TC_THREADS, t.smem, stream>>>(a);
  MQCT_CUDA_TRY(cudaGetLastError());
  return MQCT_OK;
}

int MatrixPlan::tc_check_status() {
  if (!tc) return MQCT_OK;
  int st = 0;
  MQCT_CUDA_TRY(cudaMemcpyAsync(&st, d_status.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
  if (st) {
    set_error("tcgen05 contraction aborted: a pipeline wait timed out (code %d)", st);
    cudaMemsetAsync(d_status.p, 0, sizeof(int), stream);
    return MQCT_E_DEVICE;
  }
  return MQCT_OK;
}

int MatrixPlan::error_report(const double*, mqct_err_report_t* err) {
  if (err) err->n_sampled = 0;
  return MQCT_OK;
}

}  // namespace mqct
