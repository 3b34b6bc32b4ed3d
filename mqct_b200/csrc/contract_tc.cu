// contract_tc.cu -- split-precision tensor-core contraction of the matrix build
// on sm_100a: tcgen05.mma kind::f16 with FP32 accumulators in TMEM, drained into
// FP64 sums after every short accumulation.
//
//   M[row, i] = sum_{c, alpha} w_alpha sum_{g in chunk c} X[row, g] W[g, i]
//   X = X_hi + X_lo, W = W_hi + W_lo (16-bit parts),
//   D = X_hi W_hi + X_hi W_lo + X_lo W_hi          (FP32, one K-chunk of 64 points)
//   S += w_alpha D                                  (FP64, in registers)
//
// Two 16-bit formats: BF16x3 (8 significant bits per part, ~16 bits kept) and
// F16x3 (11 bits per part, ~22 bits kept; the products of FP16 parts are exact
// in FP32).  FP16's range is narrow, so in F16x3 X is scaled by 2^14 and every
// radial column of W by the power of two that brings its largest entry to
// [2^13, 2^14); the exact inverse is applied to the FP64 sums.
//
// Accuracy: the tensor core adds the products of one MMA into its FP32
// accumulator with a rounding relative to the largest addend, so a long
// accumulation loses bits in proportion to its length and to how much its terms
// cancel.  Here an accumulator lives for one K-chunk of one alpha point (3 x 4
// MMAs of K = 16) and is then added to FP64 sums, so every sum over the grid is an
// FP64 sum of short FP32 partial sums.  The alpha weight multiplies the drained
// partial in FP64; the tensor-core operand of a K-chunk is the same for every alpha
// point of a same-m pair (the e^{i m alpha} phases of the two states cancel, so
// the integrand at every alpha point is w_alpha Re(psi_a^* psi_b) exactly), and the
// tensor cores contract it once per alpha point.
//
// Work unit = one 128-row tile of pair rows (one m-block) x one column part (at
// most 128 radial points) x one range of K-chunks.  Column parts keep two FP32
// accumulators of a part in TMEM (double buffering: the tensor cores fill one
// while the epilogue drains the other) and the FP64 sums of a part in registers.
// Warp roles (64 + 32 PE threads; PE = 16 epilogue warps when a K-chunk has several
// accumulation groups, 8 when it has one):
//   warp 0      bulk-copy (TMA) producer: per K-chunk the pre-arranged W image of
//               the part (hi and lo planes, K-major core-matrix layout) and the
//               block's rotor-basis slice, one cp.async.bulk each, mbarrier
//               complete_tx, double-buffered where shared memory allows;
//   warp 1      TMEM allocator + single-thread MMA issuer;
//   warps 2..   X producers and epilogue: per K-chunk X = Re(psi_a^* psi_b) in FP32
//               from the staged basis, split to 16-bit hi/lo parts in the
//               core-matrix layout (PE / 4 threads per tile row); then, for every
//               alpha point of the chunk, tcgen05.ld of the accumulator and the FP64
//               update of the sums (PE / 4 warps per TMEM lane quarter, each a share of the
//               part's columns); at the end of a unit the FP64 sums go to global
//               memory, one array per K range.
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
constexpr int TC_KC = 64;        // K elements per chunk (8 core-matrix columns of 8 x 16 bit)
constexpr int TC_PSI_LD = 66;    // float2 per staged basis row (64 + pad)
// Epilogue warps: a template parameter of the kernel, 8 (two per TMEM lane quarter) or 16
// (four per lane quarter, for builds with several accumulation groups per K-chunk, where
// the drain is latency-bound and more warps keep more of it in flight).
template <int PE>
struct TcShape {
  static constexpr int THREADS = 64 + 32 * PE;
  static constexpr int PRODUCERS = 32 * PE;         // X-producer / epilogue threads
  static constexpr int WPQ = PE / 4;                // epilogue warps per TMEM lane quarter
  static constexpr int NCH_MAX = PE == 8 ? 56 : 32;  // columns drained by one epilogue thread
};
constexpr int TC_A_PLANE = TC_M * TC_KC * 2;    // bytes of one 16-bit plane of an A stage
constexpr int TC_NC_MAX = 112;                  // columns of one part (TMEM buffer width)
constexpr int TC_TMEM_COLS = 256;               // allocation (a power of two >= 2 buffers)
static_assert(2 * TC_NC_MAX <= TC_TMEM_COLS, "two accumulator buffers must fit the allocation");
constexpr int TC_MAX_PARTS = 8;
constexpr int TC_SMEM_ALPHA = 64;                // alpha weights kept in shared memory
constexpr uint32_t TC_SPIN_LIMIT = kSpinLimit;  // bounded mbarrier waits

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
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
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
// One accumulation group: Q slices x three split products x four K-steps, in the order
// small products first ((A_hi, B_lo), (A_lo, B_hi), then (A_hi, B_hi)).  The descriptors are
// the chunk's base descriptors plus compile-time or per-chunk offsets (a descriptor holds the
// shared-memory address >> 4 in its low bits), so that the issuing thread does little more
// than issue: the tensor cores consume a group as fast as one thread issues it.
template <int Q>
__device__ __forceinline__ void mma_group(uint32_t td, uint64_t ad0, uint64_t bd0, uint32_t bpl16,
                                          uint32_t bkk16, uint32_t idesc, int nsl) {
  constexpr uint32_t akk16 = (uint32_t)(2 * (TC_M / 8) * 128) >> 4;
  constexpr uint32_t apl16 = (uint32_t)TC_A_PLANE >> 4;
  uint32_t acc = 0u;
#pragma unroll
  for (int pr = 1; pr <= 3; ++pr) {
    const int prod = pr % 3;
    const uint32_t ap = (prod == 2) ? 1u : 0u, bp = (prod == 1) ? 1u : 0u;
    const uint64_t adp = ad0 + ap * apl16, bdp = bd0 + bp * bpl16;
#pragma unroll
    for (int sl = 0; sl < (Q > 0 ? Q : 1); ++sl) {
      if (Q == 0 && sl >= nsl) break;
#pragma unroll
      for (int kk = 0; kk < TC_KC / 16; ++kk) {
        mma_f16(td, adp + kk * akk16, bdp + (uint64_t)(kk * bkk16), idesc, acc);
        acc = 1u;
      }
    }
    if (Q == 0) {  // a group whose size is not a compile-time case: the remaining slices
      for (int sl = 1; sl < nsl; ++sl)
#pragma unroll
        for (int kk = 0; kk < TC_KC / 16; ++kk)
          mma_f16(td, adp + kk * akk16, bdp + (uint64_t)(kk * bkk16), idesc, 1u);
    }
  }
}
// 8 consecutive TMEM columns of this warp's lane quarter (one 32-bit value per lane each);
// the values are valid after tmem_wait().
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
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
// writes the exponent s_i with max * 2^s_i in [2^13, 2^14) and the factor
// 2^-(s_i + kXScaleExp) that undoes both scalings.
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

// Column parts of the radial axis: part p covers columns [c0[p], c0[p] + nc[p]).
struct TcParts {
  int n;
  int c0[TC_MAX_PARTS];
  int nc[TC_MAX_PARTS];
};

// ---------------------------------------------------------------- operand images
// W (FP64, [g][ldw]) -> per column part p and chunk c: [plane hi/lo][kg 0..7][ng 0..nc/8-1]
// [8 rows][8 x 16 bit] at part_off(p) + c * 2 * TC_KC * nc(p), part_off(p) = n_chunks * 2 *
// TC_KC * c0(p); F16x3 scales column n by 2^wexp[n] first (exact).
template <bool kF16>
__global__ void tc_bimage_kernel(const double* __restrict__ W, int ldw, int G2, int nR, int npad,
                                 int n_chunks, TcParts parts, const int* __restrict__ wexp,
                                 unsigned short* __restrict__ img) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t per_chunk = (int64_t)TC_KC * npad;
  if (idx >= per_chunk * n_chunks) return;
  int c = (int)(idx / per_chunk);
  int rem = (int)(idx % per_chunk);
  int n = rem / TC_KC, k = rem % TC_KC;
  int p = 0;
  while (p + 1 < parts.n && parts.c0[p + 1] <= n) ++p;
  const int nl = n - parts.c0[p], nc = parts.nc[p];
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
  int kg = k >> 3, e = k & 7, ng = nl >> 3, r8 = nl & 7;
  const size_t plane = (size_t)TC_KC * nc;
  const size_t off = (size_t)n_chunks * 2 * TC_KC * parts.c0[p] + (size_t)c * 2 * plane +
                     (((size_t)kg * (nc / 8) + ng) * 8 + r8) * 8 + e;
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
  int n_units, n_parts, n_ks, n_chunks, chunks_per_ks, n_alpha_it, nbmax;
  int slices_per_drain;           // alpha points accumulated in FP32 between two drains
  int nbuf;                       // B / basis-slice buffers (1 or 2)
  uint32_t b_stage, psi_stage;    // bytes of one B / basis-slice buffer
  TcParts parts;
  const int* tile_block;          // per tile
  const int* blk_row0;            // basis row offset per block
  const int* blk_n;
  const int64_t* blk_img_off;     // float2 offset of the block's psi image
  const int* rowa;                // basis row of st1 / st2 per GEMM row
  const int* rowb;
  const float2* psi_img;
  const unsigned short* b_img;    // hi/lo planes of W, BF16 or F16 bits, per column part
  const double* walpha;           // alpha weights (n_alpha_it), or null (weight 1)
  const double* col_scale;        // per radial column: factor applied to the FP64 sums
  double* part;                   // n_ks x n_rows x ldp FP64 sums
  int64_t part_stride;
  int ldp;
  int* status;
};

// Use k of a resource with nb buffers: buffer k % nb; its "full" barrier completes
// for the (k / nb)-th time, its "empty" barrier (before reuse, k >= nb) completed
// (k / nb - 1) times before.
__device__ __forceinline__ uint32_t full_parity(uint32_t k, uint32_t nb) { return (k / nb) & 1u; }
__device__ __forceinline__ uint32_t empty_parity(uint32_t k, uint32_t nb) {
  return ((k / nb) + 1u) & 1u;
}

template <bool kF16, int PE>
__global__ void __launch_bounds__(TcShape<PE>::THREADS, 1) tc_contract_kernel(TcArgs a) {
  constexpr int TC_THREADS = TcShape<PE>::THREADS, TC_PRODUCERS = TcShape<PE>::PRODUCERS;
  constexpr int TC_KSPLIT = TC_PRODUCERS / TC_M;  // threads per tile row in X production
  constexpr int TC_WPQ = TcShape<PE>::WPQ, TC_NCH_MAX = TcShape<PE>::NCH_MAX;
  static_assert(TC_PRODUCERS % TC_M == 0 && (TC_KC / 8) % TC_KSPLIT == 0, "X production split");
  static_assert((TC_NC_MAX / 8 + TC_WPQ - 1) / TC_WPQ <= TC_NCH_MAX / 8, "drain split");
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023);
  unsigned char* sB = reinterpret_cast<unsigned char*>(base);           // nbuf x b_stage
  unsigned char* sPsi = sB + a.nbuf * a.b_stage;                         // nbuf x psi_stage
  unsigned char* sA = sPsi + a.nbuf * a.psi_stage;                       // 2 x A stage
  const uint32_t a_stage = 2u * TC_A_PLANE;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sA + 2 * a_stage);
  uint64_t* B_full = bars;          // [2]
  uint64_t* B_empty = bars + 2;     // [2]
  uint64_t* P_full = bars + 4;      // [2]
  uint64_t* P_empty = bars + 6;     // [2]
  uint64_t* A_full = bars + 8;      // [2]
  uint64_t* A_empty = bars + 10;    // [2]
  uint64_t* ACC_full = bars + 12;   // [2]
  uint64_t* ACC_empty = bars + 14;  // [2]
  uint64_t* DONE = bars + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 18);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 19);

  // the alpha weights in shared memory: the epilogue reads one per drain, and a global
  // load there would sit on the drain's critical path
  __shared__ double s_walpha[TC_SMEM_ALPHA];
  for (int i = threadIdx.x; i < TC_SMEM_ALPHA; i += TC_THREADS)
    s_walpha[i] = (a.walpha && i < a.n_alpha_it) ? a.walpha[i] : 1.0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&B_full[s], 1);
      mbar_init(&B_empty[s], 1);
      mbar_init(&P_full[s], 1);
      mbar_init(&P_empty[s], TC_PRODUCERS);
      mbar_init(&A_full[s], TC_PRODUCERS);
      mbar_init(&A_empty[s], 1);
      mbar_init(&ACC_full[s], 1);
      mbar_init(&ACC_empty[s], TC_PRODUCERS);
    }
    mbar_init(DONE, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t nbuf = (uint32_t)a.nbuf;

  if (warp == 0) {
    // ---------------- bulk-copy producer
    if (lane == 0) {
      uint32_t k = 0;  // chunk uses so far (B and basis slices move together)
      for (int u = blockIdx.x; u < a.n_units && !*abort_flag; u += gridDim.x) {
        const int ks = u % a.n_ks, pt = (u / a.n_ks) % a.n_parts, tile = u / (a.n_ks * a.n_parts);
        const int blk = a.tile_block[tile];
        const int nb = a.blk_n[blk];
        const int nc = a.parts.nc[pt];
        const uint32_t psi_bytes = (uint32_t)nb * TC_PSI_LD * 8u;
        const uint32_t b_bytes = 2u * TC_KC * (uint32_t)nc * 2u;
        const unsigned short* bsrc = a.b_img + (size_t)a.n_chunks * 2 * TC_KC * a.parts.c0[pt];
        const int c0 = ks * a.chunks_per_ks, c1 = min(a.n_chunks, c0 + a.chunks_per_ks);
        for (int c = c0; c < c1; ++c, ++k) {
          const uint32_t s = k % nbuf;
          if (k >= nbuf) {
            if (!mbar_wait(&B_empty[s], empty_parity(k, nbuf), abort_flag, a.status, 11)) break;
            if (!mbar_wait(&P_empty[s], empty_parity(k, nbuf), abort_flag, a.status, 12)) break;
          }
          mbar_expect_tx(&B_full[s], b_bytes);
          bulk_g2s(sB + s * a.b_stage, bsrc + (size_t)c * 2 * TC_KC * nc, b_bytes, &B_full[s]);
          mbar_expect_tx(&P_full[s], psi_bytes);
          bulk_g2s(sPsi + s * a.psi_stage,
                   a.psi_img + a.blk_img_off[blk] + (int64_t)c * nb * TC_PSI_LD, psi_bytes,
                   &P_full[s]);
        }
      }
      // the copies issued last must have landed before the CTA exits
      for (uint32_t j = (k > nbuf ? k - nbuf : 0); j < k; ++j) {
        const uint32_t s = j % nbuf;
        for (uint32_t it = 0; it < TC_SPIN_LIMIT && !mbar_try_wait(&B_full[s], full_parity(j, nbuf)); ++it) {}
        for (uint32_t it = 0; it < TC_SPIN_LIMIT && !mbar_try_wait(&P_full[s], full_parity(j, nbuf)); ++it) {}
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      uint32_t kc = 0, ka = 0, kacc = 0;  // chunk uses, A-stage uses, accumulator uses
      const uint32_t sA0 = smem_u32(sA), sB0 = smem_u32(sB);
      const uint32_t lbo_a = (TC_M / 8) * 128;
      for (int u = blockIdx.x; u < a.n_units && !*abort_flag; u += gridDim.x) {
        const int ks = u % a.n_ks, pt = (u / a.n_ks) % a.n_parts;
        const int nc = a.parts.nc[pt];
        const uint32_t idesc = kF16 ? idesc_f16(TC_M, nc) : idesc_bf16(TC_M, nc);
        const uint32_t lbo_b = (uint32_t)(nc / 8) * 128, bplane = (uint32_t)TC_KC * nc * 2;
        const int c0 = ks * a.chunks_per_ks, c1 = min(a.n_chunks, c0 + a.chunks_per_ks);
        bool ok = true;
        for (int c = c0; c < c1 && ok; ++c, ++kc, ++ka) {
          const uint32_t sb = kc % nbuf, sa = ka & 1u;
          ok = mbar_wait(&B_full[sb], full_parity(kc, nbuf), abort_flag, a.status, 21) &&
               mbar_wait(&A_full[sa], full_parity(ka, 2), abort_flag, a.status, 22);
          if (!ok) break;
          tc_fence_after();
          const uint32_t aoff = sA0 + sa * (2 * TC_A_PLANE);
          const uint32_t boff0 = sB0 + sb * a.b_stage;
          const uint64_t ad0 = smem_desc(aoff, lbo_a, 128), bd0 = smem_desc(boff0, lbo_b, 128);
          const uint32_t bpl16 = bplane >> 4, bkk16 = (2 * lbo_b) >> 4;
          for (int al = 0; al < a.n_alpha_it; ++al, ++kacc) {
            const uint32_t sc = kacc & 1u;
            if (kacc >= 2) {  // the epilogue must have drained this accumulator
              if (!mbar_wait(&ACC_empty[sc], empty_parity(kacc, 2), abort_flag, a.status, 23)) {
                ok = false;
                break;
              }
              tc_fence_after();
            }
            const uint32_t td = tmem + sc * TC_NC_MAX;
            const int ns_grp = min(a.slices_per_drain, a.n_alpha_it - al);
            switch (ns_grp) {
              case 1: mma_group<1>(td, ad0, bd0, bpl16, bkk16, idesc, 1); break;
              case 2: mma_group<2>(td, ad0, bd0, bpl16, bkk16, idesc, 2); break;
              case 4: mma_group<4>(td, ad0, bd0, bpl16, bkk16, idesc, 4); break;
              case 8: mma_group<8>(td, ad0, bd0, bpl16, bkk16, idesc, 8); break;
              default: mma_group<0>(td, ad0, bd0, bpl16, bkk16, idesc, ns_grp); break;
            }
            mma_commit(&ACC_full[sc]);  // the epilogue may read once these MMAs complete
            al += ns_grp - 1;
          }
          mma_commit(&A_empty[sa]);  // A and B may be overwritten once the chunk's MMAs complete
          mma_commit(&B_empty[sb]);
        }
      }
      // every MMA issued by this thread has completed before TMEM is released
      mma_commit(DONE);
      for (uint32_t it = 0; it < TC_SPIN_LIMIT && !mbar_try_wait(DONE, 0); ++it) {}
    }
  } else {
    // ---------------- X producers (warps 2 to PE + 1) and epilogue
    const int t = threadIdx.x - 64;
    const int p = t & (TC_M - 1);  // tile row generated by this thread
    const int kh = t / TC_M;       // share of the chunk's K groups formed by this thread
    const int q = warp & 3;        // TMEM lane quarter accessible to this warp
    const int h = (warp - 2) >> 2; // share of the part's columns drained by this warp
    uint32_t kc = 0, ka = 0, kacc = 0;
    double S[TC_NCH_MAX];
    for (int u = blockIdx.x; u < a.n_units && !*abort_flag; u += gridDim.x) {
      const int ks = u % a.n_ks, pt = (u / a.n_ks) % a.n_parts, tile = u / (a.n_ks * a.n_parts);
      const int blk = a.tile_block[tile];
      const int row = tile * TC_M + p;
      const int la = a.rowa[row] - a.blk_row0[blk], lb = a.rowb[row] - a.blk_row0[blk];
      // the part's batches of 8 columns split over the warps of a lane quarter
      const int nb8 = a.parts.nc[pt] / 8;
      const int b8lo = h * nb8 / TC_WPQ, b8hi = (h + 1) * nb8 / TC_WPQ;
      const int nch = 8 * (b8hi - b8lo), coff = 8 * b8lo, col0 = a.parts.c0[pt] + coff;
      const int c0 = ks * a.chunks_per_ks, c1 = min(a.n_chunks, c0 + a.chunks_per_ks);
#pragma unroll
      for (int i = 0; i < TC_NCH_MAX; ++i) S[i] = 0.0;
      // produce the operand of chunk use kcu into A stage (kau & 1) from basis slice
      // (kcu % nbuf)
      auto produce = [&](uint32_t kcu, uint32_t kau) -> bool {
        const uint32_t sp = kcu % nbuf, sa = kau & 1u;
        if (!mbar_wait(&P_full[sp], full_parity(kcu, nbuf), abort_flag, a.status, 31)) return false;
        if (kau >= 2 && !mbar_wait(&A_empty[sa], empty_parity(kau, 2), abort_flag, a.status, 32))
          return false;
        const float2* ps = reinterpret_cast<const float2*>(sPsi + sp * a.psi_stage);
        const float2* pa = ps + la * TC_PSI_LD;
        const float2* pb = ps + lb * TC_PSI_LD;
        unsigned char* hi = sA + sa * (2 * TC_A_PLANE);
        unsigned char* lo = hi + TC_A_PLANE;
#pragma unroll
        for (int kq = 0; kq < TC_KC / 8 / TC_KSPLIT; ++kq) {
          const int kg = kh * (TC_KC / 8 / TC_KSPLIT) + kq;
          float x[8];
#pragma unroll
          for (int e = 0; e < 8; e += 2) {
            const float4 va = *reinterpret_cast<const float4*>(pa + kg * 8 + e);
            const float4 vb = *reinterpret_cast<const float4*>(pb + kg * 8 + e);
            x[e] = va.x * vb.x + va.y * vb.y;
            x[e + 1] = va.z * vb.z + va.w * vb.w;
          }
          if (kF16) {
#pragma unroll
            for (int e = 0; e < 8; ++e) x[e] *= (float)(1 << kXScaleExp);  // exact
          }
          uint4 hv, lv;
          split8<kF16>(x, hv, lv);
          const uint32_t off = (uint32_t)(kg * (TC_M / 8) + (p >> 3)) * 128u + (uint32_t)(p & 7) * 16u;
          *reinterpret_cast<uint4*>(hi + off) = hv;
          *reinterpret_cast<uint4*>(lo + off) = lv;
        }
        fence_proxy_async();
        mbar_arrive(&A_full[sa]);
        mbar_arrive(&P_empty[sp]);
        return true;
      };
      // With two B / basis buffers the next chunk's operand is formed before this chunk
      // is drained, so the tensor cores go on while the epilogue works.  With one, the
      // next copy waits for this chunk's MMAs, which wait for its drains: form it after.
      const bool ahead = nbuf == 2;
      bool ok = c0 < c1 ? produce(kc, ka) : true;
      for (int c = c0; c < c1 && ok; ++c, ++kc, ++ka) {
        if (ahead && c + 1 < c1 && !produce(kc + 1, ka + 1)) {
          ok = false;
          break;
        }
        for (int al = 0; al < a.n_alpha_it; al += a.slices_per_drain, ++kacc) {
          const uint32_t sc = kacc & 1u;
          if (!mbar_wait(&ACC_full[sc], full_parity(kacc, 2), abort_flag, a.status, 33)) {
            ok = false;
            break;
          }
          tc_fence_after();
          // a group of several alpha points shares one (uniform) weight
          const double wa = al < TC_SMEM_ALPHA ? s_walpha[al] : (a.walpha ? a.walpha[al] : 1.0);
          const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + sc * TC_NC_MAX + (uint32_t)coff;
          // batches of 8 columns, software-pipelined: the next batch's TMEM load is in
          // flight while this batch is added to the FP64 sums
          constexpr int NB8 = TC_NCH_MAX / 8;
          uint32_t r[2][8];
          tmem_ld8(taddr, r[0]);
          tmem_wait();
#pragma unroll
          for (int b8 = 0; b8 < NB8; ++b8) {
            if (8 * b8 < nch) {  // the same for the whole warp
              const bool more = 8 * (b8 + 1) < nch;
              if (more) tmem_ld8(taddr + 8 * (b8 + 1), r[(b8 + 1) & 1]);
#pragma unroll
              for (int e = 0; e < 8; ++e) {
                double& acc = S[8 * b8 + e];
                acc = fma((double)__uint_as_float(r[b8 & 1][e]), wa, acc);
              }
              if (more) tmem_wait();
            }
          }
          tc_fence_before();
          mbar_arrive(&ACC_empty[sc]);
        }
        if (ok && !ahead && c + 1 < c1 && !produce(kc + 1, ka + 1)) ok = false;
      }
      if (!ok) break;
      // the unit's FP64 sums, with the exact column factors
      double* dst = a.part + (int64_t)ks * a.part_stride + (int64_t)(tile * TC_M + q * 32 + lane) * a.ldp;
#pragma unroll
      for (int i = 0; i < TC_NCH_MAX; ++i)
        if (i < nch) dst[col0 + i] = S[i] * a.col_scale[col0 + i];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TC_TMEM_COLS));
  }
}

// ---------------------------------------------------------------- host side
int MatrixPlan::tc_init() {
  MQCT_ARG_CHECK(nR <= TC_NC_MAX * TC_MAX_PARTS, "tensor-core contraction supports nR <= %d (got %d)",
                 TC_NC_MAX * TC_MAX_PARTS, nR);
  int dev = 0, cc_major = 0, cc_minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&cc_minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (cc_major != 10) {
    set_error("the tcgen05 contraction needs an sm_100 device (got sm_%d%d)", cc_major, cc_minor);
    return MQCT_E_NODEV;
  }
  tc = std::make_unique<TcInfo>();
  TcInfo& t = *tc;
  t.npad = (nR + 15) / 16 * 16;
  // column parts: as few as the TMEM buffer width allows, balanced, widths multiples of 16
  const int n16 = t.npad / 16;
  t.n_parts = (t.npad + TC_NC_MAX - 1) / TC_NC_MAX;
  for (int p = 0, c = 0; p < t.n_parts; ++p) {
    const int w = (n16 / t.n_parts + (p < n16 % t.n_parts ? 1 : 0)) * 16;
    t.part_c0[p] = c;
    t.part_nc[p] = w;
    c += w;
  }
  t.n_chunks = (G2 + TC_KC - 1) / TC_KC;
  std::vector<int> row0(h_block_row0), nb(h_block_n), bm(h_block_m);
  t.n_blocks = (int)row0.size();
  t.nbmax = 0;
  std::vector<int64_t> off(t.n_blocks);
  int64_t acc = 0;
  for (int b = 0; b < t.n_blocks; ++b) {
    off[b] = acc;
    acc += (int64_t)nb[b] * t.n_chunks * TC_PSI_LD;
    t.nbmax = std::max(t.nbmax, nb[b]);
  }
  // shared memory: B buffers, basis-slice buffers, two A stages, barriers
  int ncmax = 0;
  for (int p = 0; p < t.n_parts; ++p) ncmax = std::max(ncmax, t.part_nc[p]);
  auto up = [](size_t x) { return (x + 1023) & ~size_t(1023); };
  t.b_stage = (uint32_t)up(2ull * TC_KC * ncmax * 2);
  t.psi_stage = (uint32_t)up((size_t)t.nbmax * TC_PSI_LD * 8);
  int dev_smem = 0;
  cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  {
    // the kernel's static shared memory (the alpha weights) comes out of the same budget
    cudaFuncAttributes fa{};
    MQCT_CUDA_TRY(cudaFuncGetAttributes(&fa, tc_contract_kernel<true, 16>));
    dev_smem -= (int)fa.sharedSizeBytes;
  }
  for (t.nbuf = 2; t.nbuf >= 1; --t.nbuf) {
    t.smem = 1024 + (size_t)t.nbuf * (t.b_stage + t.psi_stage) + 2ull * 2 * TC_A_PLANE + 256;
    if (t.smem <= (size_t)dev_smem) break;
  }
  MQCT_ARG_CHECK(t.nbuf >= 1, "shared memory too small for the tcgen05 tiles (nR=%d, block %d)",
                 nR, t.nbmax);
  // one CTA per SM (the TMEM buffers and the register sums are sized for it)
  t.smem = std::max(t.smem, (size_t)dev_smem / 2 + 1024);
  MQCT_CUDA_TRY(t.blk_row0.upload(row0, stream));
  MQCT_CUDA_TRY(t.blk_n.upload(nb, stream));
  MQCT_CUDA_TRY(t.blk_m.upload(bm, stream));
  MQCT_CUDA_TRY(t.blk_img_off.upload(off, stream));
  if (n_alpha > 0) MQCT_CUDA_TRY(t.walpha.upload(h_walpha, stream));
  // alpha points per drain: a group shares one weight, so groups of more than one point
  // need equal weights (the midpoint alpha grid); 2 keeps the drains under the MMA time
  t.alpha_uniform = true;
  for (int i = 1; i < n_alpha; ++i)
    if (h_walpha[i] != h_walpha[0]) t.alpha_uniform = false;
  t.slices_per_drain = (n_alpha > 1 && t.alpha_uniform) ? 2 : 1;
  // K ranges: split the chunks only to fill the last wave of units (the FP64 sums of
  // every range are written once and added by the finalize)
  cudaDeviceGetAttribute(&t.n_sm, cudaDevAttrMultiProcessorCount, dev);
  int best_ks = 1;
  double best_eff = 0.0;
  for (int ks = 1; ks <= std::min(4, t.n_chunks); ++ks) {
    const double units = (double)n_tiles * t.n_parts * ks;
    const double waves = units / t.n_sm;
    const double eff = waves / std::ceil(waves) - 0.01 * (ks - 1);  // partial-sum traffic
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best_ks = ks;
    }
  }
  t.chunks_per_split = (t.n_chunks + best_ks - 1) / best_ks;
  tc_splits = (t.n_chunks + t.chunks_per_split - 1) / t.chunks_per_split;
  tc_ldp = t.npad;
  MQCT_CUDA_TRY(d_part.alloc((size_t)tc_splits * n_rows * tc_ldp));
  MQCT_CUDA_TRY(d_bimg.alloc((size_t)t.n_chunks * 2 * TC_KC * t.npad));
  MQCT_CUDA_TRY(d_psi32.alloc((size_t)acc));
  MQCT_CUDA_TRY(d_status.alloc(1));
  MQCT_CUDA_TRY(cudaMemsetAsync(d_status.p, 0, sizeof(int), stream));
  MQCT_CUDA_TRY(d_col_scale.alloc((size_t)t.npad));
  if (precision == MQCT_PREC_F16X3) {
    MQCT_CUDA_TRY(t.wexp.alloc((size_t)nR));
    MQCT_CUDA_TRY(cudaMemsetAsync(d_col_scale.p, 0, sizeof(double) * t.npad, stream));
    MQCT_CUDA_TRY(cudaFuncSetAttribute(tc_contract_kernel<true, 8>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
    MQCT_CUDA_TRY(cudaFuncSetAttribute(tc_contract_kernel<true, 16>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
  } else {
    std::vector<double> ones(t.npad, 1.0);
    MQCT_CUDA_TRY(d_col_scale.upload(ones, stream));
    MQCT_CUDA_TRY(cudaFuncSetAttribute(tc_contract_kernel<false, 8>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
    MQCT_CUDA_TRY(cudaFuncSetAttribute(tc_contract_kernel<false, 16>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t.smem));
  }
  return MQCT_OK;
}

int MatrixPlan::tc_execute() {
  TcInfo& t = *tc;
  const int thr = 256;
  const bool f16 = precision == MQCT_PREC_F16X3;
  TcParts parts{};
  parts.n = t.n_parts;
  for (int p = 0; p < t.n_parts; ++p) {
    parts.c0[p] = t.part_c0[p];
    parts.nc[p] = t.part_nc[p];
  }
  int64_t nb_img = (int64_t)t.n_chunks * TC_KC * t.npad;
  const unsigned nbb = (unsigned)((nb_img + thr - 1) / thr);
  if (f16) {
    tc_wscale_kernel<<<(unsigned)nR, 256, 0, stream>>>(d_W.p, ldw, G2, t.wexp.p, d_col_scale.p);
    MQCT_CUDA_TRY(cudaGetLastError());
    tc_bimage_kernel<true><<<nbb, thr, 0, stream>>>(d_W.p, ldw, G2, nR, t.npad, t.n_chunks, parts,
                                                    t.wexp.p, d_bimg.p);
  } else {
    tc_bimage_kernel<false><<<nbb, thr, 0, stream>>>(d_W.p, ldw, G2, nR, t.npad, t.n_chunks, parts,
                                                     nullptr, d_bimg.p);
  }
  MQCT_CUDA_TRY(cudaGetLastError());
  int64_t np_img = (int64_t)n_basis_rows * t.n_chunks * TC_PSI_LD;
  tc_psiimage_kernel<<<(unsigned)((np_img + thr - 1) / thr), thr, 0, stream>>>(
      d_psi.p, G2, t.n_chunks, t.blk_row0.p, t.blk_n.p, t.blk_img_off.p, t.n_blocks, d_psi32.p,
      n_basis_rows);
  MQCT_CUDA_TRY(cudaGetLastError());
  TcArgs a{};
  a.n_parts = t.n_parts;
  a.n_ks = tc_splits;
  a.n_units = n_tiles * t.n_parts * tc_splits;
  a.n_chunks = t.n_chunks;
  a.chunks_per_ks = t.chunks_per_split;
  a.n_alpha_it = n_alpha > 0 ? n_alpha : 1;
  a.slices_per_drain = std::max(1, std::min(t.slices_per_drain, a.n_alpha_it));
  a.nbmax = t.nbmax;
  a.nbuf = t.nbuf;
  a.b_stage = t.b_stage;
  a.psi_stage = t.psi_stage;
  a.parts = parts;
  a.tile_block = d_tile_block.p;
  a.blk_row0 = t.blk_row0.p;
  a.blk_n = t.blk_n.p;
  a.blk_img_off = t.blk_img_off.p;
  a.rowa = d_rowa.p;
  a.rowb = d_rowb.p;
  a.psi_img = d_psi32.p;
  a.b_img = d_bimg.p;
  a.walpha = n_alpha > 0 ? t.walpha.p : nullptr;
  a.col_scale = d_col_scale.p;
  a.part = d_part.p;
  a.part_stride = (int64_t)n_rows * tc_ldp;
  a.ldp = tc_ldp;
  a.status = d_status.p;
  int grid = std::min(a.n_units, t.n_sm);
  // sixteen epilogue warps when a K-chunk has several accumulation groups (the drains then
  // dominate: the as-written alpha grid), eight when it has one (the drain of a chunk then
  // alternates with its X production, and eight warps with more registers are faster)
  const bool many = t.pe_force ? t.pe_force == 16
                               : (a.n_alpha_it + a.slices_per_drain - 1) / a.slices_per_drain >= 2;
  t.pe_warps = many ? 16 : 8;
  if (f16) {
    if (many) tc_contract_kernel<true, 16><<<grid, TcShape<16>::THREADS, t.smem, stream>>>(a);
    else tc_contract_kernel<true, 8><<<grid, TcShape<8>::THREADS, t.smem, stream>>>(a);
  } else {
    if (many) tc_contract_kernel<false, 16><<<grid, TcShape<16>::THREADS, t.smem, stream>>>(a);
    else tc_contract_kernel<false, 8><<<grid, TcShape<8>::THREADS, t.smem, stream>>>(a);
  }
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
