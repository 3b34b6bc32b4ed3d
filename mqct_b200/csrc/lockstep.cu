// lockstep.cu -- lockstep engine of the trajectory propagation (H2): standard MQCT,
// fixed-step RK4 (DOTRAJECT, MQCT_SOURCE_CODES/propagator.f:2283-4645, with DERIVS_BK,
// MQCT_SOURCE_CODES/mqct_eqtns.f:112-499, and RK4, MQCT_SOURCE_CODES/suppl_routines.f:
// 1076-1113), for batches large enough to share the knot reads.
//
// The per-trajectory kernel (propagate.cu) reads the two knot rows of its spline
// interval for every right-hand side: 640 KB per evaluation for the 969-state table,
// served from L2 at about 5 TB/s, which bounds it.  Trajectories of a batch that sit in
// the same interval at the same moment need the same knot rows.  This engine advances
// every trajectory of the batch by one right-hand side per round (one RK4 stage) and
// groups them by the spline interval of their stage point, so that one load of the
// interval's knots serves the whole group:
//
//   ls_rhs  (one launch per round; persistent CTAs take one work item at a time from a
//           device queue): item = (interval,
//           m-block, group of up to G trajectories of that interval).  The block's knot
//           triangle at the two rows of the interval is staged in shared memory as
//           (M_lo, M_hi - M_lo, M''_lo, M''_hi) per slot, bt = D^* a of the group's
//           trajectories next to it, and the four products Z_q = K_q bt are formed by
//           threads that own one row and TB trajectories (lanes = consecutive rows, so
//           that the row updates below are coalesced; fixed order in j).  Per trajectory
//               y  = M(R) bt  = (A + B) Z_0 + B Z_1 + C1 Z_2 + C2 Z_3,
//               M'(R) bt      = Z_1 / h + D1 Z_2 + D2 Z_3
//           with the spline factors of its own R (splint_bk, MQCT_SOURCE_CODES/
//           mqct_eqtns.f:555-611).  Then, per row: the Coriolis vector u, the amplitude
//           derivative da = -i e^{iEt} y - i (dphi/2) u, the RK4 update of the row
//           (FP64 amplitudes; stage input and derivative sum in the arithmetic type),
//           and the block's share of F = Re(bt^+ M' bt), g = Im((D^* u)^+ y) and
//           pot = Re(bt^+ y), written per (trajectory, block) -- no atomics, so every
//           sum has a fixed order and the results do not depend on the grouping.
//           The item that completes a trajectory's blocks (a per-trajectory counter)
//           takes its classical step with one warp (ls_traj_step): the block shares
//           summed in block order, the classical derivative, the RK4 stage of the
//           classical variables, at the end of a step the stop rules
//           (MQCT_SOURCE_CODES/propagator.f:4011-4050); the next stage point (spline
//           interval, factors, phases e^{-iEt} per energy class); the trajectory is
//           registered in its interval's bucket for the next round.  The last CTA to
//           finish the round forms the next round's groups of up to G trajectories
//           (ls_group).  ls_init_kernel does the same for the start of a run.
//
// A finished trajectory takes one closing evaluation at its final state (the energy
// bookkeeping of MQCT_SOURCE_CODES/propagator.f:4182-4343) and retires.  The arithmetic
// of every right-hand side is that of the per-trajectory kernel in type T (products in
// T, sums of the quadratic forms in FP64, FP64 phases rounded to T), except that the
// matrix is applied as the four knot products above instead of being interpolated slot
// by slot; the M_hi - M_lo column keeps the force free of the cancellation of two
// interpolated values.  The host runs the rounds as a CUDA graph and reads the number of
// running trajectories after each graph launch.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "propagate.cuh"

namespace mqct {

constexpr int LS_CLS_THREADS = 256;

// Launch shape and work split per arithmetic type.  FP32: 16-byte slot entries, 16
// trajectories per item, 4 per thread, three CTAs of 256 threads per SM (the items of a
// round are short: several per SM in flight hide their load latencies).  FP64: 32-byte
// entries (the 81-state triangle takes 106 KB), 16 per item, 4 per thread, one CTA of 512
// threads per SM.
template <class T> struct LsCfg;
template <> struct LsCfg<float> {
  static constexpr int G = 16, TB = 4, THREADS = 256, PER_SM = 3;
  struct E { float4 a; };
};
template <> struct LsCfg<double> {
  static constexpr int G = 16, TB = 4, THREADS = 512, PER_SM = 1;
  struct E { double2 a, b; };
};
// warp units (32 rows x TB trajectories) of one item: blocks of at most 128 states
constexpr int LS_MAX_ROWS = 128;
constexpr int LS_MAX_UNITS = 16;

// Per-trajectory state (global memory).
struct LsTraj {
  Cls C, CT, K1, K23;              // state, stage point, first-stage and middle-stage sums
  double tcur, dt, eki, eqi, tmpR1, tmpR2;
  double th_c, sin_c, is2_c;       // theta of the cached sine and 1/sin^2 (planar motion)
  double dphidt, sin_t, inv_r, inv_s2;  // scalars of the stage point
  double sp[7];                    // spline factors of the stage point: A + B, B, C1, C2, 1/h, D1, D2
  int counter, status, vib, period;
  int stage;                       // 0..3 RK4 stages, 4 closing evaluation
  int active;
  int key;                         // spline interval of the stage point; nR - 1: above the grid
  int hint;                        // spline interval found last
  int s_int;                       // initial state (internal index)
};

struct LsDev {
  LsTraj* tr;
  const mqct_traj_init_t* init;
  int n_traj, n_blocks;
  int tri_cap;                     // slots of the largest block triangle
  double2* Y;                      // n x N amplitudes
  void* ACC;                       // n x N T2: k1 + 2 k2 + 2 k3
  void* AIN[2];                    // n x N T2: stage inputs (this round, next round)
  void* PH;                        // n x n_e T2: e^{-iEt} at the stage point
  double* part;                    // n x n_blocks x 3 block shares
  int* cnt;                        // per key: trajectories registered for the next round
  int* kcnt;                       // per key: trajectories of this round
  int* gstart;                     // per key: its first group of this round
  int* gkey;                       // per group of this round: its key
  int* bucket[2];                  // per key: its trajectories (n_traj places each), for the
                                   // rounds of even and odd parity
  int* tdone;                      // per trajectory: its block items finished this round
  int* n_groups;                   // groups of up to G trajectories of this round
  int* n_items;                    // groups x blocks
  int* queue;                      // ls_rhs work queue
  int* done;                       // ls_cls CTAs finished
  int* n_active;
  const int* blk_order;            // blocks by size, largest first
  double* amp;
  double* cls;
  double* diag;
};

template <class T>
__device__ void ls_traj_step(const PropDev& d, const LsDev& L, int tr, int lane, bool init, int rpar);
template <int G, int NT>
__device__ void ls_group(const PropDev& d, const LsDev& L);

__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// ---------------------------------------------------------------- ls_rhs
template <class T>
__global__ void __launch_bounds__(LsCfg<T>::THREADS, LsCfg<T>::PER_SM)
ls_rhs_kernel(PropDev d, LsDev L, int par) {
  using T2 = typename V2<T>::t;
  using Cfg = LsCfg<T>;
  using E = typename Cfg::E;
  constexpr int G = Cfg::G, TB = Cfg::TB, NW = Cfg::THREADS / 32;
  static_assert((LS_MAX_ROWS / 32) * (G / TB) <= LS_MAX_UNITS, "warp units of an item");
  extern __shared__ __align__(16) unsigned char ls_smem[];
  __shared__ int s_item[4];
  __shared__ int s_tr[G], s_stage[G];
  __shared__ T s_cf[G][7];
  __shared__ double s_dt[G], s_dphi[G];
  __shared__ double s_red[LS_MAX_UNITS][TB][3];
  __shared__ int s_fin[G];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = d.N;
  const T2* __restrict__ AIN = reinterpret_cast<const T2*>(L.AIN[par]);
  T2* __restrict__ AOUT = reinterpret_cast<T2*>(L.AIN[par ^ 1]);
  T2* __restrict__ ACC = reinterpret_cast<T2*>(L.ACC);
  const T2* __restrict__ PH = reinterpret_cast<const T2*>(L.PH);
  const T2* __restrict__ KN = reinterpret_cast<const T2*>(d.knots);
  E* K4 = reinterpret_cast<E*>(ls_smem);
  T2* bt = reinterpret_cast<T2*>(ls_smem + ((sizeof(E) * (size_t)L.tri_cap + 15) & ~size_t(15)));
  for (;;) {
    __syncthreads();  // the previous item's shared data is no longer read
    if (warp == 0) {
      // item = (block of the blk_order rank, group of up to G trajectories of one key);
      // the groups of the largest block come first.  Warp 0 fetches it and the group's
      // parameters (lane t: trajectory t).
      int it = 0;
      if (lane == 0) it = atomicAdd(L.queue, 1);
      it = __shfl_sync(0xffffffffu, it, 0);
      const int n_it = *L.n_items;
      int key = 0, b = 0, g = 0, off = 0;
      if (it < n_it) {
        const int tg = *L.n_groups;
        const int bo = it / tg, gi = it - bo * tg;
        key = L.gkey[gi];
        off = (gi - L.gstart[key]) * G;
        b = L.blk_order[bo];
        g = min(G, L.kcnt[key] - off);
        if (lane < g) {
          const int tr = L.bucket[par][(size_t)key * L.n_traj + off + lane];
          const LsTraj& S = L.tr[tr];
          s_tr[lane] = tr;
          s_stage[lane] = S.stage;
          s_dt[lane] = S.dt;
          s_dphi[lane] = S.dphidt;
#pragma unroll
          for (int q = 0; q < 7; ++q) s_cf[lane][q] = (T)S.sp[q];
        }
      }
      if (lane == 0) {
        s_item[0] = it < n_it ? 1 : 0;
        s_item[1] = key;
        s_item[2] = b;
        s_item[3] = g | (off << 6);
      }
    }
    __syncthreads();
    if (!s_item[0]) break;
    const int key = s_item[1], b = s_item[2], g = s_item[3] & 63;
    const int nb = __ldg(d.blk_n + b), r0 = __ldg(d.blk_s0 + b);
    const bool zero = key == d.nR - 1;  // above the grid: the matrix is zero
    // the block's triangle at knot rows key and key + 1: (lo, hi - lo, lo'', hi'')
    if (!zero) {
      const int64_t q0 = __ldg(d.blk_slot0 + b);
      const int nsl = nb * (nb + 1) / 2;
      const T2* Klo = KN + (int64_t)key * d.S + q0;
      const T2* Khi = Klo + d.S;
      for (int q = tid; q < nsl; q += Cfg::THREADS) {
        const T2 lo = Klo[q], hi = Khi[q];
        E e;
        if constexpr (sizeof(T) == 4) {
          e.a = make_float4(lo.x, hi.x - lo.x, lo.y, hi.y);
        } else {
          e.a = make_double2(lo.x, hi.x - lo.x);
          e.b = make_double2(lo.y, hi.y);
        }
        K4[q] = e;
      }
    }
    // bt = D^* a of the block's states: row j holds the G trajectories (unused ones zero)
    for (int idx = tid; idx < G * nb; idx += Cfg::THREADS) {
      const int j = idx / G, t = idx - j * G;
      T2 v;
      v.x = v.y = (T)0;
      if (t < g) {
        const int tr = s_tr[t];
        const T2 a = AIN[(size_t)tr * N + r0 + j];
        const T2 p = PH[(size_t)tr * d.n_e + __ldg(d.st_e + r0 + j)];
        v.x = p.x * a.x - p.y * a.y;
        v.y = p.x * a.y + p.y * a.x;
      }
      bt[idx] = v;
    }
    __syncthreads();
    // warp units: (trajectory set of TB, 32 consecutive rows)
    const int nwr = (nb + 31) >> 5, nsets = (g + TB - 1) / TB, nwu = nwr * nsets;
    for (int uw = warp; uw < nwu; uw += NW) {
      const int set = uw / nwr;
      const int i = (uw - set * nwr) * 32 + lane;
      const int ic = min(i, nb - 1);
      T zr[TB][4], zi[TB][4];
#pragma unroll
      for (int tt = 0; tt < TB; ++tt)
#pragma unroll
        for (int q = 0; q < 4; ++q) zr[tt][q] = zi[tt][q] = (T)0;
      // the row updates' operands into L1 while the products run
      if (i < nb) {
        const int gi = r0 + i;
#pragma unroll
        for (int tt = 0; tt < TB; ++tt) {
          const int t = set * TB + tt;
          if (t < g) {
            const size_t base = (size_t)s_tr[t] * N;
            prefetch_l1(L.Y + base + gi);
            prefetch_l1(ACC + base + gi);
            prefetch_l1(PH + (size_t)s_tr[t] * d.n_e + __ldg(d.st_e + gi));
            const int np_ = __ldg(d.nb_plus + gi), nm = __ldg(d.nb_minus + gi);
            if (np_ >= 0) prefetch_l1(AIN + base + np_);
            if (nm >= 0) prefetch_l1(AIN + base + nm);
          }
        }
      }
      if (!zero) {
        const int Ti = ic * (ic + 1) / 2;
        int Tj = 0;
        const T2* bset = bt + set * TB;
        for (int j = 0; j < nb; ++j) {
          const E e = K4[j <= ic ? Ti + j : Tj + ic];
          Tj += j + 1;
          T k0, k1, k2, k3;
          if constexpr (sizeof(T) == 4) {
            k0 = e.a.x; k1 = e.a.y; k2 = e.a.z; k3 = e.a.w;
          } else {
            k0 = e.a.x; k1 = e.a.y; k2 = e.b.x; k3 = e.b.y;
          }
          const T2* bj = bset + j * G;
#pragma unroll
          for (int tt = 0; tt < TB; ++tt) {
            const T2 v = bj[tt];
            zr[tt][0] += k0 * v.x; zi[tt][0] += k0 * v.y;
            zr[tt][1] += k1 * v.x; zi[tt][1] += k1 * v.y;
            zr[tt][2] += k2 * v.x; zi[tt][2] += k2 * v.y;
            zr[tt][3] += k3 * v.x; zi[tt][3] += k3 * v.y;
          }
        }
      }
      // per (row, trajectory): y, M' bt, u, da, the row's RK4 update, the shares
#pragma unroll
      for (int tt = 0; tt < TB; ++tt) {
        const int t = set * TB + tt;
        double sF = 0.0, sG = 0.0, sP = 0.0;
        if (i < nb && t < g) {
          const int tr = s_tr[t], stg = s_stage[t];
          const T cAB = s_cf[t][0], cB = s_cf[t][1], c1 = s_cf[t][2], c2 = s_cf[t][3];
          const T hinv = s_cf[t][4], d1 = s_cf[t][5], d2 = s_cf[t][6];
          const double dt = s_dt[t], dphidt = s_dphi[t];
          T2 yy, ww;
          yy.x = cAB * zr[tt][0] + cB * zr[tt][1] + c1 * zr[tt][2] + c2 * zr[tt][3];
          yy.y = cAB * zi[tt][0] + cB * zi[tt][1] + c1 * zi[tt][2] + c2 * zi[tt][3];
          ww.x = hinv * zr[tt][1] + d1 * zr[tt][2] + d2 * zr[tt][3];
          ww.y = hinv * zi[tt][1] + d1 * zi[tt][2] + d2 * zi[tt][3];
          const int gi = r0 + i;
          const size_t base = (size_t)tr * N, o = base + gi;
          const T2 b2 = bt[i * G + t];
          sP = (double)(b2.x * yy.x + b2.y * yy.y);
          if (stg == 4) {
            // closing evaluation: the quantum energy and the norm of the final amplitudes,
            // which go out in the reference state order
            const double2 yv = L.Y[o];
            const double w2 = yv.x * yv.x + yv.y * yv.y;
            sF = w2 * __ldg(d.e_val + __ldg(d.st_e + gi));
            sG = w2;
            double* amp = L.amp + base * 2;
            const int ri = __ldg(d.perm + gi);
            amp[ri] = yv.x;
            amp[N + ri] = yv.y;
          } else {
            const T2 p = PH[(size_t)tr * d.n_e + __ldg(d.st_e + gi)];
            sF = (double)(b2.x * ww.x + b2.y * ww.y);
            // u = (J_+ + J_-) a (MQCT_SOURCE_CODES/mqct_eqtns.f:447-464)
            double ur = 0.0, ui = 0.0;
            const int np_ = __ldg(d.nb_plus + gi), nm = __ldg(d.nb_minus + gi);
            if (np_ >= 0) {
              const double cp = __ldg(d.cplus + gi);
              const T2 an = AIN[base + np_];
              ur += cp * (double)an.x;
              ui += cp * (double)an.y;
            }
            if (nm >= 0) {
              const double cm = __ldg(d.cminus + gi);
              const T2 an = AIN[base + nm];
              ur += cm * (double)an.x;
              ui += cm * (double)an.y;
            }
            const T uxr = (T)ur, uxi = (T)ui;
            const T utr = p.x * uxr - p.y * uxi, uti = p.x * uxi + p.y * uxr;
            sG = (double)(utr * yy.y - uti * yy.x);
            // da = -i (e^{iEt} y + (dphi/2) u)
            const double er = (double)p.x, ei = -(double)p.y;
            const double zr_ = er * yy.x - ei * yy.y, zi_ = er * yy.y + ei * yy.x;
            const double cr = zr_ + 0.5 * dphidt * (double)uxr;
            const double ci = zi_ + 0.5 * dphidt * (double)uxi;
            const double dar = ci, dai = -cr;
            const double2 yv = L.Y[o];
            T2 nx, ac;
            if (stg == 0) {
              ac.x = (T)dar;
              ac.y = (T)dai;
              nx.x = (T)(yv.x + 0.5 * dt * dar);
              nx.y = (T)(yv.y + 0.5 * dt * dai);
              ACC[o] = ac;
            } else if (stg < 3) {
              const T2 a0 = ACC[o];
              ac.x = (T)((double)a0.x + 2.0 * dar);
              ac.y = (T)((double)a0.y + 2.0 * dai);
              ACC[o] = ac;
              const double c = stg == 1 ? 0.5 * dt : dt;
              nx.x = (T)(yv.x + c * dar);
              nx.y = (T)(yv.y + c * dai);
            } else {
              const T2 a0 = ACC[o];
              const double h6 = dt / 6.0;
              const double2 yn = make_double2(yv.x + h6 * ((double)a0.x + dar),
                                              yv.y + h6 * ((double)a0.y + dai));
              L.Y[o] = yn;
              nx.x = (T)yn.x;
              nx.y = (T)yn.y;
            }
            AOUT[o] = nx;
          }
        }
        // the warp's rows of this trajectory, fixed tree
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
          sF += __shfl_xor_sync(0xffffffffu, sF, o);
          sG += __shfl_xor_sync(0xffffffffu, sG, o);
          sP += __shfl_xor_sync(0xffffffffu, sP, o);
        }
        if (lane == 0) {
          s_red[uw][tt][0] = sF;
          s_red[uw][tt][1] = sG;
          s_red[uw][tt][2] = sP;
        }
      }
    }
    __syncthreads();
    // the shares of each trajectory: its set's warp units added in row order
    if (tid < g) {
      const int set = tid / TB, tt = tid - set * TB;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int k = 0; k < nwr; ++k) {
        a0 += s_red[set * nwr + k][tt][0];
        a1 += s_red[set * nwr + k][tt][1];
        a2 += s_red[set * nwr + k][tt][2];
      }
      double* pp = L.part + ((size_t)s_tr[tid] * L.n_blocks + b) * 3;
      pp[0] = a0;
      pp[1] = a1;
      pp[2] = a2;
      // the item that completes a trajectory's blocks takes its classical step
      __threadfence();
      s_fin[tid] = atomicAdd(L.tdone + s_tr[tid], 1) == L.n_blocks - 1;
    }
    __syncthreads();
    for (int t = warp; t < g; t += NW) {
      if (s_fin[t]) {
        __threadfence();
        if (lane == 0) L.tdone[s_tr[t]] = 0;
        ls_traj_step<T>(d, L, s_tr[t], lane, false, par ^ 1);
      }
    }
  }
  // the last CTA of the round forms the next round's groups
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(L.done, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (s_last) {
    __threadfence();
    ls_group<G, Cfg::THREADS>(d, L);
  }
}

// ---------------------------------------------------------------- ls_cls
// Classical part of a trajectory between two rounds (lane 0 of its warp) and the set-up
// of its next stage point; init: the trajectory's start instead.
template <class T>
__device__ void ls_traj_step(const PropDev& d, const LsDev& L, int tr, int lane, bool init, int rpar) {
  using T2 = typename V2<T>::t;
  LsTraj& S = L.tr[tr];
  int act = 0;
  if (lane == 0) {
    const mqct_traj_init_t& ti = L.init[tr];
    if (init) {
      const int s_int = d.inv_perm[ti.s_st - 1];
      LsTraj z{};
      z.s_int = s_int;
      z.dt = ti.dt;
      z.counter = 1;
      z.th_c = __longlong_as_double(0x7ff8000000000000ULL);
      const double k_vec = sqrt(d.mass * 2.0 * ti.e_coll);
      const double l_orb = sqrt(ti.l_real * (ti.l_real + 1.0));
      if (l_orb / k_vec > ti.r_start) {  // not propagated (status 2)
        z.status = 2;
        z.C.R = ti.r_start;
        double* cl = L.cls + (size_t)tr * 6;
        cl[0] = z.C.R; cl[1] = 0.0; cl[2] = 0.0; cl[3] = 0.0; cl[4] = 0.0; cl[5] = 0.0;
        double* dg = L.diag + (size_t)tr * 8;
        dg[0] = 0.0; dg[1] = 0.0; dg[2] = 0.0; dg[3] = 0.0; dg[4] = 2.0; dg[5] = 0.0;
        dg[6] = 0.0; dg[7] = 0.0;
        z.active = 0;
      } else {  // MQCT_SOURCE_CODES/propagator.f:2531-2566
        z.C.R = ti.r_start;
        z.C.PR = -sqrt(k_vec * k_vec - l_orb * l_orb / (ti.r_start * ti.r_start));
        z.C.th = acos(0.0);
        z.C.Pth = l_orb * sin(0.0);
        z.C.phi = 0.0;
        z.C.Pphi = l_orb * cos(0.0);
        z.CT = z.C;
        z.stage = 0;
        z.active = 1;
      }
      S = z;
      act = z.active;
    } else {
      const int s = S.stage;
      double F = 0.0, g = 0.0, pot = 0.0;
      const double* pp = L.part + (size_t)tr * L.n_blocks * 3;
      for (int b = 0; b < L.n_blocks; ++b) {
        F += __ldcg(pp + 3 * b);
        g += __ldcg(pp + 3 * b + 1);
        pot += __ldcg(pp + 3 * b + 2);
      }
      act = 1;
      if (s == 4) {  // closing evaluation done: F = quantum energy, g = norm
        const double eerr = fabs(F + kinetic(S.C, d.mass) + pot - S.eki - S.eqi);
        const Cls& c = S.C;
        double* cl = L.cls + (size_t)tr * 6;
        cl[0] = c.R; cl[1] = c.PR; cl[2] = c.th; cl[3] = c.Pth; cl[4] = c.phi; cl[5] = c.Pphi;
        double* dg = L.diag + (size_t)tr * 8;
        dg[0] = S.tcur;
        dg[1] = (double)S.counter;
        dg[2] = fabs(1.0 - g);
        dg[3] = eerr;
        dg[4] = S.status;
        dg[5] = S.period;
        dg[6] = S.vib;
        dg[7] = pot;
        S.active = 0;
        act = 0;
      } else {
        // the classical derivative at the stage point (DERIVS_BK)
        const Cls c = S.CT;
        const double im = d.inv_mass, ir = S.inv_r;
        const double ir3m = ir * ir * ir * im;
        Cls dc;
        dc.R = c.PR * im;
        dc.PR = -F + c.Pth * c.Pth * ir3m + c.Pphi * c.Pphi * ir3m * S.inv_s2;
        dc.th = 0.0;
        dc.Pth = 0.0;
        dc.phi = S.dphidt;
        dc.Pphi = S.sin_t * g;
        const double dt = S.dt, hh = dt * 0.5;
        auto axpy = [](const Cls& a, double h, const Cls& x) {
          return Cls{a.R + h * x.R, a.PR + h * x.PR, a.th + h * x.th,
                     a.Pth + h * x.Pth, a.phi + h * x.phi, a.Pphi + h * x.Pphi};
        };
        if (s == 0) {
          S.K1 = dc;
          if (S.counter == 1) {  // the initial energies (propagator.f:2695-2810)
            S.eqi = d.e_val[d.st_e[S.s_int]] + pot;
            S.eki = kinetic(S.C, d.mass);
          }
          S.CT = axpy(S.C, hh, dc);
          S.stage = 1;
        } else if (s == 1) {
          S.K23 = dc;
          S.CT = axpy(S.C, hh, dc);
          S.stage = 2;
        } else if (s == 2) {
          S.K23 = axpy(S.K23, 1.0, dc);
          S.CT = axpy(S.C, dt, dc);
          S.stage = 3;
        } else {
          const double h6 = dt / 6.0;
          Cls& cc = S.C;
          const Cls &a1 = S.K1, &a23 = S.K23, &a4 = dc;
          cc.R += h6 * (a1.R + a4.R + 2.0 * a23.R);
          cc.PR += h6 * (a1.PR + a4.PR + 2.0 * a23.PR);
          cc.th += h6 * (a1.th + a4.th + 2.0 * a23.th);
          cc.Pth += h6 * (a1.Pth + a4.Pth + 2.0 * a23.Pth);
          cc.phi += h6 * (a1.phi + a4.phi + 2.0 * a23.phi);
          cc.Pphi += h6 * (a1.Pphi + a4.Pphi + 2.0 * a23.Pphi);
          S.tcur += dt;
          // stop rules, MQCT_SOURCE_CODES/propagator.f:4011-4050
          bool run = true;
          const double uR = cc.R;
          if (S.tcur - dt > dt && S.counter > 2) {
            if ((S.tmpR2 - S.tmpR1) < 0.0 && (S.tmpR1 - uR) > 0.0) S.vib += 1;
          }
          S.tmpR2 = S.tmpR1;
          S.tmpR1 = uR;
          S.period = (int)(fabs(cc.phi) / 2.0 / kPi);
          if (ti.numb_orb_prds <= S.period) run = false;
          if (S.vib >= ti.numb_oscl_prds) run = false;
          if (ti.time_lim > 0 && S.tcur >= ti.time_lim) run = false;
          if (uR > ti.r_fin) run = false;
          if (!(uR == uR)) {
            run = false;
            S.status = 3;
          }
          if (run && ti.max_steps > 0 && S.counter >= ti.max_steps) {
            run = false;
            S.status = 1;
          }
          S.CT = cc;
          if (run) {
            S.counter += 1;
            S.stage = 0;
          } else {
            S.stage = 4;
          }
        }
      }
    }
    if (act) {
      // the next stage point: time, scalars, spline interval and factors
      const Cls c = S.CT;
      if (!(c.th == S.th_c)) {
        const double st0 = sin(c.th);
        S.th_c = c.th;
        S.sin_c = st0;
        S.is2_c = 1.0 / (st0 * st0);
      }
      S.sin_t = S.sin_c;
      S.inv_s2 = S.is2_c;
      S.inv_r = 1.0 / c.R;
      S.dphidt = c.Pphi * S.inv_r * S.inv_r * d.inv_mass * S.inv_s2;
      int hint = S.hint;
      const SplineAt sp = spline_at(d.R, d.nR, c.R, &hint);
      S.hint = hint;
      S.sp[0] = sp.aa + sp.bb;
      S.sp[1] = sp.bb;
      S.sp[2] = sp.cc1 * sp.cc5;
      S.sp[3] = sp.cc2 * sp.cc5;
      S.sp[4] = 1.0 / sp.h;
      S.sp[5] = -sp.cc3 * sp.cc6;
      S.sp[6] = sp.cc4 * sp.cc6;
      const int key = sp.zero ? d.nR - 1 : sp.klo;
      S.key = key;
      L.bucket[rpar][(size_t)key * L.n_traj + atomicAdd(L.cnt + key, 1)] = tr;
    }
  }
  act = __shfl_sync(0xffffffffu, act, 0);
  if (!act) return;
  const LsTraj& Sc = L.tr[tr];
  __syncwarp();
  const int s = Sc.stage;
  const double ts = Sc.tcur + ((s == 0 || s == 4) ? 0.0 : (s == 3 ? Sc.dt : 0.5 * Sc.dt));
  T2* ph = reinterpret_cast<T2*>(L.PH) + (size_t)tr * d.n_e;
  for (int e = lane; e < d.n_e; e += 32) {
    double sn, co;
    sincos(d.e_val[e] * ts, &sn, &co);
    T2 v;
    v.x = (T)co;
    v.y = (T)(-sn);
    ph[e] = v;
  }
}

// The last CTA of a round: the next round's groups of up to G trajectories per key (their
// trajectories are in the key's bucket), registration counters reset.
template <int G, int NT>
__device__ void ls_group(const PropDev& d, const LsDev& L) {
  __shared__ int s_sum[NT], s_gsum[NT];
  const int tid = threadIdx.x;
  const int nk = d.nR;
  const int per = (nk + NT - 1) / NT;
  const int k0 = min(nk, tid * per), k1 = min(nk, k0 + per);
  int sc = 0, sg = 0;
  for (int k = k0; k < k1; ++k) {
    const int c = __ldcg(L.cnt + k);
    sc += c;
    sg += (c + G - 1) / G;
  }
  s_sum[tid] = sc;
  s_gsum[tid] = sg;
  __syncthreads();
  // inclusive scans over the threads' chunks of keys (Hillis-Steele)
  for (int o = 1; o < NT; o <<= 1) {
    const int a = tid >= o ? s_sum[tid - o] : 0, ag = tid >= o ? s_gsum[tid - o] : 0;
    __syncthreads();
    s_sum[tid] += a;
    s_gsum[tid] += ag;
    __syncthreads();
  }
  const int total = s_sum[NT - 1], tgroups = s_gsum[NT - 1];
  int grun = tid > 0 ? s_gsum[tid - 1] : 0;
  for (int k = k0; k < k1; ++k) {
    const int c = __ldcg(L.cnt + k);
    const int ng = (c + G - 1) / G;
    L.kcnt[k] = c;
    L.gstart[k] = grun;
    for (int q = 0; q < ng; ++q) L.gkey[grun + q] = k;
    grun += ng;
    L.cnt[k] = 0;
  }
  if (tid == 0) {
    *L.n_groups = tgroups;
    *L.n_items = tgroups * L.n_blocks;
    *L.n_active = total;
    *L.queue = 0;
    *L.done = 0;
  }
}

// The start of a run: every trajectory's initial state and first stage point, registered
// for round 0; the last CTA forms round 0's groups.
template <class T>
__global__ void __launch_bounds__(LS_CLS_THREADS) ls_init_kernel(PropDev d, LsDev L) {
  const int lane = threadIdx.x & 31;
  const int tr = blockIdx.x * (LS_CLS_THREADS / 32) + (threadIdx.x >> 5);
  if (tr < L.n_traj) ls_traj_step<T>(d, L, tr, lane, true, 0);
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(L.done, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (s_last) {
    __threadfence();
    ls_group<LsCfg<T>::G, LS_CLS_THREADS>(d, L);
  }
}

// Amplitudes of the start: the unit vector of the initial state.
template <class T>
__global__ void ls_start_kernel(PropDev d, LsDev L) {
  using T2 = typename V2<T>::t;
  const size_t n = (size_t)L.n_traj * d.N;
  T2* a0 = reinterpret_cast<T2*>(L.AIN[0]);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int tr = (int)(i / d.N), s = (int)(i % d.N);
    const bool one = s == d.inv_perm[L.init[tr].s_st - 1];
    L.Y[i] = make_double2(one ? 1.0 : 0.0, 0.0);
    T2 v;
    v.x = (T)(one ? 1.0 : 0.0);
    v.y = (T)0;
    a0[i] = v;
    // trajectories that are not propagated keep the initial unit vector as result
    double* amp = L.amp + (size_t)tr * 2 * d.N;
    const int ri = d.perm[s];
    amp[ri] = one ? 1.0 : 0.0;
    amp[d.N + ri] = 0.0;
  }
}


// The trajectories still running at a graph boundary (every one at the start of an RK4
// step, or before its closing evaluation): their state into the hand-over records.
__global__ void ls_export_kernel(LsDev L, RsResume* out, int* count) {
  const int tr = blockIdx.x * blockDim.x + threadIdx.x;
  if (tr >= L.n_traj) return;
  const LsTraj& S = L.tr[tr];
  if (!S.active) return;
  RsResume r;
  r.C = S.C;
  r.tcur = S.tcur;
  r.eki = S.eki;
  r.eqi = S.eqi;
  r.tmpR1 = S.tmpR1;
  r.tmpR2 = S.tmpR2;
  r.counter = S.counter;
  r.status = S.status;
  r.vib = S.vib;
  r.period = S.period;
  r.stage = S.stage;
  r.hint = S.hint;
  r.tr = tr;
  out[atomicAdd(count, 1)] = r;
}

// ---------------------------------------------------------------- host
struct LsEngine {
  DevBuf<LsTraj> tr;
  DevBuf<double2> Y;
  DevBuf<double2> acc, ain0, ain1, ph;  // T2 arrays, sized in double2 units
  DevBuf<double> part;
  DevBuf<int> cnt, kcnt, gstart, gkey, bucket, tdone, ctr, blk_order;  // ctr: n_items, queue, done,
                                                                 // n_active, n_groups
  int cap_traj = -1, cap_arith = -1;
  int* h_active = nullptr;  // pinned, two slots
  cudaEvent_t ev_copy[2] = {nullptr, nullptr};
  cudaGraphExec_t graph = nullptr;
  LsDev graph_dev{};
  PropDev graph_pd{};
  int graph_arith = -1;
  int64_t rounds = 0;  // rounds of the last run
  ~LsEngine() {
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& e : ev_copy)
      if (e) cudaEventDestroy(e);
    if (h_active) cudaFreeHost(h_active);
  }
};

constexpr int kLsRoundsPerGraph = 64;  // even: every graph launch starts at parity 0

LsEngine* ls_create() { return new LsEngine(); }
void ls_destroy(LsEngine* e) { delete e; }
int64_t ls_rounds(const LsEngine* e) { return e ? e->rounds : 0; }

bool ls_eligible(const std::vector<int>& blk_n) {
  for (int n : blk_n)
    if (n > LS_MAX_ROWS) return false;
  return true;
}

template <class T>
static int ls_run_t(LsEngine* e, const PropDev& d, const std::vector<int>& blk_n, int n_sm,
                    cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                    const mqct_traj_init_t* d_init, const mqct_traj_init_t* h_init, int n_traj,
                    double* amp, double* cls, double* diag, int hand_below, RsResume* hand_out,
                    int* hand_n, const double2** hand_amp) {
  using T2 = typename V2<T>::t;
  using Cfg = LsCfg<T>;
  const int N = d.N, nb = (int)blk_n.size(), arith = sizeof(T) == 4 ? 1 : 2;
  int nbmax = 0;
  for (int n : blk_n) nbmax = std::max(nbmax, n);
  MQCT_ARG_CHECK(nbmax <= LS_MAX_ROWS, "lockstep engine: m-block of %d states above %d", nbmax,
                 LS_MAX_ROWS);
  const size_t t2n = (size_t)n_traj * N * sizeof(T2) / sizeof(double2) + 1;
  const int nk = d.nR;
  const size_t max_groups = (size_t)std::min(nk, n_traj) + n_traj / Cfg::G + 1;
  if (e->cap_traj < n_traj || e->cap_arith != arith) {
    if (e->graph) {
      cudaGraphExecDestroy(e->graph);
      e->graph = nullptr;
    }
    MQCT_CUDA_TRY(e->tr.alloc(n_traj));
    MQCT_CUDA_TRY(e->Y.alloc((size_t)n_traj * N));
    MQCT_CUDA_TRY(e->acc.alloc(t2n));
    MQCT_CUDA_TRY(e->ain0.alloc(t2n));
    MQCT_CUDA_TRY(e->ain1.alloc(t2n));
    MQCT_CUDA_TRY(e->ph.alloc((size_t)n_traj * d.n_e * sizeof(T2) / sizeof(double2) + 1));
    MQCT_CUDA_TRY(e->part.alloc((size_t)n_traj * nb * 3));
    MQCT_CUDA_TRY(e->gkey.alloc(max_groups));
    MQCT_CUDA_TRY(e->bucket.alloc((size_t)2 * nk * n_traj));
    MQCT_CUDA_TRY(e->tdone.alloc(n_traj));
    e->cap_traj = n_traj;
    e->cap_arith = arith;
  }
  if (!e->cnt.p || (int)e->cnt.n != nk) {
    MQCT_CUDA_TRY(e->cnt.alloc(nk));
    MQCT_CUDA_TRY(e->kcnt.alloc(nk));
    MQCT_CUDA_TRY(e->gstart.alloc(nk));
    if (e->bucket.n != (size_t)2 * nk * e->cap_traj)
      MQCT_CUDA_TRY(e->bucket.alloc((size_t)2 * nk * e->cap_traj));
  }
  if (!e->ctr.p) MQCT_CUDA_TRY(e->ctr.alloc(6));  // [5]: trajectories handed over
  {
    // blocks by size, largest first: the work queue hands out the longest items first
    std::vector<int> order(nb);
    for (int b = 0; b < nb; ++b) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return blk_n[a] > blk_n[b]; });
    MQCT_CUDA_TRY(e->blk_order.upload(order, st));
  }
  if (!e->h_active) {
    MQCT_CUDA_TRY(cudaHostAlloc((void**)&e->h_active, 2 * sizeof(int), cudaHostAllocDefault));
    MQCT_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_copy[0], cudaEventDisableTiming));
    MQCT_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_copy[1], cudaEventDisableTiming));
  }
  LsDev L{};
  L.tr = e->tr.p;
  L.init = d_init;
  L.n_traj = n_traj;
  L.n_blocks = nb;
  L.tri_cap = nbmax * (nbmax + 1) / 2;
  L.Y = e->Y.p;
  L.ACC = e->acc.p;
  L.AIN[0] = e->ain0.p;
  L.AIN[1] = e->ain1.p;
  L.PH = e->ph.p;
  L.part = e->part.p;
  L.cnt = e->cnt.p;
  L.kcnt = e->kcnt.p;
  L.gstart = e->gstart.p;
  L.gkey = e->gkey.p;
  L.bucket[0] = e->bucket.p;
  L.bucket[1] = e->bucket.p + (size_t)nk * n_traj;
  L.tdone = e->tdone.p;
  L.n_groups = e->ctr.p + 4;
  L.n_items = e->ctr.p;
  L.queue = e->ctr.p + 1;
  L.done = e->ctr.p + 2;
  L.n_active = e->ctr.p + 3;
  L.blk_order = e->blk_order.p;
  L.amp = amp;
  L.cls = cls;
  L.diag = diag;
  // the bound on the rounds: every trajectory stops by its step cap or time limit
  int64_t max_rounds = 0;
  for (int t = 0; t < n_traj; ++t) {
    const mqct_traj_init_t& a = h_init[t];
    int64_t steps = a.max_steps > 0 ? a.max_steps : INT64_MAX / 8;
    if (a.time_lim > 0) steps = std::min<int64_t>(steps, (int64_t)std::ceil(a.time_lim / a.dt) + 2);
    max_rounds = std::max(max_rounds, 4 * steps + 2);
  }
  MQCT_ARG_CHECK(max_rounds < ((int64_t)1 << 40), "trajectories without a step bound");
  const size_t smem = ((sizeof(typename Cfg::E) * (size_t)L.tri_cap + 15) & ~size_t(15)) +
                      sizeof(T2) * (size_t)Cfg::G * nbmax;
  MQCT_CUDA_TRY(cudaFuncSetAttribute(ls_rhs_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  int per_sm = 0;
  MQCT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ls_rhs_kernel<T>,
                                                              Cfg::THREADS, smem));
  MQCT_ARG_CHECK(per_sm >= 1, "lockstep engine: %zu B of shared memory per CTA do not fit", smem);
  const int grid_rhs = n_sm * per_sm;
  const int grid_cls = (n_traj + LS_CLS_THREADS / 32 - 1) / (LS_CLS_THREADS / 32);
  MQCT_CUDA_TRY(cudaMemsetAsync(e->cnt.p, 0, sizeof(int) * nk, st));
  MQCT_CUDA_TRY(cudaMemsetAsync(e->tdone.p, 0, sizeof(int) * n_traj, st));
  MQCT_CUDA_TRY(cudaMemsetAsync(e->ctr.p, 0, sizeof(int) * 5, st));
  // the graph of kLsRoundsPerGraph rounds (rebuilt when the buffers or the type change)
  const bool same = e->graph && e->graph_arith == arith &&
                    std::memcmp(&e->graph_dev, &L, sizeof(LsDev)) == 0 &&
                    std::memcmp(&e->graph_pd, &d, sizeof(PropDev)) == 0;
  if (!same) {
    if (e->graph) {
      cudaGraphExecDestroy(e->graph);
      e->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    MQCT_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < kLsRoundsPerGraph; ++r) {
      ls_rhs_kernel<T><<<grid_rhs, Cfg::THREADS, smem, st>>>(d, L, r & 1);
    }
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      MQCT_CUDA_TRY(ce);
    }
    ce = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    MQCT_CUDA_TRY(ce);
    e->graph_dev = L;
    e->graph_pd = d;
    e->graph_arith = arith;
  }
  MQCT_CUDA_TRY(cudaEventRecord(ev0, st));
  {
    const size_t n = (size_t)n_traj * N;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)n_sm * 8);
    ls_start_kernel<T><<<blocks, 256, 0, st>>>(d, L);
    MQCT_CUDA_TRY(cudaGetLastError());
  }
  ls_init_kernel<T><<<grid_cls, LS_CLS_THREADS, 0, st>>>(d, L);
  MQCT_CUDA_TRY(cudaGetLastError());
  // graph launches until no trajectory runs; the count of one launch is read while the
  // next one runs (a launch after the last trajectory finished finds no work items)
  int64_t rounds = 0;
  int k = 0;
  MQCT_CUDA_TRY(cudaGraphLaunch(e->graph, st));
  rounds += kLsRoundsPerGraph;
  MQCT_CUDA_TRY(cudaMemcpyAsync(e->h_active + k, L.n_active, sizeof(int), cudaMemcpyDeviceToHost, st));
  MQCT_CUDA_TRY(cudaEventRecord(e->ev_copy[k], st));
  MQCT_CUDA_TRY(cudaEventRecord(ev1, st));
  if (hand_n) *hand_n = 0;
  for (;;) {
    MQCT_CUDA_TRY(cudaGraphLaunch(e->graph, st));
    MQCT_CUDA_TRY(cudaMemcpyAsync(e->h_active + (k ^ 1), L.n_active, sizeof(int),
                                  cudaMemcpyDeviceToHost, st));
    MQCT_CUDA_TRY(cudaEventRecord(e->ev_copy[k ^ 1], st));
    MQCT_CUDA_TRY(cudaEventSynchronize(e->ev_copy[k]));
    if (e->h_active[k] == 0) break;
    if (hand_below > 0 && e->h_active[k] <= hand_below) {
      // few trajectories left: after the graph in flight, the running ones (each at a step
      // start or before its closing evaluation: the rounds so far are a multiple of 4) go
      // to the caller
      rounds += kLsRoundsPerGraph;
      MQCT_CUDA_TRY(cudaMemsetAsync(e->ctr.p + 5, 0, sizeof(int), st));
      ls_export_kernel<<<(n_traj + 255) / 256, 256, 0, st>>>(L, hand_out, e->ctr.p + 5);
      MQCT_CUDA_TRY(cudaGetLastError());
      int n = 0;
      MQCT_CUDA_TRY(cudaMemcpyAsync(&n, e->ctr.p + 5, sizeof(int), cudaMemcpyDeviceToHost, st));
      MQCT_CUDA_TRY(cudaStreamSynchronize(st));
      *hand_n = n;
      *hand_amp = e->Y.p;
      break;
    }
    rounds += kLsRoundsPerGraph;
    MQCT_CUDA_TRY(cudaEventRecord(ev1, st));
    k ^= 1;
    if (rounds > max_rounds + 2 * kLsRoundsPerGraph) {
      MQCT_CUDA_TRY(cudaStreamSynchronize(st));
      set_error("lockstep engine: trajectories still running after %lld rounds",
                (long long)rounds);
      return MQCT_E_DEVICE;
    }
  }
  e->rounds = rounds;
  return MQCT_OK;
}

int ls_run(LsEngine* e, const PropDev& d, bool fp32, const std::vector<int>& blk_n, int n_sm,
           cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1, const mqct_traj_init_t* d_init,
           const mqct_traj_init_t* h_init, int n_traj, double* amp, double* cls, double* diag,
           int hand_below, RsResume* hand_out, int* hand_n, const double2** hand_amp) {
  MQCT_ARG_CHECK(hand_below <= 0 || (hand_out && hand_n && hand_amp), "hand-over buffers missing");
  return fp32 ? ls_run_t<float>(e, d, blk_n, n_sm, st, ev0, ev1, d_init, h_init, n_traj, amp,
                                cls, diag, hand_below, hand_out, hand_n, hand_amp)
              : ls_run_t<double>(e, d, blk_n, n_sm, st, ev0, ev1, d_init, h_init, n_traj, amp,
                                 cls, diag, hand_below, hand_out, hand_n, hand_amp);
}

}  // namespace mqct
