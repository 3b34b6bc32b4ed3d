// resident.cu -- cluster-resident engine of the trajectory propagation (H2): standard
// MQCT, fixed-step RK4 (DOTRAJECT, MQCT_SOURCE_CODES/propagator.f:2283-4645, with
// DERIVS_BK, MQCT_SOURCE_CODES/mqct_eqtns.f:112-499, and RK4, MQCT_SOURCE_CODES/
// suppl_routines.f:1076-1113), FP32 arithmetic with FP64 amplitudes and classical
// variables.
//
// The per-trajectory kernel (propagate.cu) reads the two knot rows of its spline interval
// from L2 for every right-hand side (640 KB per evaluation for the 969-state table), and
// the aggregate L2 read rate bounds it.  A trajectory stays in one interval for many
// right-hand sides (about a dozen RK4 steps at dt = 5 a.u.), so the rows it reads are the
// same ones again and again.  This engine keeps them on chip: one trajectory is
// propagated by a thread-block cluster of CL CTAs (one per SM), and the m-blocks of the
// state space are split between the CTAs so that each holds the two knot rows of ITS
// blocks in shared memory (the cluster together holds the whole interval).  The rows are
// loaded again only when the stage point leaves the interval (one of the two rows is
// kept when the neighbour interval is entered).
//
// Per right-hand side every CTA of the cluster
//   * forms the stage point's scalars and spline factors (thread 0; the same values in
//     every CTA, from the same classical state),
//   * bt = D^* a and u = (J_+ + J_-) a for its rows, the neighbour amplitudes of u read
//     from the owning CTA's shared memory when another CTA holds them (distributed
//     shared memory),
//   * interpolates its blocks' matrix elements into a packed triangle (M) and adds its
//     part of the force Re(bt^+ M' bt), then y = M bt for its rows,
//   * forms da = -i e^{iEt} y - i (dphi/2) u and the RK4 update of its rows, and its parts
//     of F, g = Im((D^* u)^+ y) and pot = Re(bt^+ y),
//   * writes its three parts into every CTA of the cluster and waits at the cluster
//     barrier (one per right-hand side),
// after which each CTA adds the CL parts in rank order and takes the classical RK4 stage
// itself: every CTA holds the same classical state, bit for bit, so the stop decisions
// agree without another exchange.  CTA rank 0 takes the next trajectory from a device
// queue and hands its index to the others.
//
// The arithmetic of a right-hand side is that of the per-trajectory kernel in FP32 (the
// slots interpolated one by one, the same products); sums run over other partitions, so
// results agree with it to FP32 rounding.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "propagate.cuh"

namespace cg = cooperative_groups;

namespace mqct {

constexpr int RS_THREADS = 512;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_MAX_CL = 8;
constexpr int RS_MAX_BLK = 64;   // blocks per CTA
constexpr int RS_MAX_STATES = 255;  // states of one m-block (8-bit local row indices)

// Classical state of the cluster's trajectory (identical in every CTA).
struct RsCls {
  Cls C, CT, K1, K23;                 // state, stage point, first-stage and middle-stage sums
  double tcur, dt, eki, eqi, tmpR1, tmpR2;
  double th_c, sin_c, is2_c;          // theta of the cached sine and 1/sin^2
  double dphidt, sin_t, inv_r, inv_s2;
  float cf[7];                        // M: aa, bb, c1, c2;  M': 1/h, d1, d2
  int counter, status, vib, period;
  int stage;                          // 0..3 RK4 stages, 4 closing evaluation, 5 done
  int key;                            // spline interval of the stage point; nR - 1 above
  int hint;
  int s_int;
  int lo_buf;                         // knot buffer holding row key (the other: key + 1)
  int load[2];                        // knot row to load into buffer 0 / 1, or -1
  int tag[2];                         // knot row held by buffer 0 / 1, or -1
};

// One row (state) of a CTA: what its right-hand-side terms need, fixed for the tables.
struct RsRow {
  int gi;        // internal state index
  int ec;        // energy class
  int ri;        // reference state index (output order)
  int nbp, nbm;  // J_+ / J_- neighbour as rank << 16 | local row, or -1
  int ent_i;     // block entry of the CTA << 8 | row inside the block
  int to_p, to_m;  // the row whose J_+ / J_- neighbour this row is (rank << 16 | local row),
                   // or -1: where this row's stage inputs are pushed
  double cp, cm; // the coefficients of nbp and nbm
};

struct RsDev {
  const mqct_traj_init_t* init;
  int n_traj, CL, ns_cap, nr_cap, n_e;
  const int* rk_b0;       // CL + 1: first entry of each rank in rk_blk
  const int* rk_blk;      // blocks of the ranks
  const int* rk_ls0;      // local slot base of each entry (even)
  const int* rk_lr0;      // local row base of each entry
  const int* rk_rows;     // per rank: its local row count
  const int* rk_slots;    // per rank: its local slots (padded to even per block)
  const RsRow* rows;      // per rank x nr_cap
  const uint16_t* loc;    // per rank x ns_cap: local row | local column << 8 of each slot
  const double* ih;       // per interval: 1 / (R_{k+1} - R_k)
  const RsResume* resume;    // trajectories handed over by the lockstep engine, or null:
  const double2* resume_amp; // then queue entry i is resume[i] with these amplitudes
  int* queue;
  double* amp;
  double* cls;
  double* diag;
};

// Dynamic shared memory of one CTA (offsets in bytes, 16-byte aligned).
struct RsSmem {
  size_t kn0, kn1, mp, loc, y64, acc, ain0, ain1, halo0, halo1, bt, u, ph0, ph1, rows, rg, ih,
      ev, total;
};
__host__ __device__ inline RsSmem rs_layout(int ns_cap, int nr_cap, int n_e, int nR) {
  RsSmem s{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o += (bytes + 15) & ~size_t(15);
    return at;
  };
  s.kn0 = take((size_t)ns_cap * 8);
  s.kn1 = take((size_t)ns_cap * 8);
  s.mp = take((size_t)ns_cap * 4);
  s.loc = take((size_t)ns_cap * 2);
  s.y64 = take((size_t)nr_cap * 16);
  s.acc = take((size_t)nr_cap * 8);
  s.ain0 = take((size_t)nr_cap * 8);
  s.ain1 = take((size_t)nr_cap * 8);
  s.halo0 = take((size_t)nr_cap * 16);
  s.halo1 = take((size_t)nr_cap * 16);
  s.bt = take((size_t)nr_cap * 8);
  s.u = take((size_t)nr_cap * 8);
  s.ph0 = take((size_t)n_e * 8);
  s.ph1 = take((size_t)n_e * 8);
  s.rows = take((size_t)nr_cap * sizeof(RsRow));
  s.rg = take((size_t)nR * 8);
  s.ih = take((size_t)nR * 8);
  s.ev = take((size_t)n_e * 8);
  s.total = o;
  return s;
}

// Warp sums of three doubles (fixed tree) into red[3 w + q]; the block's barrier follows.
__device__ inline void rs_warp_parts(double a, double b, double c, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if (lane == 0) {
    red[3 * w] = a;
    red[3 * w + 1] = b;
    red[3 * w + 2] = c;
  }
  __syncthreads();
}

// Start of a trajectory (thread 0): MQCT_SOURCE_CODES/propagator.f:2531-2566.  Returns
// false for a trajectory that is not propagated (l / k above R_start, status 2), whose
// classical and diagnostic outputs rank 0 writes here.
__device__ inline bool rs_start(RsCls& S, const PropDev& d, const RsDev& D,
                                const mqct_traj_init_t& ti, int tr, bool rank0) {
  const int t0 = S.tag[0], t1 = S.tag[1];
  RsCls z{};
  z.tag[0] = t0;
  z.tag[1] = t1;
  z.s_int = d.inv_perm[ti.s_st - 1];
  z.dt = ti.dt;
  z.counter = 1;
  z.th_c = __longlong_as_double(0x7ff8000000000000ULL);
  const double k_vec = sqrt(d.mass * 2.0 * ti.e_coll);
  const double l_orb = sqrt(ti.l_real * (ti.l_real + 1.0));
  if (l_orb / k_vec > ti.r_start) {
    z.status = 2;
    z.stage = 5;
    if (rank0) {
      double* cl = D.cls + (size_t)tr * 6;
      cl[0] = ti.r_start; cl[1] = 0.0; cl[2] = 0.0; cl[3] = 0.0; cl[4] = 0.0; cl[5] = 0.0;
      double* dg = D.diag + (size_t)tr * 8;
      dg[0] = 0.0; dg[1] = 0.0; dg[2] = 0.0; dg[3] = 0.0; dg[4] = 2.0; dg[5] = 0.0;
      dg[6] = 0.0; dg[7] = 0.0;
    }
    S = z;
    return false;
  }
  z.C.R = ti.r_start;
  z.C.PR = -sqrt(k_vec * k_vec - l_orb * l_orb / (ti.r_start * ti.r_start));
  z.C.th = acos(0.0);
  z.C.Pth = l_orb * sin(0.0);
  z.C.phi = 0.0;
  z.C.Pphi = l_orb * cos(0.0);
  z.CT = z.C;
  z.stage = 0;
  S = z;
  return true;
}

// Spline interval and factors at x (splint_bk, MQCT_SOURCE_CODES/mqct_eqtns.f:555-611,
// as spline_at), from the grid Rg and the reciprocal interval widths ih in shared memory.
__device__ inline SplineAt rs_spline(const double* Rg, const double* ih, int nR, double x,
                                     int* hint) {
  SplineAt s;
  s.zero = x > Rg[nR - 1];
  int klo = 1, khi = nR;
  const int hk = *hint;
  if (hk >= 1 && hk < nR && Rg[hk - 1] <= x && x < Rg[hk]) {
    klo = hk;
    khi = hk + 1;
  }
  while (khi - klo > 1) {
    int k = (khi + klo) >> 1;
    if (Rg[k - 1] > x) khi = k;
    else klo = k;
  }
  *hint = klo;
  s.klo = klo - 1;
  const double h = Rg[khi - 1] - Rg[klo - 1];
  const double inv_h = ih[klo - 1];
  s.h = h;
  s.aa = (Rg[khi - 1] - x) * inv_h;
  s.bb = (x - Rg[klo - 1]) * inv_h;
  s.cc1 = s.aa * s.aa * s.aa - s.aa;
  s.cc2 = s.bb * s.bb * s.bb - s.bb;
  s.cc3 = 3 * s.aa * s.aa - 1.0;
  s.cc4 = 3 * s.bb * s.bb - 1.0;
  s.cc5 = (h * h) / 6.0;
  s.cc6 = s.cc5 * inv_h;
  return s;
}

// A trajectory handed over by the lockstep engine (thread 0): its state at the start of an
// RK4 step or before its closing evaluation.
__device__ inline void rs_resume(RsCls& S, const PropDev& d, const RsResume& r,
                                 const mqct_traj_init_t& ti) {
  const int t0 = S.tag[0], t1 = S.tag[1];
  RsCls z{};
  z.tag[0] = t0;
  z.tag[1] = t1;
  z.s_int = d.inv_perm[ti.s_st - 1];
  z.dt = ti.dt;
  z.C = r.C;
  z.CT = r.C;
  z.tcur = r.tcur;
  z.eki = r.eki;
  z.eqi = r.eqi;
  z.tmpR1 = r.tmpR1;
  z.tmpR2 = r.tmpR2;
  z.counter = r.counter;
  z.status = r.status;
  z.vib = r.vib;
  z.period = r.period;
  z.stage = r.stage;
  z.hint = r.hint;
  z.th_c = __longlong_as_double(0x7ff8000000000000ULL);
  S = z;
}

// The stage point's scalars, spline interval and factors, and the knot rows to load
// (thread 0).
__device__ inline void rs_point(RsCls& S, const PropDev& d, const double* Rg, const double* ih) {
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
  const SplineAt sp = rs_spline(Rg, ih, d.nR, c.R, &hint);
  S.hint = hint;
  S.cf[0] = (float)sp.aa;
  S.cf[1] = (float)sp.bb;
  S.cf[2] = (float)(sp.cc1 * sp.cc5);
  S.cf[3] = (float)(sp.cc2 * sp.cc5);
  S.cf[4] = (float)ih[sp.klo];
  S.cf[5] = (float)(-sp.cc3 * sp.cc6);
  S.cf[6] = (float)(sp.cc4 * sp.cc6);
  const int key = sp.zero ? d.nR - 1 : sp.klo;
  S.key = key;
  S.load[0] = S.load[1] = -1;
  if (sp.zero) return;
  const int a = key, b = key + 1;
  const int t0 = S.tag[0], t1 = S.tag[1];
  if (t0 == a) {
    S.lo_buf = 0;
    if (t1 != b) S.load[1] = b;
  } else if (t1 == a) {
    S.lo_buf = 1;
    if (t0 != b) S.load[0] = b;
  } else if (t0 == b) {
    S.lo_buf = 1;
    S.load[1] = a;
  } else if (t1 == b) {
    S.lo_buf = 0;
    S.load[0] = a;
  } else {
    S.lo_buf = 0;
    S.load[0] = a;
    S.load[1] = b;
  }
  if (S.load[0] >= 0) S.tag[0] = S.load[0];
  if (S.load[1] >= 0) S.tag[1] = S.load[1];
}

// After the cluster's sums F, g, pot of a right-hand side (thread 0 of every CTA, the
// same arithmetic in each): the classical RK4 stage, at the end of a step the stop rules
// (MQCT_SOURCE_CODES/propagator.f:4011-4050), after the closing evaluation the outputs
// (rank 0; F = quantum energy and g = norm there, the energy bookkeeping of
// MQCT_SOURCE_CODES/propagator.f:4182-4343).
__device__ inline void rs_classical(RsCls& S, const PropDev& d, const RsDev& D,
                                    const mqct_traj_init_t& ti, const double* e_val, int s_ec,
                                    int tr, bool rank0, double F, double g, double pot) {
  const int s = S.stage;
  if (s == 4) {
    if (rank0) {
      const double eerr = fabs(F + kinetic(S.C, d.mass) + pot - S.eki - S.eqi);
      const Cls& c = S.C;
      double* cl = D.cls + (size_t)tr * 6;
      cl[0] = c.R; cl[1] = c.PR; cl[2] = c.th; cl[3] = c.Pth; cl[4] = c.phi; cl[5] = c.Pphi;
      double* dg = D.diag + (size_t)tr * 8;
      dg[0] = S.tcur;
      dg[1] = (double)S.counter;
      dg[2] = fabs(1.0 - g);
      dg[3] = eerr;
      dg[4] = S.status;
      dg[5] = S.period;
      dg[6] = S.vib;
      dg[7] = pot;
    }
    S.stage = 5;
    return;
  }
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
      S.eqi = e_val[s_ec] + pot;
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

// ---------------------------------------------------------------- kernel
__device__ __forceinline__ void rs_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void rs_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Phases e^{-iEt} = (cos E t, -sin E t) of the energy classes at time t.
__device__ inline void rs_phases(float2* ph, const double* ev, int n_e, double t) {
  for (int e = threadIdx.x; e < n_e; e += RS_THREADS) {
    double sn, co;
    sincos(ev[e] * t, &sn, &co);
    ph[e] = make_float2((float)co, (float)(-sn));
  }
}

// One cluster of CL CTAs per trajectory at a time; persistent over the device queue.
__global__ void __launch_bounds__(RS_THREADS, 1) rs_kernel(PropDev d, RsDev D) {
  cg::cluster_group clu = cg::this_cluster();
  const int rank = (int)clu.block_rank();
  const int tid = threadIdx.x;
  extern __shared__ __align__(16) unsigned char rs_sm[];
  const RsSmem L = rs_layout(D.ns_cap, D.nr_cap, D.n_e, d.nR);
  float2* KN[2] = {reinterpret_cast<float2*>(rs_sm + L.kn0), reinterpret_cast<float2*>(rs_sm + L.kn1)};
  float* Mp = reinterpret_cast<float*>(rs_sm + L.mp);
  uint16_t* loc = reinterpret_cast<uint16_t*>(rs_sm + L.loc);
  double2* Y = reinterpret_cast<double2*>(rs_sm + L.y64);
  float2* ACC = reinterpret_cast<float2*>(rs_sm + L.acc);
  float2* AIN[2] = {reinterpret_cast<float2*>(rs_sm + L.ain0), reinterpret_cast<float2*>(rs_sm + L.ain1)};
  float4* HALO[2] = {reinterpret_cast<float4*>(rs_sm + L.halo0), reinterpret_cast<float4*>(rs_sm + L.halo1)};
  float2* bt = reinterpret_cast<float2*>(rs_sm + L.bt);
  float2* uv = reinterpret_cast<float2*>(rs_sm + L.u);
  float2* PH[2] = {reinterpret_cast<float2*>(rs_sm + L.ph0), reinterpret_cast<float2*>(rs_sm + L.ph1)};
  RsRow* row = reinterpret_cast<RsRow*>(rs_sm + L.rows);
  double* Rg = reinterpret_cast<double*>(rs_sm + L.rg);
  double* ih = reinterpret_cast<double*>(rs_sm + L.ih);
  double* ev = reinterpret_cast<double*>(rs_sm + L.ev);
  __shared__ RsCls S;
  __shared__ mqct_traj_init_t s_ti;
  __shared__ double red[3 * RS_WARPS + 3];
  __shared__ double part[2][RS_MAX_CL][3];
  __shared__ int s_tr, s_ec;
  __shared__ int s_n[RS_MAX_BLK], s_ls0[RS_MAX_BLK], s_lr0[RS_MAX_BLK], s_q0[RS_MAX_BLK];
  // a row's new stage input into the Coriolis neighbour slots (J_+ in .xy, J_- in .zw of
  // halo) of the rows that need it, in whichever CTA holds them: remote stores before the
  // cluster barrier, so that the next evaluation reads its neighbours locally
  auto push = [&](const RsRow& w, float2 v, float4* halo) {
    if (w.to_p >= 0) {
      const int r = w.to_p >> 16, l = w.to_p & 0xffff;
      float4* h = r == rank ? halo : clu.map_shared_rank(halo, r);
      reinterpret_cast<float2*>(h + l)[0] = v;
    }
    if (w.to_m >= 0) {
      const int r = w.to_m >> 16, l = w.to_m & 0xffff;
      float4* h = r == rank ? halo : clu.map_shared_rank(halo, r);
      reinterpret_cast<float2*>(h + l)[1] = v;
    }
  };
  const int e0 = D.rk_b0[rank], nbk = D.rk_b0[rank + 1] - e0;
  const int nr = D.rk_rows[rank], nsl_r = D.rk_slots[rank];
  for (int e = tid; e < nbk; e += RS_THREADS) {
    const int b = D.rk_blk[e0 + e];
    s_n[e] = d.blk_n[b];
    s_ls0[e] = D.rk_ls0[e0 + e];
    s_lr0[e] = D.rk_lr0[e0 + e];
    s_q0[e] = (int)d.blk_slot0[b];
  }
  // slots of the CTA's blocks (the padding slots keep zero knots: no force, unread M)
  for (int k = tid; k < D.ns_cap; k += RS_THREADS) {
    loc[k] = D.loc[(size_t)rank * D.ns_cap + k];
    KN[0][k] = make_float2(0.f, 0.f);
    KN[1][k] = make_float2(0.f, 0.f);
  }
  for (int lr = tid; lr < nr; lr += RS_THREADS) row[lr] = D.rows[(size_t)rank * D.nr_cap + lr];
  for (int k = tid; k < d.nR; k += RS_THREADS) {
    Rg[k] = d.R[k];
    ih[k] = D.ih[k];
  }
  for (int e = tid; e < D.n_e; e += RS_THREADS) ev[e] = d.e_val[e];
  if (tid == 0) {
    S.tag[0] = -1;
    S.tag[1] = -1;
  }
  int rc = 0;  // right-hand sides evaluated by the cluster (parity of the exchange buffers)
  clu.sync();
  for (;;) {
    if (rank == 0 && tid == 0) {
      const int t = atomicAdd(D.queue, 1);
      for (int r = 0; r < D.CL; ++r) *clu.map_shared_rank(&s_tr, r) = t;
    }
    clu.sync();
    const int qi = s_tr;
    if (qi >= D.n_traj) break;
    const int tr = D.resume ? D.resume[qi].tr : qi;
    if (tid == 0) {
      s_ti = D.init[tr];
      if (D.resume) {
        rs_resume(S, d, D.resume[qi], s_ti);
        rs_point(S, d, Rg, ih);
      } else if (rs_start(S, d, D, s_ti, tr, rank == 0)) {
        rs_point(S, d, Rg, ih);
      }
      s_ec = d.st_e[S.s_int];
    }
    __syncthreads();
    const bool go = S.stage != 5;
    {
      float2* a0 = AIN[rc & 1];
      double* amp = D.amp + (size_t)tr * 2 * d.N;
      for (int lr = tid; lr < nr; lr += RS_THREADS) {
        const RsRow w = row[lr];
        const double one = w.gi == S.s_int ? 1.0 : 0.0;
        // a handed-over trajectory's amplitudes, its stage input their FP32 rounding (as
        // the lockstep engine forms it at the end of a step); else the initial unit vector
        const double2 y0 = D.resume ? D.resume_amp[(size_t)tr * d.N + w.gi] : make_double2(one, 0.0);
        Y[lr] = y0;
        a0[lr] = make_float2((float)y0.x, (float)y0.y);
        push(w, a0[lr], HALO[rc & 1]);
        if (!go) {  // not propagated: the initial unit vector is the result
          amp[w.ri] = one;
          amp[d.N + w.ri] = 0.0;
        }
      }
      if (go) rs_phases(PH[rc & 1], ev, D.n_e, 0.0);
    }
    clu.sync();  // the peers read these amplitudes from the first right-hand side on
    if (!go) continue;
    while (S.stage != 5) {
      const int s = S.stage, par = rc & 1;
      const bool zero = S.key == d.nR - 1;  // above the grid: the matrix is zero
      // knot rows that the stage point's interval needs and the buffers do not hold
#pragma unroll
      for (int bsel = 0; bsel < 2; ++bsel) {
        const int krow = S.load[bsel];
        if (krow < 0) continue;
        const float2* src = reinterpret_cast<const float2*>(d.knots) + (int64_t)krow * d.S;
        float2* dst = KN[bsel];
        for (int e = 0; e < nbk; ++e) {
          const int n = s_n[e], nsl = n * (n + 1) / 2;
          const float2* se = src + s_q0[e];
          float2* de = dst + s_ls0[e];
          for (int q = tid; q < nsl; q += RS_THREADS) de[q] = __ldg(se + q);
        }
      }
      // bt = D^* a and u = (J_+ + J_-) a of this CTA's rows (MQCT_SOURCE_CODES/
      // mqct_eqtns.f:447-464); the neighbours' stage inputs were pushed into halo
      const float2* ph = PH[par];
      const float2* ain = AIN[par];
      const float4* halo = HALO[par];
      for (int lr = tid; lr < nr; lr += RS_THREADS) {
        const RsRow w = row[lr];
        const float2 a = ain[lr];
        const float2 p = ph[w.ec];
        bt[lr] = make_float2(p.x * a.x - p.y * a.y, p.x * a.y + p.y * a.x);
        const float4 hv = halo[lr];
        double ur = 0.0, ui = 0.0;
        if (w.nbp >= 0) {
          ur += w.cp * (double)hv.x;
          ui += w.cp * (double)hv.y;
        }
        if (w.nbm >= 0) {
          ur += w.cm * (double)hv.z;
          ui += w.cm * (double)hv.w;
        }
        uv[lr] = make_float2((float)ur, (float)ui);
      }
      __syncthreads();
      float force = 0.f;
      if (!zero) {
        // every slot of the CTA: M = aa lo + bb hi + c1 lo'' + c2 hi'' into the packed
        // triangles, M' = (hi - lo)/h + d1 lo'' + d2 hi'' into the force (two slots per
        // thread and step, 16-byte knot loads; padding slots hold zero knots)
        const float aa = S.cf[0], bb = S.cf[1], c1 = S.cf[2], c2 = S.cf[3];
        const float hinv = S.cf[4], d1 = S.cf[5], d2 = S.cf[6];
        const float2* K0 = KN[S.lo_buf];
        const float2* K1 = KN[S.lo_buf ^ 1];
        for (int k = 2 * tid; k < nsl_r; k += 2 * RS_THREADS) {
          const float4 lo = *reinterpret_cast<const float4*>(K0 + k);
          const float4 hi = *reinterpret_cast<const float4*>(K1 + k);
          const uint32_t l2 = *reinterpret_cast<const uint32_t*>(loc + k);
          const float m0 = aa * lo.x + bb * hi.x + c1 * lo.y + c2 * hi.y;
          const float md0 = (hi.x - lo.x) * hinv + d1 * lo.y + d2 * hi.y;
          const float m1 = aa * lo.z + bb * hi.z + c1 * lo.w + c2 * hi.w;
          const float md1 = (hi.z - lo.z) * hinv + d1 * lo.w + d2 * hi.w;
          *reinterpret_cast<float2*>(Mp + k) = make_float2(m0, m1);
          {
            const int ia = (int)(l2 & 255u), ib = (int)((l2 >> 8) & 255u);
            const float2 x = bt[ia], z = bt[ib];
            force += (ia == ib ? md0 : 2.f * md0) * (x.x * z.x + x.y * z.y);
          }
          {
            const int ia = (int)((l2 >> 16) & 255u), ib = (int)(l2 >> 24);
            const float2 x = bt[ia], z = bt[ib];
            force += (ia == ib ? md1 : 2.f * md1) * (x.x * z.x + x.y * z.y);
          }
        }
      }
      __syncthreads();
      // rows: y_i = sum_j M_ij bt_j (tpr threads per row, strided parts of the row joined by
      // shuffles within the lane group); then, by the row's first thread, the quadratic
      // forms (F from above, g = Im((D^* u)^+ y), pot = Re(bt^+ y)), the amplitude
      // derivative da = -i (e^{iEt} y + (dphi/2) u) and the row's RK4 update; the closing
      // evaluation forms the quantum energy and the norm in place of F and g
      double f = (double)force, g = 0.0, pt = 0.0;
      {
        const double dt = S.dt, dphidt = S.dphidt;
        float2* aout = AIN[par ^ 1];
        double* amp = D.amp + (size_t)tr * 2 * d.N;
        double fe = 0.0, nn = 0.0;
        const int tpr = nr * 2 > RS_THREADS ? 1 : (nr * 4 > RS_THREADS ? 2 : (nr * 8 > RS_THREADS ? 4 : 8));
        const int sub = tid % tpr, grp = tid / tpr, ng = RS_THREADS / tpr;
        for (int rb = 0; rb < nr; rb += ng) {  // the same trip count in every lane
          const int lr = rb + grp;
          float yr = 0.f, yi = 0.f;
          if (lr < nr && !zero) {
            const int ei = row[lr].ent_i;
            const int e = ei >> 8, i = ei & 255;
            const int n = s_n[e];
            const float2* z = bt + s_lr0[e];
            const float* Mb = Mp + s_ls0[e];
            for (int j = sub; j < n; j += tpr) {
              const int addr = j <= i ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
              const float m = Mb[addr];
              const float2 zz = z[j];
              yr += m * zz.x;
              yi += m * zz.y;
            }
          }
          for (int o = tpr / 2; o > 0; o >>= 1) {
            yr += __shfl_xor_sync(0xffffffffu, yr, o);
            yi += __shfl_xor_sync(0xffffffffu, yi, o);
          }
          if (lr >= nr || sub != 0) continue;
          const RsRow w = row[lr];
          const float2 p = ph[w.ec], uu = uv[lr], b2 = bt[lr];
          pt += (double)(b2.x * yr + b2.y * yi);
          if (s == 4) {
            const double2 wv = Y[lr];
            const double w2 = wv.x * wv.x + wv.y * wv.y;
            fe += w2 * ev[w.ec];
            nn += w2;
            amp[w.ri] = wv.x;
            amp[d.N + w.ri] = wv.y;
            continue;
          }
          const float utr = p.x * uu.x - p.y * uu.y, uti = p.x * uu.y + p.y * uu.x;
          g += (double)(utr * yi - uti * yr);
          const double er = (double)p.x, eim = -(double)p.y;  // e^{iEt}
          const double zr = er * yr - eim * yi, zi = er * yi + eim * yr;
          const double cr = zr + 0.5 * dphidt * (double)uu.x;
          const double ci = zi + 0.5 * dphidt * (double)uu.y;
          const double dar = ci, dai = -cr;
          const double2 yo = Y[lr];
          float2 nx;
          if (s == 0) {
            ACC[lr] = make_float2((float)dar, (float)dai);
            nx = make_float2((float)(yo.x + 0.5 * dt * dar), (float)(yo.y + 0.5 * dt * dai));
          } else if (s < 3) {
            const float2 a0 = ACC[lr];
            ACC[lr] = make_float2((float)((double)a0.x + 2.0 * dar), (float)((double)a0.y + 2.0 * dai));
            const double c = s == 1 ? 0.5 * dt : dt;
            nx = make_float2((float)(yo.x + c * dar), (float)(yo.y + c * dai));
          } else {
            const float2 a0 = ACC[lr];
            const double h6 = dt / 6.0;
            const double2 yn = make_double2(yo.x + h6 * ((double)a0.x + dar),
                                            yo.y + h6 * ((double)a0.y + dai));
            Y[lr] = yn;
            nx = make_float2((float)yn.x, (float)yn.y);
          }
          aout[lr] = nx;
          push(w, nx, HALO[par ^ 1]);
        }
        if (s == 4) {
          f = fe;
          g = nn;
        }
      }
      // this CTA's parts (warp sums, then the warps in order by one thread per quantity) into
      // every CTA of the cluster; the cluster barrier (release / acquire: the parts and the
      // stage inputs pushed above are visible after it) is split so that the next right-hand
      // side's phases, whose time is known before the classical step, are formed while the
      // other CTAs arrive
      rs_warp_parts(f, g, pt, red);
      if (tid < 3) {
        double v = 0.0;
        for (int i = 0; i < RS_WARPS; ++i) v += red[3 * i + tid];
        for (int r = 0; r < D.CL; ++r) *clu.map_shared_rank(&part[par][rank][tid], r) = v;
      }
      rs_arrive();
      if (s != 4) rs_phases(PH[par ^ 1], ev, D.n_e, s < 2 ? S.tcur + 0.5 * S.dt : S.tcur + S.dt);
      rs_wait();
      if (tid == 0) {
        double F = 0.0, G = 0.0, P = 0.0;
        for (int r = 0; r < D.CL; ++r) {
          F += part[par][r][0];
          G += part[par][r][1];
          P += part[par][r][2];
        }
        rs_classical(S, d, D, s_ti, ev, s_ec, tr, rank == 0, F, G, P);
        if (S.stage != 5) rs_point(S, d, Rg, ih);
      }
      ++rc;
      __syncthreads();
    }
  }
  clu.sync();  // no CTA leaves while another may still read its shared memory
}

// ---------------------------------------------------------------- host
struct RsEngine {
  DevBuf<int> rk_b0, rk_blk, rk_ls0, rk_lr0, rk_rows, rk_slots, queue;
  DevBuf<RsRow> rows;
  DevBuf<uint16_t> loc;
  DevBuf<double> ih;
  int CL = 0, ns_cap = 0, nr_cap = 0, n_clusters = 0;
  int cl_force = 0;           // cluster size asked for (0: the smallest that fits)
  size_t smem = 0;
  const void* key = nullptr;  // the tables the layout was made for
};

RsEngine* rs_create() { return new RsEngine(); }
void rs_destroy(RsEngine* e) { delete e; }
void rs_set_cluster(RsEngine* e, int cl) { if (e && e->cl_force != cl) { e->cl_force = cl; e->key = nullptr; } }
int rs_cluster(const RsEngine* e) { return e ? e->CL : 0; }
int rs_clusters(const RsEngine* e) { return e ? e->n_clusters : 0; }

namespace {
// The m-blocks split between CL ranks (largest first, each to the rank with the fewest
// slots so far); per rank its blocks' slots (each block from an even offset) and rows.
struct RsSplit {
  std::vector<std::vector<int>> blocks;
  int ns_cap = 0, nr_cap = 0;
};
RsSplit rs_split(const std::vector<int>& blk_n, int CL) {
  const int nb = (int)blk_n.size();
  std::vector<int> order(nb);
  for (int b = 0; b < nb; ++b) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return blk_n[a] > blk_n[b]; });
  RsSplit sp;
  sp.blocks.assign(CL, {});
  std::vector<int64_t> slots(CL, 0);
  std::vector<int> rows(CL, 0);
  for (int b : order) {
    int r = 0;
    for (int q = 1; q < CL; ++q)
      if (slots[q] < slots[r]) r = q;
    const int n = blk_n[b];
    const int64_t nsl = (int64_t)n * (n + 1) / 2;
    slots[r] += (nsl + 1) & ~int64_t(1);
    rows[r] += n;
    sp.blocks[r].push_back(b);
  }
  for (int r = 0; r < CL; ++r) {
    sp.ns_cap = (int)std::max<int64_t>(sp.ns_cap, slots[r]);
    sp.nr_cap = std::max(sp.nr_cap, rows[r]);
  }
  sp.ns_cap = std::max(2, (sp.ns_cap + 7) & ~7);
  sp.nr_cap = std::max(2, (sp.nr_cap + 1) & ~1);
  return sp;
}
}  // namespace

// Lays out the engine for the tables (cluster size, block split, shared memory) and
// reports whether it applies: standard-mode RK4 without CS is the caller's check; here
// every m-block at most RS_MAX_STATES states and a cluster of at most RS_MAX_CL CTAs
// whose shared memory holds its blocks' two knot rows.
static int rs_prepare(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
                      const std::vector<int>& blk_s0, cudaStream_t st, bool* ok) {
  *ok = false;
  if (e->key == d.knots && e->CL > 0) {
    *ok = true;
    return MQCT_OK;
  }
  e->CL = 0;
  for (int n : blk_n)
    if (n > RS_MAX_STATES) return MQCT_OK;
  int dev = 0, optin = 0;
  MQCT_CUDA_TRY(cudaGetDevice(&dev));
  MQCT_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  MQCT_CUDA_TRY(cudaFuncGetAttributes(&fa, (const void*)rs_kernel));
  const size_t room = (size_t)optin - fa.sharedSizeBytes;
  RsSplit sp;
  int CL = 0;
  size_t smem = 0;
  for (int c = e->cl_force ? e->cl_force : 2; c <= (e->cl_force ? e->cl_force : RS_MAX_CL); ++c) {
    if ((int)blk_n.size() < c) break;
    sp = rs_split(blk_n, c);
    bool fit = true;
    for (const auto& v : sp.blocks) fit = fit && (int)v.size() <= RS_MAX_BLK;
    smem = rs_layout(sp.ns_cap, sp.nr_cap, d.n_e, d.nR).total;
    if (fit && smem <= room && sp.nr_cap <= 256) {
      CL = c;
      break;
    }
  }
  if (!CL) return MQCT_OK;
  // the largest request any layout may make (plans of other tables share the function)
  MQCT_CUDA_TRY(cudaFuncSetAttribute((const void*)rs_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)room));
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(CL, 1, 1);
  cfg.blockDim = dim3(RS_THREADS, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int ncl = 0;
  MQCT_CUDA_TRY(cudaOccupancyMaxActiveClusters(&ncl, (const void*)rs_kernel, &cfg));
  if (ncl < 1) return MQCT_OK;
  // device tables: the ranks' blocks, rows and slots (local row indices of each slot)
  const int N = d.N;
  std::vector<int> st_e(N), nbp(N), nbm(N), perm(N);
  std::vector<double> cp(N), cm(N), Rh(d.nR);
  // the plan's tables, read back on its stream (they were uploaded on it)
  const cudaMemcpyKind D2H = cudaMemcpyDeviceToHost;
  MQCT_CUDA_TRY(cudaMemcpyAsync(st_e.data(), d.st_e, sizeof(int) * N, D2H, st));
  MQCT_CUDA_TRY(cudaMemcpyAsync(nbp.data(), d.nb_plus, sizeof(int) * N, D2H, st));
  MQCT_CUDA_TRY(cudaMemcpyAsync(nbm.data(), d.nb_minus, sizeof(int) * N, D2H, st));
  MQCT_CUDA_TRY(cudaMemcpyAsync(perm.data(), d.perm, sizeof(int) * N, D2H, st));
  MQCT_CUDA_TRY(cudaMemcpyAsync(cp.data(), d.cplus, sizeof(double) * N, D2H, st));
  MQCT_CUDA_TRY(cudaMemcpyAsync(cm.data(), d.cminus, sizeof(double) * N, D2H, st));
  MQCT_CUDA_TRY(cudaMemcpyAsync(Rh.data(), d.R, sizeof(double) * d.nR, D2H, st));
  MQCT_CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<double> ih(d.nR, 0.0);
  for (int k = 0; k + 1 < d.nR; ++k) ih[k] = 1.0 / (Rh[k + 1] - Rh[k]);
  std::vector<int> b0(CL + 1, 0), blk, ls0, lr0, rows(CL, 0), nslots(CL, 0), owner(N, 0);
  std::vector<RsRow> rtab((size_t)CL * sp.nr_cap);
  std::vector<uint16_t> loc((size_t)CL * sp.ns_cap, 0);
  const std::vector<int>& s0 = blk_s0;
  for (int r = 0; r < CL; ++r) {
    int so = 0, ro = 0;
    for (size_t q = 0; q < sp.blocks[r].size(); ++q) {
      const int b = sp.blocks[r][q], n = blk_n[b];
      blk.push_back(b);
      ls0.push_back(so);
      lr0.push_back(ro);
      for (int i = 0; i < n; ++i) {
        owner[s0[b] + i] = (r << 16) | (ro + i);
        RsRow& w = rtab[(size_t)r * sp.nr_cap + ro + i];
        w.gi = s0[b] + i;
        w.ent_i = ((int)q << 8) | i;
        for (int j = 0; j <= i; ++j)
          loc[(size_t)r * sp.ns_cap + so + i * (i + 1) / 2 + j] =
              (uint16_t)((ro + i) | ((ro + j) << 8));
      }
      so += ((n * (n + 1) / 2) + 1) & ~1;
      ro += n;
    }
    rows[r] = ro;
    nslots[r] = so;
    b0[r + 1] = (int)blk.size();
  }
  // per state: the row whose J_+ (J_-) neighbour it is, where its stage inputs are pushed
  // (each state is the J_+ and the J_- neighbour of at most one state)
  std::vector<int> to_p(N, -1), to_m(N, -1);
  for (int gi = 0; gi < N; ++gi) {
    if (nbp[gi] >= 0) {
      if (to_p[nbp[gi]] >= 0) return MQCT_OK;  // a second consumer: the engine does not apply
      to_p[nbp[gi]] = owner[gi];
    }
    if (nbm[gi] >= 0) {
      if (to_m[nbm[gi]] >= 0) return MQCT_OK;
      to_m[nbm[gi]] = owner[gi];
    }
  }
  for (int r = 0; r < CL; ++r)
    for (int lr = 0; lr < rows[r]; ++lr) {
      RsRow& w = rtab[(size_t)r * sp.nr_cap + lr];
      const int gi = w.gi;
      w.ec = st_e[gi];
      w.ri = perm[gi];
      w.nbp = nbp[gi] >= 0 ? owner[nbp[gi]] : -1;
      w.nbm = nbm[gi] >= 0 ? owner[nbm[gi]] : -1;
      w.to_p = to_p[gi];
      w.to_m = to_m[gi];
      w.cp = cp[gi];
      w.cm = cm[gi];
    }
  MQCT_CUDA_TRY(e->rk_b0.upload(b0, st));
  MQCT_CUDA_TRY(e->rk_blk.upload(blk, st));
  MQCT_CUDA_TRY(e->rk_ls0.upload(ls0, st));
  MQCT_CUDA_TRY(e->rk_lr0.upload(lr0, st));
  MQCT_CUDA_TRY(e->rk_rows.upload(rows, st));
  MQCT_CUDA_TRY(e->rk_slots.upload(nslots, st));
  MQCT_CUDA_TRY(e->rows.upload(rtab, st));
  MQCT_CUDA_TRY(e->loc.upload(loc, st));
  MQCT_CUDA_TRY(e->ih.upload(ih, st));
  if (!e->queue.p) MQCT_CUDA_TRY(e->queue.alloc(1));
  MQCT_CUDA_TRY(cudaStreamSynchronize(st));
  e->CL = CL;
  e->ns_cap = sp.ns_cap;
  e->nr_cap = sp.nr_cap;
  e->n_clusters = ncl;
  e->smem = smem;
  e->key = d.knots;
  *ok = true;
  return MQCT_OK;
}

bool rs_usable(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
               const std::vector<int>& blk_s0, cudaStream_t st) {
  bool ok = false;
  return rs_prepare(e, d, blk_n, blk_s0, st, &ok) == MQCT_OK && ok;
}

// One launch over n queue entries (trajectories, or hand-over records when resume is set);
// ev0 recorded before it unless null, ev1 after it.
static int rs_launch(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
                     const std::vector<int>& blk_s0, cudaStream_t st, cudaEvent_t ev0,
                     cudaEvent_t ev1, const mqct_traj_init_t* d_init, int n,
                     const RsResume* resume, const double2* resume_amp, double* amp,
                     double* cls, double* diag) {
  bool ok = false;
  int rc = rs_prepare(e, d, blk_n, blk_s0, st, &ok);
  if (rc) return rc;
  MQCT_ARG_CHECK(ok, "resident engine: the tables do not fit a cluster's shared memory");
  MQCT_ARG_CHECK(n > 0, "no trajectories");
  RsDev D{};
  D.init = d_init;
  D.n_traj = n;
  D.CL = e->CL;
  D.ns_cap = e->ns_cap;
  D.nr_cap = e->nr_cap;
  D.n_e = d.n_e;
  D.rk_b0 = e->rk_b0.p;
  D.rk_blk = e->rk_blk.p;
  D.rk_ls0 = e->rk_ls0.p;
  D.rk_lr0 = e->rk_lr0.p;
  D.rk_rows = e->rk_rows.p;
  D.rk_slots = e->rk_slots.p;
  D.rows = e->rows.p;
  D.loc = e->loc.p;
  D.ih = e->ih.p;
  D.resume = resume;
  D.resume_amp = resume_amp;
  D.queue = e->queue.p;
  D.amp = amp;
  D.cls = cls;
  D.diag = diag;
  const int ncl = std::min(e->n_clusters, n);
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = e->CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(ncl * e->CL, 1, 1);
  cfg.blockDim = dim3(RS_THREADS, 1, 1);
  cfg.dynamicSmemBytes = e->smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  MQCT_CUDA_TRY(cudaMemsetAsync(e->queue.p, 0, sizeof(int), st));
  if (ev0) MQCT_CUDA_TRY(cudaEventRecord(ev0, st));
  MQCT_CUDA_TRY(cudaLaunchKernelEx(&cfg, rs_kernel, d, D));
  MQCT_CUDA_TRY(cudaGetLastError());
  MQCT_CUDA_TRY(cudaEventRecord(ev1, st));
  return MQCT_OK;
}

int rs_run(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
           const std::vector<int>& blk_s0, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
           const mqct_traj_init_t* d_init, int n_traj, double* amp, double* cls, double* diag) {
  return rs_launch(e, d, blk_n, blk_s0, st, ev0, ev1, d_init, n_traj, nullptr, nullptr, amp,
                   cls, diag);
}

int rs_run_resume(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
                  const std::vector<int>& blk_s0, cudaStream_t st, cudaEvent_t ev1,
                  const mqct_traj_init_t* d_init, const RsResume* resume, int n,
                  const double2* resume_amp, double* amp, double* cls, double* diag) {
  MQCT_ARG_CHECK(resume && resume_amp, "hand-over records missing");
  return rs_launch(e, d, blk_n, blk_s0, st, nullptr, ev1, d_init, n, resume, resume_amp, amp,
                   cls, diag);
}

}  // namespace mqct
