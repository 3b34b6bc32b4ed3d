// propagate.cu -- batched trajectory propagation (H2).
//
// The reference integrates one trajectory at a time (DOTRAJECT,
// MQCT_SOURCE_CODES/propagator.f:2283-4645) with fixed-step RK4
// (MQCT_SOURCE_CODES/suppl_routines.f:1076-1113) of the interaction-picture
// amplitudes a and the classical variables, the right-hand side being
// DERIVS_BK (MQCT_SOURCE_CODES/mqct_eqtns.f:112-499): for every stored pair
// k=(i,j) a phase e^{-i(E_j-E_i)t}, the complex update of a_i and a_j, the
// force term and the Coriolis accumulators, then an MPI reduction per call.
//
// Here one persistent kernel holds a trajectory per CTA, takes the next one
// from a device queue when it finishes (slot retire/refill), and evaluates the
// same right-hand side in matrix form:
//     bt = D^* a  with D = diag(e^{i E_s t})          (FP64 phases)
//     y  = M(R) bt,   F = Re(bt^+ M'(R) bt)             (block-diagonal in m)
//     u  = (J_+ + J_-) a,  dP_phi/dt = sin(theta) Im((D^* u)^+ y)
//     da/dt = -i D y - i (dphi/dt / 2) u
// which is algebraically identical to the reference's pair loop (the phase of
// a pair factorises into per-state phases; its Coriolis dot product is the
// quadratic form above).
//
// Table layout: for every m-block (states of equal m12, kept contiguous in an
// internal block-major state order) the full lower triangle of the block is
// stored row-major ("slot" T(i)+j for local row i >= column j, T(i)=i(i+1)/2),
// pairs dropped by the cut-off as zeros, each block padded to 4 slots.  A knot
// row holds (M, y2) for every slot at one R.
//
// One right-hand side, for the spline interval [R_klo, R_klo+1]:
//  phase A -- every thread takes slots tid, tid+PT, ... : coalesced loads of
//    the two knot rows, M and M' by the cubic spline, M stored packed in shared
//    memory, the force term Re(bt_i^* bt_j) M'_ij accumulated in registers;
//  phase B -- every thread takes whole rows: y_i = sum_j M_ij bt_j over the
//    packed triangle (row part j <= i, then column part j > i), fixed order,
//    no atomics, deterministic.
// When the packed triangles of all blocks do not fit in shared memory the
// blocks are processed in several passes.  The RK4 amplitudes are FP64 in
// registers; the classical variables are FP64 in shared memory, advanced by
// thread 0; the table and mat-vec arithmetic T is float (FP32 mode) or double
// (FP64 mode).
#include <algorithm>
#include <cmath>
#include <map>

#include "common.cuh"
#include "propagate.cuh"

using namespace mqct;

namespace mqct {

constexpr int PT = 512;        // threads per CTA of the default launch shape
constexpr int MAX_N = 4096;    // states (N <= threads x states per thread)
constexpr int UNROLL = 4;      // slots per thread in flight in phase A
// Launch shapes: TPB threads per CTA; TPB == 256 runs two CTAs (two trajectories) per SM
// so that one trajectory's load latency overlaps the other's work.  The plan picks the
// faster shape for its tables by timing both (PropPlan::tune).

struct TrajOut {
  double* amp;
  double* cls;
  double* diag;
  // SAVE_TRAJECT records (standard mode; null: none): rec_cap records of 8 doubles per
  // trajectory, n_rec the count produced (records past rec_cap are counted, not written)
  double* rec;
  int64_t rec_cap;
  int64_t* n_rec;
};

// One SAVE_TRAJECT record (t, R, P_R, theta, P_theta, phi, P_phi, pot),
// MQCT_SOURCE_CODES/propagator.f:3458-3464 and 4329-4337.
__device__ inline void save_record(const TrajOut& o, int tr, int64_t& n, double t, const Cls& c,
                                   double pot) {
  if (n < o.rec_cap) {
    double* r = o.rec + ((size_t)tr * o.rec_cap + n) * 8;
    r[0] = t; r[1] = c.R; r[2] = c.PR; r[3] = c.th; r[4] = c.Pth; r[5] = c.phi; r[6] = c.Pphi;
    r[7] = pot;
  }
  ++n;
}

// Classical slots in shared memory: state, stage input, stage derivative, first-stage
// derivative, RK4 middle-stage sum, Cash-Karp stages 2-5, Cash-Karp result and error.
constexpr int kClsSlots = 11;

// Shared-memory layout of one CTA (dynamic).
template <class T>
struct Smem {
  Cls* c;                      // kClsSlots classical slots (see above)
  double* red;                 // reduction scratch, 3 per warp, then the 3 block sums
  SplineAt* spl;               // spline interval of the current R (one per right-hand side)
  double* scal;                // [0] sin(theta), [1] dphi/dt, [2] 1/R, [3] 1/sin^2(theta),
                               // [4..6] the last theta with its sine and 1/sin^2
  int* flag;                   // [0] next trajectory, [1] keep running, [2] CS m-block or -1,
                               // [3] the spline interval found last
  double* Rg;                  // nR grid
  double2* a_in;               // N (RHS input amplitudes)
  typename V2<T>::t* bt;       // N
  typename V2<T>::t* u;        // N
  typename V2<T>::t* y;        // N
  typename V2<T>::t* ph;       // n_e
  T* Mp;                       // packed triangles of one pass
};

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sums of three doubles, broadcast to all threads (fixed order).
template <int TPB>
__device__ inline void block_sum3(double& a, double& b, double& c, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  if (lane == 0) {
    red[3 * w] = a;
    red[3 * w + 1] = b;
    red[3 * w + 2] = c;
  }
  __syncthreads();
  // one thread adds the warp sums in warp order and publishes them (the next call's
  // partial writes go to other slots, its totals only after its first barrier)
  constexpr int W = TPB / 32;
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0, sc = 0.0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      sa += red[3 * i];
      sb += red[3 * i + 1];
      sc += red[3 * i + 2];
    }
    red[3 * W] = sa;
    red[3 * W + 1] = sb;
    red[3 * W + 2] = sc;
  }
  __syncthreads();
  a = red[3 * W];
  b = red[3 * W + 1];
  c = red[3 * W + 2];
}


constexpr int kAtCols = 6;  // splined columns of an AT path record

// Cubic-spline value of an AT path column at time t (splint,
// MQCT_SOURCE_CODES/suppl_routines.f:968-1002).
__device__ inline double at_splint(const double* rec, const double* y2, int n, int col, int ycol,
                                   double t) {
  int klo = 1, khi = n;
  while (khi - klo > 1) {
    int k = (khi + klo) >> 1;
    if (rec[8 * (k - 1)] > t) khi = k;
    else klo = k;
  }
  double xlo = rec[8 * (klo - 1)], xhi = rec[8 * (khi - 1)];
  double h = xhi - xlo, a = (xhi - t) / h, b = (t - xlo) / h;
  return a * rec[8 * (klo - 1) + col] + b * rec[8 * (khi - 1) + col] +
         ((a * a * a - a) * y2[kAtCols * (klo - 1) + ycol] + (b * b * b - b) * y2[kAtCols * (khi - 1) + ycol]) *
             (h * h) / 6.0;
}

__device__ inline float2 ldg2(const float2* p) { return __ldg(p); }
__device__ inline double2 ldg2(const double2* p) { return __ldg(p); }

// One right-hand-side evaluation at time t and classical point cin (shared
// memory).  Input amplitudes in sm.a_in (internal order).  Outputs: da for this
// thread's states, the classical derivative written to dc by thread 0 (std
// mode), and pot = Re(bt^+ y) (coupling energy), identical in all threads.
template <class T, int NS, int TPB>
__device__ void rhs(const PropDev& d, const Smem<T>& sm, double t, const Cls* cin, int ns,
                    double2 (&da)[NS], Cls* dc, double& pot) {
  using T2 = typename V2<T>::t;
  const int tid = threadIdx.x;
  const int N = d.N;
  const Cls c = *cin;
  // the point's scalars, formed once and read by every thread after the first barrier
  // (reciprocals of R, m and sin^2: two divisions per point on the serial path of
  // thread 0 in place of the reference's chained ones; the same values to rounding)
  if (tid == 0) {
    // theta stays at pi/2 in planar motion: sin(theta) and 1/sin^2 are kept while it is
    // unchanged
    if (!(c.th == sm.scal[4])) {
      const double st0 = sin(c.th);
      sm.scal[4] = c.th;
      sm.scal[5] = st0;
      sm.scal[6] = 1.0 / (st0 * st0);
    }
    const double st = sm.scal[5];
    const double inv_r = 1.0 / c.R;
    const double inv_s2 = sm.scal[6];
    sm.scal[0] = st;
    sm.scal[1] = c.Pphi * inv_r * inv_r * d.inv_mass * inv_s2;
    sm.scal[2] = inv_r;
    sm.scal[3] = inv_s2;
    *sm.spl = spline_at(sm.Rg, d.nR, c.R, sm.flag + 3);
  }
  // coupled states: only the m-block of the initial state carries amplitude, so only
  // its slots are read and only its rows formed; bt, u and y of the other rows were
  // zeroed when the trajectory started and stay zero
  const int cs_blk = sm.flag[2];
  const int cs_r0 = cs_blk >= 0 ? __ldg(d.blk_s0 + cs_blk) : 0;
  const int cs_r1 = cs_blk >= 0 ? cs_r0 + __ldg(d.blk_n + cs_blk) : N;
  // phases per energy class: (cos E t, -sin E t) = e^{-iEt}
  for (int e = tid; e < d.n_e; e += TPB) {
    double s, co;
    sincos(d.e_val[e] * t, &s, &co);
    sm.ph[e].x = (T)co;
    sm.ph[e].y = (T)(-s);
  }
  __syncthreads();
  const double sin_t = sm.scal[0], dphidt = sm.scal[1];
  const SplineAt sp = *sm.spl;
  for (int i = cs_r0 + tid; i < cs_r1; i += TPB) {
    const double2 a = sm.a_in[i];
    const T2 p = sm.ph[__ldg(d.st_e + i)];
    const T ar = (T)a.x, ai = (T)a.y;
    sm.bt[i].x = p.x * ar - p.y * ai;
    sm.bt[i].y = p.x * ai + p.y * ar;
    double ur = 0.0, ui = 0.0;
    // u = (J_+ + J_-) a; none with CS_APPROX (MQCT_SOURCE_CODES/mqct_eqtns.f:270, 362,
    // 845), which also keeps dP_phi/dt = sin(theta) Im((D^* u)^+ y) at zero
    const int np_ = d.cs ? -1 : __ldg(d.nb_plus + i), nm = d.cs ? -1 : __ldg(d.nb_minus + i);
    if (np_ >= 0) {
      const double cp = __ldg(d.cplus + i);
      ur += cp * sm.a_in[np_].x;
      ui += cp * sm.a_in[np_].y;
    }
    if (nm >= 0) {
      const double cm = __ldg(d.cminus + i);
      ur += cm * sm.a_in[nm].x;
      ui += cm * sm.a_in[nm].y;
    }
    sm.u[i].x = (T)ur;
    sm.u[i].y = (T)ui;
    if (sp.zero) {
      sm.y[i].x = (T)0;
      sm.y[i].y = (T)0;
    }
  }
  T force = (T)0;
  __syncthreads();
  if (!sp.zero) {
    // M = aa lo + bb hi + c1 lo'' + c2 hi'';  M' = (hi - lo)/h + d1 lo'' + d2 hi''
    const T aa = (T)sp.aa, bb = (T)sp.bb, c1 = (T)(sp.cc1 * sp.cc5), c2 = (T)(sp.cc2 * sp.cc5);
    const T hinv = (T)(1.0 / sp.h), d1 = (T)(-sp.cc3 * sp.cc6), d2 = (T)(sp.cc4 * sp.cc6);
    const T2* K0 = reinterpret_cast<const T2*>(d.knots) + (int64_t)sp.klo * d.S;
    const T2* K1 = K0 + d.S;
    const int p_lo = cs_blk >= 0 ? __ldg(d.blk_pass + cs_blk) : 0;
    const int p_hi = cs_blk >= 0 ? p_lo + 1 : d.n_pass;
    for (int p = p_lo; p < p_hi; ++p) {
      // s0: the pass's first slot (shared-memory base); [k0, s1): the slots read
      const int s0 = (int)d.pass_slot0[p];
      const int k0 = cs_blk >= 0 ? (int)d.blk_slot0[cs_blk] : s0;
      const int s1 = cs_blk >= 0 ? (int)d.blk_slot0[cs_blk + 1] : (int)d.pass_slot0[p + 1];
      // phase A: interpolate the pass's slots into Mp, force term
      if constexpr (sizeof(T) == 4) {
        // two adjacent slots per load (16-byte knot loads, 8-byte location loads)
        for (int kb = k0 + 2 * tid; kb < s1; kb += 2 * UNROLL * TPB) {
          float4 lo[UNROLL], hi[UNROLL];
          uint2 l[UNROLL];
#pragma unroll
          for (int q = 0; q < UNROLL; ++q) {
            const int k = kb + 2 * q * TPB;
            if (k < s1) {
              lo[q] = __ldg(reinterpret_cast<const float4*>(K0 + k));
              hi[q] = __ldg(reinterpret_cast<const float4*>(K1 + k));
              l[q] = __ldg(reinterpret_cast<const uint2*>(d.loc + k));
            }
          }
#pragma unroll
          for (int q = 0; q < UNROLL; ++q) {
            const int k = kb + 2 * q * TPB;
            if (k < s1) {
              const float m0 = aa * lo[q].x + bb * hi[q].x + c1 * lo[q].y + c2 * hi[q].y;
              const float md0 = (hi[q].x - lo[q].x) * hinv + d1 * lo[q].y + d2 * hi[q].y;
              const float m1 = aa * lo[q].z + bb * hi[q].z + c1 * lo[q].w + c2 * hi[q].w;
              const float md1 = (hi[q].z - lo[q].z) * hinv + d1 * lo[q].w + d2 * hi[q].w;
              *reinterpret_cast<float2*>(sm.Mp + (k - s0)) = make_float2(m0, m1);
              {
                const int ia = (int)(l[q].x & 0xffffu), ib = (int)(l[q].x >> 16);
                const T2 x = sm.bt[ia], z = sm.bt[ib];
                force += (ia == ib ? md0 : 2.f * md0) * (x.x * z.x + x.y * z.y);
              }
              {
                const int ia = (int)(l[q].y & 0xffffu), ib = (int)(l[q].y >> 16);
                const T2 x = sm.bt[ia], z = sm.bt[ib];
                force += (ia == ib ? md1 : 2.f * md1) * (x.x * z.x + x.y * z.y);
              }
            }
          }
        }
      } else {
        for (int kb = k0 + tid; kb < s1; kb += UNROLL * TPB) {
          T2 lo[UNROLL], hi[UNROLL];
          uint32_t l[UNROLL];
#pragma unroll
          for (int q = 0; q < UNROLL; ++q) {
            const int k = kb + q * TPB;
            if (k < s1) {
              lo[q] = ldg2(K0 + k);
              hi[q] = ldg2(K1 + k);
              l[q] = __ldg(d.loc + k);
            }
          }
#pragma unroll
          for (int q = 0; q < UNROLL; ++q) {
            const int k = kb + q * TPB;
            if (k < s1) {
              const T m = aa * lo[q].x + bb * hi[q].x + c1 * lo[q].y + c2 * hi[q].y;
              const T md = (hi[q].x - lo[q].x) * hinv + d1 * lo[q].y + d2 * hi[q].y;
              sm.Mp[k - s0] = m;
              const int ia = (int)(l[q] & 0xffffu), ib = (int)(l[q] >> 16);
              const T2 x = sm.bt[ia], z = sm.bt[ib];
              const T re = x.x * z.x + x.y * z.y;
              force += (ia == ib ? md : (T)2 * md) * re;
            }
          }
        }
      }
      __syncthreads();
      // phase B: rows of the pass, y_i = sum_j M_ij bt_j
      const int r0 = cs_blk >= 0 ? cs_r0 : d.pass_row0[p];
      const int r1 = cs_blk >= 0 ? cs_r1 : d.pass_row0[p + 1];
      const int rows = r1 - r0;
      // few rows (one m-block in CS mode): tpr threads per row, each a strided part of
      // the row, joined by shuffles within the lane group; otherwise one thread per row
      const int tpr = rows * 2 > TPB ? 1 : (rows * 4 > TPB ? 2 : (rows * 8 > TPB ? 4 : 8));
      if (tpr > 1) {
        const int sub = tid % tpr, grp = tid / tpr, ng = TPB / tpr;
        for (int rb = r0; rb < r1; rb += ng) {  // the same trip count in every lane
          const int r = rb + grp;
          T yr = (T)0, yi = (T)0;
          if (r < r1) {
            const int b = __ldg(d.st_blk + r);
            const int n = __ldg(d.blk_n + b), sb = __ldg(d.blk_s0 + b);
            const int i = r - sb;
            const T2* z = sm.bt + sb;
            const T* Mb = sm.Mp + __ldg(d.blk_mp + b);
            for (int j = sub; j < n; j += tpr) {
              const int addr = j <= i ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
              const T m = Mb[addr];
              const T2 zz = z[j];
              yr += m * zz.x;
              yi += m * zz.y;
            }
          }
          for (int o = tpr / 2; o > 0; o >>= 1) {
            yr += __shfl_xor_sync(0xffffffffu, yr, o);
            yi += __shfl_xor_sync(0xffffffffu, yi, o);
          }
          if (r < r1 && sub == 0) {
            sm.y[r].x = yr;
            sm.y[r].y = yi;
          }
        }
      } else
      for (int r = r0 + tid; r < r1; r += TPB) {
        const int b = __ldg(d.st_blk + r);
        const int n = __ldg(d.blk_n + b), sb = __ldg(d.blk_s0 + b);
        const int i = r - sb;
        const T2* z = sm.bt + sb;
        const T* Mb = sm.Mp + __ldg(d.blk_mp + b);
        int addr = i * (i + 1) / 2;
        T yr0 = (T)0, yi0 = (T)0, yr1 = (T)0, yi1 = (T)0;
        int j = 0;
        for (; j + 1 < n; j += 2) {
          const T m0 = Mb[addr];
          addr += (j < i) ? 1 : (j + 1);
          const T m1 = Mb[addr];
          addr += (j + 1 < i) ? 1 : (j + 2);
          const T2 z0 = z[j], z1 = z[j + 1];
          yr0 += m0 * z0.x;
          yi0 += m0 * z0.y;
          yr1 += m1 * z1.x;
          yi1 += m1 * z1.y;
        }
        if (j < n) {
          const T m0 = Mb[addr];
          const T2 z0 = z[j];
          yr0 += m0 * z0.x;
          yi0 += m0 * z0.y;
        }
        sm.y[r].x = yr0 + yr1;
        sm.y[r].y = yi0 + yi1;
      }
      __syncthreads();
    }
  }
  // quadratic forms: F (accumulated above), g = Im((D^* u)^+ y), pot = Re(bt^+ y)
  double g = 0.0, pt = 0.0, f = (double)force;
  for (int i = cs_r0 + tid; i < cs_r1; i += TPB) {
    const T2 p = sm.ph[__ldg(d.st_e + i)];
    const T2 uu = sm.u[i], yy = sm.y[i], b2 = sm.bt[i];
    const T utr = p.x * uu.x - p.y * uu.y, uti = p.x * uu.y + p.y * uu.x;
    g += (double)(utr * yy.y - uti * yy.x);
    pt += (double)(b2.x * yy.x + b2.y * yy.y);
  }
  block_sum3<TPB>(g, pt, f, sm.red);
  pot = pt;
  // da_i = -i e^{iE t} y_i - i (dphi/2) u_i
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    if (q >= ns) break;
    const int i = tid + q * TPB;
    const T2 p = sm.ph[__ldg(d.st_e + i)];
    const T2 yy = sm.y[i], uu = sm.u[i];
    const double er = (double)p.x, ei = -(double)p.y;  // e^{iEt}
    const double zr = er * yy.x - ei * yy.y, zi = er * yy.y + ei * yy.x;
    const double cr = zr + 0.5 * dphidt * (double)uu.x, ci = zi + 0.5 * dphidt * (double)uu.y;
    da[q] = make_double2(ci, -cr);  // -i (cr + i ci)
  }
  if (tid == 0 && d.mode == MQCT_MODE_STD) {
    const double ir = sm.scal[2], is2 = sm.scal[3], im = d.inv_mass;
    const double ir3m = ir * ir * ir * im;
    dc->R = c.PR * im;
    dc->PR = -f + c.Pth * c.Pth * ir3m + c.Pphi * c.Pphi * ir3m * is2;
    dc->th = 0.0;
    dc->Pth = 0.0;
    dc->phi = dphidt;
    dc->Pphi = sin_t * g;
  }
}

__device__ inline Cls cls_axpy(const Cls& a, double h, const Cls& b) {
  return Cls{a.R + h * b.R, a.PR + h * b.PR, a.th + h * b.th,
             a.Pth + h * b.Pth, a.phi + h * b.phi, a.Pphi + h * b.Pphi};
}

// Component i of the classical variables (R, P_R, theta, P_theta, phi, P_phi).
__device__ inline double& cls_ref(Cls& c, int i) {
  switch (i) {
    case 0: return c.R;
    case 1: return c.PR;
    case 2: return c.th;
    case 3: return c.Pth;
    case 4: return c.phi;
    default: return c.Pphi;
  }
}
__device__ inline double cls_get(const Cls& c, int i) { return cls_ref(const_cast<Cls&>(c), i); }

// Block-wide maximum, broadcast to all threads.
template <int TPB>
__device__ inline double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double m = red[0];
#pragma unroll
  for (int i = 1; i < TPB / 32; ++i) m = fmax(m, red[i]);
  __syncthreads();
  return m;
}

// Cash-Karp 5(4) coefficients (MQCT_SOURCE_CODES/suppl_routines.f:1313-1329).  A4 is
// written there as the default-real literal .6, so its value is 0.6 in single precision.
constexpr double kCkB21 = .2, kCkB31 = 3.0 / 40.0, kCkB32 = 9.0 / 40.0, kCkB41 = .3,
                 kCkB42 = -.9, kCkB43 = 1.2, kCkB51 = -11.0 / 54.0, kCkB52 = 2.5,
                 kCkB53 = -70.0 / 27.0, kCkB54 = 35.0 / 27.0, kCkB61 = 1631.0 / 55296.0,
                 kCkB62 = 175.0 / 512.0, kCkB63 = 575.0 / 13824.0, kCkB64 = 44275.0 / 110592.0,
                 kCkB65 = 253.0 / 4096.0, kCkC1 = 37.0 / 378.0, kCkC3 = 250.0 / 621.0,
                 kCkC4 = 125.0 / 594.0, kCkC6 = 512.0 / 1771.0,
                 kCkDC1 = kCkC1 - 2825.0 / 27648.0, kCkDC3 = kCkC3 - 18575.0 / 48384.0,
                 kCkDC4 = kCkC4 - 13525.0 / 55296.0, kCkDC5 = -277.0 / 14336.0,
                 kCkDC6 = kCkC6 - .25;
constexpr double kCkA4 = (double)0.6f;
constexpr int kOdeMaxSteps = 10000;  // MAXSTP of odeint


// Classical point of an AT trajectory at time t (thread 0).
__device__ inline void classical_at(const PropDev& d, int tr, double t, Cls* cc) {
  const double* rec = d.at_rec + 8 * d.at_off[tr];
  const double* y2 = d.at_y2 + kAtCols * d.at_off[tr];
  const int n = d.at_n[tr];
  cc->R = at_splint(rec, y2, n, 1, 0, t);
  cc->th = at_splint(rec, y2, n, 3, 1, t);
  cc->Pth = at_splint(rec, y2, n, 4, 2, t);
  cc->Pphi = at_splint(rec, y2, n, 6, 3, t);
  cc->PR = 0.0;
  cc->phi = 0.0;
}

// AT_ADAPT_STP (MQCT_SOURCE_CODES/propagator.f:3034-3049, 3821-3860): the next RK4 step of
// an AT trajectory from the coupling energy along its path (record column 8).  From tcur,
// probe points tmchk + tau (i + 1/2) accumulate |pot|; the step ends where
// (tau i)^4 sum|pot| / i reaches `magic`, at the first sign change of pot (after t = 0), or
// at the end of the path (then last = true).  Steps below mintm become mintm.  fa carries
// the last probed value from step to step as in the reference.  Thread 0 only.
__device__ inline double at_adapt_step(const PropDev& d, int tr, double tcur, double t_end,
                                       double magic, double& fa, bool& last) {
  const double* rec = d.at_rec + 8 * d.at_off[tr];
  const double* y2 = d.at_y2 + kAtCols * d.at_off[tr];
  const int n = d.at_n[tr];
  const double tau = 10.0, tmchk = tcur;
  double potbox = 0.0, dt = d.at_mintm;
  for (int stps = 0; stps < (1 << 26);) {  // bounded: the path ends within t_end / tau probes
    const double tmstp = tmchk + tau * (stps + 0.50);
    stps += 1;
    const double fb = at_splint(rec, y2, n, 7, 4, tmstp);
    potbox += fabs(fb);
    const double i_max = pow(tau * stps, 4.0) * potbox / stps;
    bool done = false;
    if (i_max >= magic) {
      dt = fmax(tau * (stps - 1), d.at_mintm);
      done = true;
    } else if (tmstp > t_end) {
      dt = t_end - tmchk;
      last = true;
      done = true;
    } else if (tcur > 0.0) {
      const double r = fa / fb;
      if (r < 0.0 && r == r) {
        dt = fmax(tau * (stps - 1), d.at_mintm);
        done = true;
      }
    }
    fa = fb;
    if (done) break;
  }
  return dt;
}

// Per-trajectory bookkeeping of thread 0 (shared memory).
struct Book {
  double tmpR1, tmpR2, eki, eqi;
  double at_magic, at_fa, at_dt;  // AT_ADAPT_STP state (thread 0)
  int64_t n_rec;
  int status, vib, period, run;
};

// kAdaptive: PROPAGATOR = ODEINT (adaptive Cash-Karp steps inside every step dt, or
// over the whole path in AT mode) in place of RK4 with step dt.
template <class T, int NS, bool kAdaptive, int TPB>
__global__ void __launch_bounds__(TPB, TPB == 256 ? 2 : 1)
propagate_kernel(PropDev d, const mqct_traj_init_t* __restrict__ init, int n_traj,
                 int* __restrict__ queue, TrajOut out) {
  using T2 = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = d.N, tid = threadIdx.x;
  Smem<T> sm;
  Book* bk;
  {
    unsigned char* p = smem_raw;
    auto take = [&](size_t bytes) {
      unsigned char* r = p;
      p += (bytes + 15) & ~size_t(15);
      return r;
    };
    sm.c = reinterpret_cast<Cls*>(take(sizeof(Cls) * kClsSlots));
    bk = reinterpret_cast<Book*>(take(sizeof(Book)));
    sm.red = reinterpret_cast<double*>(take(sizeof(double) * 3 * (TPB / 32 + 1)));
    sm.spl = reinterpret_cast<SplineAt*>(take(sizeof(SplineAt)));
    sm.scal = reinterpret_cast<double*>(take(64));
    sm.flag = reinterpret_cast<int*>(take(16));
    sm.Rg = reinterpret_cast<double*>(take(sizeof(double) * d.nR));
    sm.a_in = reinterpret_cast<double2*>(take(sizeof(double2) * N));
    sm.bt = reinterpret_cast<T2*>(take(sizeof(T2) * N));
    sm.u = reinterpret_cast<T2*>(take(sizeof(T2) * N));
    sm.y = reinterpret_cast<T2*>(take(sizeof(T2) * N));
    sm.ph = reinterpret_cast<T2*>(take(sizeof(T2) * d.n_e));
    sm.Mp = reinterpret_cast<T*>(take(sizeof(T) * (size_t)d.mp_cap));
  }
  for (int i = tid; i < d.nR; i += TPB) sm.Rg[i] = d.R[i];
  if (tid == 0) {
    sm.scal[4] = __longlong_as_double(0x7ff8000000000000ULL);  // no theta yet
    sm.flag[3] = 0;                                            // no interval yet
  }
  Cls* const C = sm.c;       // current state
  Cls* const CT = sm.c + 1;  // classical point of the stage
  Cls* const KC = sm.c + 2;  // classical derivative of the stage
  Cls* const K1 = sm.c + 3;  // first-stage derivative
  Cls* const K23 = sm.c + 4; // sum of the second and third stages
  Cls* const KS = sm.c + 5;  // Cash-Karp stages 2..5 (KS[0..3])
  Cls* const CO = sm.c + 9;  // Cash-Karp result
  Cls* const CE = sm.c + 10; // Cash-Karp error estimate
  const int ns = (N + TPB - 1 - tid) / TPB;  // states owned by this thread
  const bool at = d.mode == MQCT_MODE_AT;
  for (;;) {
    __syncthreads();
    if (tid == 0) sm.flag[0] = atomicAdd(queue, 1);
    __syncthreads();
    const int tr = sm.flag[0];
    if (tr >= n_traj) break;
    const mqct_traj_init_t* ti = init + tr;
    double2 y[NS], k[NS], k1[NS], k23[NS];
    const int s_int = d.inv_perm[ti->s_st - 1];
#pragma unroll
    for (int q = 0; q < NS; ++q)
      y[q] = make_double2((q < ns && tid + q * TPB == s_int) ? 1.0 : 0.0, 0.0);
    double tcur = at ? d.at_rec[8 * d.at_off[tr]] : 0.0;
    const double t_end = at ? d.at_rec[8 * (d.at_off[tr] + d.at_n[tr] - 1)] : 0.0;
    double dt = ti->dt;
    long long counter = 0;
    if (tid == 0) {
      const double k_vec = sqrt(d.mass * 2.0 * ti->e_coll);
      const double l_orb = sqrt(ti->l_real * (ti->l_real + 1.0));
      *bk = Book{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0, 0, 0, 0, 1};
      if (at && d.at_adapt) {
        // the step-size scale of AT_ADAPT_STP, once per trajectory
        const double u_cm = ti->e_coll / kCmToHartree;
        double tmp3 = -exp(2.0 * kPi * (u_cm - 202.0) / 20.0);
        if (fabs(tmp3) > 1e16) tmp3 = -1e16;
        const double tmp4 = 0.30 + 0.80 * tmp3 / (1.0 - tmp3) - 4.250 * tmp3 / pow(1.0 - tmp3, 2.0);
        const double tol = d.at_tol * pow(u_cm / 300.0, tmp4);
        bk->at_magic = ti->e_coll * pow(t_end * tol, 4.0);
      }
      *C = Cls{};
      sm.flag[2] = d.cs ? d.st_blk[s_int] : -1;
      if (!at && l_orb / k_vec > ti->r_start) {
        bk->status = 2;  // impact parameter beyond the starting distance: not propagated
        bk->run = 0;
        C->R = ti->r_start;
      } else if (!at) {  // initial conditions, MQCT_SOURCE_CODES/propagator.f:2531-2566
        C->R = ti->r_start;
        C->PR = -sqrt(k_vec * k_vec - l_orb * l_orb / (ti->r_start * ti->r_start));
        C->th = acos(0.0);
        C->Pth = l_orb * sin(0.0);
        C->phi = 0.0;
        C->Pphi = l_orb * cos(0.0);
      }
    }
    __syncthreads();
    if (d.cs)
      for (int i = tid; i < N; i += TPB) {
        sm.bt[i] = T2{(T)0, (T)0};
        sm.u[i] = T2{(T)0, (T)0};
        sm.y[i] = T2{(T)0, (T)0};
      }
    const bool skipped = bk->run == 0;
    double dt_step = dt;  // ODEINT's carried step (dt_step / dt_corrected)
    // hooks of the first right-hand side of a step: the SAVE_TRAJECT record and,
    // on the first step, the initial energies (MQCT_SOURCE_CODES/propagator.f:2695-2810)
    auto first_rhs = [&](double potv) {
      if (tid == 0 && out.rec && !at) save_record(out, tr, bk->n_rec, tcur, *C, potv);
      if (counter == 1 && !at) {
        double q0 = 0.0, z1 = 0.0, z2 = 0.0;
#pragma unroll
        for (int q = 0; q < NS; ++q)
          if (q < ns) {
            const int i = tid + q * TPB;
            q0 += (y[q].x * y[q].x + y[q].y * y[q].y) * d.e_val[d.st_e[i]];
          }
        block_sum3<TPB>(q0, z1, z2, sm.red);
        if (tid == 0) {
          bk->eqi = q0 + potv;
          bk->eki = kinetic(*C, d.mass);
        }
      }
    };
    while (bk->run) {
      ++counter;
      bool last = false;
      double h6 = 0.0;
      if constexpr (kAdaptive) {
        // ---- ODEINT (MQCT_SOURCE_CODES/suppl_routines.f:1229-1435; called per step dt at
        // propagator.f:3933, over the whole AT path at :3900).  All threads take the same
        // control decisions from block-wide values.
        // bikram_int (bk_int / bk_int_adia, MQCT_SOURCE_CODES/suppl_routines.f:1468-1856):
        // one call over [t, TIME_LIM] (standard) or the whole path (AT) that stops after
        // any step at which R > R_fin, the R oscillations or the orbits reach their caps
        const double x1 = tcur, x2 = at ? t_end : (d.bk_int ? ti->time_lim : tcur + dt);
        double x = x1, h = dt_step, hnext = dt_step;
        double bk_r1 = 0.0, bk_r2 = 0.0;
        int bk_vib = 0;
        double2 k2[NS], k3[NS], k4[NS], k5[NS], yo[NS], ye[NS];
        // stage input: amplitudes y + h * (combination) into a_in, classical into CT
        auto set_stage = [&](double ts, auto comb, auto ccomb) {
#pragma unroll
          for (int q = 0; q < NS; ++q)
            if (q < ns) sm.a_in[tid + q * TPB] = comb(q);
          if (tid == 0) {
            if (at) classical_at(d, tr, ts, CT);
            else {
              Cls c;
              for (int i = 0; i < 6; ++i) cls_ref(c, i) = ccomb(i);
              *CT = c;
            }
          }
          __syncthreads();
        };
        for (int nstp = 1; nstp <= kOdeMaxSteps; ++nstp) {
          double potv;
          set_stage(x, [&](int q) { return y[q]; }, [&](int i) { return cls_get(*C, i); });
          rhs<T, NS, TPB>(d, sm, x, CT, ns, k1, KC, potv);
          if (tid == 0) *K1 = *KC;
          if (nstp == 1) first_rhs(potv);
          if (nstp == kOdeMaxSteps) {
            // the last allowed step: RK4 over what remains (odeint's last_step branch)
            const double hr = x2 - x, hh = hr * 0.5, h6r = hr / 6.0, xh = x + hh;
            set_stage(xh, [&](int q) { return make_double2(y[q].x + hh * k1[q].x, y[q].y + hh * k1[q].y); },
                      [&](int i) { return cls_get(*C, i) + hh * cls_get(*K1, i); });
            rhs<T, NS, TPB>(d, sm, xh, CT, ns, k2, KC, potv);
            if (tid == 0) KS[0] = *KC;
            set_stage(xh, [&](int q) { return make_double2(y[q].x + hh * k2[q].x, y[q].y + hh * k2[q].y); },
                      [&](int i) { return cls_get(*C, i) + hh * cls_get(KS[0], i); });
            rhs<T, NS, TPB>(d, sm, xh, CT, ns, k3, KC, potv);
            if (tid == 0) KS[1] = *KC;
            set_stage(x + hr, [&](int q) { return make_double2(y[q].x + hr * k3[q].x, y[q].y + hr * k3[q].y); },
                      [&](int i) { return cls_get(*C, i) + hr * cls_get(KS[1], i); });
            rhs<T, NS, TPB>(d, sm, x + hr, CT, ns, k4, KC, potv);
#pragma unroll
            for (int q = 0; q < NS; ++q)
              if (q < ns) {
                const double2 m = make_double2(k2[q].x + k3[q].x, k2[q].y + k3[q].y);
                y[q] = make_double2(y[q].x + h6r * (k1[q].x + k4[q].x + 2.0 * m.x),
                                    y[q].y + h6r * (k1[q].y + k4[q].y + 2.0 * m.y));
              }
            if (tid == 0 && !at)
              for (int i = 0; i < 6; ++i)
                cls_ref(*C, i) += h6r * (cls_get(*K1, i) + cls_get(*KC, i) +
                                         2.0 * (cls_get(KS[0], i) + cls_get(KS[1], i)));
            __syncthreads();
            x = x2;
            break;
          }
          const double hs = h;  // the error scale uses the step before it is cut
          if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
          for (;;) {  // rkqs: Cash-Karp trial steps until the error is within eps
            set_stage(x + .2 * h,
                      [&](int q) { return make_double2(y[q].x + kCkB21 * h * k1[q].x, y[q].y + kCkB21 * h * k1[q].y); },
                      [&](int i) { return cls_get(*C, i) + kCkB21 * h * cls_get(*K1, i); });
            rhs<T, NS, TPB>(d, sm, x + .2 * h, CT, ns, k2, KC, potv);
            if (tid == 0) KS[0] = *KC;
            set_stage(x + .3 * h,
                      [&](int q) {
                        return make_double2(y[q].x + h * (kCkB31 * k1[q].x + kCkB32 * k2[q].x),
                                            y[q].y + h * (kCkB31 * k1[q].y + kCkB32 * k2[q].y));
                      },
                      [&](int i) {
                        return cls_get(*C, i) + h * (kCkB31 * cls_get(*K1, i) + kCkB32 * cls_get(KS[0], i));
                      });
            rhs<T, NS, TPB>(d, sm, x + .3 * h, CT, ns, k3, KC, potv);
            if (tid == 0) KS[1] = *KC;
            set_stage(x + kCkA4 * h,
                      [&](int q) {
                        return make_double2(
                            y[q].x + h * (kCkB41 * k1[q].x + kCkB42 * k2[q].x + kCkB43 * k3[q].x),
                            y[q].y + h * (kCkB41 * k1[q].y + kCkB42 * k2[q].y + kCkB43 * k3[q].y));
                      },
                      [&](int i) {
                        return cls_get(*C, i) + h * (kCkB41 * cls_get(*K1, i) + kCkB42 * cls_get(KS[0], i) +
                                                     kCkB43 * cls_get(KS[1], i));
                      });
            rhs<T, NS, TPB>(d, sm, x + kCkA4 * h, CT, ns, k4, KC, potv);
            if (tid == 0) KS[2] = *KC;
            set_stage(x + 1.0 * h,
                      [&](int q) {
                        return make_double2(y[q].x + h * (kCkB51 * k1[q].x + kCkB52 * k2[q].x +
                                                          kCkB53 * k3[q].x + kCkB54 * k4[q].x),
                                            y[q].y + h * (kCkB51 * k1[q].y + kCkB52 * k2[q].y +
                                                          kCkB53 * k3[q].y + kCkB54 * k4[q].y));
                      },
                      [&](int i) {
                        return cls_get(*C, i) + h * (kCkB51 * cls_get(*K1, i) + kCkB52 * cls_get(KS[0], i) +
                                                     kCkB53 * cls_get(KS[1], i) + kCkB54 * cls_get(KS[2], i));
                      });
            rhs<T, NS, TPB>(d, sm, x + 1.0 * h, CT, ns, k5, KC, potv);
            if (tid == 0) KS[3] = *KC;
            set_stage(x + .875 * h,
                      [&](int q) {
                        return make_double2(
                            y[q].x + h * (kCkB61 * k1[q].x + kCkB62 * k2[q].x + kCkB63 * k3[q].x +
                                          kCkB64 * k4[q].x + kCkB65 * k5[q].x),
                            y[q].y + h * (kCkB61 * k1[q].y + kCkB62 * k2[q].y + kCkB63 * k3[q].y +
                                          kCkB64 * k4[q].y + kCkB65 * k5[q].y));
                      },
                      [&](int i) {
                        return cls_get(*C, i) + h * (kCkB61 * cls_get(*K1, i) + kCkB62 * cls_get(KS[0], i) +
                                                     kCkB63 * cls_get(KS[1], i) + kCkB64 * cls_get(KS[2], i) +
                                                     kCkB65 * cls_get(KS[3], i));
                      });
            rhs<T, NS, TPB>(d, sm, x + .875 * h, CT, ns, k, KC, potv);  // k = stage 6
            double em = 0.0;
#pragma unroll
            for (int q = 0; q < NS; ++q)
              if (q < ns) {
                yo[q] = make_double2(
                    y[q].x + h * (kCkC1 * k1[q].x + kCkC3 * k3[q].x + kCkC4 * k4[q].x + kCkC6 * k[q].x),
                    y[q].y + h * (kCkC1 * k1[q].y + kCkC3 * k3[q].y + kCkC4 * k4[q].y + kCkC6 * k[q].y));
                ye[q] = make_double2(h * (kCkDC1 * k1[q].x + kCkDC3 * k3[q].x + kCkDC4 * k4[q].x +
                                          kCkDC5 * k5[q].x + kCkDC6 * k[q].x),
                                     h * (kCkDC1 * k1[q].y + kCkDC3 * k3[q].y + kCkDC4 * k4[q].y +
                                          kCkDC5 * k5[q].y + kCkDC6 * k[q].y));
                em = fmax(em, fabs(ye[q].x / (fabs(y[q].x) + fabs(hs * k1[q].x) + 1e-30)));
                em = fmax(em, fabs(ye[q].y / (fabs(y[q].y) + fabs(hs * k1[q].y) + 1e-30)));
              }
            if (tid == 0 && !at) {
              Cls o, e;
              for (int i = 0; i < 6; ++i) {
                const double c1 = cls_get(*K1, i), c3 = cls_get(KS[1], i), c4 = cls_get(KS[2], i),
                             c5 = cls_get(KS[3], i), c6 = cls_get(*KC, i), c0 = cls_get(*C, i);
                cls_ref(o, i) = c0 + h * (kCkC1 * c1 + kCkC3 * c3 + kCkC4 * c4 + kCkC6 * c6);
                cls_ref(e, i) = h * (kCkDC1 * c1 + kCkDC3 * c3 + kCkDC4 * c4 + kCkDC5 * c5 + kCkDC6 * c6);
                em = fmax(em, fabs(cls_get(e, i) / (fabs(c0) + fabs(hs * c1) + 1e-30)));
              }
              *CO = o;
              *CE = e;
            }
            if (h <= d.ode_hmin) break;  // at or below the minimum step: accepted as it is
            em = block_max<TPB>(em, sm.red) / d.ode_eps;
            if (em > 1.0) {
              const double htemp = 0.9 * h * pow(em, -0.25);
              h = fmax(fabs(htemp), 0.1 * fabs(h));
              continue;
            }
            hnext = em > 1.89e-4 ? 0.9 * h * pow(em, -0.2) : 5.0 * h;
            break;
          }
          x = x + h;
#pragma unroll
          for (int q = 0; q < NS; ++q)
            if (q < ns) y[q] = yo[q];
          if (tid == 0 && !at) *C = *CO;
          if (d.bk_int) {
            if (tid == 0) {
              // R and phi of the step's end: the classical state, or the AT path's splines
              const double* rec = at ? d.at_rec + 8 * d.at_off[tr] : nullptr;
              const double* y2p = at ? d.at_y2 + kAtCols * d.at_off[tr] : nullptr;
              const double rr = at ? at_splint(rec, y2p, d.at_n[tr], 1, 0, x) : C->R;
              const double ph = at ? at_splint(rec, y2p, d.at_n[tr], 5, 5, x) : C->phi;
              bool stop = rr > ti->r_fin;
              if (!stop) {
                if (nstp > 2 && (bk_r2 - bk_r1) < 0.0 && (bk_r1 - rr) > 0.0) ++bk_vib;
                bk_r2 = bk_r1;
                bk_r1 = rr;
                stop = bk_vib >= ti->numb_oscl_prds;
                if (!stop) {
                  bk->period = (int)(fabs(ph) / 2.0 / kPi);
                  stop = ti->numb_orb_prds <= bk->period;
                }
              }
              bk->vib = bk_vib;
              sm.flag[1] = stop ? 1 : 0;
            }
            __syncthreads();
            if (sm.flag[1]) break;
          }
          __syncthreads();
          if ((x - x2) * (x2 - x1) >= 0.0) break;
          if (fabs(hnext) < d.ode_hmin) hnext = d.ode_hmin;
          h = hnext;
        }
        dt_step = hnext;
        if (at || d.bk_int) {
          last = true;
          dt = x - tcur;  // the path's end, or where bk_int stopped
        }
      } else {
      if (at && d.at_adapt) {
        if (tid == 0) {
          bool lst = false;
          bk->at_dt = at_adapt_step(d, tr, tcur, t_end, bk->at_magic, bk->at_fa, lst);
          bk->run = lst ? 0 : 1;
        }
        __syncthreads();
        dt = bk->at_dt;
        last = bk->run == 0;
        __syncthreads();
      } else if (at && tcur + dt >= t_end) {
        dt = t_end - tcur;
        last = true;
      }
      const double hh = dt * 0.5;
      h6 = dt / 6.0;
      // RK4 (MQCT_SOURCE_CODES/suppl_routines.f:1076-1113): stage s evaluates
      // at t + {0, h/2, h/2, h} and y + {0, h/2 k1, h/2 k2, h k3}
      for (int st = 0; st < 4; ++st) {
        const double cst = st == 0 ? 0.0 : (st == 3 ? dt : hh);
        const double tst = tcur + cst;
#pragma unroll
        for (int q = 0; q < NS; ++q)
          if (q < ns)
            sm.a_in[tid + q * TPB] =
                st == 0 ? y[q] : make_double2(y[q].x + cst * k[q].x, y[q].y + cst * k[q].y);
        if (tid == 0) {
          if (at) classical_at(d, tr, tst, CT);
          else *CT = st == 0 ? *C : cls_axpy(*C, cst, *KC);
        }
        __syncthreads();
        double potv;
        rhs<T, NS, TPB>(d, sm, tst, CT, ns, k, KC, potv);
        if (st == 0) {
#pragma unroll
          for (int q = 0; q < NS; ++q) k1[q] = k[q];
          if (tid == 0) *K1 = *KC;
          first_rhs(potv);  // record of the state before the step; initial energies
        } else if (st == 1) {
#pragma unroll
          for (int q = 0; q < NS; ++q) k23[q] = k[q];
          if (tid == 0) *K23 = *KC;
        } else if (st == 2) {
#pragma unroll
          for (int q = 0; q < NS; ++q) k23[q] = make_double2(k23[q].x + k[q].x, k23[q].y + k[q].y);
          if (tid == 0) *K23 = cls_axpy(*K23, 1.0, *KC);
        }
      }
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (q < ns)
          y[q] = make_double2(y[q].x + h6 * (k1[q].x + k[q].x + 2.0 * k23[q].x),
                              y[q].y + h6 * (k1[q].y + k[q].y + 2.0 * k23[q].y));
      }
      if (kAdaptive && at && !d.bk_int) tcur = t_end;
      else tcur += dt;
      if (tid == 0) {
        bool run = !last;
        if (!at) {
          Cls& c = *C;
          if constexpr (!kAdaptive) {  // the RK4 step of the classical variables
            const Cls &a1 = *K1, &a23 = *K23, &a4 = *KC;
            c.R += h6 * (a1.R + a4.R + 2.0 * a23.R);
            c.PR += h6 * (a1.PR + a4.PR + 2.0 * a23.PR);
            c.th += h6 * (a1.th + a4.th + 2.0 * a23.th);
            c.Pth += h6 * (a1.Pth + a4.Pth + 2.0 * a23.Pth);
            c.phi += h6 * (a1.phi + a4.phi + 2.0 * a23.phi);
            c.Pphi += h6 * (a1.Pphi + a4.Pphi + 2.0 * a23.Pphi);
          }
          // stop rules, MQCT_SOURCE_CODES/propagator.f:4011-4050
          const double uR = c.R;
          if (tcur - dt > dt && counter > 2) {
            if ((bk->tmpR2 - bk->tmpR1) < 0.0 && (bk->tmpR1 - uR) > 0.0) bk->vib += 1;
          }
          bk->tmpR2 = bk->tmpR1;
          bk->tmpR1 = uR;
          bk->period = (int)(fabs(c.phi) / 2.0 / kPi);
          if (ti->numb_orb_prds <= bk->period) run = false;
          if (bk->vib >= ti->numb_oscl_prds) run = false;
          if (ti->time_lim > 0 && tcur >= ti->time_lim) run = false;
          if (uR > ti->r_fin) run = false;
          if (!(uR == uR)) {
            run = false;
            bk->status = 3;
          }
        }
        if (run && ti->max_steps > 0 && counter >= ti->max_steps) {
          run = false;
          bk->status = 1;
        }
        bk->run = run ? 1 : 0;
      }
      __syncthreads();
    }
    double pot_end = 0.0, eerr = 0.0;
    if (!at && !skipped) {  // final energy bookkeeping, MQCT_SOURCE_CODES/propagator.f:4182-4343
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (q < ns) sm.a_in[tid + q * TPB] = y[q];
      if (tid == 0) *CT = *C;
      __syncthreads();
      rhs<T, NS, TPB>(d, sm, tcur, CT, ns, k, KC, pot_end);
      double eqf = 0.0, z1 = 0.0, z2 = 0.0;
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (q < ns) {
          const int i = tid + q * TPB;
          eqf += (y[q].x * y[q].x + y[q].y * y[q].y) * d.e_val[d.st_e[i]];
        }
      block_sum3<TPB>(eqf, z1, z2, sm.red);
      eerr = fabs(eqf + kinetic(*C, d.mass) + pot_end - bk->eki - bk->eqi);
      // the closing record carries the final state stamped one step later
      if (tid == 0 && out.rec) save_record(out, tr, bk->n_rec, tcur + dt, *C, pot_end);
    }
    double nrm = 0.0, z1 = 0.0, z2 = 0.0;
#pragma unroll
    for (int q = 0; q < NS; ++q)
      if (q < ns) nrm += y[q].x * y[q].x + y[q].y * y[q].y;
    block_sum3<TPB>(nrm, z1, z2, sm.red);
    double* amp = out.amp + (size_t)tr * 2 * N;
#pragma unroll
    for (int q = 0; q < NS; ++q)
      if (q < ns) {
        const int i = d.perm[tid + q * TPB];
        amp[i] = y[q].x;
        amp[N + i] = y[q].y;
      }
    if (tid == 0) {
      const Cls& c = *C;
      double* cl = out.cls + (size_t)tr * 6;
      cl[0] = c.R; cl[1] = c.PR; cl[2] = c.th; cl[3] = c.Pth; cl[4] = c.phi; cl[5] = c.Pphi;
      double* dg = out.diag + (size_t)tr * 8;
      dg[0] = tcur;
      dg[1] = (double)counter;
      dg[2] = bk->status == 2 ? 0.0 : fabs(1.0 - nrm);
      dg[3] = eerr;
      dg[4] = bk->status;
      dg[5] = bk->period;
      dg[6] = bk->vib;
      dg[7] = pot_end;
      if (out.n_rec) out.n_rec[tr] = bk->n_rec;
    }
  }
}

// ------------------------------------------------------------------ plan
struct PropPlan {
  int arith = MQCT_PROP_FP32;
  int N = 0, P = 0, nR = 0, n_blocks = 0, n_e = 0, n_pass = 0, mp_cap = 0;
  int64_t S = 0;
  double mass = 0.0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<double> d_R, d_e_val, d_cplus, d_cminus;
  DevBuf<int> d_pass_row0, d_st_blk, d_blk_n, d_blk_s0, d_blk_mp, d_st_e, d_nbp, d_nbm, d_perm,
      d_inv, d_queue, d_status;
  DevBuf<int64_t> d_pass_slot0, d_blk_slot0;
  DevBuf<int> d_blk_pass;
  DevBuf<uint32_t> d_loc;
  DevBuf<float2> d_knots32;
  DevBuf<double2> d_knots64;
  DevBuf<mqct_traj_init_t> d_init;
  DevBuf<double> d_amp, d_cls, d_diag;
  // AT
  DevBuf<int64_t> d_at_off;
  DevBuf<int> d_at_n;
  DevBuf<double> d_at_rec, d_at_y2;
  int n_sm = 148, dev_smem = 0, sm_smem = 0;
  int ns = 1;        // states per thread, power of two
  int tpb = PT;      // threads per CTA of the launch shape
  int per_sm = 1;    // CTAs (trajectories) per SM the shape is laid out for
  bool tuned = false;
  float tune_ms[2] = {0.f, 0.f};  // probe times of the shapes (512 x 1, 256 x 2)
  // host copies of the block structure (the pass layout is rebuilt per shape)
  std::vector<int> h_blk_n, h_blk_s0;
  std::vector<int64_t> h_blk_slot0;

  int method = MQCT_INTEG_RK4;
  double ode_eps = 1e-6, ode_hmin = 0.0;
  // engine choice (MQCT_ENGINE_*), the engine of the last run and the lockstep engine
  int engine = MQCT_ENGINE_AUTO;
  int last_engine = 0;
  LsEngine* ls = nullptr;
  RsEngine* rs = nullptr;
  int rs_cl = 0;  // cluster size asked for the resident engine (0: the smallest that fits)
  bool cs = false;  // CS_APPROX for every run of the plan
  int bk_int = 0;                       // bikram_int (ODEINT with per-step stop rules)
  int at_adapt = 0;                     // AT_ADAPT_STP (RK4 steps of AT runs)
  double at_tol = 0.5, at_mintm = 0.0;  // AT_ADAPTOL, TIME_STEP

  template <class T, bool A, int TB>
  static const void* pick_tb(int ns) {
    if constexpr (TB == 512) {
      switch (ns) {
        case 1: return (const void*)propagate_kernel<T, 1, A, 512>;
        case 2: return (const void*)propagate_kernel<T, 2, A, 512>;
        case 4: return (const void*)propagate_kernel<T, 4, A, 512>;
        default: return (const void*)propagate_kernel<T, 8, A, 512>;
      }
    } else {
      switch (ns) {
        case 1:
        case 2: return (const void*)propagate_kernel<T, 2, A, 256>;
        case 4: return (const void*)propagate_kernel<T, 4, A, 256>;
        case 8: return (const void*)propagate_kernel<T, 8, A, 256>;
        default: return (const void*)propagate_kernel<T, 16, A, 256>;
      }
    }
  }
  const void* kernel_ptr() const {
    if (method == MQCT_INTEG_ODEINT)  // the adaptive kernel keeps the one-CTA shape
      return arith == MQCT_PROP_FP32 ? pick_tb<float, true, 512>(ns) : pick_tb<double, true, 512>(ns);
    if (tpb == 256)
      return arith == MQCT_PROP_FP32 ? pick_tb<float, false, 256>(ns) : pick_tb<double, false, 256>(ns);
    return arith == MQCT_PROP_FP32 ? pick_tb<float, false, 512>(ns) : pick_tb<double, false, 512>(ns);
  }

  int set_integrator(const mqct_integrator_t* in) {
    MQCT_ARG_CHECK(in, "null integrator");
    MQCT_ARG_CHECK(in->method == MQCT_INTEG_RK4 || in->method == MQCT_INTEG_ODEINT ||
                       in->method == MQCT_INTEG_AT_ADAPT || in->method == MQCT_INTEG_BK_INT,
                   "unknown integrator %d", in->method);
    at_adapt = 0;
    bk_int = in->method == MQCT_INTEG_BK_INT ? 1 : 0;
    if (in->method == MQCT_INTEG_AT_ADAPT) {
      // RK4 whose AT steps follow AT_ADAPT_STP; eps = AT_ADAPTOL, hmin = TIME_STEP
      MQCT_ARG_CHECK(in->eps > 0.0 && in->hmin > 0.0,
                     "AT_ADAPT_STP needs AT_ADAPTOL (eps) > 0 and TIME_STEP (hmin) > 0");
      at_adapt = 1;
      at_tol = in->eps;
      at_mintm = in->hmin;
      method = MQCT_INTEG_RK4;
      MQCT_CUDA_TRY(cudaFuncSetAttribute(kernel_ptr(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes()));
      return MQCT_OK;
    }
    if (in->method == MQCT_INTEG_ODEINT || in->method == MQCT_INTEG_BK_INT) {
      MQCT_ARG_CHECK(in->eps > 0.0 && in->hmin >= 0.0, "ODEINT needs eps > 0 and hmin >= 0");
      // the error control resolves every component to relative eps of |y| + |h dy/dt|;
      // FP32 rounding of the right-hand side (matrix, phases) leaves an error estimate
      // for small amplitudes that does not shrink with h, so the steps collapse
      MQCT_ARG_CHECK(arith == MQCT_PROP_FP64,
                     "ODEINT needs FP64 arithmetic (FP32 rounding of the right-hand side "
                     "defeats its error control on small amplitudes)");
    }
    method = in->method == MQCT_INTEG_BK_INT ? MQCT_INTEG_ODEINT : in->method;
    ode_eps = in->eps;
    ode_hmin = in->hmin;
    if (method == MQCT_INTEG_ODEINT && tpb != PT) return set_shape(PT, 1);
    MQCT_CUDA_TRY(cudaFuncSetAttribute(kernel_ptr(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_bytes()));
    return MQCT_OK;
  }
  size_t tsize() const { return arith == MQCT_PROP_FP32 ? 4 : 8; }

  // Shared memory without the packed-triangle area.
  size_t smem_fixed() const {
    const size_t t2 = 2 * tsize();
    auto a = [](size_t x) { return (x + 15) & ~size_t(15); };
    return a(sizeof(Cls) * kClsSlots) + a(sizeof(Book)) + a(sizeof(double) * 3 * (tpb / 32 + 1)) +
           a(sizeof(SplineAt)) + a(64) + a(16) +
           a(8 * (size_t)nR) +
           a(16 * (size_t)N) + 3 * a(t2 * N) + a(t2 * n_e);
  }
  size_t smem_bytes() const { return smem_fixed() + ((tsize() * (size_t)mp_cap + 15) & ~size_t(15)); }

  int init(const mqct_tables_t* tab, int32_t ar) {
    MQCT_ARG_CHECK(tab && tab->j12 && tab->m12 && tab->ej && tab->ind_mat && tab->R &&
                       tab->mat && tab->y2,
                   "null table argument");
    MQCT_ARG_CHECK(ar == MQCT_PROP_FP32 || ar == MQCT_PROP_FP64, "unknown arithmetic %d", ar);
    MQCT_ARG_CHECK(tab->n_states > 0 && tab->n_states <= MAX_N,
                   "n_states %d beyond the kernel limit %d", tab->n_states, MAX_N);
    MQCT_ARG_CHECK(tab->P > 0 && tab->P < (1 << 30) && tab->nR >= 2, "bad P/nR");
    MQCT_ARG_CHECK(tab->mass_au > 0, "mass must be positive");
    for (int i = 0; i + 1 < tab->nR; ++i)
      MQCT_ARG_CHECK(tab->R[i + 1] > tab->R[i], "R grid must increase");
    arith = ar;
    N = tab->n_states;
    P = (int)tab->P;
    nR = tab->nR;
    mass = tab->mass_au;
    MQCT_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    MQCT_CUDA_TRY(cudaEventCreate(&ev0));
    MQCT_CUDA_TRY(cudaEventCreate(&ev1));
    int dev = 0;
    MQCT_CUDA_TRY(cudaGetDevice(&dev));
    MQCT_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    MQCT_CUDA_TRY(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    MQCT_CUDA_TRY(cudaDeviceGetAttribute(&sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    // m-blocks; internal order = blocks in ascending m, reference order inside
    std::map<int, std::vector<int>> by_m;
    for (int s = 0; s < N; ++s) by_m[tab->m12[s]].push_back(s);
    std::vector<int> local(N), blk_of(N), blk_n, blk_s0, perm, inv(N), st_blk(N);
    std::vector<int64_t> blk_slot0;
    int64_t slots = 0;
    for (auto& kv : by_m) {
      const int b = (int)blk_n.size();
      const int n = (int)kv.second.size();
      blk_n.push_back(n);
      blk_s0.push_back((int)perm.size());
      blk_slot0.push_back(slots);
      slots += (((int64_t)n * (n + 1) / 2) + 3) & ~int64_t(3);
      for (int l = 0; l < n; ++l) {
        const int s = kv.second[l];
        local[s] = l;
        blk_of[s] = b;
        st_blk[perm.size()] = b;
        inv[s] = (int)perm.size();
        perm.push_back(s);
      }
    }
    n_blocks = (int)blk_n.size();
    S = slots;
    MQCT_ARG_CHECK(S < ((int64_t)1 << 30), "%lld table slots beyond the kernel limit", (long long)S);
    // energy classes (needed for the shared-memory size)
    std::vector<double> e_val;
    std::vector<int> st_e(N);
    for (int ii = 0; ii < N; ++ii) {
      const int s = perm[ii];
      int c = -1;
      for (size_t q = 0; q < e_val.size(); ++q)
        if (e_val[q] == tab->ej[s]) {
          c = (int)q;
          break;
        }
      if (c < 0) {
        c = (int)e_val.size();
        e_val.push_back(tab->ej[s]);
      }
      st_e[ii] = c;
    }
    n_e = (int)e_val.size();
    h_blk_n = blk_n;
    h_blk_s0 = blk_s0;
    h_blk_slot0 = blk_slot0;
    {
      const int rc = layout();
      if (rc) return rc;
    }
    // slots of the stored pairs; every other slot keeps zero knots
    std::vector<int> slot_pair(S, -1);
    std::vector<uint32_t> loc(S, 0u);
    for (int b = 0; b < n_blocks; ++b)
      for (int i = 0; i < blk_n[b]; ++i)
        for (int j = 0; j <= i; ++j)
          loc[blk_slot0[b] + (int64_t)i * (i + 1) / 2 + j] =
              (uint32_t)(blk_s0[b] + i) | ((uint32_t)(blk_s0[b] + j) << 16);
    for (int k = 0; k < P; ++k) {
      const int s1 = tab->ind_mat[2 * k] - 1, s2 = tab->ind_mat[2 * k + 1] - 1;
      MQCT_ARG_CHECK(s1 >= 0 && s1 < N && s2 >= 0 && s2 < N, "ind_mat out of range at k=%d", k + 1);
      MQCT_ARG_CHECK(tab->m12[s1] == tab->m12[s2], "pair with different m12 at k=%d", k + 1);
      const int b = blk_of[s1];
      const int i = std::max(local[s1], local[s2]), j = std::min(local[s1], local[s2]);
      const int64_t slot = blk_slot0[b] + (int64_t)i * (i + 1) / 2 + j;
      MQCT_ARG_CHECK(slot_pair[slot] < 0, "pair %d repeats pair %d", k + 1, slot_pair[slot] + 1);
      slot_pair[slot] = k;
    }
    if (arith == MQCT_PROP_FP32) {
      std::vector<float2> kn((size_t)nR * S, make_float2(0.f, 0.f));
      for (int64_t q = 0; q < S; ++q)
        if (slot_pair[q] >= 0)
          for (int r = 0; r < nR; ++r) {
            const size_t src = (size_t)slot_pair[q] * nR + r;
            kn[(size_t)r * S + q] = make_float2((float)tab->mat[src], (float)tab->y2[src]);
          }
      MQCT_CUDA_TRY(d_knots32.upload(kn, stream));
      MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    } else {
      std::vector<double2> kn((size_t)nR * S, make_double2(0.0, 0.0));
      for (int64_t q = 0; q < S; ++q)
        if (slot_pair[q] >= 0)
          for (int r = 0; r < nR; ++r) {
            const size_t src = (size_t)slot_pair[q] * nR + r;
            kn[(size_t)r * S + q] = make_double2(tab->mat[src], tab->y2[src]);
          }
      MQCT_CUDA_TRY(d_knots64.upload(kn, stream));
      MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    // Coriolis neighbours: the reference couples a state with its successor and
    // predecessor in the reference state order (sqrt2 / sqrt1,
    // MQCT_SOURCE_CODES/mqct_eqtns.f:447-464); the coefficient vanishes where
    // the neighbour has another j12.
    std::vector<double> cp(N, 0.0), cm(N, 0.0);
    std::vector<int> nbp(N, -1), nbm(N, -1);
    for (int ii = 0; ii < N; ++ii) {
      const int s = perm[ii];
      const double J = tab->j12[s], m = tab->m12[s];
      if (s + 1 < N) {
        nbp[ii] = inv[s + 1];
        cp[ii] = sqrt(J * (J + 1.0) - (m + 1.0) * m);
      }
      if (s > 0) {
        nbm[ii] = inv[s - 1];
        cm[ii] = sqrt(J * (J + 1.0) - (m - 1.0) * m);
      }
    }
    MQCT_CUDA_TRY(d_R.upload(tab->R, nR, stream));
    MQCT_CUDA_TRY(d_e_val.upload(e_val, stream));
    MQCT_CUDA_TRY(d_cplus.upload(cp, stream));
    MQCT_CUDA_TRY(d_cminus.upload(cm, stream));
    MQCT_CUDA_TRY(d_nbp.upload(nbp, stream));
    MQCT_CUDA_TRY(d_nbm.upload(nbm, stream));
    MQCT_CUDA_TRY(d_st_blk.upload(st_blk, stream));
    MQCT_CUDA_TRY(d_blk_n.upload(blk_n, stream));
    MQCT_CUDA_TRY(d_blk_s0.upload(blk_s0, stream));
    {
      std::vector<int64_t> bs0(blk_slot0);
      bs0.push_back(S);
      MQCT_CUDA_TRY(d_blk_slot0.upload(bs0, stream));
    }
    MQCT_CUDA_TRY(d_loc.upload(loc, stream));
    MQCT_CUDA_TRY(d_st_e.upload(st_e, stream));
    MQCT_CUDA_TRY(d_perm.upload(perm, stream));
    MQCT_CUDA_TRY(d_inv.upload(inv, stream));
    MQCT_CUDA_TRY(d_queue.alloc(1));
    MQCT_CUDA_TRY(d_status.alloc(1));
    MQCT_CUDA_TRY(cudaMemsetAsync(d_status.p, 0, sizeof(int), stream));
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  // Pass layout for the current shape: consecutive m-blocks whose packed triangles fit
  // the shared memory one CTA of the shape may take (the SM's shared memory divided by
  // the CTAs per SM); uploads the pass tables and sets the kernel's launch limit.
  int layout() {
    ns = 1;
    while (ns * tpb < N) ns *= 2;
    const size_t fixed = smem_fixed();
    const size_t budget = std::min<size_t>((size_t)dev_smem,
                                           (size_t)sm_smem / (size_t)per_sm - 1024) & ~size_t(15);
    MQCT_ARG_CHECK(fixed + 1024 <= budget,
                   "shared memory of the state vectors (%zu B) beyond the per-CTA budget %zu", fixed,
                   budget);
    const int64_t cap = (int64_t)((budget - fixed) / tsize()) & ~int64_t(3);
    std::vector<int64_t> pass_slot0;
    std::vector<int> pass_row0, blk_mp(n_blocks), blk_pass(n_blocks);
    int64_t max_pass = 0;
    for (int b = 0; b < n_blocks; ++b) {
      const int64_t bs = (b + 1 < n_blocks ? h_blk_slot0[b + 1] : S) - h_blk_slot0[b];
      MQCT_ARG_CHECK(bs <= cap, "m-block of %d states does not fit in shared memory", h_blk_n[b]);
      if (pass_slot0.empty() || h_blk_slot0[b] + bs - pass_slot0.back() > cap) {
        pass_slot0.push_back(h_blk_slot0[b]);
        pass_row0.push_back(h_blk_s0[b]);
      }
      blk_mp[b] = (int)(h_blk_slot0[b] - pass_slot0.back());
      blk_pass[b] = (int)pass_slot0.size() - 1;
      max_pass = std::max(max_pass, h_blk_slot0[b] + bs - pass_slot0.back());
    }
    n_pass = (int)pass_slot0.size();
    pass_slot0.push_back(S);
    pass_row0.push_back(N);
    mp_cap = (int)max_pass;
    MQCT_CUDA_TRY(d_pass_row0.upload(pass_row0, stream));
    MQCT_CUDA_TRY(d_pass_slot0.upload(pass_slot0, stream));
    MQCT_CUDA_TRY(d_blk_mp.upload(blk_mp, stream));
    MQCT_CUDA_TRY(d_blk_pass.upload(blk_pass, stream));
    MQCT_CUDA_TRY(cudaFuncSetAttribute(kernel_ptr(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_bytes()));
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  int set_shape(int t, int c) {
    tpb = t;
    per_sm = c;
    return layout();
  }

  // Autotuning of the launch shape: both shapes (512 threads x 1 CTA per SM, 256 threads x
  // 2 CTAs per SM, each with its own pass layout) run a probe batch -- the first
  // trajectories of the caller's set, enough to fill the GPU twice, each capped at
  // kTuneSteps steps, results discarded -- and the faster one is kept for the plan.
  static constexpr int kTuneSteps = 32;
  int tune(const mqct_traj_init_t* init, int64_t n_traj, int mode) {
    if (method != MQCT_INTEG_RK4 || n_traj <= 0) return MQCT_OK;
    const int64_t n = std::min<int64_t>(n_traj, 4LL * n_sm);
    std::vector<mqct_traj_init_t> probe(init, init + n);
    for (auto& t : probe) {
      t.max_steps = kTuneSteps;
      t.time_lim = 0.0;
    }
    DevBuf<mqct_traj_init_t> d_probe;
    DevBuf<double> amp, cls, diag;
    MQCT_CUDA_TRY(d_probe.upload(probe.data(), (size_t)n, stream));
    MQCT_CUDA_TRY(amp.alloc((size_t)n * 2 * N));
    MQCT_CUDA_TRY(cls.alloc((size_t)n * 6));
    MQCT_CUDA_TRY(diag.alloc((size_t)n * 8));
    const int shapes[2][2] = {{512, 1}, {256, 2}};
    int best = 0;
    for (int k = 0; k < 2; ++k) {
      int rc = set_shape(shapes[k][0], shapes[k][1]);
      if (rc) return rc;
      float ms = 0.f;
      for (int rep = 0; rep < 2; ++rep) {  // the first launch of a shape loads its code
        rc = launch(d_probe.p, n, mode, amp.p, cls.p, diag.p);
        if (rc) return rc;
        MQCT_CUDA_TRY(cudaEventSynchronize(ev1));
        MQCT_CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
      }
      tune_ms[k] = ms;
      if (ms < tune_ms[best]) best = k;
    }
    tuned = true;
    return set_shape(shapes[best][0], shapes[best][1]);
  }

  PropDev dev_view(int mode) const {
    PropDev d{};
    d.N = N; d.nR = nR; d.n_e = n_e; d.n_pass = n_pass; d.S = S;
    d.R = d_R.p; d.pass_row0 = d_pass_row0.p; d.pass_slot0 = d_pass_slot0.p;
    d.st_blk = d_st_blk.p; d.blk_n = d_blk_n.p; d.blk_s0 = d_blk_s0.p; d.blk_mp = d_blk_mp.p;
    d.blk_slot0 = d_blk_slot0.p; d.blk_pass = d_blk_pass.p;
    d.loc = d_loc.p; d.st_e = d_st_e.p; d.e_val = d_e_val.p;
    d.nb_plus = d_nbp.p; d.nb_minus = d_nbm.p; d.cplus = d_cplus.p; d.cminus = d_cminus.p;
    d.perm = d_perm.p; d.inv_perm = d_inv.p;
    d.knots = arith == MQCT_PROP_FP32 ? (const void*)d_knots32.p : (const void*)d_knots64.p;
    d.mass = mass;
    d.inv_mass = 1.0 / mass;
    d.mode = mode & MQCT_MODE_AT;
    d.cs = ((mode & MQCT_MODE_CS) != 0) || cs;
    d.mp_cap = mp_cap;
    d.ode_eps = ode_eps;
    d.ode_hmin = ode_hmin;
    d.at_off = d_at_off.p; d.at_n = d_at_n.p; d.at_rec = d_at_rec.p; d.at_y2 = d_at_y2.p;
    d.at_adapt = at_adapt;
    d.bk_int = bk_int;
    d.at_tol = at_tol;
    d.at_mintm = at_mintm;
    return d;
  }

  // Algorithmic table bytes of one RK4 step: 4 right-hand sides, each reading
  // two knot rows and the slot locations.
  double bytes_per_step() const { return 4.0 * (double)S * (4.0 * tsize() + 4.0); }

  int launch(const mqct_traj_init_t* d_init_p, int64_t n_traj, int mode, double* amp,
             double* cls, double* diag, double* rec = nullptr, int64_t rec_cap = 0,
             int64_t* n_rec = nullptr) {
    MQCT_ARG_CHECK(n_traj > 0 && n_traj < (1 << 30), "n_traj out of range");
    last_engine = MQCT_ENGINE_PER_TRAJECTORY;
    MQCT_CUDA_TRY(cudaMemsetAsync(d_queue.p, 0, sizeof(int), stream));
    PropDev d = dev_view(mode);
    TrajOut o{amp, cls, diag, rec, rec_cap, n_rec};
    int n_traj_i = (int)n_traj;
    const size_t sb = smem_bytes();
    int per_sm = 1;
    const void* fn = kernel_ptr();
    MQCT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, tpb, sb));
    const int grid = (int)std::min<int64_t>(n_traj, (int64_t)n_sm * std::max(per_sm, 1));
    void* args[] = {&d, (void*)&d_init_p, &n_traj_i, &d_queue.p, &o};
    MQCT_CUDA_TRY(cudaEventRecord(ev0, stream));
    MQCT_CUDA_TRY(cudaLaunchKernel(fn, dim3(grid), dim3(tpb), args, sb, stream));
    MQCT_CUDA_TRY(cudaEventRecord(ev1, stream));
    return MQCT_OK;
  }

  int set_at(const mqct_at_paths_t* at, int64_t n_traj) {
    MQCT_ARG_CHECK(at && at->rec_off && at->n_rec && at->rec, "AT mode needs paths");
    int64_t total = 0;
    for (int64_t t = 0; t < n_traj; ++t) {
      MQCT_ARG_CHECK(at->n_rec[t] >= 4, "AT path %lld has fewer than 4 records", (long long)t);
      total = std::max(total, at->rec_off[t] + at->n_rec[t]);
    }
    // spline second derivatives of R, theta, P_theta, P_phi over t with
    // finite-difference end slopes (MQCT_SOURCE_CODES/propagator.f:3116-3125)
    std::vector<double> y2((size_t)total * kAtCols, 0.0), u;
    const int cols[kAtCols] = {1, 3, 4, 6, 7, 5};
    for (int64_t t = 0; t < n_traj; ++t) {
      const double* r = at->rec + 8 * at->rec_off[t];
      const int n = at->n_rec[t];
      for (int i = 0; i + 1 < n; ++i)
        MQCT_ARG_CHECK(r[8 * (i + 1)] > r[8 * i], "AT path %lld: time not increasing", (long long)t);
      u.assign(n, 0.0);
      for (int a = 0; a < kAtCols; ++a) {
        double* yy = y2.data() + kAtCols * at->rec_off[t];
        auto X = [&](int i) { return r[8 * i]; };
        auto Y = [&](int i) { return r[8 * i + cols[a]]; };
        const double yp1 = (Y(1) - Y(0)) / (X(1) - X(0));
        const double ypn = (Y(n - 1) - Y(n - 2)) / (X(n - 1) - X(n - 2));
        yy[a] = -0.5;
        u[0] = (3.0 / (X(1) - X(0))) * ((Y(1) - Y(0)) / (X(1) - X(0)) - yp1);
        for (int i = 1; i < n - 1; ++i) {
          const double sig = (X(i) - X(i - 1)) / (X(i + 1) - X(i - 1));
          const double p = sig * yy[kAtCols * (i - 1) + a] + 2.0;
          yy[kAtCols * i + a] = (sig - 1.0) / p;
          u[i] = (6.0 * ((Y(i + 1) - Y(i)) / (X(i + 1) - X(i)) - (Y(i) - Y(i - 1)) / (X(i) - X(i - 1))) /
                      (X(i + 1) - X(i - 1)) -
                  sig * u[i - 1]) /
                 p;
        }
        const double un =
            (3.0 / (X(n - 1) - X(n - 2))) * (ypn - (Y(n - 1) - Y(n - 2)) / (X(n - 1) - X(n - 2)));
        yy[kAtCols * (n - 1) + a] = (un - 0.5 * u[n - 2]) / (0.5 * yy[kAtCols * (n - 2) + a] + 1.0);
        for (int i = n - 2; i >= 0; --i) yy[kAtCols * i + a] = yy[kAtCols * i + a] * yy[kAtCols * (i + 1) + a] + u[i];
      }
    }
    MQCT_CUDA_TRY(d_at_off.upload(at->rec_off, n_traj, stream));
    MQCT_CUDA_TRY(d_at_n.upload(at->n_rec, n_traj, stream));
    MQCT_CUDA_TRY(d_at_rec.upload(at->rec, (size_t)total * 8, stream));
    MQCT_CUDA_TRY(d_at_y2.upload(y2, stream));
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  // The lockstep engine takes standard-mode RK4 runs without CS or SAVE_TRAJECT records
  // when every m-block has at most 128 states: always with MQCT_ENGINE_LOCKSTEP, from
  // kLockstepMinBatch trajectories with MQCT_ENGINE_AUTO.  Smaller batches share few knot
  // rows per interval, and every lockstep round costs its fixed latency however few
  // trajectories remain: on the 969-state asymmetric-top tables the per-trajectory kernel
  // is faster at 512 trajectories (5.0 s against 7.1 s), the lockstep engine at 4 096
  // (22.7 s against 24.1 s).
  static constexpr int64_t kLockstepMinBatch = 4096;
  bool use_lockstep(int mode, int64_t n_traj, bool records) const {
    if (engine == MQCT_ENGINE_PER_TRAJECTORY || records || mode != MQCT_MODE_STD || cs ||
        method != MQCT_INTEG_RK4 || !ls_eligible(h_blk_n))
      return false;
    return engine == MQCT_ENGINE_LOCKSTEP || engine == MQCT_ENGINE_LOCKSTEP_TAIL ||
           n_traj >= kLockstepMinBatch;
  }
  // The resident engine takes the runs the lockstep engine could take (FP32 only) when the
  // tables fit a cluster: always with MQCT_ENGINE_RESIDENT, up to kResidentMaxBatch
  // trajectories with MQCT_ENGINE_AUTO.  It gives each trajectory a cluster of CTAs, so a
  // trajectory's steps take less time than on the per-trajectory kernel, but fewer run at
  // once: on the 969-state asymmetric-top tables it is faster for 33 trajectories (0.64 s
  // against 1.97 s), 512 (4.55 s against 6.04 s) and 1024 (8.9 s against 10.7 s), slower
  // for 4096 (35.9 s against 24.2 s).  With the cluster size left to the plan, a batch that
  // fits the clusters of eight CTAs runs on them (shorter steps), a larger one on the
  // smallest cluster that holds the tables (more clusters).
  static constexpr int64_t kResidentMaxBatch = 1024;
  int rs_clusters8 = -1;  // clusters of eight CTAs resident on the device (-1: not asked yet)
  int last_rs[2] = {0, 0};  // cluster size and clusters of the last resident run
  bool use_resident(int mode, int64_t n_traj, bool records) {
    if (engine == MQCT_ENGINE_PER_TRAJECTORY || engine == MQCT_ENGINE_LOCKSTEP ||
        engine == MQCT_ENGINE_LOCKSTEP_TAIL || records ||
        mode != MQCT_MODE_STD || cs || method != MQCT_INTEG_RK4 || arith != MQCT_PROP_FP32)
      return false;
    if (engine == MQCT_ENGINE_AUTO && n_traj > kResidentMaxBatch) return false;
    if (!rs) rs = rs_create();
    const PropDev d = dev_view(MQCT_MODE_STD);
    int cl = rs_cl;
    if (!cl) {
      if (rs_clusters8 < 0) {
        rs_set_cluster(rs, 8);
        rs_clusters8 = rs_usable(rs, d, h_blk_n, h_blk_s0, stream) ? rs_clusters(rs) : 0;
      }
      cl = n_traj <= rs_clusters8 ? 8 : 0;
    }
    rs_set_cluster(rs, cl);
    return rs_usable(rs, d, h_blk_n, h_blk_s0, stream);
  }
  int run_resident(const mqct_traj_init_t* d_init_p, int64_t n_traj, double* amp, double* cls,
                   double* diag) {
    MQCT_ARG_CHECK(n_traj > 0 && n_traj < (1LL << 31), "n_traj out of range");
    last_engine = MQCT_ENGINE_RESIDENT;
    last_rs[0] = rs_cluster(rs);
    last_rs[1] = rs_clusters(rs);
    return rs_run(rs, dev_view(MQCT_MODE_STD), h_blk_n, h_blk_s0, stream, ev0, ev1, d_init_p,
                  (int)n_traj, amp, cls, diag);
  }
  // With MQCT_ENGINE_AUTO an FP32 lockstep run hands its last trajectories to the resident
  // engine: once at most kHandPerCluster per resident cluster still run, the lockstep
  // rounds, whose fixed cost no longer has trajectories to share it, stop, and each of the
  // remaining ones continues on a cluster of its own from the start of its RK4 step (the
  // long tail of the slowest trajectories: 58 k steps for the longest of the 4 096
  // benchmark trajectories against 9.6 k for the median).
  static constexpr int kHandPerCluster = 6;
  DevBuf<RsResume> d_hand;
  int last_handed = 0;  // trajectories the last lockstep run handed to the resident engine
  int run_lockstep(const mqct_traj_init_t* d_init_p, const mqct_traj_init_t* h_init,
                   int64_t n_traj, double* amp, double* cls, double* diag) {
    MQCT_ARG_CHECK(n_traj > 0 && n_traj < (1 << 24), "n_traj out of range for the lockstep engine");
    if (!ls) ls = ls_create();
    last_engine = MQCT_ENGINE_LOCKSTEP;
    last_handed = 0;
    const PropDev d = dev_view(MQCT_MODE_STD);
    int hand_below = 0;
    if ((engine == MQCT_ENGINE_AUTO || engine == MQCT_ENGINE_LOCKSTEP_TAIL) &&
        arith == MQCT_PROP_FP32) {
      if (!rs) rs = rs_create();
      rs_set_cluster(rs, rs_cl);
      if (rs_usable(rs, d, h_blk_n, h_blk_s0, stream)) {
        hand_below = kHandPerCluster * rs_clusters(rs);
        if (d_hand.n < (size_t)n_traj) MQCT_CUDA_TRY(d_hand.alloc((size_t)n_traj));
      }
    }
    int handed = 0;
    const double2* hand_amp = nullptr;
    int rc = ls_run(ls, d, arith == MQCT_PROP_FP32, h_blk_n, n_sm, stream, ev0, ev1, d_init_p,
                    h_init, (int)n_traj, amp, cls, diag, hand_below, d_hand.p, &handed,
                    &hand_amp);
    if (hand_below > 0) last_engine = MQCT_ENGINE_LOCKSTEP_TAIL;
    if (rc || handed == 0) return rc;
    last_handed = handed;
    last_rs[0] = rs_cluster(rs);
    last_rs[1] = rs_clusters(rs);
    return rs_run_resume(rs, d, h_blk_n, h_blk_s0, stream, ev1, d_init_p, d_hand.p, handed,
                         hand_amp, amp, cls, diag);
  }

  ~PropPlan() {
    if (ls) ls_destroy(ls);
    if (rs) rs_destroy(rs);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

static int validate_init(const mqct_traj_init_t* init, int64_t n, int N, int mode,
                         bool bk_int = false) {
  mode &= MQCT_MODE_AT;
  for (int64_t t = 0; t < n; ++t) {
    const mqct_traj_init_t& a = init[t];
    MQCT_ARG_CHECK(a.s_st >= 1 && a.s_st <= N, "trajectory %lld: s_st out of range", (long long)t);
    MQCT_ARG_CHECK(a.dt > 0, "trajectory %lld: dt must be positive", (long long)t);
    if (mode == MQCT_MODE_STD) {
      MQCT_ARG_CHECK(a.e_coll > 0 && a.l_real >= 0 && a.r_start > 0, "trajectory %lld: bad E/l/R",
                     (long long)t);
      MQCT_ARG_CHECK(a.max_steps > 0 || a.time_lim > 0,
                     "trajectory %lld: needs a step cap or a time limit", (long long)t);
      MQCT_ARG_CHECK(!bk_int || a.time_lim > 0,
                     "trajectory %lld: bk_int integrates up to TIME_LIM, which must be > 0",
                     (long long)t);
    }
  }
  return MQCT_OK;
}

// Host-buffer run: upload the initial conditions, launch, copy the results back
// (and the SAVE_TRAJECT records when rec_out is given).  In standard mode the
// trajectories go to the device queue longest first (estimated steps
// 2 r_start / (v dt), v the initial speed), so that the CTAs finish together instead
// of waiting for a slow trajectory taken last; the results return in the caller's
// order and do not depend on the order (one trajectory per CTA, no shared state).
static int run_host(PropPlan* p, const mqct_traj_init_t* init, int64_t n_traj, int mode,
                    double* amp_out, double* cls_out, double* diag_out,
                    double* rec_out = nullptr, int64_t rec_cap = 0, int64_t* n_rec_out = nullptr) {
  int rc = validate_init(init, n_traj, p->N, mode, p->bk_int != 0);
  if (rc) return rc;
  std::vector<int64_t> order(n_traj);
  for (int64_t t = 0; t < n_traj; ++t) order[t] = t;
  const bool reorder = (mode & MQCT_MODE_AT) == 0 && n_traj > 1;
  if (reorder) {
    std::vector<double> est(n_traj);
    for (int64_t t = 0; t < n_traj; ++t) {
      const mqct_traj_init_t& a = init[t];
      const double v = std::sqrt(2.0 * a.e_coll / p->mass);
      est[t] = 2.0 * a.r_start / (v * a.dt);
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t x, int64_t y) { return est[x] > est[y]; });
  }
  std::vector<mqct_traj_init_t> sorted(n_traj);
  for (int64_t t = 0; t < n_traj; ++t) sorted[t] = init[order[t]];
  const bool resident = p->use_resident(mode, n_traj, rec_out != nullptr);
  const bool lockstep = !resident && p->use_lockstep(mode, n_traj, rec_out != nullptr);
  if (!lockstep && !resident && !p->tuned && p->method == MQCT_INTEG_RK4 && n_traj >= 2LL * p->n_sm) {
    rc = p->tune(sorted.data(), n_traj, mode);
    if (rc) return rc;
  }
  MQCT_CUDA_TRY(p->d_init.upload(sorted.data(), n_traj, p->stream));
  MQCT_CUDA_TRY(p->d_amp.alloc((size_t)n_traj * 2 * p->N));
  MQCT_CUDA_TRY(p->d_cls.alloc((size_t)n_traj * 6));
  MQCT_CUDA_TRY(p->d_diag.alloc((size_t)n_traj * 8));
  if (resident) {
    rc = p->run_resident(p->d_init.p, n_traj, p->d_amp.p, p->d_cls.p, p->d_diag.p);
    if (rc) return rc;
  } else if (lockstep) {
    rc = p->run_lockstep(p->d_init.p, sorted.data(), n_traj, p->d_amp.p, p->d_cls.p, p->d_diag.p);
    if (rc) return rc;
  }
  DevBuf<double> d_rec;
  DevBuf<int64_t> d_nrec;
  if (rec_out) {
    MQCT_CUDA_TRY(d_rec.alloc((size_t)n_traj * rec_cap * 8));
    MQCT_CUDA_TRY(d_nrec.alloc((size_t)n_traj));
  }
  if (!lockstep && !resident) {
    rc = p->launch(p->d_init.p, n_traj, mode, p->d_amp.p, p->d_cls.p, p->d_diag.p, d_rec.p,
                   rec_cap, d_nrec.p);
    if (rc) return rc;
  }
  const size_t na = (size_t)2 * p->N;
  std::vector<double> amp(reorder ? (size_t)n_traj * na : 0), cls(reorder ? n_traj * 6 : 0),
      diag(reorder ? n_traj * 8 : 0), rec(reorder && rec_out ? (size_t)n_traj * rec_cap * 8 : 0);
  std::vector<int64_t> nrec(reorder && rec_out ? n_traj : 0);
  double* h_amp = reorder ? amp.data() : amp_out;
  double* h_cls = reorder ? cls.data() : cls_out;
  double* h_diag = reorder ? diag.data() : diag_out;
  double* h_rec = reorder ? rec.data() : rec_out;
  int64_t* h_nrec = reorder ? nrec.data() : n_rec_out;
  if (rec_out) {
    MQCT_CUDA_TRY(cudaMemcpyAsync(h_rec, d_rec.p, sizeof(double) * n_traj * rec_cap * 8,
                                  cudaMemcpyDeviceToHost, p->stream));
    MQCT_CUDA_TRY(cudaMemcpyAsync(h_nrec, d_nrec.p, sizeof(int64_t) * n_traj,
                                  cudaMemcpyDeviceToHost, p->stream));
  }
  MQCT_CUDA_TRY(cudaMemcpyAsync(h_amp, p->d_amp.p, sizeof(double) * n_traj * na,
                                cudaMemcpyDeviceToHost, p->stream));
  MQCT_CUDA_TRY(cudaMemcpyAsync(h_cls, p->d_cls.p, sizeof(double) * n_traj * 6,
                                cudaMemcpyDeviceToHost, p->stream));
  MQCT_CUDA_TRY(cudaMemcpyAsync(h_diag, p->d_diag.p, sizeof(double) * n_traj * 8,
                                cudaMemcpyDeviceToHost, p->stream));
  MQCT_CUDA_TRY(cudaStreamSynchronize(p->stream));
  if (reorder) {
    for (int64_t t = 0; t < n_traj; ++t) {
      const int64_t o = order[t];
      std::copy(amp.begin() + t * na, amp.begin() + (t + 1) * na, amp_out + o * na);
      std::copy(cls.begin() + t * 6, cls.begin() + (t + 1) * 6, cls_out + o * 6);
      std::copy(diag.begin() + t * 8, diag.begin() + (t + 1) * 8, diag_out + o * 8);
      if (rec_out) {
        const size_t rn = (size_t)rec_cap * 8;
        std::copy(rec.begin() + t * rn, rec.begin() + (t + 1) * rn, rec_out + o * rn);
        n_rec_out[o] = nrec[t];
      }
    }
  }
  return MQCT_OK;
}

}  // namespace mqct

extern "C" {

int mqct_prop_plan_create(const mqct_tables_t* tab, int32_t arith, mqct_prop_plan** plan) {
  MQCT_ARG_CHECK(plan, "null plan pointer");
  *plan = nullptr;
  if (mqct_device_count() <= 0) {
    set_error("no CUDA device available");
    return MQCT_E_NODEV;
  }
  auto* p = new PropPlan();
  int rc = p->init(tab, arith);
  if (rc) {
    delete p;
    return rc;
  }
  *plan = reinterpret_cast<mqct_prop_plan*>(p);
  return MQCT_OK;
}

int mqct_prop_plan_run_device(mqct_prop_plan* plan, const mqct_traj_init_t* d_init,
                              int64_t n_traj, double* d_amp, double* d_cls, double* d_diag) {
  MQCT_ARG_CHECK(plan && d_init && d_amp && d_cls && d_diag, "null argument");
  PropPlan* p = reinterpret_cast<PropPlan*>(plan);
  if (p->use_resident(MQCT_MODE_STD, n_traj, false)) {
    std::vector<mqct_traj_init_t> h((size_t)n_traj);
    MQCT_CUDA_TRY(cudaMemcpyAsync(h.data(), d_init, sizeof(mqct_traj_init_t) * n_traj,
                                  cudaMemcpyDeviceToHost, p->stream));
    MQCT_CUDA_TRY(cudaStreamSynchronize(p->stream));
    const int rc = validate_init(h.data(), n_traj, p->N, MQCT_MODE_STD);
    if (rc) return rc;
    return p->run_resident(d_init, n_traj, d_amp, d_cls, d_diag);
  }
  if (p->use_lockstep(MQCT_MODE_STD, n_traj, false)) {
    // the lockstep engine bounds its rounds by the trajectories' step caps and time limits
    MQCT_ARG_CHECK(n_traj > 0 && n_traj < (1 << 24), "n_traj out of range for the lockstep engine");
    std::vector<mqct_traj_init_t> h((size_t)n_traj);
    MQCT_CUDA_TRY(cudaMemcpyAsync(h.data(), d_init, sizeof(mqct_traj_init_t) * n_traj,
                                  cudaMemcpyDeviceToHost, p->stream));
    MQCT_CUDA_TRY(cudaStreamSynchronize(p->stream));
    const int rc = validate_init(h.data(), n_traj, p->N, MQCT_MODE_STD);
    if (rc) return rc;
    return p->run_lockstep(d_init, h.data(), n_traj, d_amp, d_cls, d_diag);
  }
  return p->launch(d_init, n_traj, MQCT_MODE_STD, d_amp, d_cls, d_diag);
}

int mqct_prop_plan_run(mqct_prop_plan* plan, const mqct_traj_init_t* init, int64_t n_traj,
                       double* amp_out, double* cls_out, double* diag_out) {
  MQCT_ARG_CHECK(plan && init && amp_out && cls_out && diag_out, "null argument");
  return run_host(reinterpret_cast<PropPlan*>(plan), init, n_traj, MQCT_MODE_STD, amp_out,
                  cls_out, diag_out);
}

int mqct_prop_plan_sync(mqct_prop_plan* plan) {
  MQCT_ARG_CHECK(plan, "null plan");
  MQCT_CUDA_TRY(cudaStreamSynchronize(reinterpret_cast<PropPlan*>(plan)->stream));
  return MQCT_OK;
}

double mqct_prop_plan_bytes_per_step(const mqct_prop_plan* plan) {
  if (!plan) return 0.0;
  return reinterpret_cast<const PropPlan*>(plan)->bytes_per_step();
}

int mqct_prop_plan_timing(mqct_prop_plan* plan, float* ms) {
  MQCT_ARG_CHECK(plan && ms, "null argument");
  PropPlan* p = reinterpret_cast<PropPlan*>(plan);
  MQCT_CUDA_TRY(cudaEventSynchronize(p->ev1));
  MQCT_CUDA_TRY(cudaEventElapsedTime(ms, p->ev0, p->ev1));
  return MQCT_OK;
}

void mqct_prop_plan_destroy(mqct_prop_plan* plan) { delete reinterpret_cast<PropPlan*>(plan); }

int mqct_prop_plan_tune(mqct_prop_plan* plan, const mqct_traj_init_t* init, int64_t n_traj,
                        int32_t mode) {
  MQCT_ARG_CHECK(plan && init && n_traj > 0, "null or empty argument");
  PropPlan* p = reinterpret_cast<PropPlan*>(plan);
  int rc = validate_init(init, n_traj, p->N, mode);
  if (rc) return rc;
  return p->tune(init, n_traj, mode);
}

int mqct_prop_plan_shape(const mqct_prop_plan* plan, int32_t* threads, int32_t* ctas_per_sm,
                         float* probe_ms) {
  MQCT_ARG_CHECK(plan && threads && ctas_per_sm, "null argument");
  const PropPlan* p = reinterpret_cast<const PropPlan*>(plan);
  *threads = p->tpb;
  *ctas_per_sm = p->per_sm;
  if (probe_ms) {
    probe_ms[0] = p->tuned ? p->tune_ms[0] : 0.f;
    probe_ms[1] = p->tuned ? p->tune_ms[1] : 0.f;
  }
  return MQCT_OK;
}

int mqct_prop_plan_set_engine(mqct_prop_plan* plan, int32_t engine) {
  MQCT_ARG_CHECK(plan, "null plan");
  MQCT_ARG_CHECK(engine == MQCT_ENGINE_AUTO || engine == MQCT_ENGINE_PER_TRAJECTORY ||
                     engine == MQCT_ENGINE_LOCKSTEP || engine == MQCT_ENGINE_RESIDENT ||
                     engine == MQCT_ENGINE_LOCKSTEP_TAIL,
                 "unknown engine %d", engine);
  reinterpret_cast<PropPlan*>(plan)->engine = engine;
  return MQCT_OK;
}

int mqct_prop_plan_handed(const mqct_prop_plan* plan, int32_t* n) {
  MQCT_ARG_CHECK(plan && n, "null argument");
  const PropPlan* p = reinterpret_cast<const PropPlan*>(plan);
  *n = p->last_engine == MQCT_ENGINE_LOCKSTEP_TAIL ? p->last_handed : 0;
  return MQCT_OK;
}

int mqct_prop_plan_set_cluster(mqct_prop_plan* plan, int32_t ctas) {
  MQCT_ARG_CHECK(plan, "null plan");
  MQCT_ARG_CHECK(ctas == 0 || (ctas >= 2 && ctas <= 8), "cluster size %d not 0 or 2..8", ctas);
  reinterpret_cast<PropPlan*>(plan)->rs_cl = ctas;
  return MQCT_OK;
}

int mqct_prop_plan_cluster(mqct_prop_plan* plan, int32_t* ctas, int32_t* clusters) {
  MQCT_ARG_CHECK(plan, "null plan");
  PropPlan* p = reinterpret_cast<PropPlan*>(plan);
  if (ctas) *ctas = 0;
  if (clusters) *clusters = 0;
  if (p->arith != MQCT_PROP_FP32) return MQCT_OK;
  if (p->last_engine == MQCT_ENGINE_RESIDENT) {
    if (ctas) *ctas = p->last_rs[0];
    if (clusters) *clusters = p->last_rs[1];
    return MQCT_OK;
  }
  if (!p->rs) p->rs = rs_create();
  rs_set_cluster(p->rs, p->rs_cl);
  if (!rs_usable(p->rs, p->dev_view(MQCT_MODE_STD), p->h_blk_n, p->h_blk_s0, p->stream))
    return MQCT_OK;
  if (ctas) *ctas = rs_cluster(p->rs);
  if (clusters) *clusters = rs_clusters(p->rs);
  return MQCT_OK;
}

int mqct_prop_plan_engine(const mqct_prop_plan* plan, int32_t* engine, int64_t* rounds) {
  MQCT_ARG_CHECK(plan, "null plan");
  const PropPlan* p = reinterpret_cast<const PropPlan*>(plan);
  if (engine) *engine = p->last_engine;
  if (rounds)
    *rounds = (p->last_engine == MQCT_ENGINE_LOCKSTEP || p->last_engine == MQCT_ENGINE_LOCKSTEP_TAIL)
                  ? ls_rounds(p->ls)
                  : 0;
  return MQCT_OK;
}

int mqct_prop_plan_set_coupled_states(mqct_prop_plan* plan, int32_t cs) {
  MQCT_ARG_CHECK(plan, "null plan");
  reinterpret_cast<PropPlan*>(plan)->cs = cs != 0;
  return MQCT_OK;
}

int mqct_prop_plan_set_integrator(mqct_prop_plan* plan, const mqct_integrator_t* integ) {
  MQCT_ARG_CHECK(plan, "null plan");
  return reinterpret_cast<PropPlan*>(plan)->set_integrator(integ);
}

int mqct_propagate_batch_integ(const mqct_tables_t* tab, const mqct_traj_init_t* init,
                               int64_t n_traj, int32_t mode, const mqct_at_paths_t* at,
                               int32_t arith, const mqct_integrator_t* integ, double* amp_out,
                               double* cls_out, double* diag_out) {
  MQCT_ARG_CHECK(init && amp_out && cls_out && diag_out && integ, "null argument");
  MQCT_ARG_CHECK((mode & ~MQCT_MODE_CS) == MQCT_MODE_STD || (mode & ~MQCT_MODE_CS) == MQCT_MODE_AT,
                 "unknown mode %d", mode);
  mqct_prop_plan* h = nullptr;
  int rc = mqct_prop_plan_create(tab, arith, &h);
  if (rc) return rc;
  PropPlan* p = reinterpret_cast<PropPlan*>(h);
  rc = p->set_integrator(integ);
  if (!rc) rc = validate_init(init, n_traj, p->N, mode);
  if (!rc && (mode & MQCT_MODE_AT)) rc = p->set_at(at, n_traj);
  if (!rc) rc = run_host(p, init, n_traj, mode, amp_out, cls_out, diag_out);
  mqct_prop_plan_destroy(h);
  return rc;
}

int mqct_propagate_batch(const mqct_tables_t* tab, const mqct_traj_init_t* init, int64_t n_traj,
                         int32_t mode, const mqct_at_paths_t* at, int32_t arith,
                         double* amp_out, double* cls_out, double* diag_out) {
  MQCT_ARG_CHECK(init && amp_out && cls_out && diag_out, "null argument");
  MQCT_ARG_CHECK((mode & ~MQCT_MODE_CS) == MQCT_MODE_STD || (mode & ~MQCT_MODE_CS) == MQCT_MODE_AT,
                 "unknown mode %d", mode);
  mqct_prop_plan* h = nullptr;
  int rc = mqct_prop_plan_create(tab, arith, &h);
  if (rc) return rc;
  PropPlan* p = reinterpret_cast<PropPlan*>(h);
  rc = validate_init(init, n_traj, p->N, mode);
  if (!rc && (mode & MQCT_MODE_AT)) rc = p->set_at(at, n_traj);
  if (!rc) rc = run_host(p, init, n_traj, mode, amp_out, cls_out, diag_out);
  mqct_prop_plan_destroy(h);
  return rc;
}

int mqct_propagate_batch_rec(const mqct_tables_t* tab, const mqct_traj_init_t* init,
                             int64_t n_traj, int32_t arith, int64_t max_rec, double* amp_out,
                             double* cls_out, double* diag_out, double* rec_out,
                             int64_t* n_rec_out) {
  MQCT_ARG_CHECK(init && amp_out && cls_out && diag_out && rec_out && n_rec_out, "null argument");
  MQCT_ARG_CHECK(max_rec > 0 && max_rec < ((int64_t)1 << 32), "max_rec out of range");
  mqct_prop_plan* h = nullptr;
  int rc = mqct_prop_plan_create(tab, arith, &h);
  if (rc) return rc;
  PropPlan* p = reinterpret_cast<PropPlan*>(h);
  rc = run_host(p, init, n_traj, MQCT_MODE_STD, amp_out, cls_out, diag_out, rec_out, max_rec,
                n_rec_out);
  mqct_prop_plan_destroy(h);
  return rc;
}

}  // extern "C"
