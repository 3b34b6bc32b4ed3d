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
// quadratic form above).  M(R) and M'(R) come from the cubic spline on the
// stored knots; each m-block is staged densely in shared memory and reduced
// with warp shuffles (deterministic order).  The RK4 state and the classical
// variables stay FP64; the table/mat-vec arithmetic T is float (FP32 mode) or
// double (FP64 mode).
#include <algorithm>
#include <cmath>
#include <map>

#include "common.cuh"

using namespace mqct;

namespace mqct {

constexpr int PT = 256;        // threads per CTA
constexpr int MAX_NS = 16;     // states per thread (N <= PT * MAX_NS = 4096)

template <class T> struct V2;
template <> struct V2<float> { using t = float2; };
template <> struct V2<double> { using t = double2; };

struct PropDev {
  int N, P, nR, n_blocks, n_e, nmax;
  const double* R;          // nR
  const int* blk_off;       // n_blocks+1 offsets into pairs
  const int* blk_n;         // states per block
  const int* blk_s0;        // offset into blk_states
  const int* blk_states;    // global state index per (block, local)
  const int* pair_loc;      // ia | ib << 16 (block-local)
  const int* st_e;          // energy class per state
  const double* e_val;      // energy per class, Hartree
  const double* cplus;      // per state coefficient of a_{i+1}
  const double* cminus;     // per state coefficient of a_{i-1}
  const void* knots;        // nR x P of (M, y2) in T precision
  double mass;
  int mode;                 // MQCT_MODE_*
  // AT paths
  const int64_t* at_off;
  const int* at_n;
  const double* at_rec;     // records of 8
  const double* at_y2;      // per record 4 second derivatives (R, theta, P_theta, P_phi)
};

struct TrajOut {
  double* amp;
  double* cls;
  double* diag;
};

// Shared-memory layout of one CTA (dynamic).
template <class T>
struct Smem {
  typename V2<T>::t* bt;     // N
  typename V2<T>::t* u;      // N
  typename V2<T>::t* y;      // N
  typename V2<T>::t* ph;     // n_e
  T* Md;                     // nmax^2
  double2* a_in;             // N (RHS input)
  double* red;               // reduction scratch
  int* flag;
};

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of two doubles; result broadcast to all threads.
__device__ inline void block_sum2(double& a, double& b, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  if (lane == 0) {
    red[2 * w] = a;
    red[2 * w + 1] = b;
  }
  __syncthreads();
  double sa = 0.0, sb = 0.0;
#pragma unroll
  for (int i = 0; i < PT / 32; ++i) {
    sa += red[2 * i];
    sb += red[2 * i + 1];
  }
  a = sa;
  b = sb;
  __syncthreads();
}

// Spline coefficients at R (splint_bk, MQCT_SOURCE_CODES/mqct_eqtns.f:555-611;
// above R_n the matrix is zero, MQCT_SOURCE_CODES/mqct_eqtns.f:545-549).
struct SplineAt {
  int klo;
  bool zero;
  double aa, bb, cc1, cc2, cc3, cc4, cc5, cc6, h;
};
__device__ inline SplineAt spline_at(const double* R, int nR, double x) {
  SplineAt s;
  s.zero = x > R[nR - 1];
  int klo = 1, khi = nR;
  while (khi - klo > 1) {
    int k = (khi + klo) >> 1;
    if (R[k - 1] > x) khi = k;
    else klo = k;
  }
  s.klo = klo - 1;
  double h = R[khi - 1] - R[klo - 1];
  s.h = h;
  s.aa = (R[khi - 1] - x) / h;
  s.bb = (x - R[klo - 1]) / h;
  s.cc1 = s.aa * s.aa * s.aa - s.aa;
  s.cc2 = s.bb * s.bb * s.bb - s.bb;
  s.cc3 = 3 * s.aa * s.aa - 1.0;
  s.cc4 = 3 * s.bb * s.bb - 1.0;
  s.cc5 = (h * h) / 6.0;
  s.cc6 = s.cc5 / h;
  return s;
}

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
         ((a * a * a - a) * y2[4 * (klo - 1) + ycol] + (b * b * b - b) * y2[4 * (khi - 1) + ycol]) *
             (h * h) / 6.0;
}

struct Cls {
  double R, PR, th, Pth, phi, Pphi;
};

// One right-hand-side evaluation.  Input amplitudes in sm.a_in (all states);
// outputs: da for this thread's states (registers), the classical derivative
// (std mode), and pot = Re(bt^+ y) (coupling energy).
template <class T, int NS>
__device__ void rhs(const PropDev& d, const Smem<T>& sm, double t, const Cls& c, int ns,
                    double2 (&da)[NS], Cls& dc, double& pot) {
  using T2 = typename V2<T>::t;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = d.N;
  const double sin_t = sin(c.th);
  const double dphidt = c.Pphi / c.R / c.R / d.mass / (sin_t * sin_t);
  // phases per energy class: (cos E t, -sin E t) = e^{-iEt}
  for (int e = tid; e < d.n_e; e += PT) {
    double s, co;
    sincos(d.e_val[e] * t, &s, &co);
    sm.ph[e].x = (T)co;
    sm.ph[e].y = (T)(-s);
  }
  __syncthreads();
  for (int i = tid; i < N; i += PT) {
    double2 a = sm.a_in[i];
    T2 p = sm.ph[d.st_e[i]];
    T ar = (T)a.x, ai = (T)a.y;
    sm.bt[i].x = p.x * ar - p.y * ai;
    sm.bt[i].y = p.x * ai + p.y * ar;
    double ur = 0.0, ui = 0.0;
    if (i + 1 < N) {
      ur += d.cplus[i] * sm.a_in[i + 1].x;
      ui += d.cplus[i] * sm.a_in[i + 1].y;
    }
    if (i > 0) {
      ur += d.cminus[i] * sm.a_in[i - 1].x;
      ui += d.cminus[i] * sm.a_in[i - 1].y;
    }
    sm.u[i].x = (T)ur;
    sm.u[i].y = (T)ui;
  }
  const SplineAt sp = spline_at(d.R, d.nR, c.R);
  const T2* K0 = reinterpret_cast<const T2*>(d.knots) + (size_t)sp.klo * d.P;
  const T2* K1 = K0 + d.P;
  const T aa = (T)sp.aa, bb = (T)sp.bb, cc1 = (T)sp.cc1, cc2 = (T)sp.cc2, cc3 = (T)sp.cc3,
          cc4 = (T)sp.cc4, cc5 = (T)sp.cc5, cc6 = (T)sp.cc6, hinv = (T)(1.0 / sp.h);
  T force = (T)0;
  __syncthreads();
  for (int b = 0; b < d.n_blocks; ++b) {
    const int n = d.blk_n[b], p0 = d.blk_off[b], p1 = d.blk_off[b + 1];
    const int* st = d.blk_states + d.blk_s0[b];
    for (int q = tid; q < n * n; q += PT) sm.Md[q] = (T)0;
    __syncthreads();
    if (!sp.zero) {
      for (int k = p0 + tid; k < p1; k += PT) {
        T2 lo = K0[k], hi = K1[k];
        T m = aa * lo.x + bb * hi.x + (cc1 * lo.y + cc2 * hi.y) * cc5;
        T md = (hi.x - lo.x) * hinv + (-cc3 * lo.y + cc4 * hi.y) * cc6;
        int loc = d.pair_loc[k];
        int ia = loc & 0xffff, ib = loc >> 16;
        sm.Md[ia * n + ib] = m;
        sm.Md[ib * n + ia] = m;
        T2 x = sm.bt[st[ia]], z = sm.bt[st[ib]];
        T re = x.x * z.x + x.y * z.y;
        force += (ia == ib ? (T)1 : (T)2) * md * re;
      }
    }
    __syncthreads();
    for (int r = warp; r < n; r += PT / 32) {
      T yr = (T)0, yi = (T)0;
      for (int j = lane; j < n; j += 32) {
        T m = sm.Md[r * n + j];
        T2 z = sm.bt[st[j]];
        yr += m * z.x;
        yi += m * z.y;
      }
      yr = warp_sum(yr);
      yi = warp_sum(yi);
      if (lane == 0) {
        sm.y[st[r]].x = yr;
        sm.y[st[r]].y = yi;
      }
    }
    __syncthreads();
  }
  // quadratic forms: F = Re(bt^+ M' bt) (accumulated above), g = Im(ut^+ y),
  // pot = Re(bt^+ y)
  double g = 0.0, pt = 0.0;
  for (int i = tid; i < N; i += PT) {
    T2 p = sm.ph[d.st_e[i]];
    T2 uu = sm.u[i], yy = sm.y[i], bb2 = sm.bt[i];
    T utr = p.x * uu.x - p.y * uu.y, uti = p.x * uu.y + p.y * uu.x;  // D^* u
    g += (double)(utr * yy.y - uti * yy.x);
    pt += (double)(bb2.x * yy.x + bb2.y * yy.y);
  }
  double f = (double)force;
  block_sum2(g, pt, sm.red);
  double dummy = 0.0;
  block_sum2(f, dummy, sm.red);
  pot = pt;
  // da_i = -i e^{iE t} y_i - i (dphi/2) u_i
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    if (q >= ns) break;
    int i = tid + q * PT;
    T2 p = sm.ph[d.st_e[i]];
    T2 yy = sm.y[i], uu = sm.u[i];
    double er = (double)p.x, ei = -(double)p.y;  // e^{iEt}
    double zr = er * yy.x - ei * yy.y, zi = er * yy.y + ei * yy.x;
    double cr = zr + 0.5 * dphidt * (double)uu.x, ci = zi + 0.5 * dphidt * (double)uu.y;
    da[q] = make_double2(ci, -cr);  // -i (cr + i ci)
  }
  if (d.mode == MQCT_MODE_STD) {
    double R = c.R, m = d.mass;
    dc.R = c.PR / m;
    dc.PR = -f + c.Pth / R / R / m * c.Pth / R + c.Pphi / R / R / m * c.Pphi / R / (sin_t * sin_t);
    dc.th = 0.0;
    dc.Pth = 0.0;
    dc.phi = c.Pphi / R / R / m / (sin_t * sin_t);
    dc.Pphi = sin_t * g;
  }
}

template <class T, int NS>
__global__ void __launch_bounds__(PT, 1)
propagate_kernel(PropDev d, const mqct_traj_init_t* __restrict__ init, int n_traj,
                 int* __restrict__ queue, TrajOut out) {
  using T2 = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = d.N, tid = threadIdx.x;
  Smem<T> sm;
  {
    unsigned char* p = smem_raw;
    sm.a_in = reinterpret_cast<double2*>(p);
    p += sizeof(double2) * N;
    sm.bt = reinterpret_cast<T2*>(p);
    p += sizeof(T2) * N;
    sm.u = reinterpret_cast<T2*>(p);
    p += sizeof(T2) * N;
    sm.y = reinterpret_cast<T2*>(p);
    p += sizeof(T2) * N;
    sm.ph = reinterpret_cast<T2*>(p);
    p += sizeof(T2) * ((d.n_e + 1) & ~1);
    sm.red = reinterpret_cast<double*>(p);
    p += sizeof(double) * 2 * (PT / 32);
    sm.flag = reinterpret_cast<int*>(p);
    p += 16;
    sm.Md = reinterpret_cast<T*>(p);
  }
  const int ns = (N + PT - 1 - tid) / PT;  // states owned by this thread
  for (;;) {
    if (tid == 0) sm.flag[0] = atomicAdd(queue, 1);
    __syncthreads();
    const int tr = sm.flag[0];
    __syncthreads();
    if (tr >= n_traj) break;
    const mqct_traj_init_t ti = init[tr];
    double2 y[NS], dydx[NS], dyt[NS], dym[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) y[q] = make_double2(0.0, 0.0);
    _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns)
      if (tid + q * PT == ti.s_st - 1) y[q].x = 1.0;
    Cls c{}, dcl{}, dct{}, dcm{}, ct{};
    const double k_vec = sqrt(d.mass * 2.0 * ti.e_coll);
    const double l_orb = sqrt(ti.l_real * (ti.l_real + 1.0));
    int status = 0;
    double tcur = 0.0, pot0 = 0.0, pot_end = 0.0, eki = 0.0, eqi = 0.0, eerr = 0.0;
    long long counter = 0;
    int vib = 0, period = 0;
    const bool at = d.mode == MQCT_MODE_AT;
    const double* arec = nullptr;
    const double* ay2 = nullptr;
    int an = 0;
    if (at) {
      arec = d.at_rec + 8 * d.at_off[tr];
      ay2 = d.at_y2 + 4 * d.at_off[tr];
      an = d.at_n[tr];
      tcur = arec[0];
    }
    auto classical_at = [&](double t, Cls& cc) {
      cc.R = at_splint(arec, ay2, an, 1, 0, t);
      cc.th = at_splint(arec, ay2, an, 3, 1, t);
      cc.Pth = at_splint(arec, ay2, an, 4, 2, t);
      cc.Pphi = at_splint(arec, ay2, an, 6, 3, t);
      cc.PR = 0.0;
      cc.phi = 0.0;
    };
    auto load_in = [&](const double2 (&v)[NS]) {
#pragma unroll
      for (int q = 0; q < NS; ++q)
        if (q < ns) sm.a_in[tid + q * PT] = v[q];
      __syncthreads();
    };
    if (!at && l_orb / k_vec > ti.r_start) {
      status = 2;
      c.R = ti.r_start;
    } else {
      if (!at) {
        c.R = ti.r_start;
        c.PR = -sqrt(k_vec * k_vec - l_orb * l_orb / (ti.r_start * ti.r_start));
        c.th = acos(0.0);
        c.Pth = l_orb * sin(0.0);
        c.phi = 0.0;
        c.Pphi = l_orb * cos(0.0);
      }
      double tmpR1 = 0.0, tmpR2 = 0.0;
      bool run = true;
      double dt = ti.dt;
      const double t_end = at ? arec[8 * (an - 1)] : 0.0;
      while (run) {
        ++counter;
        if (at && tcur + dt >= t_end) {
          dt = t_end - tcur;
          run = false;
        }
        const double hh = dt * 0.5, h6 = dt / 6.0, xh = tcur + hh;
        // k1 at (t, y)
        load_in(y);
        Cls cin = c;
        if (at) classical_at(tcur, cin);
        double potv;
        rhs<T, NS>(d, sm, tcur, cin, ns, dydx, dcl, potv);
        if (counter == 1 && !at) {
          pot0 = potv;
          double q0 = 0.0, dummy = 0.0;
          _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns) {
            int i = tid + q * PT;
            q0 += (y[q].x * y[q].x + y[q].y * y[q].y) * d.e_val[d.st_e[i]];
          }
          block_sum2(q0, dummy, sm.red);
          eqi = q0 + pot0;
          eki = c.PR * c.PR / 2.0 / d.mass + c.Pth * c.Pth / 2.0 / d.mass / (c.R * c.R) +
                c.Pphi * c.Pphi / 2.0 / d.mass / (c.R * c.R) / (sin(c.th) * sin(c.th));
        }
        // k2 at (t + h/2, y + h/2 k1)
        double2 yt[NS];
        _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns)
          yt[q] = make_double2(y[q].x + hh * dydx[q].x, y[q].y + hh * dydx[q].y);
        if (!at) {
          ct = Cls{c.R + hh * dcl.R, c.PR + hh * dcl.PR, c.th + hh * dcl.th,
                   c.Pth + hh * dcl.Pth, c.phi + hh * dcl.phi, c.Pphi + hh * dcl.Pphi};
        } else {
          classical_at(xh, ct);
        }
        load_in(yt);
        rhs<T, NS>(d, sm, xh, ct, ns, dyt, dct, potv);
        // k3 at (t + h/2, y + h/2 k2)
        _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns)
          yt[q] = make_double2(y[q].x + hh * dyt[q].x, y[q].y + hh * dyt[q].y);
        if (!at) {
          ct = Cls{c.R + hh * dct.R, c.PR + hh * dct.PR, c.th + hh * dct.th,
                   c.Pth + hh * dct.Pth, c.phi + hh * dct.phi, c.Pphi + hh * dct.Pphi};
        }
        load_in(yt);
        rhs<T, NS>(d, sm, xh, ct, ns, dym, dcm, potv);
        // k4 at (t + h, y + h k3)
        _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns) {
          yt[q] = make_double2(y[q].x + dt * dym[q].x, y[q].y + dt * dym[q].y);
          dym[q] = make_double2(dyt[q].x + dym[q].x, dyt[q].y + dym[q].y);
        }
        if (!at) {
          ct = Cls{c.R + dt * dcm.R, c.PR + dt * dcm.PR, c.th + dt * dcm.th,
                   c.Pth + dt * dcm.Pth, c.phi + dt * dcm.phi, c.Pphi + dt * dcm.Pphi};
          dcm = Cls{dct.R + dcm.R, dct.PR + dcm.PR, dct.th + dcm.th, dct.Pth + dcm.Pth,
                    dct.phi + dcm.phi, dct.Pphi + dcm.Pphi};
        } else {
          classical_at(tcur + dt, ct);
        }
        load_in(yt);
        rhs<T, NS>(d, sm, tcur + dt, ct, ns, dyt, dct, potv);
        _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns)
          y[q] = make_double2(y[q].x + h6 * (dydx[q].x + dyt[q].x + 2.0 * dym[q].x),
                              y[q].y + h6 * (dydx[q].y + dyt[q].y + 2.0 * dym[q].y));
        if (!at) {
          c.R += h6 * (dcl.R + dct.R + 2.0 * dcm.R);
          c.PR += h6 * (dcl.PR + dct.PR + 2.0 * dcm.PR);
          c.th += h6 * (dcl.th + dct.th + 2.0 * dcm.th);
          c.Pth += h6 * (dcl.Pth + dct.Pth + 2.0 * dcm.Pth);
          c.phi += h6 * (dcl.phi + dct.phi + 2.0 * dcm.phi);
          c.Pphi += h6 * (dcl.Pphi + dct.Pphi + 2.0 * dcm.Pphi);
          // stop rules, MQCT_SOURCE_CODES/propagator.f:4011-4050
          const double uR = c.R;
          if (tcur > dt && counter > 2) {
            if ((tmpR2 - tmpR1) < 0.0 && (tmpR1 - uR) > 0.0) vib += 1;
          }
          tmpR2 = tmpR1;
          tmpR1 = uR;
          tcur += dt;
          period = (int)(fabs(c.phi) / 2.0 / kPi);
          if (ti.numb_orb_prds <= period) run = false;
          if (vib >= ti.numb_oscl_prds) run = false;
          if (ti.time_lim > 0 && tcur >= ti.time_lim) run = false;
          if (uR > ti.r_fin) run = false;
          if (!(uR == uR)) {
            run = false;
            status = 3;
          }
        } else {
          tcur += dt;
        }
        if (run && ti.max_steps > 0 && counter >= ti.max_steps) {
          run = false;
          status = 1;
        }
      }
      if (!at) {  // final energy bookkeeping, MQCT_SOURCE_CODES/propagator.f:4182-4343
        load_in(y);
        double2 dd[NS];
        Cls dcx;
        rhs<T, NS>(d, sm, tcur, c, ns, dd, dcx, pot_end);
        double eqf = 0.0, dummy = 0.0;
        _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns) {
          int i = tid + q * PT;
          eqf += (y[q].x * y[q].x + y[q].y * y[q].y) * d.e_val[d.st_e[i]];
        }
        block_sum2(eqf, dummy, sm.red);
        double ef = c.PR * c.PR / 2.0 / d.mass + c.Pth * c.Pth / 2.0 / d.mass / (c.R * c.R) +
                    c.Pphi * c.Pphi / 2.0 / d.mass / (c.R * c.R) / (sin(c.th) * sin(c.th));
        eerr = fabs(eqf + ef + pot_end - eki - eqi);
      }
    }
    double nrm = 0.0, dummy = 0.0;
    _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns) nrm += y[q].x * y[q].x + y[q].y * y[q].y;
    block_sum2(nrm, dummy, sm.red);
    double* amp = out.amp + (size_t)tr * 2 * N;
    _Pragma("unroll") for (int q = 0; q < NS; ++q) if (q < ns) {
      int i = tid + q * PT;
      amp[i] = y[q].x;
      amp[N + i] = y[q].y;
    }
    if (tid == 0) {
      double* cl = out.cls + (size_t)tr * 6;
      cl[0] = c.R; cl[1] = c.PR; cl[2] = c.th; cl[3] = c.Pth; cl[4] = c.phi; cl[5] = c.Pphi;
      double* dg = out.diag + (size_t)tr * 8;
      dg[0] = tcur;
      dg[1] = (double)counter;
      dg[2] = status == 2 ? 0.0 : fabs(1.0 - nrm);
      dg[3] = eerr;
      dg[4] = status;
      dg[5] = period;
      dg[6] = vib;
      dg[7] = pot_end;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ plan
struct PropPlan {
  int arith = MQCT_PROP_FP32;
  int N = 0, P = 0, nR = 0, n_blocks = 0, n_e = 0, nmax = 0;
  double mass = 0.0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<double> d_R, d_e_val, d_cplus, d_cminus;
  DevBuf<int> d_blk_off, d_blk_n, d_blk_s0, d_blk_states, d_pair_loc, d_st_e, d_queue;
  DevBuf<float2> d_knots32;
  DevBuf<double2> d_knots64;
  DevBuf<mqct_traj_init_t> d_init;
  DevBuf<double> d_amp, d_cls, d_diag;
  // AT
  DevBuf<int64_t> d_at_off;
  DevBuf<int> d_at_n;
  DevBuf<double> d_at_rec, d_at_y2;
  int n_sm = 148;
  int ns = 1;  // states per thread, power of two

  template <class T>
  static const void* pick(int ns) {
    switch (ns) {
      case 1: return (const void*)propagate_kernel<T, 1>;
      case 2: return (const void*)propagate_kernel<T, 2>;
      case 4: return (const void*)propagate_kernel<T, 4>;
      case 8: return (const void*)propagate_kernel<T, 8>;
      default: return (const void*)propagate_kernel<T, 16>;
    }
  }
  const void* kernel_ptr() const {
    return arith == MQCT_PROP_FP32 ? pick<float>(ns) : pick<double>(ns);
  }

  size_t smem_bytes() const {
    size_t t = arith == MQCT_PROP_FP32 ? 8 : 16;
    size_t b = sizeof(double2) * N + 3 * t * N + t * ((n_e + 1) & ~1) + 16 * (PT / 32) + 16;
    b = (b + 15) & ~size_t(15);
    return b + (t / 2) * (size_t)nmax * nmax;
  }

  int init(const mqct_tables_t* tab, int32_t ar) {
    MQCT_ARG_CHECK(tab && tab->j12 && tab->m12 && tab->ej && tab->ind_mat && tab->R &&
                       tab->mat && tab->y2,
                   "null table argument");
    MQCT_ARG_CHECK(ar == MQCT_PROP_FP32 || ar == MQCT_PROP_FP64, "unknown arithmetic %d", ar);
    MQCT_ARG_CHECK(tab->n_states > 0 && tab->n_states <= PT * MAX_NS,
                   "n_states %d beyond the kernel limit %d", tab->n_states, PT * MAX_NS);
    MQCT_ARG_CHECK(tab->P > 0 && tab->P < (1 << 30) && tab->nR >= 2, "bad P/nR");
    MQCT_ARG_CHECK(tab->mass_au > 0, "mass must be positive");
    for (int i = 0; i + 1 < tab->nR; ++i) MQCT_ARG_CHECK(tab->R[i + 1] > tab->R[i], "R grid must increase");
    arith = ar;
    N = tab->n_states;
    P = (int)tab->P;
    nR = tab->nR;
    mass = tab->mass_au;
    MQCT_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    MQCT_CUDA_TRY(cudaEventCreate(&ev0));
    MQCT_CUDA_TRY(cudaEventCreate(&ev1));
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    // blocks by m
    std::map<int, std::vector<int>> by_m;
    for (int s = 0; s < N; ++s) by_m[tab->m12[s]].push_back(s);
    std::vector<int> local(N), blk_of(N), blk_n, blk_s0, blk_states;
    for (auto& kv : by_m) {
      int b = (int)blk_n.size();
      blk_n.push_back((int)kv.second.size());
      blk_s0.push_back((int)blk_states.size());
      for (size_t l = 0; l < kv.second.size(); ++l) {
        local[kv.second[l]] = (int)l;
        blk_of[kv.second[l]] = b;
        blk_states.push_back(kv.second[l]);
      }
      nmax = std::max(nmax, (int)kv.second.size());
    }
    n_blocks = (int)blk_n.size();
    MQCT_ARG_CHECK(nmax < 65536, "block too large");
    std::vector<std::vector<int>> bk(n_blocks);
    for (int k = 0; k < P; ++k) {
      int i = tab->ind_mat[2 * k] - 1, j = tab->ind_mat[2 * k + 1] - 1;
      MQCT_ARG_CHECK(i >= 0 && i < N && j >= 0 && j < N, "ind_mat out of range at k=%d", k + 1);
      MQCT_ARG_CHECK(tab->m12[i] == tab->m12[j], "pair with different m12 at k=%d", k + 1);
      bk[blk_of[i]].push_back(k);
    }
    std::vector<int> blk_off(n_blocks + 1, 0), pair_loc, order;
    for (int b = 0; b < n_blocks; ++b) {
      blk_off[b] = (int)order.size();
      for (int k : bk[b]) {
        int i = tab->ind_mat[2 * k] - 1, j = tab->ind_mat[2 * k + 1] - 1;
        pair_loc.push_back(local[i] | (local[j] << 16));
        order.push_back(k);
      }
    }
    blk_off[n_blocks] = (int)order.size();
    // knots (M, y2) per R, pairs in block order
    if (arith == MQCT_PROP_FP32) {
      std::vector<float2> kn((size_t)nR * P);
      for (int r = 0; r < nR; ++r)
        for (int q = 0; q < P; ++q) {
          size_t src = (size_t)order[q] * nR + r;
          kn[(size_t)r * P + q] = make_float2((float)tab->mat[src], (float)tab->y2[src]);
        }
      MQCT_CUDA_TRY(d_knots32.upload(kn, stream));
      MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    } else {
      std::vector<double2> kn((size_t)nR * P);
      for (int r = 0; r < nR; ++r)
        for (int q = 0; q < P; ++q) {
          size_t src = (size_t)order[q] * nR + r;
          kn[(size_t)r * P + q] = make_double2(tab->mat[src], tab->y2[src]);
        }
      MQCT_CUDA_TRY(d_knots64.upload(kn, stream));
      MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    // energy classes and Coriolis coefficients
    std::vector<double> e_val;
    std::vector<int> st_e(N);
    for (int s = 0; s < N; ++s) {
      int c = -1;
      for (size_t q = 0; q < e_val.size(); ++q)
        if (e_val[q] == tab->ej[s]) { c = (int)q; break; }
      if (c < 0) {
        c = (int)e_val.size();
        e_val.push_back(tab->ej[s]);
      }
      st_e[s] = c;
    }
    n_e = (int)e_val.size();
    std::vector<double> cp(N, 0.0), cm(N, 0.0);
    for (int s = 0; s < N; ++s) {
      double J = tab->j12[s], m = tab->m12[s];
      // reference sqrt2 / sqrt1 (MQCT_SOURCE_CODES/mqct_eqtns.f:447-448)
      if (s + 1 < N) cp[s] = sqrt(J * (J + 1.0) - (m + 1.0) * m);
      if (s > 0) cm[s] = sqrt(J * (J + 1.0) - (m - 1.0) * m);
    }
    MQCT_CUDA_TRY(d_R.upload(tab->R, nR, stream));
    MQCT_CUDA_TRY(d_e_val.upload(e_val, stream));
    MQCT_CUDA_TRY(d_cplus.upload(cp, stream));
    MQCT_CUDA_TRY(d_cminus.upload(cm, stream));
    MQCT_CUDA_TRY(d_blk_off.upload(blk_off, stream));
    MQCT_CUDA_TRY(d_blk_n.upload(blk_n, stream));
    MQCT_CUDA_TRY(d_blk_s0.upload(blk_s0, stream));
    MQCT_CUDA_TRY(d_blk_states.upload(blk_states, stream));
    MQCT_CUDA_TRY(d_pair_loc.upload(pair_loc, stream));
    MQCT_CUDA_TRY(d_st_e.upload(st_e, stream));
    MQCT_CUDA_TRY(d_queue.alloc(1));
    size_t sb = smem_bytes();
    MQCT_ARG_CHECK(sb <= 227 * 1024, "shared memory %zu B beyond the 227 KB limit", sb);
    ns = 1;
    while (ns * PT < N) ns *= 2;
    const void* fn = kernel_ptr();
    MQCT_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb));
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  PropDev dev_view(int mode) const {
    PropDev d{};
    d.N = N; d.P = P; d.nR = nR; d.n_blocks = n_blocks; d.n_e = n_e; d.nmax = nmax;
    d.R = d_R.p; d.blk_off = d_blk_off.p; d.blk_n = d_blk_n.p; d.blk_s0 = d_blk_s0.p;
    d.blk_states = d_blk_states.p; d.pair_loc = d_pair_loc.p; d.st_e = d_st_e.p;
    d.e_val = d_e_val.p; d.cplus = d_cplus.p; d.cminus = d_cminus.p;
    d.knots = arith == MQCT_PROP_FP32 ? (const void*)d_knots32.p : (const void*)d_knots64.p;
    d.mass = mass;
    d.mode = mode;
    d.at_off = d_at_off.p; d.at_n = d_at_n.p; d.at_rec = d_at_rec.p; d.at_y2 = d_at_y2.p;
    return d;
  }

  int launch(const mqct_traj_init_t* d_init_p, int64_t n_traj, int mode, double* amp,
             double* cls, double* diag) {
    MQCT_ARG_CHECK(n_traj > 0 && n_traj < (1 << 30), "n_traj out of range");
    MQCT_CUDA_TRY(cudaMemsetAsync(d_queue.p, 0, sizeof(int), stream));
    PropDev d = dev_view(mode);
    TrajOut o{amp, cls, diag};
    int n_traj_i = (int)n_traj;
    size_t sb = smem_bytes();
    int per_sm = 1;
    const void* fn = kernel_ptr();
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PT, sb);
    int grid = (int)std::min<int64_t>(n_traj, (int64_t)n_sm * std::max(per_sm, 1));
    void* args[] = {&d, (void*)&d_init_p, &n_traj_i, &d_queue.p, &o};
    MQCT_CUDA_TRY(cudaEventRecord(ev0, stream));
    MQCT_CUDA_TRY(cudaLaunchKernel(fn, dim3(grid), dim3(PT), args, sb, stream));
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
    std::vector<double> y2((size_t)total * 4, 0.0), u;
    const int cols[4] = {1, 3, 4, 6};
    for (int64_t t = 0; t < n_traj; ++t) {
      const double* r = at->rec + 8 * at->rec_off[t];
      int n = at->n_rec[t];
      for (int i = 0; i + 1 < n; ++i)
        MQCT_ARG_CHECK(r[8 * (i + 1)] > r[8 * i], "AT path %lld: time not increasing", (long long)t);
      u.assign(n, 0.0);
      for (int a = 0; a < 4; ++a) {
        double* yy = y2.data() + 4 * at->rec_off[t];
        auto X = [&](int i) { return r[8 * i]; };
        auto Y = [&](int i) { return r[8 * i + cols[a]]; };
        double yp1 = (Y(1) - Y(0)) / (X(1) - X(0));
        double ypn = (Y(n - 1) - Y(n - 2)) / (X(n - 1) - X(n - 2));
        yy[a] = -0.5;
        u[0] = (3.0 / (X(1) - X(0))) * ((Y(1) - Y(0)) / (X(1) - X(0)) - yp1);
        for (int i = 1; i < n - 1; ++i) {
          double sig = (X(i) - X(i - 1)) / (X(i + 1) - X(i - 1));
          double p = sig * yy[4 * (i - 1) + a] + 2.0;
          yy[4 * i + a] = (sig - 1.0) / p;
          u[i] = (6.0 * ((Y(i + 1) - Y(i)) / (X(i + 1) - X(i)) - (Y(i) - Y(i - 1)) / (X(i) - X(i - 1))) /
                      (X(i + 1) - X(i - 1)) -
                  sig * u[i - 1]) /
                 p;
        }
        double un = (3.0 / (X(n - 1) - X(n - 2))) * (ypn - (Y(n - 1) - Y(n - 2)) / (X(n - 1) - X(n - 2)));
        yy[4 * (n - 1) + a] = (un - 0.5 * u[n - 2]) / (0.5 * yy[4 * (n - 2) + a] + 1.0);
        for (int i = n - 2; i >= 0; --i) yy[4 * i + a] = yy[4 * i + a] * yy[4 * (i + 1) + a] + u[i];
      }
    }
    MQCT_CUDA_TRY(d_at_off.upload(at->rec_off, n_traj, stream));
    MQCT_CUDA_TRY(d_at_n.upload(at->n_rec, n_traj, stream));
    MQCT_CUDA_TRY(d_at_rec.upload(at->rec, (size_t)total * 8, stream));
    MQCT_CUDA_TRY(d_at_y2.upload(y2, stream));
    MQCT_CUDA_TRY(cudaStreamSynchronize(stream));
    return MQCT_OK;
  }

  ~PropPlan() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

static int validate_init(const mqct_traj_init_t* init, int64_t n, int N, int mode) {
  for (int64_t t = 0; t < n; ++t) {
    const mqct_traj_init_t& a = init[t];
    MQCT_ARG_CHECK(a.s_st >= 1 && a.s_st <= N, "trajectory %lld: s_st out of range", (long long)t);
    MQCT_ARG_CHECK(a.dt > 0, "trajectory %lld: dt must be positive", (long long)t);
    if (mode == MQCT_MODE_STD) {
      MQCT_ARG_CHECK(a.e_coll > 0 && a.l_real >= 0 && a.r_start > 0, "trajectory %lld: bad E/l/R",
                     (long long)t);
      MQCT_ARG_CHECK(a.max_steps > 0 || a.time_lim > 0,
                     "trajectory %lld: needs a step cap or a time limit", (long long)t);
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
  return reinterpret_cast<PropPlan*>(plan)->launch(d_init, n_traj, MQCT_MODE_STD, d_amp, d_cls,
                                                   d_diag);
}

int mqct_prop_plan_run(mqct_prop_plan* plan, const mqct_traj_init_t* init, int64_t n_traj,
                       double* amp_out, double* cls_out, double* diag_out) {
  MQCT_ARG_CHECK(plan && init && amp_out && cls_out && diag_out, "null argument");
  PropPlan* p = reinterpret_cast<PropPlan*>(plan);
  int rc = validate_init(init, n_traj, p->N, MQCT_MODE_STD);
  if (rc) return rc;
  MQCT_CUDA_TRY(p->d_init.upload(init, n_traj, p->stream));
  MQCT_CUDA_TRY(p->d_amp.alloc((size_t)n_traj * 2 * p->N));
  MQCT_CUDA_TRY(p->d_cls.alloc((size_t)n_traj * 6));
  MQCT_CUDA_TRY(p->d_diag.alloc((size_t)n_traj * 8));
  rc = p->launch(p->d_init.p, n_traj, MQCT_MODE_STD, p->d_amp.p, p->d_cls.p, p->d_diag.p);
  if (rc) return rc;
  MQCT_CUDA_TRY(cudaMemcpyAsync(amp_out, p->d_amp.p, sizeof(double) * n_traj * 2 * p->N,
                                cudaMemcpyDeviceToHost, p->stream));
  MQCT_CUDA_TRY(cudaMemcpyAsync(cls_out, p->d_cls.p, sizeof(double) * n_traj * 6,
                                cudaMemcpyDeviceToHost, p->stream));
  MQCT_CUDA_TRY(cudaMemcpyAsync(diag_out, p->d_diag.p, sizeof(double) * n_traj * 8,
                                cudaMemcpyDeviceToHost, p->stream));
  MQCT_CUDA_TRY(cudaStreamSynchronize(p->stream));
  return MQCT_OK;
}

int mqct_prop_plan_sync(mqct_prop_plan* plan) {
  MQCT_ARG_CHECK(plan, "null plan");
  MQCT_CUDA_TRY(cudaStreamSynchronize(reinterpret_cast<PropPlan*>(plan)->stream));
  return MQCT_OK;
}

double mqct_prop_plan_bytes_per_step(const mqct_prop_plan* plan) {
  if (!plan) return 0.0;
  const PropPlan* p = reinterpret_cast<const PropPlan*>(plan);
  return (p->arith == MQCT_PROP_FP32 ? 16.0 : 32.0) * p->P;
}

int mqct_prop_plan_timing(mqct_prop_plan* plan, float* ms) {
  MQCT_ARG_CHECK(plan && ms, "null argument");
  PropPlan* p = reinterpret_cast<PropPlan*>(plan);
  MQCT_CUDA_TRY(cudaEventSynchronize(p->ev1));
  MQCT_CUDA_TRY(cudaEventElapsedTime(ms, p->ev0, p->ev1));
  return MQCT_OK;
}

void mqct_prop_plan_destroy(mqct_prop_plan* plan) { delete reinterpret_cast<PropPlan*>(plan); }

int mqct_propagate_batch(const mqct_tables_t* tab, const mqct_traj_init_t* init, int64_t n_traj,
                         int32_t mode, const mqct_at_paths_t* at, int32_t arith,
                         double* amp_out, double* cls_out, double* diag_out) {
  MQCT_ARG_CHECK(init && amp_out && cls_out && diag_out, "null argument");
  MQCT_ARG_CHECK(mode == MQCT_MODE_STD || mode == MQCT_MODE_AT, "unknown mode %d", mode);
  mqct_prop_plan* h = nullptr;
  int rc = mqct_prop_plan_create(tab, arith, &h);
  if (rc) return rc;
  PropPlan* p = reinterpret_cast<PropPlan*>(h);
  rc = validate_init(init, n_traj, p->N, mode);
  if (!rc && mode == MQCT_MODE_AT) rc = p->set_at(at, n_traj);
  if (!rc) {
    if (mode == MQCT_MODE_STD) {
      rc = mqct_prop_plan_run(h, init, n_traj, amp_out, cls_out, diag_out);
    } else {
      cudaError_t e = p->d_init.upload(init, n_traj, p->stream);
      if (e == cudaSuccess) e = p->d_amp.alloc((size_t)n_traj * 2 * p->N);
      if (e == cudaSuccess) e = p->d_cls.alloc((size_t)n_traj * 6);
      if (e == cudaSuccess) e = p->d_diag.alloc((size_t)n_traj * 8);
      if (e != cudaSuccess) {
        set_error("%s", cudaGetErrorString(e));
        rc = MQCT_E_CUDA;
      }
      if (!rc) rc = p->launch(p->d_init.p, n_traj, MQCT_MODE_AT, p->d_amp.p, p->d_cls.p, p->d_diag.p);
      if (!rc) {
        cudaMemcpyAsync(amp_out, p->d_amp.p, sizeof(double) * n_traj * 2 * p->N,
                        cudaMemcpyDeviceToHost, p->stream);
        cudaMemcpyAsync(cls_out, p->d_cls.p, sizeof(double) * n_traj * 6, cudaMemcpyDeviceToHost,
                        p->stream);
        cudaMemcpyAsync(diag_out, p->d_diag.p, sizeof(double) * n_traj * 8,
                        cudaMemcpyDeviceToHost, p->stream);
        e = cudaStreamSynchronize(p->stream);
        if (e != cudaSuccess) {
          set_error("propagation failed: %s", cudaGetErrorString(e));
          rc = MQCT_E_CUDA;
        }
      }
    }
  }
  mqct_prop_plan_destroy(h);
  return rc;
}

}  // extern "C"
