// propagate.cuh -- definitions shared by the two propagation engines: the
// per-trajectory persistent kernel (propagate.cu) and the lockstep engine that
// advances all trajectories of a batch one right-hand side at a time, grouped by spline
// interval (lockstep.cu).
#pragma once

#include <vector>

#include "common.cuh"

namespace mqct {

template <class T> struct V2;
template <> struct V2<float> { using t = float2; };
template <> struct V2<double> { using t = double2; };

struct PropDev {
  int N, nR, n_e, n_pass;
  int64_t S;                   // slots per knot row (all blocks, padded)
  const double* R;             // nR
  const int* pass_row0;        // first internal state of each pass (n_pass + 1)
  const int64_t* pass_slot0;   // first slot of each pass (n_pass + 1)
  const int* st_blk;           // block of each internal state
  const int* blk_n;            // states per block
  const int* blk_s0;           // first internal state of the block
  const int* blk_mp;           // offset of the block's triangle inside its pass
  const int64_t* blk_slot0;    // first slot of each block (n_blocks + 1)
  const int* blk_pass;         // pass holding each block
  const uint32_t* loc;         // per slot: internal (row | column << 16)
  const int* st_e;             // energy class per internal state
  const double* e_val;         // energy per class, Hartree
  const int* nb_plus;          // internal index of the reference-order successor, or -1
  const int* nb_minus;         // internal index of the reference-order predecessor, or -1
  const double* cplus;         // coefficient of the successor's amplitude
  const double* cminus;        // coefficient of the predecessor's amplitude
  const int* perm;             // internal -> reference state index
  const int* inv_perm;         // reference -> internal state index
  const void* knots;           // nR x S of (M, y2) in T precision
  double mass, inv_mass;
  int mode;                    // MQCT_MODE_STD or MQCT_MODE_AT
  int cs;                      // coupled-states approximation: no Coriolis terms
  int mp_cap;                  // packed slots that fit in shared memory
  double ode_eps, ode_hmin;    // ODEINT accuracy and minimum step (adaptive kernel)
  // AT paths
  const int64_t* at_off;
  const int* at_n;
  const double* at_rec;        // records of 8
  const double* at_y2;         // per record kAtCols second derivatives (R, theta, P_theta,
                               // P_phi, pot, phi)
  int bk_int;                  // bikram_int: one adaptive call with per-step stop rules
  int at_adapt;                // AT_ADAPT_STP: RK4 steps from the path's coupling energy
  double at_tol, at_mintm;     // AT_ADAPTOL and TIME_STEP (the smallest step)
};

// Classical variables (R, P_R, theta, P_theta, phi, P_phi).
struct Cls {
  double R, PR, th, Pth, phi, Pphi;
};


// Spline coefficients at R (splint_bk, MQCT_SOURCE_CODES/mqct_eqtns.f:555-611;
// above R_n the matrix is zero, MQCT_SOURCE_CODES/mqct_eqtns.f:545-549; below
// R_1 the first interval's cubic, the net effect of :534-551).
struct SplineAt {
  int klo;
  bool zero;
  double aa, bb, cc1, cc2, cc3, cc4, cc5, cc6, h;
};
// *hint: the interval found last (klo); when x is still inside it the bisection, whose
// result it is, is skipped.
__device__ inline SplineAt spline_at(const double* R, int nR, double x, int* hint) {
  SplineAt s;
  s.zero = x > R[nR - 1];
  int klo = 1, khi = nR;
  const int hk = *hint;
  if (hk >= 1 && hk < nR && R[hk - 1] <= x && x < R[hk]) {
    klo = hk;
    khi = hk + 1;
  }
  while (khi - klo > 1) {
    int k = (khi + klo) >> 1;
    if (R[k - 1] > x) khi = k;
    else klo = k;
  }
  *hint = klo;
  s.klo = klo - 1;
  double h = R[khi - 1] - R[klo - 1];
  const double inv_h = 1.0 / h;
  s.h = h;
  s.aa = (R[khi - 1] - x) * inv_h;
  s.bb = (x - R[klo - 1]) * inv_h;
  s.cc1 = s.aa * s.aa * s.aa - s.aa;
  s.cc2 = s.bb * s.bb * s.bb - s.bb;
  s.cc3 = 3 * s.aa * s.aa - 1.0;
  s.cc4 = 3 * s.bb * s.bb - 1.0;
  s.cc5 = (h * h) / 6.0;
  s.cc6 = s.cc5 * inv_h;
  return s;
}

__device__ inline double kinetic(const Cls& c, double mass) {
  return c.PR * c.PR / 2.0 / mass + c.Pth * c.Pth / 2.0 / mass / (c.R * c.R) +
         c.Pphi * c.Pphi / 2.0 / mass / (c.R * c.R) / (sin(c.th) * sin(c.th));
}

// A running trajectory handed from the lockstep engine to the resident engine at the
// start of an RK4 step (stage 0) or before its closing evaluation (stage 4): its classical
// state, bookkeeping and index; its FP64 amplitudes stay in the lockstep engine's array.
struct RsResume {
  Cls C;
  double tcur, eki, eqi, tmpR1, tmpR2;
  int counter, status, vib, period, stage, hint, tr;
};

// Lockstep engine (lockstep.cu): standard mode, RK4, no CS; every m-block of at most 128
// states.  ls_run propagates n_traj trajectories whose initial conditions are on the
// device (d_init) and on the host (h_init, for the bound on the rounds), writing the
// outputs of the per-trajectory kernel; ev0 / ev1 bracket the device work on stream st.
// With hand_below > 0 it stops at the first graph boundary after the running trajectories
// fell to hand_below or fewer and writes those that still run into hand_out (device, n_traj
// places), their count into *hand_n (host; 0 when the run ended in the engine) and the
// engine's FP64 amplitude array (n_traj x N, internal order) into *hand_amp.
struct LsEngine;
LsEngine* ls_create();
void ls_destroy(LsEngine* e);
bool ls_eligible(const std::vector<int>& blk_n);
int64_t ls_rounds(const LsEngine* e);
int ls_run(LsEngine* e, const PropDev& d, bool fp32, const std::vector<int>& blk_n, int n_sm,
           cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1, const mqct_traj_init_t* d_init,
           const mqct_traj_init_t* h_init, int n_traj, double* amp, double* cls, double* diag,
           int hand_below = 0, RsResume* hand_out = nullptr, int* hand_n = nullptr,
           const double2** hand_amp = nullptr);

// Cluster-resident engine (resident.cu): standard mode, RK4, no CS, FP32; one thread-block
// cluster per trajectory holds the knot rows of its spline interval in shared memory.
// rs_usable lays the engine out for the tables (once per table) and reports whether they
// fit; rs_run launches it on stream st, ev0 / ev1 bracketing the kernel.
struct RsEngine;
RsEngine* rs_create();
void rs_destroy(RsEngine* e);
void rs_set_cluster(RsEngine* e, int cl);
int rs_cluster(const RsEngine* e);
int rs_clusters(const RsEngine* e);
bool rs_usable(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
               const std::vector<int>& blk_s0, cudaStream_t st);
int rs_run(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
           const std::vector<int>& blk_s0, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
           const mqct_traj_init_t* d_init, int n_traj, double* amp, double* cls, double* diag);
// The n trajectories a lockstep run handed over (resume, device; their amplitudes in
// resume_amp, n_traj x N internal order, indexed by the trajectories' own indices):
// continued to their end, outputs at their own indices; only ev1 is recorded (after the
// kernel).
int rs_run_resume(RsEngine* e, const PropDev& d, const std::vector<int>& blk_n,
                  const std::vector<int>& blk_s0, cudaStream_t st, cudaEvent_t ev1,
                  const mqct_traj_init_t* d_init, const RsResume* resume, int n,
                  const double2* resume_amp, double* amp, double* cls, double* diag);

}  // namespace mqct
