/*
 * mqct_b200.h -- C ABI of the B200-native MQCT hot paths.
 *
 * Two entry points replace the reference's two hot loops:
 *   mqct_build_matrix    <- the DO k / DO i / CALL INTEGRATOR_TEMP loop and the
 *                           spline loop of MATRIX_MAKE
 *                           (MQCT_SOURCE_CODES/matrix_ini.f:1920-2016,
 *                            integrand MQCT_SOURCE_CODES/pot_comp.f:1790-3737)
 *   mqct_propagate_batch <- the DO itraject / CALL DOTRAJECT loop of PROPAGATE
 *                           (MQCT_SOURCE_CODES/propagator.f:885-899, DOTRAJECT
 *                            :2283-4645, RHS MQCT_SOURCE_CODES/mqct_eqtns.f:112-985)
 * plus the matrix-file formats of the SAVE_MTRX/READ_MTRX flow
 * (MTRX_UF.DAT: MQCT_SOURCE_CODES/matrix_ini.f:6640-6780 and :5794-6630).
 *
 * Conventions shared with the reference so a Fortran iso_c_binding shim can
 * pass its arrays unchanged:
 *   - ind_mat is the reference's ind_mat(2,P): pairs (st1, st2), 1-based,
 *     st2 <= st1, equal m12 (MQCT_SOURCE_CODES/matrix_ini.f:553-627);
 *   - Mat_el / Mat_el_der are column-major (n_R, P): element k at R index i is
 *     mat[k*nR + i]; energies in Hartree, distances in bohr;
 *   - all buffers are owned by the caller (host memory unless a function says
 *     "device"); the library never frees caller memory;
 *   - every function returns MQCT_OK (0) or a negative MQCT_E_* code and never
 *     exits; mqct_last_error() gives a message for the calling thread.
 * The library needs a CUDA device; there is no CPU fallback.
 */
#ifndef MQCT_B200_H
#define MQCT_B200_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define MQCT_OK 0
#define MQCT_E_ARG (-1)       /* invalid argument / inconsistent sizes        */
#define MQCT_E_CUDA (-2)      /* CUDA runtime error                           */
#define MQCT_E_NODEV (-3)     /* no CUDA device / extension not usable        */
#define MQCT_E_IO (-4)        /* file I/O or malformed matrix file            */
#define MQCT_E_RANGE (-5)     /* size beyond a documented limit               */
#define MQCT_E_DEVICE (-6)    /* a device-side check failed (status word set) */

/* SYS_TYPE values handled (MQCT_SOURCE_CODES/iotest.f $BASIS SYS_TYPE). */
#define MQCT_SYS_DIATOM_ATOM 1
#define MQCT_SYS_ASYM_ATOM 4
#define MQCT_SYS_ASYM_DIATOM 8
#define MQCT_SYS_ASYM_ASYM 0

/* Contraction precision of the matrix build. */
#define MQCT_PREC_FP64 0      /* plain FP64 CUDA-core form                    */
#define MQCT_PREC_BF16X3 1    /* tcgen05 kind::f16, BF16 hi/lo split, FP32 acc */
#define MQCT_PREC_F16X3 2     /* tcgen05 kind::f16, FP16 hi/lo split with power-of-two
                                 scaling, FP32 acc (~22 significant bits per operand) */

/* Propagation arithmetic. */
#define MQCT_PROP_FP64 0      /* FP64 amplitudes and tables                   */
#define MQCT_PROP_FP32 1      /* FP32 amplitude RHS and tables, FP64 phases,
                                 FP64 classical variables and RK4 state        */

/* Propagation modes. */
#define MQCT_MODE_STD 0       /* Ehrenfest MQCT: classical and quantum coupled */
#define MQCT_MODE_AT 1        /* AT-MQCT: classical path given                 */
#define MQCT_MODE_CS 2        /* flag, OR-ed with either mode: the coupled-states
                                 approximation (CS_APPROX = YES): no Coriolis
                                 coupling of m12 blocks, no Coriolis torque
                                 (MQCT_SOURCE_CODES/mqct_eqtns.f:208-210, 270,
                                 362, 787, 845)                                */

const char* mqct_last_error(void);
int mqct_version(void);                 /* MAJOR*10000 + MINOR*100 + PATCH */
int mqct_device_count(void);

/* Collision system after INI_ARRAYS (MQCT_SOURCE_CODES/matrix_ini.f:1-806). */
typedef struct mqct_sys_t {
  int32_t sys_type;          /* MQCT_SYS_*                                       */
  int32_t n_channels;
  const int32_t* j1;         /* per channel: j (types 1, 3, 4) or j1 (5, 7, 8, 0) */
  const int32_t* ka1;
  const int32_t* kc1;
  const int32_t* j2;         /* types 5, 7, 8, 0                                 */
  const int32_t* ka2;        /* type 0                                           */
  const int32_t* kc2;
  const double* vec1;        /* rotor-1 eigenvectors, channel-major, stride ldv,
                                components K=-j..j (M_VECTORS of
                                MQCT_SOURCE_CODES/pot_comp.f:121-175)            */
  const double* vec2;        /* rotor-2 eigenvectors (type 0)                    */
  int32_t ldv;
  int32_t n_states;
  const int32_t* indx_chann; /* per state, 1-based channel                       */
  const int32_t* j12;
  const int32_t* m12;
  const int32_t* parity;     /* per state exchange parity parity_state (+1/-1) of
                                identical partners (IDENTICAL = YES, SYS_TYPE 0),
                                MQCT_SOURCE_CODES/matrix_ini.f:482-530; NULL when the
                                partners are distinguishable                      */
} mqct_sys_t;

/* Angular quadrature (INI_POT_STORAGE, MQCT_SOURCE_CODES/pot_comp.f:333-1788):
 * GL beta grids on [0,pi]; gamma/alpha grids midpoint-equidistant on [0,2pi]
 * when eq_gamma (EQ_ANG_GRID=YES, the default) else GL.  Type 4 with
 * n_alpha = 0 integrates alpha analytically (factor 2*pi) as the reference
 * does; n_alpha > 0 contracts an explicit alpha grid. */
typedef struct mqct_grid_t {
  int32_t n_beta, n_gamma, n_alpha;
  int32_t n_beta2, n_alpha2, n_gamma2;   /* type 0 */
  int32_t eq_gamma;
} mqct_grid_t;

/* Potential energy surface (the USER_DEFINED_PES plugin, called through the
 * per-type wrappers of MQCT_SOURCE_CODES/pes_sys_type.f:2-97).  Values in
 * cm^-1, R in bohr.
 *   TABLE:    caller-evaluated V on the angular grid, table[iR*G + g] with
 *             g = i_beta*n_gamma + i_gamma (type 4; the surface of an atom +
 *             rigid rotor does not depend on alpha), g = i_beta (type 1, G =
 *             n_beta) or, for type 0, the 5-D index over (alpha2, beta1, beta2,
 *             gamma1, gamma2) with gamma2 fastest.  The analogue of the
 *             reference's VGRID_UF.DAT path;
 *   LEGENDRE: V(R,beta) = sum_l [A_l e^{-b_l R} - C_l/R^6] P_l(cos beta),
 *             params = [A_0..A_{n-1}, b_0.., C_0..];
 *   SITES1:   rigid-rotor sites + atom, per term [site, D, a, re, C6, rd]:
 *             D(e^{-2a(r-re)} - 2e^{-a(r-re)}) - C6 (1 - e^{-(r/rd)^6}) / r^6;
 *   SITES2:   two rigid rotors (type 0): rotor 1 at the origin with Euler
 *             angles (0, beta1, gamma1), rotor 2 at R z with (alpha2, beta2,
 *             gamma2) (the argument mapping of MQCT_SOURCE_CODES/pes_sys_type.f:90-97),
 *             per term [site1, site2, D, a, re, C6, rd]. */
#define MQCT_PES_TABLE 0
#define MQCT_PES_LEGENDRE 1
#define MQCT_PES_SITES1 2
#define MQCT_PES_SITES2 3
typedef struct mqct_pes_t {
  int32_t kind;
  int32_t n_terms;
  const double* params;
  int32_t n_sites1, n_sites2;
  const double* sites1;      /* xyz per site, bohr */
  const double* sites2;
  const double* table;
} mqct_pes_t;

/* Accuracy report of a split-precision build against an FP64 build of sampled
 * elements (optional, may be NULL). */
typedef struct mqct_err_report_t {
  int32_t n_sampled;         /* in: elements to sample (0 = none)              */
  double max_abs_err;        /* out, Hartree                                   */
  double max_rel_err;        /* out, |d|/max(|M|, 1e-8 max|M| of the element)  */
  double rms_rel_err;        /* out                                            */
} mqct_err_report_t;

/* Matrix build (SYS_TYPE 1, 3, 4, 9 and 0; SYS_TYPE 3 reads k from sys->ka1 and eps
 * from sys->kc1, SYS_TYPE 9 its second rotor's k from sys->ka2 and eps from sys->kc2,
 * and both form the symmetric-top vectors themselves): M_k(R_i) = C sum_g w_g V(R_i,g) Re(psi_st1(g)* psi_st2(g))
 * (MQCT_SOURCE_CODES/pot_comp.f:1947-1952, 2535-2557, 3709-3721), converted to
 * Hartree, MIJ_CUTOFF truncation at R~r_cut1/r_cut2
 * (MQCT_SOURCE_CODES/matrix_ini.f:1969-1997, columns whose max |M| there is
 * below mij_cutoff_cm are zeroed and flagged in skipped[k]) and clamped-spline
 * second derivatives with finite-difference end slopes (:2005-2016).
 * Mat_el, Mat_el_y2: host, nR*P doubles; skipped: host, P int32 (may be NULL). */
int mqct_build_matrix(const mqct_sys_t* sys, const int32_t* ind_mat, int64_t P,
                      const double* R, int32_t nR, const mqct_grid_t* grid,
                      const mqct_pes_t* pes, int32_t precision, double mij_cutoff_cm,
                      double r_cut1, double r_cut2, double* Mat_el, double* Mat_el_y2,
                      int32_t* skipped, mqct_err_report_t* err);
/* mqct_build_matrix keeps the plan and device buffers of its last call (one entry,
 * guarded by a lock): a call whose inputs all equal the last call's (compared by two
 * 64-bit digests of every array and scalar) copies the inputs to the device again and
 * runs the kept plan, skipping the set-up and the device allocations.  This releases
 * that entry (the plan and its device memory); the next call builds anew.  No
 * counterpart in the reference. */
void mqct_release_cached_build(void);

/* Matrix build from PES expansion terms (the READ_EXPANSION path: READ_EXPANSION_TERMS
 * + EXPANSION_MATRIX_ELEMENT, MQCT_SOURCE_CODES/pot_comp.f:6276-6395, 6465-8749), for
 * SYS_TYPE 1 (diatom + atom, case 1 at :6551-6622), SYS_TYPE 3 (symmetric top + atom,
 * case 3 at :6846-6954; the channel's k in sys->ka1, its parity eps in sys->kc1, vec1
 * unused; its -nju branch carries -(-1)^nju as written there, type 4's carries 1),
 * SYS_TYPE 4 (asymmetric top + atom, case 4 at :6955-7075), SYS_TYPE 5 (two diatoms, distinguishable partners, case 5 at
 * :7076-7386; j2 per channel in sys->j2, vec1 unused), SYS_TYPE 7 (symmetric top + diatom, case 7 at :7593-7824; the channel's k in
 * sys->ka1, its parity eps in sys->kc1, vec1 unused), SYS_TYPE 8 (asymmetric top +
 * diatom, case 8 at :7826-8058), SYS_TYPE 9 (asymmetric top + symmetric top, case 9 at
 * :8059-8256; the second rotor's k in sys->ka2, its eps in sys->kc2, vec2 unused) and
 * SYS_TYPE 0 (two asymmetric tops, distinguishable partners, case 0 at :8257-8672).  The arrays are the reference's own:
 *   a_top  A_TOP(5, nterms): per term 5 int32, (l, -, ...) for SYS_TYPE 1, (l, nju, -,
 *          ...) for SYS_TYPE 3 and 4, (l1, l2, l, -, -) for SYS_TYPE 5, (l1, nju1, l2, l, -) for SYS_TYPE 7 and 8, (l1, nju1, l2,
 *          nju2, l) for SYS_TYPE 9 and 0 (:6276-6338);
 *   terms  expansion_terms(n_r_coll, nterms): terms[t * nR + iR], R fastest, in the
 *          energy unit of the PES_EXPAN_TERMS.DAT file;
 *   e_unit conv_unit_e, the Hartree value of that unit (MQCT_SOURCE_CODES/matrix_ini.f:918-921:
 *          1/eVtown/autoeV for CM-1, 1/kcal for KCAL, 1/autokelv/autoeV for K).
 * Output as mqct_build_matrix: Mat_el in Hartree, MIJ_CUTOFF (mij_cutoff_cm, cm^-1)
 * and the spline y2.  j1, j2 <= 30, l1, l2 <= 30, l <= 60, n_terms <= 4096. */
int mqct_build_matrix_expansion(const mqct_sys_t* sys, const int32_t* ind_mat, int64_t P,
                                const double* R, int32_t nR, int32_t n_terms,
                                const int32_t* a_top, const double* terms, double e_unit,
                                double mij_cutoff_cm, double r_cut1, double r_cut2,
                                double* Mat_el, double* Mat_el_y2, int32_t* skipped);

/* The expansion build as a plan: _create validates the system, uploads it and forms
 * the R-independent angular coefficients (EXPANSION_MATRIX_ELEMENT's angular_part,
 * one per pair and term) on the device; _execute then forms Mat_el from radial terms
 * already on the device (d_terms[t * nR + iR] in units of e_unit Hartree), applies
 * MIJ_CUTOFF and fits the spline into device buffers (d_mat, d_y2: nR * P doubles,
 * d_y2 may be NULL; d_skipped: P int32), asynchronously on the plan's stream; _sync
 * waits for it; _timing gives the device milliseconds of the angular set-up and of
 * the last execute.  One plan serves any number of term sets on the same R grid. */
typedef struct mqct_expansion_plan mqct_expansion_plan;
int mqct_expansion_plan_create(const mqct_sys_t* sys, const int32_t* ind_mat, int64_t P,
                               const double* R, int32_t nR, int32_t n_terms, const int32_t* a_top,
                               double mij_cutoff_cm, double r_cut1, double r_cut2,
                               mqct_expansion_plan** plan);
int mqct_expansion_plan_execute(mqct_expansion_plan* plan, const double* d_terms, double e_unit,
                                double* d_mat, double* d_y2, int32_t* d_skipped);
int mqct_expansion_plan_sync(mqct_expansion_plan* plan);
int mqct_expansion_plan_timing(mqct_expansion_plan* plan, float* ms_angular, float* ms_execute);
void mqct_expansion_plan_destroy(mqct_expansion_plan* plan);

/* Device-resident form of the same build for callers that keep the matrix on
 * the GPU: a plan uploads the system once; execute writes Mat_el and y2 into
 * device buffers (nR*P doubles each, may be NULL for y2) on the plan's stream. */
typedef struct mqct_matrix_plan mqct_matrix_plan;
int mqct_matrix_plan_create(const mqct_sys_t* sys, const int32_t* ind_mat, int64_t P,
                            const double* R, int32_t nR, const mqct_grid_t* grid,
                            const mqct_pes_t* pes, int32_t precision, double mij_cutoff_cm,
                            double r_cut1, double r_cut2, mqct_matrix_plan** plan);
int mqct_matrix_plan_execute(mqct_matrix_plan* plan, double* d_mat, double* d_y2,
                             int32_t* d_skipped);
int mqct_matrix_plan_sync(mqct_matrix_plan* plan);
/* Flops of the contraction actually executed per build (2*P*nR*K times the
 * number of split-precision products). */
double mqct_matrix_plan_flops(const mqct_matrix_plan* plan);
/* Split-precision plans (no counterpart in the reference): the tensor-core accumulators
 * are added to FP64 sums after every group of slices_per_drain alpha points of a
 * 64-point grid chunk (1..64; more than 1 needs equal alpha weights; the plan's choice is
 * 2 on an equal-weight alpha grid, else 1).  mqct_matrix_plan_layout reports that choice,
 * the number of grid-chunk ranges whose FP64 sums the finalize adds, and the number of
 * radial column parts (0 for the FP64 form). */
int mqct_matrix_plan_set_drain(mqct_matrix_plan* plan, int32_t slices_per_drain);
int mqct_matrix_plan_layout(const mqct_matrix_plan* plan, int32_t* slices_per_drain,
                            int32_t* k_ranges, int32_t* column_parts);
/* Epilogue layout of the tensor-core contraction (no reference counterpart): 8 warps (two
 * per TMEM lane quarter, more registers each) or 16 (four per lane quarter, more of the
 * latency-bound drain in flight).  By default the launch takes 16 when a K-chunk has several
 * accumulation groups and 8 otherwise; mqct_matrix_plan_tune runs four executes with each
 * (into the caller's device outputs, which receive the build), takes the minimum contraction
 * time of the last three and keeps the faster layout.  The two
 * layouts give bitwise identical results (every column's sum has the same order).
 * mqct_matrix_plan_epilogue reports the layout the next execute uses and, after tuning,
 * the contraction times of the two (tune_ms[2], may be NULL).  The FP64 form has no such
 * layout (tune returns at once, epilogue reports 0). */
int mqct_matrix_plan_tune(mqct_matrix_plan* plan, double* d_mat, double* d_y2,
                          int32_t* d_skipped);
int mqct_matrix_plan_epilogue(const mqct_matrix_plan* plan, int32_t* warps, float* tune_ms);
/* Force the layout (8 or 16 warps) for the following executes, or 0 for the default rule. */
int mqct_matrix_plan_set_epilogue(mqct_matrix_plan* plan, int32_t warps);
/* CUDA-event timings (ms) of the last execute, recorded on the plan's stream:
 * t3[0] basis + PES tables, t3[1] contraction, t3[2] finalize (units, cutoff,
 * spline).  Waits for the execute to finish. */
int mqct_matrix_plan_timing(mqct_matrix_plan* plan, float* t3);
void mqct_matrix_plan_destroy(mqct_matrix_plan* plan);

/* Learned surrogate of an analytic PES (no counterpart in the reference, which
 * evaluates its PES plugin at every grid point): a multilayer perceptron
 * V(R, angles) with n_hidden_layers SiLU layers of `hidden` units on the
 * features (R - c)/s and cos, sin of (beta1, gamma1, alpha2, beta2, gamma2),
 * trained on the GPU (FP32, Adam, cosine-decayed learning rate) on n_samples
 * seeded points of the PES with R uniform in [r_min, r_max] and the angles
 * uniform on the grid's domain.  sys_type selects the angles used and the PES
 * argument mapping (1: LEGENDRE or SITES1; 4: SITES1 or LEGENDRE; 0: SITES2).
 * A surrogate is not re-entrant: one call at a time. */
typedef struct mqct_surrogate mqct_surrogate;
int mqct_surrogate_create(int32_t sys_type, const mqct_pes_t* pes, int32_t hidden,
                          int32_t n_hidden_layers, uint64_t seed, double r_min, double r_max,
                          mqct_surrogate** out);
/* loss_per_epoch: epochs entries (MSE of the last batch, target units) or NULL;
 * val_rmse: RMSE on a held-out seeded set (target units) or NULL. */
int mqct_surrogate_train(mqct_surrogate* sur, int64_t n_samples, int32_t epochs, int32_t batch,
                         double lr, double* loss_per_epoch, double* val_rmse);
/* V (cm^-1) at n points args[6 i + (0..5)] = (R, beta1, gamma1, alpha2, beta2, gamma2). */
int mqct_surrogate_predict(mqct_surrogate* sur, const double* args, int64_t n, double* v_out);
int64_t mqct_surrogate_n_params(const mqct_surrogate* sur);
/* Parameters, flat: per layer W (in x out, row-major) then b (out). */
int mqct_surrogate_get_params(mqct_surrogate* sur, float* out);
/* Mean squared error of the network on n feature rows X (n x 11) against targets
 * y, and its gradient with respect to the flat parameters (the training step's
 * backward pass). */
int mqct_surrogate_loss_grad(mqct_surrogate* sur, const float* X, const float* y, int32_t n,
                             double* loss, float* grad_out);
void mqct_surrogate_destroy(mqct_surrogate* sur);
/* Use a trained surrogate for the PES table of a plan's builds.  Every execute
 * evaluates the network on the whole (grid x R) table, evaluates the exact PES on
 * n_check grid points per radial point, and re-evaluates the whole grid exactly at
 * every radial point where some checked |V_net - V| exceeds rel_bound |V| +
 * abs_bound_cm.  The surrogate must outlive the plan's executes; NULL detaches. */
int mqct_matrix_plan_set_surrogate(mqct_matrix_plan* plan, mqct_surrogate* sur, double rel_bound,
                                   double abs_bound_cm, int32_t n_check);
/* After an execute: radial points re-evaluated exactly, and the largest checked
 * |V_net - V| / (rel_bound |V| + abs_bound_cm). */
int mqct_matrix_plan_surrogate_stats(mqct_matrix_plan* plan, int32_t* n_exact_r, double* max_ratio);

/* Spline fit of device-resident matrix columns without any device allocation
 * (this entry point has no counterpart in the reference, which fits its splines
 * on the host).  d_R: nR grid points, d_mat: P x nR values (column k at
 * k * nR), d_skipped: optional per-column flags (y2 = 0 where set), d_y2: P x nR
 * output; all device pointers; stream: a cudaStream_t or NULL.  The grid-only
 * coefficients live in a fixed device array of the library, so nR is limited
 * to 399 (MQCT_E_RANGE beyond).  The first call on each device (with that
 * device current) looks up the array's address and keeps it for the life of
 * the process; make that first call before any stream capture.  After a
 * cudaDeviceReset the library's device arrays are reloaded at new addresses, so
 * a process that resets a device must not call this entry point again.  Calls
 * that may overlap in time (other streams or host threads) share the array and
 * race: the caller serialises them. */
int mqct_spline_y2_noalloc(const double* d_R, int32_t nR, const double* d_mat,
                           const int32_t* d_skipped, int64_t P, double* d_y2, void* stream);

/* Propagation tables after READ_MIJ / MATRIX_MAKE: the retained pairs only
 * (elements dropped by MIJ_CUTOFF removed, MQCT_SOURCE_CODES/matrix_ini.f:4309-4378),
 * Mat_el already shifted when MIJ_SHIFT is on (:4270-4273). */
typedef struct mqct_tables_t {
  int32_t n_states;
  const int32_t* j12;
  const int32_t* m12;
  const double* ej;          /* Hartree, per state                              */
  int64_t P;
  const int32_t* ind_mat;    /* 2*P, 1-based                                    */
  int32_t nR;
  const double* R;
  const double* mat;         /* P x nR, Hartree                                 */
  const double* y2;          /* spline second derivatives, same layout          */
  double mass_au;            /* reduced mass in electron masses                 */
} mqct_tables_t;

/* One trajectory (DOTRAJECT initial conditions MQCT_SOURCE_CODES/propagator.f:2435-2566
 * and stop rules :4033-4050). */
typedef struct mqct_traj_init_t {
  double e_coll;             /* collision energy, Hartree                       */
  double l_real;             /* orbital angular momentum quantum number         */
  int32_t s_st;              /* initial state, 1-based                          */
  double dt;                 /* RK4 step, a.u.                                  */
  double r_start;            /* R at t=0 (RMAX)                                 */
  double r_fin;              /* stop when R > r_fin                             */
  int32_t numb_orb_prds;     /* stop after this many orbits (reference default 1) */
  int32_t numb_oscl_prds;    /* stop after this many R oscillations (default 1) */
  double time_lim;           /* <= 0: none                                      */
  int64_t max_steps;         /* device step cap; reaching it sets status 1      */
} mqct_traj_init_t;

/* AT-MQCT classical paths: per trajectory n_rec[t] records of
 * (t, R, P_R, theta, P_theta, phi, P_phi, pot), concatenated in rec with
 * offsets rec_off[t] (in records). */
typedef struct mqct_at_paths_t {
  const int64_t* rec_off;
  const int32_t* n_rec;
  const double* rec;
} mqct_at_paths_t;

/* Batched propagation.  amp_out: n_traj x 2N (Re a, Im a); cls_out: n_traj x 6
 * (R, P_R, theta, P_theta, phi, P_phi); diag_out: n_traj x 8 (t_end, steps,
 * |1-norm|, |energy error| Hartree, status, orbits, oscillations, coupling
 * energy at the end).  status: 0 finished, 1 step cap reached, 2 not
 * propagated (impact parameter beyond RMAX), 3 non-finite state.  mode:
 * MQCT_MODE_STD or MQCT_MODE_AT, either OR-ed with MQCT_MODE_CS for the
 * coupled-states approximation (states of other m12 than the initial state's keep
 * zero amplitude, as the reference's skipped pairs leave them). */
int mqct_propagate_batch(const mqct_tables_t* tab, const mqct_traj_init_t* init,
                         int64_t n_traj, int32_t mode, const mqct_at_paths_t* at,
                         int32_t arith, double* amp_out, double* cls_out, double* diag_out);

/* Device-resident propagation plan (tables uploaded once; trajectories given
 * per call).  run() uses host trajectory/out buffers; run_device() takes device
 * buffers for init (n_traj mqct_traj_init_t) and outputs. */
/* The same in standard mode with SAVE_TRAJECT = YES (the classical paths of the
 * first AT-MQCT run, MQCT_SOURCE_CODES/propagator.f:2866-2880, 3458-3464, 4329-4337):
 * rec_out (host, n_traj * max_rec * 8 doubles) receives per trajectory the records
 * (t, R, P_R, theta, P_theta, phi, P_phi, pot) of the state at the top of every
 * RK4 step, pot the coupling energy, then one record of the final state stamped
 * t_final + dt; n_rec_out[t] = records produced (those past max_rec are counted,
 * not written).  Record t of a trajectory is at rec_out[(t * max_rec + r) * 8]. */
int mqct_propagate_batch_rec(const mqct_tables_t* tab, const mqct_traj_init_t* init,
                             int64_t n_traj, int32_t arith, int64_t max_rec, double* amp_out,
                             double* cls_out, double* diag_out, double* rec_out,
                             int64_t* n_rec_out);

/* Time integrator of the propagation (PROPAGATOR = RK4 | ODEINT of $SYSTEM,
 * MQCT_SOURCE_CODES/iotest.f:2628-2640, 2676-2681).  ODEINT is the reference's adaptive
 * Cash-Karp scheme (rkqs / rkck / odeint, MQCT_SOURCE_CODES/suppl_routines.f:1229-1435):
 * in standard mode every step dt of DOTRAJECT is covered by adaptive steps with
 * relative accuracy eps (eps_odeint) and minimum step hmin (min_t_stp), the step
 * size carried from one dt to the next (propagator.f:3933-3941); in AT mode one such
 * call covers the whole saved path (propagator.f:3900-3908).  The stop rules, records
 * and energy bookkeeping stay per step dt.  ODEINT requires MQCT_PROP_FP64: its error
 * control resolves every amplitude to relative eps, below the FP32 rounding of the
 * right-hand side, so FP32 steps would collapse (MQCT_E_ARG).  As in the reference,
 * the error scale |y| + |h dy/dt| + 1e-30 also covers amplitudes at rounding level:
 * with hmin = 0 the step can collapse where their rounding noise dominates, and a
 * step at or below hmin is accepted without a new step proposal, so once the step
 * reaches hmin it stays there; a small positive hmin bounds the cost. */
#define MQCT_INTEG_RK4 0
#define MQCT_INTEG_ODEINT 1
/* AT_ADAPT_STP = YES (MQCT_SOURCE_CODES/propagator.f:3034-3049, 3821-3860): RK4 whose
 * steps in AT mode follow the coupling energy along the saved path; eps carries
 * AT_ADAPTOL (reference default 0.5), hmin the unscaled TIME_STEP (the smallest step).
 * Standard-mode runs keep their fixed dt. */
#define MQCT_INTEG_AT_ADAPT 2
/* PROPAGATOR = ODEINT with bikram_int (bk_int / bk_int_adia,
 * MQCT_SOURCE_CODES/suppl_routines.f:1468-1856, called at propagator.f:3889-3900,
 * 3925-3931): one adaptive Cash-Karp call over [0, TIME_LIM] (standard mode; dt is
 * its first step) or over the whole saved path (AT mode) that stops after any step at
 * which R > R_fin or the oscillation or orbit caps are reached (in AT mode R and phi
 * from the path's splines); eps and hmin as for ODEINT; FP64 arithmetic. */
#define MQCT_INTEG_BK_INT 3
typedef struct mqct_integrator_t {
  int32_t method;   /* MQCT_INTEG_* */
  double eps;       /* ODEINT accuracy (> 0) */
  double hmin;      /* ODEINT minimum step, a.u. (>= 0) */
} mqct_integrator_t;
/* mqct_propagate_batch with an integrator other than RK4. */
int mqct_propagate_batch_integ(const mqct_tables_t* tab, const mqct_traj_init_t* init,
                               int64_t n_traj, int32_t mode, const mqct_at_paths_t* at,
                               int32_t arith, const mqct_integrator_t* integ, double* amp_out,
                               double* cls_out, double* diag_out);

/* INELAST_CALC on the device (MQCT_SOURCE_CODES/propagator.f:4752-4851) from device
 * amplitudes d_amp (n_traj x 2 n_states, the layout of mqct_propagate_batch's amp_out;
 * trajectory t covers the l bin [L_MIN + t DL, L_MIN + (t + 1) DL)): per trajectory the
 * channel probabilities d_prob (n_traj x n_channels), the J-resolved cross sections
 * d_partial ((J_up - J_down + 1) x n_channels, PARTIAL_CROSS_SECTIONS_J.out) and their
 * sums d_sigma (n_channels, M_PROJ_CROSSECTIONS.out), all in Angstrom^2, for the initial
 * j12 = j_ini; the l of partial wave J maps to trajectory (l - L_MIN) / DL (TRAJ_ORB,
 * :5127-5134).  indx_chann (host, per state, 1-based) must be channel-major; at most
 * 2048 channels.  Runs on `stream` (cudaStream_t, NULL: the default stream), allocates
 * nothing and returns without synchronising. */
int mqct_cross_sections_device(const double* d_amp, int64_t n_traj, int32_t n_states,
                               const int32_t* indx_chann, int32_t n_channels, int32_t j_ini,
                               int32_t J_down, int32_t J_up, int32_t L_min, int32_t dl,
                               double k_vec, double* d_prob, double* d_partial, double* d_sigma,
                               void* stream);

typedef struct mqct_prop_plan mqct_prop_plan;
int mqct_prop_plan_create(const mqct_tables_t* tab, int32_t arith, mqct_prop_plan** plan);
int mqct_prop_plan_run(mqct_prop_plan* plan, const mqct_traj_init_t* init, int64_t n_traj,
                       double* amp_out, double* cls_out, double* diag_out);
int mqct_prop_plan_run_device(mqct_prop_plan* plan, const mqct_traj_init_t* d_init,
                              int64_t n_traj, double* d_amp, double* d_cls, double* d_diag);
int mqct_prop_plan_sync(mqct_prop_plan* plan);
/* Algorithmic table bytes of one RK4 step of one trajectory: 4 right-hand sides,
 * each reading two knot rows of (M, y2) and the slot locations over S slots (the
 * full lower triangle of every m-block): 4 * S * (4 * sizeof(T) + 4). */
double mqct_prop_plan_bytes_per_step(const mqct_prop_plan* plan);
/* CUDA-event time (ms) of the last propagation kernel on the plan's stream. */
int mqct_prop_plan_timing(mqct_prop_plan* plan, float* ms);
void mqct_prop_plan_destroy(mqct_prop_plan* plan);
/* Select the plan's integrator for the following runs (default RK4). */
int mqct_prop_plan_set_integrator(mqct_prop_plan* plan, const mqct_integrator_t* integ);
/* CS_APPROX for the following runs of the plan (cs != 0), as MQCT_MODE_CS does for
 * one batch call. */
int mqct_prop_plan_set_coupled_states(mqct_prop_plan* plan, int32_t cs);
/* Launch-shape autotuning of the RK4 kernel (no counterpart in the reference, which
 * runs one trajectory per MPI rank): the shapes 512 threads x 1 CTA per SM and 256
 * threads x 2 CTAs per SM (each with its own split of the m-blocks into shared-memory
 * passes) are timed on the first min(n_traj, 4 x SMs) of these trajectories, each capped
 * at 32 steps, results discarded, and the faster shape is kept for the plan's runs.
 * mqct_prop_plan_run tunes by itself on its first batch of at least 2 x SMs
 * trajectories.  mqct_prop_plan_shape reports the shape (threads per CTA, CTAs per SM)
 * and, after tuning, the probe times in ms (probe_ms[2], may be NULL). */
int mqct_prop_plan_tune(mqct_prop_plan* plan, const mqct_traj_init_t* init, int64_t n_traj,
                        int32_t mode);
int mqct_prop_plan_shape(const mqct_prop_plan* plan, int32_t* threads, int32_t* ctas_per_sm,
                         float* probe_ms);
/* Propagation engines (no counterpart in the reference, which integrates one trajectory
 * per MPI rank).  MQCT_ENGINE_PER_TRAJECTORY: the persistent kernel that holds one
 * trajectory per CTA (every mode and integrator).  MQCT_ENGINE_LOCKSTEP: all trajectories
 * of the batch advance one RK4 stage per round, grouped by the spline interval of their
 * stage point, so that a group shares one load of the interval's knot rows; standard
 * mode, RK4, no CS approximation, no SAVE_TRAJECT records, m-blocks of at most 128
 * states (other runs take the per-trajectory kernel).  Its right-hand side applies the
 * spline as four knot products (M_lo, M_hi - M_lo, M''_lo, M''_hi) per interval instead of
 * interpolating slot by slot: the same arithmetic type, other rounding.  Its device-buffer
 * runs (mqct_prop_plan_run_device) read the initial conditions back for the bound on the
 * rounds and return when the batch is done.  MQCT_ENGINE_AUTO (default): the lockstep
 * engine for eligible batches of at least 4096 trajectories, the resident engine (below)
 * for eligible FP32 batches of at most 1024, and for eligible FP32 batches of at least 4096
 * MQCT_ENGINE_LOCKSTEP_TAIL: the lockstep engine until at most six trajectories per
 * resident cluster still run, then the resident engine, which continues each of them from
 * the start of its RK4 step (mqct_prop_plan_handed reports how many the last run handed
 * over; FP64 plans and tables the resident engine does not take run the plain lockstep
 * engine).  MQCT_ENGINE_RESIDENT: one
 * thread-block cluster per trajectory, the m-blocks split between its CTAs, each holding
 * the two knot rows of its blocks in shared memory (reloaded when the stage point leaves
 * the spline interval); the CTAs exchange their parts of the quadratic forms and the
 * neighbour amplitudes of the Coriolis vector through distributed shared memory once per
 * right-hand side.  FP32 plans, standard mode, RK4, no CS, no records, m-blocks of at
 * most 255 states, and the tables must fit the shared memory of a cluster of at most 8
 * CTAs (other runs take the engine the AUTO rule picks).  Its arithmetic is that of the
 * per-trajectory kernel (slot-by-slot interpolation), with other summation orders.
 * MQCT_ENGINE_AUTO takes it for eligible FP32 batches of at most 1024 trajectories (fewer
 * trajectories at once, each faster: the faster engine for such batches).
 * mqct_prop_plan_engine reports the engine of the last run and, for the lockstep engine,
 * the rounds it ran (rounds may be NULL). */
#define MQCT_ENGINE_AUTO 0
#define MQCT_ENGINE_PER_TRAJECTORY 1
#define MQCT_ENGINE_LOCKSTEP 2
#define MQCT_ENGINE_RESIDENT 3
#define MQCT_ENGINE_LOCKSTEP_TAIL 4
int mqct_prop_plan_set_engine(mqct_prop_plan* plan, int32_t engine);
int mqct_prop_plan_engine(const mqct_prop_plan* plan, int32_t* engine, int64_t* rounds);
/* Cluster size of the resident engine: 0 (default) eight CTAs for a batch that the
 * clusters of eight hold at once, else the smallest of 2..8 CTAs whose shared memory holds
 * the tables; or a size in 2..8 (used when the tables fit it).  mqct_prop_plan_cluster
 * reports the cluster size and the clusters resident on the device: those of the last run
 * when it took the resident engine, else those of the setting (0 meaning the smallest
 * size) for the plan's tables; both 0 when the engine does not apply to the plan. */
int mqct_prop_plan_set_cluster(mqct_prop_plan* plan, int32_t ctas);
int mqct_prop_plan_handed(const mqct_prop_plan* plan, int32_t* n);
int mqct_prop_plan_cluster(mqct_prop_plan* plan, int32_t* ctas, int32_t* clusters);

/* Host-side helpers mirroring INI_ARRAYS / EIGEN_VEC / the R grid. */
int mqct_asym_top_level(double A, double B, double C, int32_t j, int32_t ka, int32_t kc,
                        double* energy, double* vec);
int mqct_count_states(int32_t sys_type, int32_t n_channels, const int32_t* j1,
                      const int32_t* j2);
int mqct_enumerate_states(int32_t sys_type, int32_t n_channels, const int32_t* j1,
                          const int32_t* j2, int32_t* indx_chann, int32_t* j12, int32_t* m12);
int64_t mqct_count_pairs(int32_t n_states, const int32_t* m12);
int64_t mqct_fill_ind_mat(int32_t n_states, const int32_t* m12, int32_t* ind_mat);
/* Identical partners (SYS_TYPE 0, IDENTICAL = YES; MQCT_SOURCE_CODES/matrix_ini.f:482-530,
 * 553-627): per channel, for p = 1 and (unless both rotors are in the same level) p = 2,
 * the states (j12, m12) with exchange parity (-1)^(p-1), -1 for odd j12 of a same-level
 * channel; pairs only between states of equal parity.  Same argument conventions as
 * above; parity receives +1/-1 per state. */
int mqct_count_states_identical(int32_t n_channels, const int32_t* j1, const int32_t* ka1,
                                const int32_t* kc1, const int32_t* j2, const int32_t* ka2,
                                const int32_t* kc2);
int mqct_enumerate_states_identical(int32_t n_channels, const int32_t* j1, const int32_t* ka1,
                                    const int32_t* kc1, const int32_t* j2, const int32_t* ka2,
                                    const int32_t* kc2, int32_t* indx_chann, int32_t* j12,
                                    int32_t* m12, int32_t* parity);
int64_t mqct_count_pairs_identical(int32_t n_states, const int32_t* m12, const int32_t* parity);
int64_t mqct_fill_ind_mat_identical(int32_t n_states, const int32_t* m12, const int32_t* parity,
                                    int32_t* ind_mat);
int mqct_r_grid(int32_t n, double rmin, double rmax, int32_t equidistant, double* R);

/* MTRX_UF.DAT (Fortran unformatted sequential, 4-byte record markers):
 * header (coll_type, n_channels, n_states, P, nR), n_states state records of
 * state_rec_len int32, P records (k, st1, st2), nR records (i, R), then per k
 * a record (k) and a record Mat_el(:,k). */
int mqct_write_mtrx_uf(const char* path, int32_t coll_type, int32_t n_channels,
                       int32_t n_states, const int32_t* state_rec, int32_t state_rec_len,
                       int64_t P, const int32_t* ind_mat, int32_t nR, const double* R,
                       const double* mat);
int mqct_read_mtrx_uf_header(const char* path, int32_t* coll_type, int32_t* n_channels,
                             int32_t* n_states, int64_t* P, int32_t* nR,
                             int32_t* state_rec_len);
int mqct_read_mtrx_uf(const char* path, int32_t state_rec_len, int32_t* state_rec,
                      int32_t* ind_mat, double* R, double* mat);

/* Formatted MTRX.DAT (SAVE_MTRX / READ_MTRX with UNFORMAT = NO): PRINT_MIJ and READ_MIJ,
 * MQCT_SOURCE_CODES/matrix_ini.f:4692-4877 and 5794-6630.  Five header counts, the
 * state table (the columns of state_rec, SYS_TYPE 1, 3, 4, 5, 7, 8, 9 or 0 for the writer), the
 * pairs, the R grid (e19.12) and one line (k, iR, Mij) per element (e19.12).  The
 * header reader returns the counts and the number of state columns. */
int mqct_write_mtrx_dat(const char* path, int32_t coll_type, int32_t n_channels,
                        int32_t n_states, const int32_t* state_rec, int32_t state_rec_len,
                        int64_t P, const int32_t* ind_mat, int32_t nR, const double* R,
                        const double* mat);
int mqct_read_mtrx_dat_header(const char* path, int32_t* coll_type, int32_t* n_channels,
                              int32_t* n_states, int64_t* P, int32_t* nR,
                              int32_t* state_rec_len);
int mqct_read_mtrx_dat(const char* path, int32_t state_rec_len, int32_t* state_rec,
                       int32_t* ind_mat, double* R, double* mat);

/* PES_EXPAN_TERMS.DAT (READ_EXPANSION_TERMS, MQCT_SOURCE_CODES/pot_comp.f:6344-6388): a
 * header line, then per R point R and n_terms coefficients.  R[iR] and
 * terms[t * nR + iR] (the expansion_terms(n_r_coll, nterms) layout that
 * mqct_build_matrix_expansion takes); values in the file's energy unit. */
int mqct_read_expansion_terms(const char* path, int32_t nR, int32_t n_terms, double* R,
                              double* terms);
/* The PES_EXPAN_TERMS.DAT writer of CALC_EXPANSION_TERMS
 * (MQCT_SOURCE_CODES/pot_comp.f:5918-6270), SYS_TYPE 7, 8 and 0: appends R[iR] and
 * terms[t * nR + iR] to path, the header line first when the file holds at most one
 * line (runs over consecutive R ranges, IR_BGN / IR_FIN, share one file). */
int mqct_write_expansion_terms(const char* path, int32_t sys_type, int32_t n_terms,
                               const int32_t* a_top, int32_t nR, const double* R,
                               const double* terms);

/* The per-energy result files, appended block by block as the reference appends them:
 *   mqct_write_opacity: OPACITY_FUNCTIONS_L.out and (path_total, may be NULL)
 *     TOTAL_PROBABILITIES_L.out (MQCT_SOURCE_CODES/propagator.f:5837-5896): per trajectory
 *     l / k_vec, l and the channel probabilities prob[t * n_ch + c]; the totals file the
 *     sum over channels and the sum without chann_ini (1-based);
 *   mqct_write_partial_j: PARTIAL_CROSS_SECTIONS_J.out (:4845-4868), per total J the
 *     J-resolved cross sections partial[i * n_ch + c] in Angstrom^2;
 *   mqct_write_m_proj: M_PROJ_CROSSECTIONS.out (:4870-4880), the cross sections of one
 *     initial state without the Billing correction, Angstrom^2;
 *   mqct_write_cross_sections: one energy block of CROSS_SECTIONS.out
 *     (MQCT_SOURCE_CODES/print_output.f:46-101): sigma(U) = sigma_f / U * E_bill, E_bill
 *     and sigma_f for the channels with exists[c] != 0 (all when exists is NULL), the
 *     probability and, with with_e_err, energy conservation errors in percent;
 *     mqct_write_cross_sections_footer: the closing trajectory count (:117-118). */
int mqct_write_opacity(const char* path, const char* path_total, int32_t s_st, int32_t j12,
                       int32_t m12, int32_t i_ener, double U_cm, int32_t n_traj, const int32_t* l,
                       double k_vec, int32_t n_ch, const double* prob, int32_t chann_ini);
int mqct_write_partial_j(const char* path, int32_t s_st, int32_t j12, int32_t m12,
                         int32_t i_ener, double U_cm, int32_t n_J, const int32_t* J, int32_t n_ch,
                         const double* partial);
int mqct_write_m_proj(const char* path, int32_t s_st, int32_t i_ener, int32_t j12, int32_t m12,
                      int32_t n_ch, const double* sigma);
int mqct_write_cross_sections(const char* path, double U_cm, int32_t chann_ini, int32_t n_ch,
                              const int32_t* exists, const double* sigma_f, const double* E_bill,
                              double p_err_pct, int32_t with_e_err, double e_err_pct);
int mqct_write_cross_sections_footer(const char* path, int32_t n_traj_total);
/* The elastic-scattering files of ELAST_CALC (MQCT_SOURCE_CODES/propagator.f:5897-5943):
 *   mqct_write_deflection: one block of DEFLECTION_FUNCTION.out, per trajectory l, l / k,
 *     the deflection angle and the scattering phase (rad), the finish time (a.u.), the
 *     energy and norm errors (percent), the orbiting periods and the oscillations of R;
 *   mqct_write_diff_cross: one block of DIFF_CROSS.out, the angles (given in rad, written
 *     in degrees) and the elastic differential cross section (Angstrom^2).
 * The deflection angles, phases and cross sections themselves are host arithmetic on the
 * propagation's outputs (mqct_b200.deflection_angles, scattering_phases,
 * elastic_cross_section, differential_cross_section). */
int mqct_write_deflection(const char* path, int32_t s_st, int32_t j12, int32_t m12,
                          int32_t i_ener, double U_cm, int32_t n_traj, const int32_t* l,
                          double k_vec, const double* deflection, const double* phase,
                          const double* finish_time, const double* e_err_pct,
                          const double* p_err_pct, const int32_t* periods,
                          const int32_t* oscillations);
int mqct_write_diff_cross(const char* path, int32_t i_ener, int32_t s_st, int32_t j12,
                          int32_t m12, int32_t n_angles, const double* theta_rad,
                          const double* dcs);
/* SPLINED_DEFLECTION_OPACITY_L.out of PROB_SPLINE runs (MQCT_SOURCE_CODES/propagator.f:
 * 6063-6110): per integer l (l[i], i < n_l) l / k, l, the splined deflection function and
 * the splined channel probabilities prob[i * n_ch + c] (mqct_b200.splined_opacity). */
int mqct_write_splined_opacity(const char* path, int32_t n_l, const int32_t* l, double k_vec,
                               const double* deflection, int32_t n_ch, const double* prob);

/* CALC_EXPANSION_TERMS (MQCT_SOURCE_CODES/pot_comp.f:4695-6274; replaces the R-grid
 * loop of :5174-5765 and EXPANSION_TERM, :3739-3896), SYS_TYPE 1, 3, 4, 7, 8, 9 and 0: the
 * quadrature projection of the PES tabulated on the angular grid onto the expansion
 * terms,
 *   terms[t * nR + iR]    = sum_g V Re(EXPANSION_TERM_t) w(g)    (intgrlr)
 *   terms_im[t * nR + iR] = sum_g V Im(EXPANSION_TERM_t) w(g)    (intgrli)
 * with the weights and grids of INI_POT_STORAGE: grid->n_beta = beta1 and
 * grid->n_beta2 = beta2 (Gauss-Legendre on [0, pi]); grid->n_alpha2 = alpha2,
 * grid->n_gamma = gamma1 and, for SYS_TYPE 0, grid->n_gamma2 = gamma2 (on [0, 2 pi],
 * midpoint-equidistant when eq_gamma, else Gauss-Legendre); grid->n_alpha unused.
 * V in the reference's V_3_2 / V_TRANSFER order, V[iR][alpha2][beta1][beta2][gamma1]
 * (SYS_TYPE 7, 8) or V[iR][alpha2][beta1][beta2][gamma1][gamma2] (SYS_TYPE 9 and 0), in the
 * unit the terms are wanted in.  For a rotor and an atom (cases 1, 3 and 4, :4973-5104;
 * case 3 is case 4) V is V_2_1, V[iR][beta] (SYS_TYPE 1, grid->n_beta), or V_3_1,
 * V[iR][beta][gamma] (SYS_TYPE 3 and 4, grid->n_beta and grid->n_gamma), and a_top
 * holds (l, -, ...) or (l, nju, -, ...), nju >= 0.  a_top: A_TOP(5, nterms), (l1, nju1,
 * l2, l, -) for 7 and 8, (l1, nju1, l2, nju2, l) for 0, checked as the reference checks a term list
 * (triangle rule, nju1 >= 0, nju2 >= 0 when nju1 = 0, no term twice up to the sign of
 * the nju's; with identical != 0, SYS_TYPE 0 only, also l1 >= l2, |nju1| >= |nju2|
 * when l1 = l2 and no term twice up to the exchange of the partners): MQCT_E_ARG
 * otherwise.  The plan forms the per-term tables once; _execute projects device V
 * (d_V) into device d_terms and d_terms_im (may be NULL) on the plan's stream,
 * asynchronously; _timing gives the device milliseconds of the three contractions
 * (gamma, alpha2, beta) of the last single-pass execute.  mqct_project_terms is the
 * one-shot form on host buffers. */
typedef struct mqct_projection_plan mqct_projection_plan;
int mqct_projection_plan_create(int32_t sys_type, int32_t n_terms, const int32_t* a_top,
                                const mqct_grid_t* grid, int32_t identical,
                                mqct_projection_plan** plan);
int mqct_projection_plan_execute(mqct_projection_plan* plan, const double* d_V, int32_t nR,
                                 double* d_terms, double* d_terms_im);
int mqct_projection_plan_sync(mqct_projection_plan* plan);
int mqct_projection_plan_timing(mqct_projection_plan* plan, float* ms_gamma, float* ms_alpha,
                                float* ms_terms);
void mqct_projection_plan_destroy(mqct_projection_plan* plan);
int mqct_project_terms(int32_t sys_type, int32_t n_terms, const int32_t* a_top,
                       const mqct_grid_t* grid, int32_t identical, int32_t nR, const double* V,
                       double* terms, double* terms_im);

#ifdef __cplusplus
}
#endif
#endif
