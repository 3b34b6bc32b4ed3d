/*
 * mqct_oracle.h -- CPU FP64 oracle for the MQCT matrix-build and propagation
 * hot paths.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain-C restatement of the
 * reference algorithm (MarquetteQuantum/MQCT, Fortran).  It is the checker
 * that the CUDA product is compared against; only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it.  The product never links it.
 *
 * Every routine cites the reference file:line it restates
 * (paths relative to the MQCT repository; SRC = MQCT_SOURCE_CODES).
 *
 * Conventions: indices that cross this ABI in ind_mat / indx_chann are
 * 1-based (as in the reference); matrices are stored R-fastest
 * (mat[k*nR + iR]), i.e. the Fortran column-major Mat_el(n_r, P).
 */
#ifndef MQCT_ORACLE_H
#define MQCT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- numerics (SRC/suppl_routines.f) ---------------- */
void   orc_gauleg(int n, double* x, double* w);
double orc_plgndr(int l, int m, double x);
void   orc_jacobi_poly(int n, double a, double b, double x, double* cx);
double orc_w3js(int j1, int j2, int j3, int m1, int m2, int m3); /* doubled args */
double orc_cg(int j1, int j2, int j3, int m1, int m2, int m3);
void   orc_spline(const double* x, const double* y, int n, double yp1, double ypn, double* y2);
void   orc_splint(const double* xa, const double* ya, const double* y2a, int n,
                  double x, double* y, double* yprime);

/* ---------------- rotor functions ---------------- */
void orc_djkm(int j, int k, int m, double alpha, double beta, double gamma,
              double* re, double* im);
void orc_wf_diat(int j, int m, double theta, double phi, double* re, double* im);
/* Rigid asymmetric-top level (j, ka, kc): energy (same units as A,B,C) and the
 * (2j+1) symmetric-top coefficients ordered K=-j..j.  Returns 0 or <0. */
int  orc_asym_top(double A, double B, double C, int j, int ka, int kc,
                  double* energy, double* vec);
void orc_wf_sym(int j, int k, int eps, int m, double alpha, double beta, double gamma,
                double* re, double* im);
void orc_wf_asym(int j, const double* coeff, int m, double alpha, double beta,
                 double gamma, double* re, double* im);

/* ---------------- system / states (SRC/matrix_ini.f) ---------------- */
typedef struct orc_system {
  int32_t sys_type;      /* 1 diatom+atom, 4 asym top+atom, 7 sym top+diatom,
                            8 asym top+diatom, 0 asym+asym */
  int32_t n_channels;
  const int32_t* j1;     /* per channel: j (type 1,4) or j1 (type 8,0) */
  const int32_t* ka1;    /* type 7: k of the symmetric top */
  const int32_t* kc1;    /* type 7: eps (parity) */
  const int32_t* j2;     /* type 8, 0 */
  const int32_t* ka2;    /* type 0 */
  const int32_t* kc2;
  const double* e_ch;    /* channel energies, cm^-1 */
  const double* vec1;    /* eigenvectors of rotor 1, per channel, stride ldv (K=-j..j) */
  const double* vec2;    /* eigenvectors of rotor 2 (type 0) */
  int32_t ldv;
} orc_system;

int orc_count_states(const orc_system* sys);
/* Fills indx_chann (1-based), j12, m12, Ej (cm^-1) for n states. */
int orc_enumerate_states(const orc_system* sys, int32_t* indx_chann, int32_t* j12,
                         int32_t* m12, double* ej);
int64_t orc_count_pairs(int n_states, const int32_t* m12);
int64_t orc_ind_mat(int n_states, const int32_t* m12, int32_t* ind_mat /* 2*P */);

void orc_rgrid(int n, double rmin, double rmax, int equidistant, double* R);

/* ---------------- synthetic PES (the plugin USER_DEFINED_PES) ---------------- */
enum { ORC_PES_LEGENDRE = 1, ORC_PES_SITES1 = 2, ORC_PES_SITES2 = 3, ORC_PES_TABLE = 0 };
typedef struct orc_pes {
  int32_t kind;
  int32_t n_terms;
  const double* p;       /* kind-specific parameter block, see oracle source */
  int32_t n_sites1, n_sites2;
  const double* sites1;  /* xyz per site, body frame of rotor 1 */
  const double* sites2;
  const double* table;   /* kind TABLE: V[iR][g] over the full angular grid */
} orc_pes;
/* USER_DEFINED_PES(V,R,rvib,rvib2,alpha,beta,gamma,aalpha,bbeta,ggamma) */
double orc_pes_eval(const orc_pes* pes, double R, double alpha, double beta, double gamma,
                    double aalpha, double bbeta, double ggamma);

/* ---------------- matrix build (SRC/matrix_ini.f MATRIX_MAKE, SRC/pot_comp.f) ---- */
typedef struct orc_grid {
  int32_t n_beta, n_gamma, n_alpha;      /* type 1: n_beta; type 4: beta x gamma (x alpha) */
  int32_t n_beta2, n_alpha2, n_gamma2;   /* type 0: beta1=n_beta, gamma1=n_gamma */
  int32_t eq_gamma;                      /* EQ_ANG_GRID (default 1): midpoint gamma/alpha grids */
} orc_grid;

/* Full build: Mat_el (Hartree) and spline second derivatives, MIJ_CUTOFF
 * truncation.  literal != 0 re-evaluates the rotor wavefunctions at every
 * grid point for every (k, R) exactly as INTEGRATOR_TEMP does (the reference
 * cost); literal == 0 tabulates them once (same arithmetic per point).
 * k_begin/k_end restrict the elements computed (others left untouched).
 * n_threads <= 0 uses all OpenMP threads.  Returns 0 or <0. */
int orc_build_matrix(const orc_system* sys, int n_states, const int32_t* indx_chann,
                     const int32_t* j12, const int32_t* m12, int64_t P,
                     const int32_t* ind_mat, int nR, const double* R,
                     const orc_grid* grid, const orc_pes* pes,
                     double mij_cut_cm, double r_cut1, double r_cut2, int literal,
                     int64_t k_begin, int64_t k_end, int n_threads,
                     double* mat, double* y2, int32_t* skipped);
/* Only the quadrature (no cutoff/spline), values in cm^-1, for timing samples. */
int orc_integrate_elements(const orc_system* sys, int n_states, const int32_t* indx_chann,
                           const int32_t* j12, const int32_t* m12, int64_t P,
                           const int32_t* ind_mat, int nR, const double* R,
                           const orc_grid* grid, const orc_pes* pes, int literal,
                           int64_t k_begin, int64_t k_end, int iR_begin, int iR_end,
                           int n_threads, double* mat);

/* ---------------- MTRX_UF.DAT / MTRX.DAT (SRC/matrix_ini.f) ---------------- */
int orc_write_mtrx_uf(const char* path, int coll_type, int n_channels, int n_states,
                      const int32_t* state_rec, int state_rec_len, int64_t P,
                      const int32_t* ind_mat, int nR, const double* R, const double* mat);
/* Formatted MTRX.DAT reader (header counts first, then arrays). */
int orc_read_mtrx_dat_header(const char* path, int* coll_type, int* n_channels,
                             int* n_states, int64_t* P, int* nR);
int orc_read_mtrx_dat(const char* path, int n_state_cols, int32_t* state_cols,
                      int32_t* ind_mat, double* R, double* mat);

/* ---------------- propagation (SRC/mqct_eqtns.f, SRC/propagator.f) ---------- */
typedef struct orc_tables {
  int32_t n_states;
  const int32_t* j12;
  const int32_t* m12;
  const double* ej;        /* Hartree */
  int64_t P;
  const int32_t* ind_mat;  /* 2*P, 1-based, only the retained (non-truncated) pairs */
  int32_t nR;
  const double* R;
  const double* mat;       /* P x nR (R fastest), Hartree */
  const double* y2;        /* spline second derivatives, same layout */
  double mass_au;          /* reduced mass, electron masses */
} orc_tables;

typedef struct orc_traj {
  double e_coll;           /* Hartree */
  double l_real;           /* orbital angular momentum quantum number (float) */
  int32_t s_st;            /* initial state, 1-based */
  double dt;               /* atomic units */
  double r_start;          /* R at t=0 (RMAX) */
  double r_fin;            /* stop when R > r_fin */
  int32_t numb_orb_prds;   /* stop after this many orbits (default 1) */
  int32_t numb_oscl_prds;  /* stop after this many R oscillations (default 1) */
  double time_lim;         /* <=0: none */
  int64_t max_steps;
  int32_t method;          /* 0: RK4 (PROPAGATOR = RK4), 1: adaptive Cash-Karp (ODEINT),
                              2: AT mode RK4 with AT_ADAPT_STP steps, 3: standard mode
                              ODEINT with bikram_int: one bk_int call over [0, time_lim]
                              with the stop rules after every adaptive step, dt the
                              first step (int_1st_stp) */
  double eps;              /* ODEINT accuracy (eps_odeint); method 2: AT_ADAPTOL */
  double hmin;             /* ODEINT minimum step (min_t_stp); method 2: TIME_STEP */
  int32_t cs;              /* CS_APPROX = YES: coupled-states approximation */
} orc_traj;

/* Per-trajectory output: amp[2N] (Re, Im), cls[6] = (R,P_R,theta,P_theta,phi,P_phi),
 * diag[8] = (t_end, steps, norm_err, energy_err, status, orbit_cnt, vib_cnt, pot_end). */
int orc_dotraject(const orc_tables* tab, const orc_traj* tr, double* amp, double* cls,
                  double* diag);
int orc_propagate_batch(const orc_tables* tab, int n_traj, const orc_traj* trajs,
                        int n_threads, double* amp, double* cls, double* diag);
/* DOTRAJECT with the SAVE_TRAJECT records (8 doubles each: t, R, P_R, theta,
 * P_theta, phi, P_phi, pot) of the state at the top of every step plus the final
 * state stamped t_final + dt; *n_rec = records produced (written up to max_rec). */
int orc_dotraject_rec(const orc_tables* tab, const orc_traj* tr, double* amp, double* cls,
                      double* diag, double* rec, int64_t max_rec, int64_t* n_rec);
/* AT-MQCT: classical path given as n_at records (t,R,P_R,theta,P_theta,phi,P_phi,pot). */
int orc_dotraject_at(const orc_tables* tab, const orc_traj* tr, int n_at,
                     const double* at_rec, double* amp, double* diag);
/* One RHS evaluation of DERIVS_BK (for unit checks); q, dqdt have 2N+8 entries. */
int orc_derivs(const orc_tables* tab, double t, const double* q, double* dqdt);

/* INELAST_CALC for one initial (j, m) block with integer l = L_MIN..L_MAX step 1:
 * prob[n_traj*n_channels] -> sigma_bohr2[n_channels] (pi/k^2 * sum (2J+1)/(2j+1) P). */
int orc_inelast(int n_channels, int j_ini, int J_down, int J_up, int L_min, int n_traj,
                const double* prob, double k_vec, double* sigma);
/* The same with trajectories every dl values of l (trajectory id = (l - L_min)/dl). */
int orc_inelast_dl(int n_channels, int j_ini, int J_down, int J_up, int L_min, int dl,
                   int n_traj, const double* prob, double k_vec, double* sigma);

/* PES-expansion matrix elements of SYS_TYPE 8 (asymmetric top + diatom),
 * SRC/pot_comp.f:7826-8058 (EXPANSION_MATRIX_ELEMENT, case 8): per stored pair k
 * (stp = ind_mat[2k], stpp = ind_mat[2k+1]) and R point, the sum over terms t of
 * terms[iR * n_terms + t] (cm^-1) times the R-independent angular coefficient of
 * (l1, nju1, l2, l) = labels[4t .. 4t+3]; mat[k * nR + iR] in Hartree. */
int orc_expansion_matrix_type8(const orc_system* sys, const int32_t* indx_chann,
                               const int32_t* j12, const int32_t* m12, int64_t P,
                               const int32_t* ind_mat, int n_terms, const int32_t* labels,
                               int nR, const double* terms, double* mat);

/* SYS_TYPE 0 (two asymmetric tops, distinguishable), SRC/pot_comp.f:8257-8746:
 * labels[5t .. 5t+4] = (l1, nju1, l2, nju2, l) (the A_TOP columns), terms in the
 * file's energy unit, e_unit = Hartree per that unit. */
int orc_expansion_matrix_type0(const orc_system* sys, const int32_t* indx_chann,
                               const int32_t* j12, const int32_t* m12, int64_t P,
                               const int32_t* ind_mat, int n_terms, const int32_t* labels,
                               int nR, const double* terms, double e_unit, double* mat);

/* SYS_TYPE 7 (symmetric top + diatom), SRC/pot_comp.f:7593-7824: the channel's k in
 * sys->ka1 and eps in sys->kc1; labels[4t .. 4t+3] = (l1, nju1, l2, l). */
int orc_expansion_matrix_type7(const orc_system* sys, const int32_t* indx_chann,
                               const int32_t* j12, const int32_t* m12, int64_t P,
                               const int32_t* ind_mat, int n_terms, const int32_t* labels,
                               int nR, const double* terms, double e_unit, double* mat);

/* SYS_TYPE 0 with identical partners (IDENTICAL = YES, IDENTICAL_PES = YES),
 * SRC/pot_comp.f:8257-8746: parity[s] = the exchange parity of state s (+1/-1); the
 * system needs ka1, kc1, ka2, kc2, vec1 and vec2. */
int orc_expansion_matrix_type0_identical(const orc_system* sys, const int32_t* indx_chann,
                                         const int32_t* j12, const int32_t* m12,
                                         const int32_t* parity, int64_t P,
                                         const int32_t* ind_mat, int n_terms,
                                         const int32_t* labels, int nR, const double* terms,
                                         double e_unit, double* mat);
/* Inversion parity p1 p2 of a channel from its rotor vectors (SRC/pot_comp.f:70-110). */
int orc_parity_inversion(const double* v1, int j1, const double* v2, int j2);

/* EXPANSION_MATRIX_ELEMENT for a rotor and an atom, SYS_TYPE 1, 3 and 4
 * (SRC/pot_comp.f:6551-7075); terms nR x n_terms in units of e_unit Hartree, a_top 5
 * per term (l, nju, ...). */
int orc_expansion_matrix_atom(const orc_system* sys, const int32_t* indx_chann,
                              const int32_t* j12, const int32_t* m12, int64_t P,
                              const int32_t* ind_mat, int n_terms, const int32_t* a_top, int nR,
                              const double* terms, double e_unit, double* mat);

/* EXPANSION_TERM and CALC_EXPANSION_TERMS for SYS_TYPE 7, 8 and 0
 * (SRC/pot_comp.f:3739-3896, 4695-6274): the term's angular function, and the
 * quadrature projection of V[iR][alpha2][beta1][beta2][gamma1][gamma2] onto the terms
 * (a_top 5 per term), terms[t * nR + iR]. */
void orc_expansion_term(int sys_type, int l, int l1, int l2, int nju1, int nju2, double beta1,
                        double gamma1, double alpha2, double beta2, double gamma2, double* wfr,
                        double* wfi);
int orc_project_terms(int sys_type, int n_terms, const int32_t* a_top, int n_alpha2,
                      int n_beta1, int n_beta2, int n_gamma1, int n_gamma2, int eq_gamma, int nR,
                      const double* V, double* terms, double* terms_im);

/* CALC_EXPANSION_TERMS for SYS_TYPE 1 (V[iR][beta]) and 4 (V[iR][beta][gamma])
 * (SRC/pot_comp.f:4973-4999, 5054-5104); terms[t * nR + iR]. */
int orc_project_terms_atom(int sys_type, int n_terms, const int32_t* a_top, int n_beta,
                           int n_gamma, int eq_gamma, int nR, const double* V, double* terms,
                           double* terms_im);

#ifdef __cplusplus
}
#endif
#endif
