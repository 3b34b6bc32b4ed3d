/*
 * mqct_oracle.c -- CPU FP64 oracle for the MQCT hot paths.
 *
 * TEST INFRASTRUCTURE ONLY (see mqct_oracle.h).  Plain-C restatement of the
 * reference Fortran (MarquetteQuantum/MQCT) written from the mathematics and
 * the reference's algorithms; each routine names the file:line it follows.
 * Parity is pinned by tests against the reference's own example outputs
 * (EXAMPLES_IO) and closed-form known answers.
 */
#include "mqct_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Physical constants, SRC/iotest.f:19-25 and SRC/propagator.f:46. */
#define ORC_AUTOEV 27.21113845
#define ORC_EVTOWN 8065.5448
#define ORC_PI 3.14159265358979323846

/* ---------------------------------------------------------------------- */
/* LOGFACT table: SRC/pot_comp.f:311-322 (INI_FACT), log(n!) by summation. */
#define LOGFACT_N 400
static double g_logfact[LOGFACT_N + 1];
static int g_logfact_ready = 0;
static void orc_init_logfact(void) {
  if (g_logfact_ready) return;
  g_logfact[0] = 0.0;
  for (int i = 1; i <= LOGFACT_N; ++i) g_logfact[i] = g_logfact[i - 1] + log((double)i);
  g_logfact_ready = 1;
}
__attribute__((constructor)) static void orc_ctor(void) { orc_init_logfact(); }

/* C_N_K binomial via LOGFACT, SRC/pot_comp.f:324-331. */
static double orc_cnk(int n, int k) {
  return exp(g_logfact[n] - g_logfact[n - k] - g_logfact[k]);
}

static double orc_ipow(double x, int n) { /* Fortran x**n with integer n >= 0 */
  double r = 1.0;
  for (int i = 0; i < n; ++i) r *= x;
  return r;
}

/* ---------------------------------------------------------------------- */
/* Gauss-Legendre nodes/weights on [-1,1]: SRC/suppl_routines.f:157-204 (gauleg):
 * Newton iteration on P_n from z0 = cos(pi(i-1/4)/(n+1/2)), |dz| <= 3e-15. */
void orc_gauleg(int n, double* x, double* w) {
  const double eps = 3.0e-15;
  int m = (n + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = cos(ORC_PI * (i - 0.25) / (n + 0.5));
    double z1, pp;
    for (;;) {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= n; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (!(fabs(z - z1) > eps)) break;
    }
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

/* Associated Legendre P_l^m(x) with Condon-Shortley phase:
 * SRC/suppl_routines.f:207-243 (plgndr). */
double orc_plgndr(int l, int m, double x) {
  double pmm = 1.0;
  if (m > 0) {
    double somx2 = sqrt((1.0 - x) * (1.0 + x));
    double fact = 1.0;
    for (int i = 1; i <= m; ++i) {
      pmm = -pmm * fact * somx2;
      fact += 2.0;
    }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2 * m + 1) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0.0;
  for (int ll = m + 2; ll <= l; ++ll) {
    pll = (x * (2 * ll - 1) * pmmp1 - (ll + m - 1) * pmm) / (ll - m);
    pmm = pmmp1;
    pmmp1 = pll;
  }
  return pll;
}

/* Jacobi polynomials P_0..P_n^(a,b)(x), three-term recurrence:
 * SRC/suppl_routines.f:1-148 (jacobi_poly). */
void orc_jacobi_poly(int n, double a, double b, double x, double* cx) {
  if (n < 0) return;
  cx[0] = 1.0;
  if (n == 0) return;
  cx[1] = (1.0 + 0.5 * (a + b)) * x + 0.5 * (a - b);
  for (int i = 2; i <= n; ++i) {
    double r = (double)i;
    double c1 = 2.0 * r * (r + a + b) * (2.0 * r - 2.0 + a + b);
    double c2 = (2.0 * r - 1.0 + a + b) * (2.0 * r + a + b) * (2.0 * r - 2.0 + a + b);
    double c3 = (2.0 * r - 1.0 + a + b) * (a + b) * (a - b);
    double c4 = -2.0 * (r - 1.0 + a) * (r - 1.0 + b) * (2.0 * r + a + b);
    cx[i] = ((c3 + c2 * x) * cx[i - 1] + c4 * cx[i - 2]) / c1;
  }
}

/* Wigner 3j symbol, Racah sum with doubled arguments:
 * SRC/suppl_routines.f:270-314 (W3JS). */
double orc_w3js(int j1, int j2, int j3, int m1, int m2, int m3) {
  if (m1 + m2 + m3 != 0) return 0.0;
  int ia = j1 + j2;
  if (j3 > ia) return 0.0;
  int ib = j1 - j2;
  if (j3 < abs(ib)) return 0.0;
  int jsum = j3 + ia, ic = j1 - m1, id = j2 - m2;
  if (jsum % 2 || ic % 2 || id % 2) return 0.0;
  if (abs(m1) > j1 || abs(m2) > j2 || abs(m3) > j3) return 0.0;
  int ie = j3 - j2 + m1, iff = j3 - j1 - m2;
  int zmin = 0;
  if (-ie > zmin) zmin = -ie;
  if (-iff > zmin) zmin = -iff;
  int ig = ia - j3, ih = j2 + m2;
  int zmax = ig;
  if (ih < zmax) zmax = ih;
  if (ic < zmax) zmax = ic;
  double cc = 0.0;
  for (int z = zmin; z <= zmax; z += 2) {
    double denom = exp(g_logfact[z / 2] + g_logfact[(ig - z) / 2] + g_logfact[(ic - z) / 2] +
                       g_logfact[(ih - z) / 2] + g_logfact[(ie + z) / 2] + g_logfact[(iff + z) / 2]);
    if (z % 4 != 0) denom = -denom;
    cc += 1.0 / denom;
  }
  double cc1 = exp(g_logfact[ig / 2] + g_logfact[(j3 + ib) / 2] + g_logfact[(j3 - ib) / 2] -
                   g_logfact[(jsum + 2) / 2]);
  double cc2 = exp(g_logfact[(j1 + m1) / 2] + g_logfact[ic / 2] + g_logfact[ih / 2] +
                   g_logfact[id / 2] + g_logfact[(j3 - m3) / 2] + g_logfact[(j3 + m3) / 2]);
  cc = cc * sqrt(cc1 * cc2);
  if ((ib - m3) % 4 != 0) cc = -cc;
  return cc;
}

/* Clebsch-Gordan <j1 m1 j2 m2|j3 m3>: SRC/suppl_routines.f:246-252 (CG). */
double orc_cg(int j1, int j2, int j3, int m1, int m2, int m3) {
  int e = -j1 + j2 - m3;
  double sgn = (e % 2 == 0) ? 1.0 : -1.0;
  return orc_w3js(2 * j1, 2 * j2, 2 * j3, 2 * m1, 2 * m2, -2 * m3) * sqrt(2.0 * j3 + 1.0) * sgn;
}

/* Cubic spline second derivatives with end slopes yp1/ypn (natural if >.99e30):
 * SRC/suppl_routines.f:914-965 (spline). */
void orc_spline(const double* x, const double* y, int n, double yp1, double ypn, double* y2) {
  double* u = (double*)malloc(sizeof(double) * (size_t)n);
  if (yp1 > 0.99e30) {
    y2[0] = 0.0;
    u[0] = 0.0;
  } else {
    y2[0] = -0.5;
    u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
  }
  for (int i = 1; i < n - 1; ++i) {
    double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    double p = sig * y2[i - 1] + 2.0;
    y2[i] = (sig - 1.0) / p;
    u[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])) /
                (x[i + 1] - x[i - 1]) -
            sig * u[i - 1]) /
           p;
  }
  double qn, un;
  if (ypn > 0.99e30) {
    qn = 0.0;
    un = 0.0;
  } else {
    qn = 0.5;
    un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
  }
  y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
  free(u);
}

/* Spline evaluation with derivative, bisection bracket:
 * SRC/suppl_routines.f:968-1002 (splint). */
void orc_splint(const double* xa, const double* ya, const double* y2a, int n, double x,
                double* y, double* yprime) {
  int klo = 1, khi = n;
  while (khi - klo > 1) {
    int k = (khi + klo) / 2;
    if (xa[k - 1] > x) khi = k;
    else klo = k;
  }
  double h = xa[khi - 1] - xa[klo - 1];
  double a = (xa[khi - 1] - x) / h;
  double b = (x - xa[klo - 1]) / h;
  *y = a * ya[klo - 1] + b * ya[khi - 1] +
       ((a * a * a - a) * y2a[klo - 1] + (b * b * b - b) * y2a[khi - 1]) * (h * h) / 6.0;
  *yprime = -ya[klo - 1] / h + ya[khi - 1] / h +
            (-(3.0 * a * a - 1.0) * y2a[klo - 1] / h + (3.0 * b * b - 1.0) * y2a[khi - 1] / h) *
                (h * h) / 6.0;
}

/* ---------------------------------------------------------------------- */
/* Wigner D-function as used by the reference: d(beta) from the Jacobi form
 * with the reference's (n, a, lambda) case selection, times
 * (cos + i sin)(k*gamma + m*alpha).  SRC/pot_comp.f:256-309 (Djkm). */
void orc_djkm(int j, int k, int m, double alpha, double beta, double gamma, double* re,
              double* im) {
  int n = j + k, a = 0, lambda = 0;
  if (j - k < n) n = j - k;
  if (j + m < n) n = j + m;
  if (j - m < n) n = j - m;
  if (n == j + m) { a = k - m; lambda = 0; }
  if (n == j - m) { a = m - k; lambda = k - m; }
  if (n == j + k) { a = m - k; lambda = k - m; }
  if (n == j - k) { a = k - m; lambda = 0; }
  int b = 2 * j - 2 * n - a;
  double cx[2 * 64 + 2];
  orc_jacobi_poly(n, (double)a, (double)b, cos(beta), cx);
  double sgn = ((lambda % 2) == 0) ? 1.0 : -1.0;
  double dkm = cx[n] * sgn * sqrt(orc_cnk(2 * j - n, n + a)) / sqrt(orc_cnk(n + b, b)) *
               orc_ipow(sin(beta / 2.0), a) * orc_ipow(cos(beta / 2.0), b);
  *re = dkm * cos(k * gamma + m * alpha);
  *im = dkm * sin(k * gamma + m * alpha);
}

/* Normalised spherical harmonic of the rigid diatom:
 * SRC/basis_wave_functions.f:153-175 (WF_DIAT_TOP). */
void orc_wf_diat(int j, int m, double theta, double phi, double* re, double* im) {
  int am = abs(m);
  double pl = orc_plgndr(j, am, cos(theta));
  double nrm = sqrt((2.0 * j + 1.0) / 4.0 / ORC_PI * exp(g_logfact[j - am] - g_logfact[j + am]));
  double wr = pl * nrm * cos(m * phi);
  double wi = pl * nrm * sin(m * phi);
  if (m < 0 && (am % 2)) {
    wr = -wr;
    wi = -wi;
  }
  *re = wr;
  *im = wi;
}

/* Asymmetric-top wavefunction sum_K c_K sqrt((2j+1)/8pi^2) D^j_{K m}:
 * SRC/basis_wave_functions.f:83-116 (WF_ASYM_TOP). */
void orc_wf_asym(int j, const double* coeff, int m, double alpha, double beta, double gamma,
                 double* re, double* im) {
  double wr = 0.0, wi = 0.0;
  double nrm = sqrt((2.0 * j + 1.0) / 8.0 / (ORC_PI * ORC_PI));
  for (int i = 1; i <= 2 * j + 1; ++i) {
    int dk = i - j - 1;
    double dwr, dwi;
    orc_djkm(j, dk, m, alpha, beta, gamma, &dwr, &dwi);
    dwr *= nrm;
    dwi *= nrm;
    wr += dwr * coeff[i - 1];
    wi += dwi * coeff[i - 1];
  }
  *re = wr;
  *im = wi;
}

/* Symmetric-top wavefunction of the level (j, k, eps):
 * (D^j_{k m} + (1 - 2 eps) D^j_{-k m}) sqrt((2j+1)/8pi^2), divided by 2 for k = 0 and by
 * sqrt(2) otherwise: SRC/basis_wave_functions.f:118-151 (WF_SYM_TOP). */
void orc_wf_sym(int j, int k, int eps, int m, double alpha, double beta, double gamma,
                double* re, double* im) {
  double dwr, dwi, wr, wi;
  orc_djkm(j, k, m, alpha, beta, gamma, &dwr, &dwi);
  wr = dwr;
  wi = dwi;
  orc_djkm(j, -k, m, alpha, beta, gamma, &dwr, &dwi);
  wr += dwr * (1.0 - 2 * eps);
  wi += dwi * (1.0 - 2 * eps);
  const double nrm = sqrt((2.0 * j + 1.0) / 8.0 / (ORC_PI * ORC_PI));
  const double f = (k == 0) ? 0.5 : 1.0 / sqrt(2.0);
  *re = wr * f * nrm;
  *im = wi * f * nrm;
}

/* Rigid-rotor Hamiltonian element in the symmetric-top basis, z = c axis:
 * SRC/asym_top.f:103-137 (hamilt_kyro). */
static double orc_hamilt(int j, int k1, int k2, double A, double B, double C) {
  double jj = j * (j + 1.0);
  if (k1 != k2) {
    if (k1 == k2 - 2 || k1 == k2 + 2) {
      int kav = (k1 + k2) / 2;
      double jxy = sqrt((j + 1.0) * j - kav * k1) * sqrt((j + 1.0) * j - kav * k2) / 2.0;
      return 0.5 * (A - B) * jxy;
    }
    return 0.0;
  }
  return 0.5 * (A + B) * jj + (C - 0.5 * (A + B)) * (double)(k1 * k1);
}

/* Cyclic Jacobi eigensolver for a small dense symmetric matrix (row-major a[n*n]);
 * eigenvalues in w, eigenvectors as columns of v (row-major v[i*n+col]). */
static void orc_jacobi_eig(int n, double* a, double* w, double* v) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) v[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i) {
      diag += a[i * n + i] * a[i * n + i];
      for (int j = i + 1; j < n; ++j) off += a[i * n + j] * a[i * n + j];
    }
    if (off <= 1e-32 * (diag + 1e-300)) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[p * n + q];
        if (fabs(apq) < 1e-300) continue;
        double app = a[p * n + p], aqq = a[q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) w[i] = a[i * n + i];
}

/* Level (j, ka, kc): ascending eigenvalue number j + (ka - kc), the labelling of
 * SRC/asym_top.f:139-173 (STATE) used by EIGEN_VAL/EIGEN_VEC
 * (SRC/asym_top.f:1-101, 280-388).  The eigenvector sign is fixed so that its
 * first non-negligible component (lowest K) is positive. */
int orc_asym_top(double A, double B, double C, int j, int ka, int kc, double* energy,
                 double* vec) {
  int n = 2 * j + 1;
  if (j < 0 || ka < 0 || kc < 0 || ka > j || kc > j) return -1;
  if (ka + kc != j && ka + kc != j + 1) return -2;
  int tau = ka - kc;
  if (tau < -j || tau > j) return -3;
  /* STATE: K_A = [0,1,1,2,2,...], index i = j + tau + 1 must reproduce ka. */
  int idx = j + tau + 1; /* 1-based */
  int ka_chk = idx / 2;
  if (ka_chk != ka) return -4;
  double* h = (double*)malloc(sizeof(double) * n * n);
  double* vv = (double*)malloc(sizeof(double) * n * n);
  double* w = (double*)malloc(sizeof(double) * n);
  int* ord = (int*)malloc(sizeof(int) * n);
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) h[a * n + b] = orc_hamilt(j, a - j, b - j, A, B, C);
  orc_jacobi_eig(n, h, w, vv);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 1; i < n; ++i) { /* insertion sort ascending */
    int t = ord[i], p = i - 1;
    while (p >= 0 && w[ord[p]] > w[t]) { ord[p + 1] = ord[p]; --p; }
    ord[p + 1] = t;
  }
  int col = ord[idx - 1];
  *energy = w[col];
  int first = -1;
  for (int k = 0; k < n; ++k) {
    vec[k] = vv[k * n + col];
    if (first < 0 && fabs(vec[k]) > 1e-10) first = k;
  }
  if (first >= 0 && vec[first] < 0)
    for (int k = 0; k < n; ++k) vec[k] = -vec[k];
  free(h); free(vv); free(w); free(ord);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* States: SRC/matrix_ini.f:60-209 (count) and 261-544 (fill), distinguishable
 * particles.  Types 1/3/4: m=-j..j per channel; types 5/7/8/0: j12=|j1-j2|..j1+j2, m12. */
int orc_count_states(const orc_system* sys) {
  int st = 0;
  for (int i = 0; i < sys->n_channels; ++i) {
    switch (sys->sys_type) {
      case 1: case 3: case 4: st += 2 * sys->j1[i] + 1; break;
      case 5: case 7: case 8: case 9: case 0: {
        int a = sys->j1[i], b = sys->j2[i];
        for (int js = abs(a - b); js <= a + b; ++js) st += 2 * js + 1;
        break;
      }
      default: return -1;
    }
  }
  return st;
}

int orc_enumerate_states(const orc_system* sys, int32_t* indx_chann, int32_t* j12, int32_t* m12,
                         double* ej) {
  int st = 0;
  for (int i = 0; i < sys->n_channels; ++i) {
    if (sys->sys_type == 1 || sys->sys_type == 3 || sys->sys_type == 4) {
      int j = sys->j1[i];
      for (int m = -j; m <= j; ++m) {
        indx_chann[st] = i + 1; j12[st] = j; m12[st] = m; ej[st] = sys->e_ch[i]; ++st;
      }
    } else if (sys->sys_type == 5 || sys->sys_type == 7 || sys->sys_type == 8 ||
               sys->sys_type == 9 || sys->sys_type == 0) {
      int a = sys->j1[i], b = sys->j2[i];
      for (int js = abs(a - b); js <= a + b; ++js)
        for (int m = -js; m <= js; ++m) {
          indx_chann[st] = i + 1; j12[st] = js; m12[st] = m; ej[st] = sys->e_ch[i]; ++st;
        }
    } else {
      return -1;
    }
  }
  return st;
}

/* ind_mat: all (st1, st2) with st2 <= st1 and equal m12, st1 outer:
 * SRC/matrix_ini.f:553-627. */
int64_t orc_count_pairs(int n, const int32_t* m12) {
  int64_t p = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b <= a; ++b)
      if (m12[a] == m12[b]) ++p;
  return p;
}
int64_t orc_ind_mat(int n, const int32_t* m12, int32_t* ind) {
  int64_t p = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b <= a; ++b)
      if (m12[a] == m12[b]) {
        ind[2 * p] = a + 1;
        ind[2 * p + 1] = b + 1;
        ++p;
      }
  return p;
}

/* R grid: equidistant (SRC/matrix_ini.f:976-980) or the 3-segment
 * "optimized" grid (SRC/matrix_ini.f:957-973). */
void orc_rgrid(int n, double rmin, double rmax, int equidistant, double* R) {
  if (equidistant) {
    double dr = (rmax - rmin) / (n - 1.0);
    for (int i = 1; i <= n; ++i) R[i - 1] = rmin + dr * (i - 1.0);
    return;
  }
  int n1 = n / 3, n2 = n / 2 + 1;
  R[0] = rmin;
  R[n - 1] = rmax;
  double dr = (rmax - rmin) / (n - 1.0);
  for (int i = 1; i <= n1; ++i) R[i - 1] = rmin + dr * (i - 1.0) / 3.0;
  for (int i = n1 + 1; i <= n2; ++i) R[i - 1] = R[n1 - 1] + dr * (i - n1);
  dr = (rmax - R[n2 - 1]) / (n - n2);
  for (int i = n2; i <= n; ++i) R[i - 1] = R[n2 - 1] + dr * (i - n2);
}

/* ---------------------------------------------------------------------- */
/* Synthetic PES family (stand-ins for the USER_DEFINED_PES plugin of PES_DIRECTORIES).
 *  LEGENDRE: V(R,beta) = sum_l [A_l exp(-b_l R) - C_l/R^6] P_l(cos beta),
 *            p = [A_0..A_{n-1}, b_0.., C_0..].
 *  SITES1:   atom at R*(sin b cos g, sin b sin g, cos b) in the rotor frame
 *            (b,g = PES beta/gamma arguments); per term
 *            p = [site, D, a, re, C6, rd]:
 *            D(e^{-2a(r-re)} - 2e^{-a(r-re)}) - C6 (1-e^{-(r/rd)^6}) / r^6.
 *  SITES2:   rotor 1 at the origin with Euler (alpha=0?,beta,gamma), rotor 2 at
 *            R*z with Euler (aalpha,bbeta,ggamma); p = [s1, s2, D, a, re, C6, rd].
 */
static void orc_euler_rot(double a, double b, double g, double* M) {
  /* R = Rz(a) Ry(b) Rz(g), row-major */
  double ca = cos(a), sa = sin(a), cb = cos(b), sb = sin(b), cg = cos(g), sg = sin(g);
  M[0] = ca * cb * cg - sa * sg; M[1] = -ca * cb * sg - sa * cg; M[2] = ca * sb;
  M[3] = sa * cb * cg + ca * sg; M[4] = -sa * cb * sg + ca * cg; M[5] = sa * sb;
  M[6] = -sb * cg;               M[7] = sb * sg;                 M[8] = cb;
}
static double orc_site_term(double r, const double* t) {
  double D = t[0], a = t[1], re = t[2], c6 = t[3], rd = t[4];
  double e = exp(-a * (r - re));
  double r2 = r * r, r6 = r2 * r2 * r2;
  double x = r / rd, x2 = x * x, x6 = x2 * x2 * x2;
  return D * (e * e - 2.0 * e) - c6 * (1.0 - exp(-x6)) / r6;
}
double orc_pes_eval(const orc_pes* pes, double R, double alpha, double beta, double gamma,
                    double aalpha, double bbeta, double ggamma) {
  int n = pes->n_terms;
  const double* p = pes->p;
  if (pes->kind == ORC_PES_LEGENDRE) {
    double x = cos(beta), v = 0.0;
    double r2 = R * R, r6 = r2 * r2 * r2;
    for (int l = 0; l < n; ++l) {
      double pl = orc_plgndr(l, 0, x);
      v += (p[l] * exp(-p[n + l] * R) - p[2 * n + l] / r6) * pl;
    }
    return v;
  }
  if (pes->kind == ORC_PES_SITES1) {
    double ux = sin(beta) * cos(gamma), uy = sin(beta) * sin(gamma), uz = cos(beta);
    double ax = R * ux, ay = R * uy, az = R * uz;
    double v = 0.0;
    for (int t = 0; t < n; ++t) {
      const double* q = p + 6 * t;
      const double* s = pes->sites1 + 3 * (int)q[0];
      double dx = ax - s[0], dy = ay - s[1], dz = az - s[2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      v += orc_site_term(r, q + 1);
    }
    return v;
  }
  if (pes->kind == ORC_PES_SITES2) {
    double M1[9], M2[9];
    orc_euler_rot(alpha, beta, gamma, M1);
    orc_euler_rot(aalpha, bbeta, ggamma, M2);
    double v = 0.0;
    for (int t = 0; t < n; ++t) {
      const double* q = p + 7 * t;
      const double* s1 = pes->sites1 + 3 * (int)q[0];
      const double* s2 = pes->sites2 + 3 * (int)q[1];
      double x1[3], x2[3];
      for (int c = 0; c < 3; ++c) {
        x1[c] = M1[3 * c] * s1[0] + M1[3 * c + 1] * s1[1] + M1[3 * c + 2] * s1[2];
        x2[c] = M2[3 * c] * s2[0] + M2[3 * c + 1] * s2[1] + M2[3 * c + 2] * s2[2];
      }
      x2[2] += R;
      double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      v += orc_site_term(r, q + 2);
    }
    return v;
  }
  return NAN;
}

/* ---------------------------------------------------------------------- */
/* Angular grids of INI_POT_STORAGE.  Type 1: GL beta on [0,pi]
 * (SRC/pot_comp.f:374-394).  Type 4: GL beta x gamma, gamma midpoint-equidistant
 * on [0,2pi] with weight 2/n when EQ_ANG_GRID (default) else GL
 * (SRC/pot_comp.f:586-635).  The optional alpha grid (type 4 with n_alpha>0)
 * replaces the analytic 2*pi alpha factor by the same midpoint rule. */
typedef struct {
  int nb, ng, na;
  double xbl, xgl, xal;       /* half-lengths */
  double *bx, *bw, *gx, *gw, *ax, *aw;
  /* type 0 extra axes */
  int nbb, naa, ngg;
  double xbbl, xaal, xggl;
  double *bbx, *bbw, *aax, *aaw, *ggx, *ggw;
} orc_agrid;

static void orc_axis_gl(int n, double lo, double hi, double** x, double** w, double* half) {
  double* t = (double*)malloc(sizeof(double) * n);
  double* u = (double*)malloc(sizeof(double) * n);
  orc_gauleg(n, t, u);
  double xm = 0.5 * (hi + lo), xl = 0.5 * (hi - lo);
  for (int i = 0; i < n; ++i) t[i] = xm + xl * t[i];
  *x = t; *w = u; *half = xl;
}
static void orc_axis_mid(int n, double lo, double hi, double** x, double** w, double* half) {
  double* t = (double*)malloc(sizeof(double) * n);
  double* u = (double*)malloc(sizeof(double) * n);
  double xl = 0.5 * (hi - lo);
  for (int i = 1; i <= n; ++i) {
    t[i - 1] = lo + (i - 0.50) * 2.0 * xl / n;
    u[i - 1] = 2.0 / n;
  }
  *x = t; *w = u; *half = xl;
}
static void orc_make_agrid(int sys_type, const orc_grid* g, orc_agrid* a) {
  memset(a, 0, sizeof(*a));
  a->nb = g->n_beta;
  orc_axis_gl(g->n_beta, 0.0, ORC_PI, &a->bx, &a->bw, &a->xbl);
  if (sys_type == 3 || sys_type == 4 || sys_type == 9 || sys_type == 0) {
    a->ng = g->n_gamma;
    if (g->eq_gamma) orc_axis_mid(g->n_gamma, 0.0, 2 * ORC_PI, &a->gx, &a->gw, &a->xgl);
    else orc_axis_gl(g->n_gamma, 0.0, 2 * ORC_PI, &a->gx, &a->gw, &a->xgl);
  }
  if (sys_type == 4 && g->n_alpha > 0) {
    a->na = g->n_alpha;
    orc_axis_mid(g->n_alpha, 0.0, 2 * ORC_PI, &a->ax, &a->aw, &a->xal);
  }
  if (sys_type == 0 || sys_type == 9) {
    a->nbb = g->n_beta2;
    orc_axis_gl(g->n_beta2, 0.0, ORC_PI, &a->bbx, &a->bbw, &a->xbbl);
    a->naa = g->n_alpha2;
    a->ngg = g->n_gamma2;
    if (g->eq_gamma) {
      orc_axis_mid(g->n_alpha2, 0.0, 2 * ORC_PI, &a->aax, &a->aaw, &a->xaal);
      orc_axis_mid(g->n_gamma2, 0.0, 2 * ORC_PI, &a->ggx, &a->ggw, &a->xggl);
    } else {
      orc_axis_gl(g->n_alpha2, 0.0, 2 * ORC_PI, &a->aax, &a->aaw, &a->xaal);
      orc_axis_gl(g->n_gamma2, 0.0, 2 * ORC_PI, &a->ggx, &a->ggw, &a->xggl);
    }
  }
}
static void orc_free_agrid(orc_agrid* a) {
  free(a->bx); free(a->bw); free(a->gx); free(a->gw); free(a->ax); free(a->aw);
  free(a->bbx); free(a->bbw); free(a->aax); free(a->aaw); free(a->ggx); free(a->ggw);
}
static int64_t orc_agrid_size(int sys_type, const orc_agrid* a) {
  if (sys_type == 1) return a->nb;
  if (sys_type == 3 || sys_type == 4) return (int64_t)a->nb * a->ng * (a->na > 0 ? a->na : 1);
  if (sys_type == 0 || sys_type == 9)
    return (int64_t)a->naa * a->nb * a->nbb * a->ng * a->ngg;
  return -1;
}

/* Wavefunction of state st (0-based) at a grid point, dispatching on type:
 * type 1 WF_DIAT_TOP(j,m,beta,0); type 4 WF_ASYM_TOP(...,alpha,beta,gamma);
 * type 3 WF_SYM_TOP(j,k,eps,m,...,0,beta,gamma) (SRC/pot_comp.f:2296-2302);
 * type 0 WF_ASYM_TOP_ASYM_TOP (SRC/basis_wave_functions.f:1-41). */
static void orc_wf_state(const orc_system* sys, int ch, int j12, int m12, double al, double be,
                         double ga, double aal, double bbe, double gga, double* re, double* im) {
  if (sys->sys_type == 1) {
    orc_wf_diat(sys->j1[ch], m12, be, 0.0, re, im);
  } else if (sys->sys_type == 4) {
    orc_wf_asym(sys->j1[ch], sys->vec1 + (size_t)ch * sys->ldv, m12, al, be, ga, re, im);
  } else if (sys->sys_type == 3) {
    orc_wf_sym(sys->j1[ch], sys->ka1[ch], sys->kc1[ch], m12, 0.0, be, ga, re, im);
  } else { /* type 0; type 9 WF_ASYM_TOP_SYM_TOP (SRC/basis_wave_functions.f:42-82) */
    int j1 = sys->j1[ch], j2 = sys->j2[ch];
    double wr = 0.0, wi = 0.0;
    for (int m1 = -j1; m1 <= j1; ++m1) {
      int m2 = m12 - m1;
      if (abs(m2) > j2) continue;
      double dr1, di1, dr2, di2;
      orc_wf_asym(j1, sys->vec1 + (size_t)ch * sys->ldv, m1, al, be, ga, &dr1, &di1);
      if (sys->sys_type == 9)
        orc_wf_sym(j2, sys->ka2[ch], sys->kc2[ch], m2, aal, bbe, gga, &dr2, &di2);
      else
        orc_wf_asym(j2, sys->vec2 + (size_t)ch * sys->ldv, m2, aal, bbe, gga, &dr2, &di2);
      double cg = orc_cg(j1, j2, j12, m1, m2, m12);
      wr += cg * (dr1 * dr2 - di1 * di2);
      wi += cg * (dr1 * di2 + di1 * dr2);
    }
    *re = wr;
    *im = wi;
  }
}

/* Grid point g -> angles and the product of weights/Jacobian of the reference
 * integrand (SRC/pot_comp.f:1947-1952, 2535-2557, 3663-3721). */
typedef struct { double al, be, ga, aal, bbe, gga, wt; } orc_gpt;
static orc_gpt orc_grid_point(int sys_type, const orc_agrid* a, int64_t g) {
  orc_gpt p;
  memset(&p, 0, sizeof(p));
  if (sys_type == 1) {
    p.be = a->bx[g];
    p.wt = a->bw[g] * sin(p.be) * a->xbl * 2.0 * ORC_PI;
  } else if (sys_type == 3 || sys_type == 4) {  /* type 3: beta, gamma (:2259-2303) */
    int na = a->na > 0 ? a->na : 1;
    int ia = (int)(g % na);
    int64_t r = g / na;
    int ig = (int)(r % a->ng), ib = (int)(r / a->ng);
    p.be = a->bx[ib];
    p.ga = a->gx[ig];
    if (a->na > 0) {
      p.al = a->ax[ia];
      p.wt = a->bw[ib] * a->gw[ig] * a->aw[ia] * sin(p.be) * a->xbl * a->xgl * a->xal;
    } else {
      p.wt = a->bw[ib] * a->gw[ig] * sin(p.be) * a->xbl * a->xgl * 2.0 * ORC_PI;
    }
  } else {
    /* loop order alpha2, beta1, beta2, gamma1, gamma2 (gamma2 fastest) */
    int i6 = (int)(g % a->ngg);
    int64_t r = g / a->ngg;
    int i5 = (int)(r % a->ng); r /= a->ng;
    int i4 = (int)(r % a->nbb); r /= a->nbb;
    int i3 = (int)(r % a->nb); r /= a->nb;
    int i2 = (int)r;
    p.be = a->bx[i3]; p.bbe = a->bbx[i4]; p.ga = a->gx[i5]; p.aal = a->aax[i2]; p.gga = a->ggx[i6];
    p.wt = a->bw[i3] * a->gw[i5] * sin(p.be) * a->aaw[i2] * a->bbw[i4] * a->ggw[i6] * sin(p.bbe) *
           a->xbl * a->xgl * a->xaal * a->xbbl * a->xggl * 2.0 * ORC_PI;
  }
  return p;
}

/* PES at a grid point with the per-type argument mapping of SRC/pes_sys_type.f:
 * type 1 (R,beta) :2-9; type 4 (-beta,-gamma) :32-37; type 0 (0,b,g,aa,bb,gg) :90-97. */
static double orc_pes_at(int sys_type, const orc_pes* pes, double R, const orc_gpt* p,
                         int iR, int64_t g, int64_t ng) {
  if (pes->kind == ORC_PES_TABLE) return pes->table[(size_t)iR * ng + g];
  if (sys_type == 1) return orc_pes_eval(pes, R, 0.0, p->be, 0.0, 0.0, 0.0, 0.0);
  if (sys_type == 3 || sys_type == 4)  /* V_POT_TOP_ATOM, SYS_TYPE 3 and 4 */
    return orc_pes_eval(pes, R, 0.0, -p->be, -p->ga, 0.0, 0.0, 0.0);
  return orc_pes_eval(pes, R, 0.0, p->be, p->ga, p->aal, p->bbe, p->gga);
}

#define ORC_CM_TO_HARTREE (1.0 / ORC_EVTOWN / ORC_AUTOEV)

int orc_integrate_elements(const orc_system* sys, int n_states, const int32_t* indx_chann,
                           const int32_t* j12, const int32_t* m12, int64_t P,
                           const int32_t* ind_mat, int nR, const double* R,
                           const orc_grid* grid, const orc_pes* pes, int literal,
                           int64_t k_begin, int64_t k_end, int iR_begin, int iR_end,
                           int n_threads, double* mat) {
  (void)P;
  if (sys->sys_type == 3 && (!sys->ka1 || !sys->kc1)) return -1;
  if (sys->sys_type == 9 && (!sys->ka2 || !sys->kc2 || !sys->vec1)) return -1;
  orc_agrid a;
  orc_make_agrid(sys->sys_type, grid, &a);
  int64_t ng = orc_agrid_size(sys->sys_type, &a);
  if (ng <= 0) { orc_free_agrid(&a); return -1; }
  orc_gpt* pts = (orc_gpt*)malloc(sizeof(orc_gpt) * (size_t)ng);
  for (int64_t g = 0; g < ng; ++g) pts[g] = orc_grid_point(sys->sys_type, &a, g);
  /* V table over (R, grid): INI_POT_STORAGE */
  double* V = (double*)malloc(sizeof(double) * (size_t)ng * (iR_end - iR_begin));
  for (int iR = iR_begin; iR < iR_end; ++iR)
    for (int64_t g = 0; g < ng; ++g)
      V[(size_t)(iR - iR_begin) * ng + g] = orc_pes_at(sys->sys_type, pes, R[iR], &pts[g], iR, g, ng);
  /* Optional tabulation of psi_s(g) (same per-point arithmetic as the literal form). */
  double* wr = NULL;
  double* wi = NULL;
  if (!literal) {
    wr = (double*)malloc(sizeof(double) * (size_t)ng * n_states);
    wi = (double*)malloc(sizeof(double) * (size_t)ng * n_states);
#pragma omp parallel for schedule(dynamic) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
    for (int s = 0; s < n_states; ++s)
      for (int64_t g = 0; g < ng; ++g) {
        const orc_gpt* p = &pts[g];
        orc_wf_state(sys, indx_chann[s] - 1, j12[s], m12[s], p->al, p->be, p->ga, p->aal, p->bbe,
                     p->gga, &wr[(size_t)s * ng + g], &wi[(size_t)s * ng + g]);
      }
  }
#pragma omp parallel for schedule(dynamic) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
  for (int64_t k = k_begin; k < k_end; ++k) {
    int s1 = ind_mat[2 * k] - 1, s2 = ind_mat[2 * k + 1] - 1;
    for (int iR = iR_begin; iR < iR_end; ++iR) {
      const double* Vr = V + (size_t)(iR - iR_begin) * ng;
      double acc = 0.0;
      for (int64_t g = 0; g < ng; ++g) {
        const orc_gpt* p = &pts[g];
        double dr1, di1, dr2, di2;
        if (literal) {
          orc_wf_state(sys, indx_chann[s1] - 1, j12[s1], m12[s1], p->al, p->be, p->ga, p->aal,
                       p->bbe, p->gga, &dr1, &di1);
          orc_wf_state(sys, indx_chann[s2] - 1, j12[s2], m12[s2], p->al, p->be, p->ga, p->aal,
                       p->bbe, p->gga, &dr2, &di2);
        } else {
          dr1 = wr[(size_t)s1 * ng + g]; di1 = wi[(size_t)s1 * ng + g];
          dr2 = wr[(size_t)s2 * ng + g]; di2 = wi[(size_t)s2 * ng + g];
        }
        acc += (dr1 * dr2 + di1 * di2) * p->wt * Vr[g];
      }
      mat[(size_t)k * nR + iR] = acc;
    }
  }
  free(V); free(pts); free(wr); free(wi);
  orc_free_agrid(&a);
  return 0;
}

static int orc_nearest(int n, const double* R, double r) { /* first minloc |R-r| */
  int best = 0;
  double d = fabs(R[0] - r);
  for (int i = 1; i < n; ++i)
    if (fabs(R[i] - r) < d) { d = fabs(R[i] - r); best = i; }
  return best;
}

/* MATRIX_MAKE direct-integration flow: quadrature -> Hartree
 * (SRC/matrix_ini.f:1948-1955), MIJ_CUTOFF at R~r_cut1/r_cut2 (:1969-1997),
 * clamped spline with finite-difference end slopes (:2005-2016). */
int orc_build_matrix(const orc_system* sys, int n_states, const int32_t* indx_chann,
                     const int32_t* j12, const int32_t* m12, int64_t P, const int32_t* ind_mat,
                     int nR, const double* R, const orc_grid* grid, const orc_pes* pes,
                     double mij_cut_cm, double r_cut1, double r_cut2, int literal,
                     int64_t k_begin, int64_t k_end, int n_threads, double* mat, double* y2,
                     int32_t* skipped) {
  int rc = orc_integrate_elements(sys, n_states, indx_chann, j12, m12, P, ind_mat, nR, R, grid,
                                  pes, literal, k_begin, k_end, 0, nR, n_threads, mat);
  if (rc) return rc;
  int ir1 = orc_nearest(nR, R, r_cut1), ir2 = orc_nearest(nR, R, r_cut2);
  double cut = mij_cut_cm / ORC_EVTOWN / ORC_AUTOEV;
  for (int64_t k = k_begin; k < k_end; ++k) {
    double* col = mat + (size_t)k * nR;
    for (int i = 0; i < nR; ++i) col[i] *= ORC_CM_TO_HARTREE;
    double mx = fabs(col[ir1]);
    if (fabs(col[ir2]) > mx) mx = fabs(col[ir2]);
    if (mx < cut) {
      for (int i = 0; i < nR; ++i) { col[i] = 0.0; y2[(size_t)k * nR + i] = 0.0; }
      skipped[k] = 1;
      continue;
    }
    skipped[k] = 0;
    double d0 = (col[1] - col[0]) / (R[1] - R[0]);
    double d1 = (col[nR - 1] - col[nR - 2]) / (R[nR - 1] - R[nR - 2]);
    orc_spline(R, col, nR, d0, d1, y2 + (size_t)k * nR);
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Fortran unformatted sequential records: int32 length markers around each
 * WRITE.  Layout of PRINT_MIJ_USER, SRC/matrix_ini.f:6640-6770. */
static void orc_rec(FILE* f, const void* data, int32_t nbytes) {
  fwrite(&nbytes, 4, 1, f);
  fwrite(data, 1, (size_t)nbytes, f);
  fwrite(&nbytes, 4, 1, f);
}
int orc_write_mtrx_uf(const char* path, int coll_type, int n_channels, int n_states,
                      const int32_t* state_rec, int state_rec_len, int64_t P,
                      const int32_t* ind_mat, int nR, const double* R, const double* mat) {
  FILE* f = fopen(path, "wb");
  if (!f) return -1;
  int32_t v;
  v = coll_type; orc_rec(f, &v, 4);
  v = n_channels; orc_rec(f, &v, 4);
  v = n_states; orc_rec(f, &v, 4);
  v = (int32_t)P; orc_rec(f, &v, 4);
  v = nR; orc_rec(f, &v, 4);
  for (int s = 0; s < n_states; ++s) orc_rec(f, state_rec + (size_t)s * state_rec_len, 4 * state_rec_len);
  for (int64_t k = 0; k < P; ++k) {
    int32_t t[3] = {(int32_t)(k + 1), ind_mat[2 * k], ind_mat[2 * k + 1]};
    orc_rec(f, t, 12);
  }
  for (int i = 0; i < nR; ++i) {
    unsigned char buf[12];
    int32_t ii = i + 1;
    memcpy(buf, &ii, 4);
    memcpy(buf + 4, &R[i], 8);
    orc_rec(f, buf, 12);
  }
  for (int64_t k = 0; k < P; ++k) {
    int32_t kk = (int32_t)(k + 1);
    orc_rec(f, &kk, 4);
    orc_rec(f, mat + (size_t)k * nR, 8 * nR);
  }
  fclose(f);
  return 0;
}

/* Formatted MTRX.DAT (PRINT_MIJ, SRC/matrix_ini.f:4692-4891): five "KEY= n"
 * header lines, a states table, "MIJ_INDEX" pairs, "#iR" R values and
 * "#k_matel #iR Mij" rows. */
int orc_read_mtrx_dat_header(const char* path, int* coll_type, int* n_channels, int* n_states,
                             int64_t* P, int* nR) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  char line[512];
  long long pp = 0;
  int ok = 0;
  if (fgets(line, sizeof line, f) && sscanf(line, "COLLISION_TYPE= %d", coll_type) == 1) ++ok;
  if (fgets(line, sizeof line, f) && sscanf(line, "NUMBER_OF_CHANLS= %d", n_channels) == 1) ++ok;
  if (fgets(line, sizeof line, f) && sscanf(line, "NUMBER_OF_STATES= %d", n_states) == 1) ++ok;
  if (fgets(line, sizeof line, f) && sscanf(line, "MATRIX_SIZE= %lld", &pp) == 1) ++ok;
  if (fgets(line, sizeof line, f) && sscanf(line, "R_GRID_SIZE= %d", nR) == 1) ++ok;
  fclose(f);
  *P = pp;
  return ok == 5 ? 0 : -2;
}
int orc_read_mtrx_dat(const char* path, int n_state_cols, int32_t* state_cols, int32_t* ind_mat,
                      double* R, double* mat) {
  int ct, nch, ns, nR;
  int64_t P;
  if (orc_read_mtrx_dat_header(path, &ct, &nch, &ns, &P, &nR)) return -1;
  FILE* f = fopen(path, "r");
  char line[1024];
  for (int i = 0; i < 5; ++i) fgets(line, sizeof line, f);
  fgets(line, sizeof line, f); /* states header */
  for (int s = 0; s < ns; ++s) {
    if (!fgets(line, sizeof line, f)) { fclose(f); return -3; }
    char* p = line;
    for (int c = 0; c < n_state_cols; ++c) state_cols[(size_t)s * n_state_cols + c] = (int32_t)strtol(p, &p, 10);
  }
  fgets(line, sizeof line, f); /* MIJ_INDEX header */
  for (int64_t k = 0; k < P; ++k) {
    long long kk; int a, b;
    if (!fgets(line, sizeof line, f) || sscanf(line, "%lld %d %d", &kk, &a, &b) != 3) { fclose(f); return -4; }
    ind_mat[2 * k] = a; ind_mat[2 * k + 1] = b;
  }
  fgets(line, sizeof line, f); /* #iR header */
  for (int i = 0; i < nR; ++i) {
    int ii; double r;
    if (!fgets(line, sizeof line, f) || sscanf(line, "%d %lf", &ii, &r) != 2) { fclose(f); return -5; }
    R[i] = r;
  }
  fgets(line, sizeof line, f); /* #k_matel header */
  for (int64_t k = 0; k < P; ++k)
    for (int i = 0; i < nR; ++i) {
      long long kk; int ii; double v;
      if (!fgets(line, sizeof line, f) || sscanf(line, "%lld %d %lf", &kk, &ii, &v) != 3) { fclose(f); return -6; }
      mat[(size_t)(kk - 1) * nR + (ii - 1)] = v;
    }
  fclose(f);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Propagation.  State vector q (0-based): q[0..N-1] Re a, q[N..2N-1] Im a,
 * q[2N]=R, q[2N+1]=P_R, q[2N+2]=theta, q[2N+3]=P_theta, q[2N+4]=phi,
 * q[2N+5]=P_phi, q[2N+6]=q[2N+7]=0 (zero sinks): SRC/mqct_eqtns.f:123,148-161. */
typedef struct {
  const orc_tables* tab;
  int n_u;                 /* unique Delta E count */
  double* du;              /* unique Delta E values */
  int32_t* uidx;           /* per pair */
  double* misc;            /* 4 per pair (Coriolis factors) */
  double *m, *dm, *phi_amp, *sc;
  int cs;                  /* coupled states: only pairs of the initial m12, no Coriolis */
  int cs_m;                /* m12 of the initial state */
} orc_rhs_ws;

/* resize: unique Delta E table (last match within 1e-12 in single precision wins)
 * and the Coriolis factors misc_bk, SRC/mqct_eqtns.f:1-110. */
static void orc_ws_init(orc_rhs_ws* w, const orc_tables* t) {
  int64_t P = t->P;
  w->tab = t;
  w->du = (double*)malloc(sizeof(double) * (size_t)(P > 0 ? P : 1));
  w->uidx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(P > 0 ? P : 1));
  w->misc = (double*)malloc(sizeof(double) * 4 * (size_t)(P > 0 ? P : 1));
  w->m = (double*)malloc(sizeof(double) * (size_t)(P > 0 ? P : 1));
  w->dm = (double*)malloc(sizeof(double) * (size_t)(P > 0 ? P : 1));
  w->phi_amp = (double*)malloc(sizeof(double) * (size_t)(P > 0 ? P : 1));
  w->sc = (double*)malloc(sizeof(double) * 2 * (size_t)(P > 0 ? P : 1));
  w->cs = 0;
  w->cs_m = 0;
  const double tol = (double)(float)1.0e-12;
  int n_u = 0;
  for (int64_t k = 0; k < P; ++k) {
    int i = t->ind_mat[2 * k] - 1, j = t->ind_mat[2 * k + 1] - 1;
    double de = t->ej[j] - t->ej[i];
    int hit = -1;
    for (int u = 0; u < n_u; ++u)
      if (fabs(de - w->du[u]) < tol) hit = u;
    if (hit < 0) { w->du[n_u] = de; hit = n_u++; }
    w->uidx[k] = hit;
    double jj = t->j12[j], mi = t->m12[i];
    double m1 = mi + 1.0, m0 = mi - 1.0;
    w->misc[4 * k + 0] = sqrt(jj * (jj + 1.0) - m1 * (m1 - 1.0));
    w->misc[4 * k + 1] = sqrt(jj * (jj + 1.0) - m0 * (m0 + 1.0));
    double ji = t->j12[i], mj = t->m12[j];
    m1 = mj + 1; m0 = mj - 1;
    w->misc[4 * k + 2] = sqrt(ji * (ji + 1.0) - m1 * (m1 - 1.0));
    w->misc[4 * k + 3] = sqrt(ji * (ji + 1.0) - m0 * (m0 + 1.0));
  }
  w->n_u = n_u;
}
static void orc_ws_free(orc_rhs_ws* w) {
  free(w->du); free(w->uidx); free(w->misc); free(w->m); free(w->dm); free(w->phi_amp); free(w->sc);
}

/* potential_data_bk + splint_bk, SRC/mqct_eqtns.f:501-611: zero above R_n,
 * cubic spline with derivative otherwise.  Below R_1 the reference computes a
 * linear extrapolation (:534-543) but does not return, so splint_bk overwrites
 * it with the cubic of the first interval (bisection gives klo=1, khi=2); that
 * effective behaviour is what is restated here. */
static void orc_matrix_at(const orc_tables* t, double x, double* m, double* dm) {
  int nR = t->nR;
  const double* R = t->R;
  int64_t P = t->P;
  if (x > R[nR - 1]) {
    for (int64_t k = 0; k < P; ++k) { m[k] = 0.0; dm[k] = 0.0; }
    return;
  }
  int klo = 1, khi = nR;
  while (khi - klo > 1) {
    int kk = (khi + klo) / 2;
    if (R[kk - 1] > x) khi = kk;
    else klo = kk;
  }
  double h = R[khi - 1] - R[klo - 1];
  double aa = (R[khi - 1] - x) / h, bb = (x - R[klo - 1]) / h;
  double cc1 = aa * aa * aa - aa, cc2 = bb * bb * bb - bb;
  double cc3 = 3 * aa * aa - 1.0, cc4 = 3 * bb * bb - 1.0;
  double cc5 = (h * h) / 6.0, cc6 = cc5 / h;
  for (int64_t k = 0; k < P; ++k) {
    const double* c = t->mat + (size_t)k * nR;
    const double* y = t->y2 + (size_t)k * nR;
    double mlo = c[klo - 1], mhi = c[khi - 1], ylo = y[klo - 1], yhi = y[khi - 1];
    m[k] = aa * mlo + bb * mhi + (cc1 * ylo + cc2 * yhi) * cc5;
    dm[k] = (mhi - mlo) / h + (-cc3 * ylo + cc4 * yhi) * cc6;
  }
}

/* DERIVS_BK for distinguishable particles, full CC, planar motion
 * (POLAR_ANGLE=NO): SRC/mqct_eqtns.f:112-499.  With CS_APPROX (coupled states) the
 * pairs whose m12 differs from the initial state's are skipped (:208-210) and so are
 * the Coriolis terms of P_phi and of the amplitudes (:270, :362, :845). */
static void orc_derivs_ws(orc_rhs_ws* w, double t, const double* q, double* dq) {
  const orc_tables* tb = w->tab;
  int N = tb->n_states;
  int64_t P = tb->P;
  double mass = tb->mass_au;
  for (int i = 0; i < 2 * N + 8; ++i) dq[i] = 0.0;
  double Rrr = q[2 * N];
  double tet = q[2 * N + 2];
  double sin_tet = sin(tet);
  double dPhidT = q[2 * N + 5] / q[2 * N] / q[2 * N] / mass / (sin_tet * sin_tet);
  orc_matrix_at(tb, Rrr, w->m, w->dm);
  for (int u = 0; u < w->n_u; ++u) {
    w->sc[2 * u] = sin(t * w->du[u]);
    w->sc[2 * u + 1] = cos(t * w->du[u]);
  }
  const int Z1 = 2 * N + 6, Z2 = 2 * N + 7; /* zero sinks */
  for (int64_t k = 0; k < P; ++k) {
    int i = tb->ind_mat[2 * k] - 1, j = tb->ind_mat[2 * k + 1] - 1;
    w->phi_amp[k] = 0.0;
    if (w->cs && tb->m12[i] != w->cs_m) continue;
    double M = w->m[k], Md = w->dm[k];
    double d_f = (i == j) ? 1.0 : 2.0;
    double iphase = w->sc[2 * w->uidx[k]], rphase = w->sc[2 * w->uidx[k] + 1];
    double rfp = -d_f * iphase, ifp = d_f * rphase;
    dq[i] += (q[j] * rfp + q[j + N] * ifp) * M / 2.0;
    dq[i + N] += (q[j + N] * rfp - q[j] * ifp) * M / 2.0;
    dq[j] -= (q[i] * rfp - q[i + N] * ifp) * M / 2.0;
    dq[j + N] -= (q[i + N] * rfp + q[i] * ifp) * M / 2.0;
    dq[2 * N + 1] -= ((q[i] * q[j] + q[i + N] * q[j + N]) * rphase -
                      (q[i + N] * q[j] - q[i] * q[j + N]) * iphase) * d_f * Md;
    if (w->cs) continue;
    const double* mc = w->misc + 4 * k;
    double amp = 0.0;
    {
      int jj = tb->j12[j], mm = tb->m12[i];
      int s1, s11, s0, s00;
      if (abs(mm + 1) <= jj) { s1 = j + 1; s11 = s1 + N; } else { s1 = Z1; s11 = Z2; }
      if (abs(mm - 1) <= jj) { s0 = j - 1; s00 = s0 + N; } else { s0 = Z1; s00 = Z2; }
      amp = amp - sin_tet * rfp / 2.0 *
                      (mc[0] * (q[i] * q[s1] + q[i + N] * q[s11]) +
                       mc[1] * (q[i] * q[s0] + q[i + N] * q[s00])) -
            sin_tet * (-ifp) / 2.0 *
                (mc[0] * (q[i + N] * q[s1] - q[i] * q[s11]) +
                 mc[1] * (q[i + N] * q[s0] - q[i] * q[s00]));
    }
    {
      int jj = tb->j12[i], mm = tb->m12[j];
      int s1, s11, s0, s00;
      if (abs(mm + 1) <= jj) { s1 = i + 1; s11 = s1 + N; } else { s1 = Z1; s11 = Z2; }
      if (abs(mm - 1) <= jj) { s0 = i - 1; s00 = s0 + N; } else { s0 = Z1; s00 = Z2; }
      amp = amp - sin_tet * (-rfp) / 2.0 *
                      (mc[2] * (q[s1] * q[j] + q[s11] * q[j + N]) +
                       mc[3] * (q[s0] * q[j] + q[s00] * q[j + N]));
      amp = amp - sin_tet * (-ifp) / 2.0 *
                      (mc[2] * (q[s1] * q[j + N] - q[s11] * q[j]) +
                       mc[3] * (q[s0] * q[j + N] - q[s00] * q[j]));
    }
    w->phi_amp[k] = amp;
  }
  double dot = 0.0;
  for (int64_t k = 0; k < P; ++k) dot += w->m[k] * w->phi_amp[k];
  dq[2 * N + 5] = w->cs ? 0.0 : dot;
  for (int i = 0; i < N && !w->cs; ++i) {
    double jj = tb->j12[i], mm = tb->m12[i];
    double m1 = mm + 1.0, m0 = mm - 1.0;
    double sqrt1 = sqrt(jj * (jj + 1.0) - m0 * (m0 + 1.0));
    double sqrt2 = sqrt(jj * (jj + 1.0) - m1 * (m1 - 1.0));
    if (i > 0) {
      dq[i] += dPhidT / 2.0 * sqrt1 * q[i - 1 + N];
      dq[i + N] -= dPhidT / 2.0 * sqrt1 * q[i - 1];
    }
    if (i < N - 1) {
      dq[i] += dPhidT / 2.0 * sqrt2 * q[i + 1 + N];
      dq[i + N] -= dPhidT / 2.0 * sqrt2 * q[i + 1];
    }
  }
  dq[2 * N] = q[2 * N + 1] / mass;
  dq[2 * N + 4] = q[2 * N + 5] / q[2 * N] / q[2 * N] / mass / (sin_tet * sin_tet);
  dq[2 * N + 1] = dq[2 * N + 1] + q[2 * N + 3] / q[2 * N] / q[2 * N] / mass * q[2 * N + 3] / q[2 * N] +
                  q[2 * N + 5] / q[2 * N] / q[2 * N] / mass * q[2 * N + 5] / q[2 * N] / (sin_tet * sin_tet);
}

int orc_derivs(const orc_tables* tab, double t, const double* q, double* dqdt) {
  orc_rhs_ws w;
  orc_ws_init(&w, tab);
  orc_derivs_ws(&w, t, q, dqdt);
  orc_ws_free(&w);
  return 0;
}

/* Classical RK4 step: SRC/suppl_routines.f:1076-1113 (rk4). */
typedef void (*orc_rhs_fn)(void* ctx, double t, const double* y, double* dy);
static void orc_rk4(int n, double* y, const double* dydx, double x, double h, orc_rhs_fn f,
                    void* ctx, double* yt, double* dyt, double* dym) {
  double hh = h * 0.5, h6 = h / 6.0, xh = x + hh;
  for (int i = 0; i < n; ++i) yt[i] = y[i] + hh * dydx[i];
  f(ctx, xh, yt, dyt);
  for (int i = 0; i < n; ++i) yt[i] = y[i] + hh * dyt[i];
  f(ctx, xh, yt, dym);
  for (int i = 0; i < n; ++i) {
    yt[i] = y[i] + h * dym[i];
    dym[i] = dyt[i] + dym[i];
  }
  f(ctx, x + h, yt, dyt);
  for (int i = 0; i < n; ++i) y[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
}
/* Adaptive step-size control, SRC/suppl_routines.f:1229-1435 (rkqs, rkck, odeint as
 * the reference modified them): Cash-Karp 5(4) steps, error max_i |yerr_i / yscal_i|
 * / eps with yscal_i = |y_i| + |h dydx_i| + 1e-30, shrink 0.9 h err^-1/4 (at least
 * h/10), grow 0.9 h err^-1/5 or 5 h below err 1.89e-4; a step at or below hmin is
 * accepted as it is; the step is cut to land on x2; at most 10000 steps, the last
 * one an RK4 step over the remainder. */
static const double ORC_CK_A4 = (double)0.6f; /* A4 = .6 is a default-real literal there */
static void orc_rkck(int n, const double* y, const double* dydx, double x, double h,
                     orc_rhs_fn f, void* ctx, double* yout, double* yerr, double* ak,
                     double* yt) {
  const double B21 = .2, B31 = 3.0 / 40.0, B32 = 9.0 / 40.0, B41 = .3, B42 = -.9, B43 = 1.2,
               B51 = -11.0 / 54.0, B52 = 2.5, B53 = -70.0 / 27.0, B54 = 35.0 / 27.0,
               B61 = 1631.0 / 55296.0, B62 = 175.0 / 512.0, B63 = 575.0 / 13824.0,
               B64 = 44275.0 / 110592.0, B65 = 253.0 / 4096.0, C1 = 37.0 / 378.0,
               C3 = 250.0 / 621.0, C4 = 125.0 / 594.0, C6 = 512.0 / 1771.0,
               DC1 = C1 - 2825.0 / 27648.0, DC3 = C3 - 18575.0 / 48384.0,
               DC4 = C4 - 13525.0 / 55296.0, DC5 = -277.0 / 14336.0, DC6 = C6 - .25;
  double *ak2 = ak, *ak3 = ak + n, *ak4 = ak + 2 * n, *ak5 = ak + 3 * n, *ak6 = ak + 4 * n;
  for (int i = 0; i < n; ++i) yt[i] = y[i] + B21 * h * dydx[i];
  f(ctx, x + .2 * h, yt, ak2);
  for (int i = 0; i < n; ++i) yt[i] = y[i] + h * (B31 * dydx[i] + B32 * ak2[i]);
  f(ctx, x + .3 * h, yt, ak3);
  for (int i = 0; i < n; ++i) yt[i] = y[i] + h * (B41 * dydx[i] + B42 * ak2[i] + B43 * ak3[i]);
  f(ctx, x + ORC_CK_A4 * h, yt, ak4);
  for (int i = 0; i < n; ++i)
    yt[i] = y[i] + h * (B51 * dydx[i] + B52 * ak2[i] + B53 * ak3[i] + B54 * ak4[i]);
  f(ctx, x + 1.0 * h, yt, ak5);
  for (int i = 0; i < n; ++i)
    yt[i] = y[i] + h * (B61 * dydx[i] + B62 * ak2[i] + B63 * ak3[i] + B64 * ak4[i] + B65 * ak5[i]);
  f(ctx, x + .875 * h, yt, ak6);
  for (int i = 0; i < n; ++i) yout[i] = y[i] + h * (C1 * dydx[i] + C3 * ak3[i] + C4 * ak4[i] + C6 * ak6[i]);
  for (int i = 0; i < n; ++i)
    yerr[i] = h * (DC1 * dydx[i] + DC3 * ak3[i] + DC4 * ak4[i] + DC5 * ak5[i] + DC6 * ak6[i]);
}
static void orc_rkqs(int n, double* y, const double* dydx, double* x, double htry, double eps,
                     const double* yscal, double* hnext, double hmin, orc_rhs_fn f, void* ctx,
                     double* ytemp, double* yerr, double* ak, double* yt) {
  double h = htry;
  for (;;) {
    orc_rkck(n, y, dydx, *x, h, f, ctx, ytemp, yerr, ak, yt);
    if (h <= hmin) break; /* accepted as it is; hnext keeps its value */
    double errmax = 0.0;
    for (int i = 0; i < n; ++i) errmax = fmax(errmax, fabs(yerr[i] / yscal[i]));
    errmax = errmax / eps;
    if (errmax > 1.0) {
      const double htemp = 0.9 * h * pow(errmax, -0.25);
      h = copysign(fmax(fabs(htemp), 0.1 * fabs(h)), h);
      continue;
    }
    *hnext = errmax > 1.89e-4 ? 0.9 * h * pow(errmax, -0.2) : 5.0 * h;
    break;
  }
  *x = *x + h;
  for (int i = 0; i < n; ++i) y[i] = ytemp[i];
}
static void orc_rk4(int n, double* y, const double* dydx, double x, double h, orc_rhs_fn f,
                    void* ctx, double* yt, double* dyt, double* dym);
/* ystart advanced from x1 to x2; h1 the first trial step, *hnext_io receives the last
 * proposed step (dt_corrected); returns the number of steps taken. */
static int orc_odeint(int n, double* ystart, double x1, double x2, double eps, double h1,
                      double hmin, orc_rhs_fn f, void* ctx, double* hnext_io) {
  const int MAXSTP = 10000;
  double* w = (double*)calloc((size_t)n * 11, sizeof(double));
  double *y = w, *dydx = w + n, *yscal = w + 2 * n, *ytemp = w + 3 * n, *yerr = w + 4 * n,
         *yt = w + 5 * n, *ak = w + 6 * n;
  double x = x1, h = copysign(h1, x2 - x1), hnext = h;
  int nstp;
  for (int i = 0; i < n; ++i) y[i] = ystart[i];
  for (nstp = 1; nstp <= MAXSTP; ++nstp) {
    f(ctx, x, y, dydx);
    if (nstp < MAXSTP) {
      for (int i = 0; i < n; ++i) yscal[i] = fabs(y[i]) + fabs(h * dydx[i]) + 1e-30;
      if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
      orc_rkqs(n, y, dydx, &x, h, eps, yscal, &hnext, hmin, f, ctx, ytemp, yerr, ak, yt);
    } else {  /* the last allowed step: RK4 over what remains */
      orc_rk4(n, y, dydx, x, x2 - x, f, ctx, yt, ytemp, yerr);
      x = x2 + copysign(1e-30, x2 - x1);
    }
    if ((x - x2) * (x2 - x1) >= 0.0) break;
    if (fabs(hnext) < hmin) hnext = copysign(hmin, x2 - x1);
    h = hnext;
  }
  for (int i = 0; i < n; ++i) ystart[i] = y[i];
  *hnext_io = hnext;
  free(w);
  return nstp;
}

/* bk_int (SRC/suppl_routines.f:1468-1653): odeint over [x1, x2] (the whole trajectory)
 * that stops after any step at which R > cut_r, the R oscillation count reaches
 * numb_oscl or the orbit count int(|phi| / 2 pi) reaches numb_orb; R and phi are
 * y[ir], y[iphi].  Returns the steps taken; *f_time is the time reached. */
typedef void (*orc_probe_fn)(void* pctx, double x, const double* y, double* R, double* phi);
static int orc_bk_int(int n, double* ystart, double x1, double x2, double eps, double h1,
                      double hmin, orc_rhs_fn f, void* ctx, double* hnext_io, double* f_time,
                      double cut_r, orc_probe_fn probe, void* pctx, int numb_oscl, int numb_orb,
                      int* vib_out, int* period_out) {
  const int MAXSTP = 10000;
  double* w = (double*)calloc((size_t)n * 11, sizeof(double));
  double *y = w, *dydx = w + n, *yscal = w + 2 * n, *ytemp = w + 3 * n, *yerr = w + 4 * n,
         *yt = w + 5 * n, *ak = w + 6 * n;
  double x = x1, h = copysign(h1, x2 - x1), hnext = h;
  double tmp_R1 = 0.0, tmp_R2 = 0.0;
  int vib = 0, period = 0, nstp;
  int stopped = 0;
  for (int i = 0; i < n; ++i) y[i] = ystart[i];
  for (nstp = 1; nstp <= MAXSTP; ++nstp) {
    f(ctx, x, y, dydx);
    if (nstp < MAXSTP) {
      for (int i = 0; i < n; ++i) yscal[i] = fabs(y[i]) + fabs(h * dydx[i]) + 1e-30;
      if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
      orc_rkqs(n, y, dydx, &x, h, eps, yscal, &hnext, hmin, f, ctx, ytemp, yerr, ak, yt);
      double rr, ph;
      probe(pctx, x, y, &rr, &ph);
      if (rr > cut_r) { stopped = 1; break; }
      if (nstp > 2 && (tmp_R2 - tmp_R1) < 0.0 && (tmp_R1 - rr) > 0.0) vib += 1;
      tmp_R2 = tmp_R1;
      tmp_R1 = rr;
      if (vib >= numb_oscl) { stopped = 1; break; }
      period = (int)(fabs(ph) / 2.0 / ORC_PI);
      if (numb_orb <= period) { stopped = 1; break; }
    } else {  /* the last allowed step: RK4 over what remains */
      orc_rk4(n, y, dydx, x, x2 - x, f, ctx, yt, ytemp, yerr);
      x = x2 + copysign(1e-30, x2 - x1);
    }
    if ((x - x2) * (x2 - x1) >= 0.0) break;
    if (fabs(hnext) < hmin) hnext = copysign(hmin, x2 - x1);
    h = hnext;
  }
  (void)stopped;
  for (int i = 0; i < n; ++i) ystart[i] = y[i];
  *hnext_io = hnext;
  *f_time = x;
  *vib_out = vib;
  *period_out = period;
  free(w);
  return nstp;
}

static void orc_rhs_std(void* ctx, double t, const double* y, double* dy) {
  orc_derivs_ws((orc_rhs_ws*)ctx, t, y, dy);
}
/* bk_int's R and phi in standard mode: the classical variables of the state. */
static void orc_probe_std(void* pctx, double x, const double* y, double* R, double* phi) {
  (void)x;
  const int N = *(const int*)pctx;
  *R = y[2 * N];
  *phi = y[2 * N + 4];
}

/* Coupling energy sum_k d_f M_k Re(a_i* a_j e^{-i dE t}) (SRC/propagator.f:2725-2788). */
static double orc_pot(orc_rhs_ws* w, double t, double R, const double* q) {
  const orc_tables* tb = w->tab;
  int N = tb->n_states;
  orc_matrix_at(tb, R, w->m, w->dm);
  double pot = 0.0;
  for (int64_t k = 0; k < tb->P; ++k) {
    int i = tb->ind_mat[2 * k] - 1, j = tb->ind_mat[2 * k + 1] - 1;
    double d = (i == j) ? 1.0 : 2.0;
    double du = w->du[w->uidx[k]];
    double ip = sin(t * du), rp = cos(t * du);
    pot += d * w->m[k] * ((q[i] * q[j] + q[i + N] * q[j + N]) * rp - (q[i + N] * q[j] - q[i] * q[j + N]) * ip);
  }
  return pot;
}

/* DOTRAJECT, standard MQCT with fixed-step RK4: initial conditions
 * SRC/propagator.f:2435-2566, energies :2695-2810, loop :3205-4050,
 * final bookkeeping :4182-4383. */
/* rec (optional, 8 doubles per record, max_rec records): the SAVE_TRAJECT
 * records of the reference (SRC/propagator.f:3458-3464, 4329-4337): at the top
 * of every step (t, R, P_R, theta, P_theta, phi, P_phi, pot) of the state before
 * the step, pot the coupling energy; after the last step one more record of the
 * final state stamped t_final + dt.  *n_rec receives the record count (the
 * records past max_rec are counted but not written). */
static int orc_dotraject_impl(const orc_tables* tab, const orc_traj* tr, double* amp, double* cls,
                              double* diag, double* rec, int64_t max_rec, int64_t* n_rec) {
  int N = tab->n_states;
  int64_t nr = 0;
  int n = 2 * N + 8;
  double mass = tab->mass_au;
  double* q = (double*)calloc((size_t)n, sizeof(double));
  double* dq = (double*)calloc((size_t)n, sizeof(double));
  double* yt = (double*)calloc((size_t)n, sizeof(double));
  double* dyt = (double*)calloc((size_t)n, sizeof(double));
  double* dym = (double*)calloc((size_t)n, sizeof(double));
  orc_rhs_ws w;
  orc_ws_init(&w, tab);
  w.cs = tr->cs;
  w.cs_m = tab->m12[tr->s_st - 1];
  double k_vec = sqrt(mass * 2.0 * tr->e_coll);
  double l_orb = sqrt(tr->l_real * (tr->l_real + 1.0));
  double R_st = tr->r_start;
  int status = 0;
  q[tr->s_st - 1] = 1.0;
  double tcur = 0.0;
  int64_t counter = 0;
  int vib = 0, period = 0;
  double pot_end = 0.0;
  double eror = 0.0, norm_err = 0.0;
  if (l_orb / k_vec > R_st) {
    status = 2; /* not propagated: impact parameter beyond RMAX */
    q[2 * N] = R_st;
  } else {
    q[2 * N] = R_st;
    q[2 * N + 1] = -sqrt(k_vec * k_vec - l_orb * l_orb / (R_st * R_st));
    q[2 * N + 2] = acos(0.0);
    q[2 * N + 3] = l_orb * sin(0.0);
    q[2 * N + 4] = 0.0;
    q[2 * N + 5] = l_orb * cos(0.0);
    double Eqi = 0.0;
    for (int i = 0; i < N; ++i) Eqi += (q[i] * q[i] + q[i + N] * q[i + N]) * tab->ej[i];
    Eqi += orc_pot(&w, tcur, q[2 * N], q);
    double pr = q[2 * N + 1], l = q[2 * N + 3], ql = q[2 * N + 2], qphi = q[2 * N + 5], R = q[2 * N];
    double Eki = pr * pr / 2.0 / mass + l * l / 2.0 / mass / (R * R) +
                 qphi * qphi / 2.0 / mass / (R * R) / (sin(ql) * sin(ql));
    double tmp_R1 = 0.0, tmp_R2 = 0.0;
    double dt_step = tr->dt; /* ODEINT's carried step (dt_step / dt_corrected) */
    int run = 1;
    while (run) {
      ++counter;
      if (q[2 * N] != q[2 * N]) { status = 3; break; }
      if (rec) {
        if (nr < max_rec) {
          double* r = rec + 8 * nr;
          r[0] = tcur;
          for (int c = 0; c < 6; ++c) r[1 + c] = q[2 * N + c];
          r[7] = orc_pot(&w, tcur, q[2 * N], q);
        }
        ++nr;
      }
      if (tr->method == 3) {  /* ODEINT with bikram_int: one bk_int call (:3925-3931) */
        double hn, ft;
        orc_bk_int(n, q, tcur, tr->time_lim, tr->eps, tr->dt, tr->hmin, orc_rhs_std, &w, &hn, &ft,
                   tr->r_fin, orc_probe_std, &N, tr->numb_oscl_prds, tr->numb_orb_prds, &vib,
                   &period);
        tcur = ft;  /* :4172 */
        break;
      }
      if (tr->method == 1) {  /* PROPAGATOR = ODEINT: adaptive steps over [t, t + dt] */
        double hn;
        orc_odeint(n, q, tcur, tcur + tr->dt, tr->eps, dt_step, tr->hmin, orc_rhs_std, &w, &hn);
        dt_step = hn;
      } else {
        orc_derivs_ws(&w, tcur, q, dq);
        orc_rk4(n, q, dq, tcur, tr->dt, orc_rhs_std, &w, yt, dyt, dym);
      }
      double uR = q[2 * N], uphi = q[2 * N + 4];
      if (tcur > (0.0 + tr->dt) && counter > 2) {
        if ((tmp_R2 - tmp_R1) < 0.0 && (tmp_R1 - uR) > 0.0) vib += 1;
      }
      tmp_R2 = tmp_R1;
      tmp_R1 = uR;
      tcur += tr->dt;
      period = (int)(fabs(uphi) / 2.0 / ORC_PI);
      if (tr->numb_orb_prds <= period) run = 0;
      if (vib >= tr->numb_oscl_prds) run = 0;
      if (tr->time_lim > 0 && tcur >= tr->time_lim) run = 0;
      if (uR > tr->r_fin) run = 0;
      if (tr->max_steps > 0 && counter >= tr->max_steps && run) { run = 0; status = 1; }
    }
    double Eqf = 0.0, Pt = 0.0;
    for (int i = 0; i < N; ++i) {
      double p = q[i] * q[i] + q[i + N] * q[i + N];
      Eqf += p * tab->ej[i];
      Pt += p;
    }
    pr = q[2 * N + 1]; l = q[2 * N + 3]; ql = q[2 * N + 2]; qphi = q[2 * N + 5]; R = q[2 * N];
    double Ef = pr * pr / 2.0 / mass + l * l / 2.0 / mass / (R * R) +
                qphi * qphi / 2.0 / mass / (R * R) / (sin(ql) * sin(ql));
    pot_end = orc_pot(&w, tcur, R, q);
    eror = fabs(Eqf + Ef + pot_end - Eki - Eqi);
    norm_err = fabs(1.0 - Pt);
    if (rec) {
      if (nr < max_rec) {
        double* r = rec + 8 * nr;
        r[0] = tcur + tr->dt;
        for (int c = 0; c < 6; ++c) r[1 + c] = q[2 * N + c];
        r[7] = pot_end;
      }
      ++nr;
    }
  }
  if (n_rec) *n_rec = nr;
  for (int i = 0; i < 2 * N; ++i) amp[i] = q[i];
  for (int c = 0; c < 6; ++c) cls[c] = q[2 * N + c];
  diag[0] = tcur; diag[1] = (double)counter; diag[2] = norm_err; diag[3] = eror;
  diag[4] = status; diag[5] = period; diag[6] = vib; diag[7] = pot_end;
  orc_ws_free(&w);
  free(q); free(dq); free(yt); free(dyt); free(dym);
  return 0;
}

int orc_dotraject(const orc_tables* tab, const orc_traj* tr, double* amp, double* cls,
                  double* diag) {
  return orc_dotraject_impl(tab, tr, amp, cls, diag, NULL, 0, NULL);
}
int orc_dotraject_rec(const orc_tables* tab, const orc_traj* tr, double* amp, double* cls,
                      double* diag, double* rec, int64_t max_rec, int64_t* n_rec) {
  return orc_dotraject_impl(tab, tr, amp, cls, diag, rec, max_rec, n_rec);
}

int orc_propagate_batch(const orc_tables* tab, int n_traj, const orc_traj* trajs, int n_threads,
                        double* amp, double* cls, double* diag) {
  int N = tab->n_states;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads > 0 ? n_threads : omp_get_max_threads())
  for (int t = 0; t < n_traj; ++t)
    orc_dotraject(tab, &trajs[t], amp + (size_t)t * 2 * N, cls + (size_t)t * 6, diag + (size_t)t * 8);
  return 0;
}

/* AT-MQCT second run: classical path from the saved trajectory splined over t
 * (end slopes from finite differences), amplitudes by DERIVS_BK_adia with RK4;
 * the last step is truncated to the final saved time.
 * SRC/propagator.f:3094-3132, 3862-3881; SRC/mqct_eqtns.f:720-985. */
typedef struct {
  orc_rhs_ws* w;
  int n_at;
  const double* t;
  double* col[4];   /* R, theta, P_theta, P_phi */
  double* col2[4];
  double* phi;      /* phi and its spline (bk_int_adia's orbit count) */
  double* phi2;
} orc_at_ctx;
/* bk_int_adia's R and phi: the saved path's splines at x (SRC/suppl_routines.f:1760-1761). */
static void orc_probe_at(void* pctx, double x, const double* y, double* R, double* phi) {
  (void)y;
  orc_at_ctx* c = (orc_at_ctx*)pctx;
  double yp;
  orc_splint(c->t, c->col[0], c->col2[0], c->n_at, x, R, &yp);
  orc_splint(c->t, c->phi, c->phi2, c->n_at, x, phi, &yp);
}
static void orc_rhs_at(void* vctx, double t, const double* q, double* dq) {
  orc_at_ctx* c = (orc_at_ctx*)vctx;
  orc_rhs_ws* w = c->w;
  const orc_tables* tb = w->tab;
  int N = tb->n_states;
  double v[4], yp;
  for (int a = 0; a < 4; ++a) orc_splint(c->t, c->col[a], c->col2[a], c->n_at, t, &v[a], &yp);
  double Rrr = v[0], tet = v[1], pphi = v[3];
  double sin_tet = sin(tet);
  double dPhidT = pphi / Rrr / Rrr / tb->mass_au / (sin_tet * sin_tet);
  for (int i = 0; i < 2 * N; ++i) dq[i] = 0.0;
  orc_matrix_at(tb, Rrr, w->m, w->dm);
  for (int u = 0; u < w->n_u; ++u) {
    w->sc[2 * u] = sin(t * w->du[u]);
    w->sc[2 * u + 1] = cos(t * w->du[u]);
  }
  for (int64_t k = 0; k < tb->P; ++k) {
    int i = tb->ind_mat[2 * k] - 1, j = tb->ind_mat[2 * k + 1] - 1;
    if (w->cs && tb->m12[i] != w->cs_m) continue; /* SRC/mqct_eqtns.f:787-789 */
    double M = w->m[k];
    double d_f = (i == j) ? 1.0 : 2.0;
    double iphase = w->sc[2 * w->uidx[k]], rphase = w->sc[2 * w->uidx[k] + 1];
    double rfp = -d_f * iphase, ifp = d_f * rphase;
    dq[i] += (q[j] * rfp + q[j + N] * ifp) * M / 2.0;
    dq[i + N] += (q[j + N] * rfp - q[j] * ifp) * M / 2.0;
    dq[j] -= (q[i] * rfp - q[i + N] * ifp) * M / 2.0;
    dq[j + N] -= (q[i + N] * rfp + q[i] * ifp) * M / 2.0;
  }
  for (int i = 0; i < N && !w->cs; ++i) { /* no Coriolis with CS_APPROX (:845) */
    double jj = tb->j12[i], mm = tb->m12[i];
    double m1 = mm + 1.0, m0 = mm - 1.0;
    double sqrt1 = sqrt(jj * (jj + 1.0) - m0 * (m0 + 1.0));
    double sqrt2 = sqrt(jj * (jj + 1.0) - m1 * (m1 - 1.0));
    if (i > 0) {
      dq[i] += dPhidT / 2.0 * sqrt1 * q[i - 1 + N];
      dq[i + N] -= dPhidT / 2.0 * sqrt1 * q[i - 1];
    }
    if (i < N - 1) {
      dq[i] += dPhidT / 2.0 * sqrt2 * q[i + 1 + N];
      dq[i + N] -= dPhidT / 2.0 * sqrt2 * q[i + 1];
    }
  }
}
int orc_dotraject_at(const orc_tables* tab, const orc_traj* tr, int n_at, const double* rec,
                     double* amp, double* diag) {
  int N = tab->n_states, n = 2 * N;
  orc_rhs_ws w;
  orc_ws_init(&w, tab);
  w.cs = tr->cs;
  w.cs_m = tab->m12[tr->s_st - 1];
  orc_at_ctx c;
  c.w = &w;
  c.n_at = n_at;
  double* t = (double*)malloc(sizeof(double) * n_at);
  for (int i = 0; i < n_at; ++i) t[i] = rec[8 * i];
  c.t = t;
  const int cols[4] = {1, 3, 4, 6}; /* R, theta, P_theta, P_phi in the record */
  for (int a = 0; a < 4; ++a) {
    c.col[a] = (double*)malloc(sizeof(double) * n_at);
    c.col2[a] = (double*)malloc(sizeof(double) * n_at);
    for (int i = 0; i < n_at; ++i) c.col[a][i] = rec[8 * i + cols[a]];
    double yp1 = (c.col[a][1] - c.col[a][0]) / (t[1] - t[0]);
    double ypn = (c.col[a][n_at - 1] - c.col[a][n_at - 2]) / (t[n_at - 1] - t[n_at - 2]);
    orc_spline(t, c.col[a], n_at, yp1, ypn, c.col2[a]);
  }
  c.phi = (double*)malloc(sizeof(double) * n_at);
  c.phi2 = (double*)malloc(sizeof(double) * n_at);
  for (int i = 0; i < n_at; ++i) c.phi[i] = rec[8 * i + 5];
  {
    double yp1 = (c.phi[1] - c.phi[0]) / (t[1] - t[0]);
    double ypn = (c.phi[n_at - 1] - c.phi[n_at - 2]) / (t[n_at - 1] - t[n_at - 2]);
    orc_spline(t, c.phi, n_at, yp1, ypn, c.phi2);
  }
  double* q = (double*)calloc((size_t)n, sizeof(double));
  double* dq = (double*)calloc((size_t)n, sizeof(double));
  double* yt = (double*)calloc((size_t)n, sizeof(double));
  double* dyt = (double*)calloc((size_t)n, sizeof(double));
  double* dym = (double*)calloc((size_t)n, sizeof(double));
  q[tr->s_st - 1] = 1.0;
  double tcur = t[0], dt = tr->dt;
  double t_end = t[n_at - 1];
  int64_t counter = 0;
  int run = 1;
  /* AT_ADAPT_STP (method 2): the step of every RK4 step from the coupling energy along
   * the path (column 8 of the records), SRC/propagator.f:3034-3049 and 3821-3860;
   * eps = AT_ADAPTOL, hmin = TIME_STEP (the smallest step). */
  double* pot = NULL;
  double* pot2 = NULL;
  double magic = 0.0, fa = 0.0;
  if (tr->method == 2) {
    pot = (double*)malloc(sizeof(double) * n_at);
    pot2 = (double*)malloc(sizeof(double) * n_at);
    for (int i = 0; i < n_at; ++i) pot[i] = rec[8 * i + 7];
    double yp1 = (pot[1] - pot[0]) / (t[1] - t[0]);
    double ypn = (pot[n_at - 1] - pot[n_at - 2]) / (t[n_at - 1] - t[n_at - 2]);
    orc_spline(t, pot, n_at, yp1, ypn, pot2);
    const double u_cm = tr->e_coll * ORC_EVTOWN * ORC_AUTOEV;
    const double tmp1 = -0.80, tmp2 = 4.250, damp = 20.0;
    double tmp3 = -exp(2.0 * ORC_PI * (u_cm - 202.0) / damp);
    if (fabs(tmp3) > 1e16) tmp3 = -1e16;
    const double tmp4 = 0.30 - tmp1 * tmp3 / (1.0 - tmp3) - tmp2 * tmp3 / pow(1.0 - tmp3, 2.0);
    const double tol = tr->eps * pow(u_cm / 300.0, tmp4);
    magic = tr->e_coll * pow(t_end * tol, 4.0);
  }
  if (tr->method == 3) {  /* ODEINT with bikram_int: bk_int_adia over the path (:3889-3896) */
    double hn, ft;
    int vib = 0, period = 0;
    orc_bk_int(n, q, tcur, t_end, tr->eps, dt, tr->hmin, orc_rhs_at, &c, &hn, &ft, tr->r_fin,
               orc_probe_at, &c, tr->numb_oscl_prds, tr->numb_orb_prds, &vib, &period);
    tcur = ft;
    counter = 1;
    run = 0;
  }
  if (tr->method == 1) {  /* ODEINT: one adaptive call over the whole path (:3888-3905) */
    double hn;
    orc_odeint(n, q, tcur, t_end, tr->eps, dt, tr->hmin, orc_rhs_at, &c, &hn);
    tcur = t_end;
    counter = 1;
    run = 0;
  }
  while (run) {
    ++counter;
    if (tr->method == 2) {
      const double tau = 10.0, mintm = tr->hmin, tmchk = tcur;
      double potbox = 0.0;
      for (int stps = 0;;) {
        const double tmstp = tmchk + tau * (stps + 0.50);
        stps += 1;
        double fb, yp;
        orc_splint(t, pot, pot2, n_at, tmstp, &fb, &yp);
        potbox += fabs(fb);
        const double i_max = pow(tau * stps, 4.0) * potbox / stps;
        int done = 0;
        if (i_max >= magic) {
          dt = tau * (stps - 1);
          if (dt < mintm) dt = mintm;
          done = 1;
        } else if (tmstp > t_end) {
          dt = t_end - tmchk;
          run = 0;
          done = 1;
        } else if (tcur > 0.0) {
          const double r = fa / fb;
          if (r < 0.0 && r == r) {
            dt = tau * (stps - 1);
            if (dt < mintm) dt = mintm;
            done = 1;
          }
        }
        fa = fb;
        if (done) break;
      }
    } else if ((tcur + dt) >= t_end) {
      dt = t_end - tcur;
      run = 0;
    }
    orc_rhs_at(&c, tcur, q, dq);
    orc_rk4(n, q, dq, tcur, dt, orc_rhs_at, &c, yt, dyt, dym);
    tcur += dt;
    if (tr->max_steps > 0 && counter >= tr->max_steps) break;
  }
  double Pt = 0.0;
  for (int i = 0; i < N; ++i) Pt += q[i] * q[i] + q[i + N] * q[i + N];
  for (int i = 0; i < n; ++i) amp[i] = q[i];
  diag[0] = tcur; diag[1] = (double)counter; diag[2] = fabs(1.0 - Pt); diag[3] = 0.0;
  diag[4] = 0; diag[5] = 0; diag[6] = 0; diag[7] = 0;
  for (int a = 0; a < 4; ++a) { free(c.col[a]); free(c.col2[a]); }
  free(pot); free(pot2); free(c.phi); free(c.phi2);
  free(t); free(q); free(dq); free(yt); free(dyt); free(dym);
  orc_ws_free(&w);
  return 0;
}

/* INELAST_CALC, SRC/propagator.f:4776-4841 with DL=1 (trajectory of l is
 * index l - L_MIN): sigma_f = pi/k^2 sum_J sum_{l=|J-j|}^{J+j} (2J+1)/(2j+1) P_f(l). */
int orc_inelast(int n_channels, int j_ini, int J_down, int J_up, int L_min, int n_traj,
                const double* prob, double k_vec, double* sigma) {
  return orc_inelast_dl(n_channels, j_ini, J_down, J_up, L_min, 1, n_traj, prob, k_vec, sigma);
}
/* With a step DL in l: trajectory id = (l - L_MIN) / DL (TRAJ_ORB flag 1,
 * SRC/propagator.f:5127-5134), so every l of a bin takes the probability of the
 * bin's trajectory, l = (id + 1/2) DL + L_MIN truncated (:5163-5167). */
int orc_inelast_dl(int n_channels, int j_ini, int J_down, int J_up, int L_min, int dl,
                   int n_traj, const double* prob, double k_vec, double* sigma) {
  if (dl < 1) return -1;
  for (int f = 0; f < n_channels; ++f) {
    double s = 0.0;
    for (int J = J_down; J <= J_up; ++J)
      for (int l = abs(J - j_ini); l <= J + j_ini; ++l) {
        int id = (l - L_min) / dl;
        if (id < 0 || id >= n_traj) continue;
        s += prob[(size_t)id * n_channels + f] * (2.0 * J + 1.0) / (k_vec * k_vec) /
             (2.0 * j_ini + 1) * ORC_PI;
      }
    sigma[f] = s;
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* SRC/pot_comp.f:7826-8058 (EXPANSION_MATRIX_ELEMENT, SYS_TYPE 8).  For the pair
 * (p = stp, pp = stpp) with total m:
 *   A_t = sqrt((2l1+1)(2l2+1))/(4 pi) <j2'' 0 l2 0|j2' 0> M1 M3,
 *   M1  = sum over nju = nju1 and (if nju1 != 0) -nju1 with the phase
 *         (-1)^(l1+l2+l+nju1) for the second, of
 *         sum_{k1'} <j1'' k1'-nju l1 nju|j1' k1'> c'_{k1'} c''_{k1'-nju}   (:7948-7974),
 *   M3  = sum_{m'} <j1' m' j2' m-m'|j12' m> sum_{me} <l1 me l2 -me|l 0>
 *         <j1'' m'' j2'' m-m''|j12'' m> <j1'' m'' l1 me|j1' m'>
 *         <j2'' m-m'' l2 -me|j2' m-m'>,  m'' = m' - me                    (:7982-8018),
 *   M_k(R) = sqrt((2j1''+1)/(2j1'+1)) sqrt((2j2''+1)/(2j2'+1)) sum_t T_t(R) A_t
 * with the triangle rules of :7923-7925. */
static int orc_triangle(int a, int b, int c) { return c >= abs(a - b) && c <= a + b; }

int orc_expansion_matrix_type8(const orc_system* sys, const int32_t* indx_chann,
                               const int32_t* j12, const int32_t* m12, int64_t P,
                               const int32_t* ind_mat, int n_terms, const int32_t* labels,
                               int nR, const double* terms, double* mat) {
  if (sys->sys_type != 8 || !sys->j2 || !sys->vec1) return -1;
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < P; ++k) {
    const int sp = ind_mat[2 * k] - 1, spp = ind_mat[2 * k + 1] - 1;
    const int cp = indx_chann[sp] - 1, cpp = indx_chann[spp] - 1;
    const int j1p = sys->j1[cp], j2p = sys->j2[cp], j1pp = sys->j1[cpp], j2pp = sys->j2[cpp];
    const int j12p = j12[sp], j12pp = j12[spp], m = m12[sp];
    const double* vp = sys->vec1 + (size_t)cp * sys->ldv;
    const double* vpp = sys->vec1 + (size_t)cpp * sys->ldv;
    const double coef12 = sqrt((2.0 * j1pp + 1.0) / (2.0 * j1p + 1.0)) *
                          sqrt((2.0 * j2pp + 1.0) / (2.0 * j2p + 1.0));
    double* out = mat + (size_t)k * nR;
    for (int i = 0; i < nR; ++i) out[i] = 0.0;
    for (int t = 0; t < n_terms; ++t) {
      const int l1 = labels[4 * t], nju1 = labels[4 * t + 1], l2 = labels[4 * t + 2],
                l = labels[4 * t + 3];
      if (!orc_triangle(j1pp, l1, j1p) || !orc_triangle(l1, l2, l) || !orc_triangle(j2pp, l2, j2p))
        continue;
      const double coef3 = sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0)) / (4.0 * ORC_PI);
      const double cg_j2 = orc_cg(j2pp, l2, j2p, 0, 0, 0);
      double m1 = 0.0;
      for (int planar = 0; planar < (nju1 == 0 ? 1 : 2); ++planar) {
        const int nju = planar ? -nju1 : nju1;
        const double phase = planar ? (((l1 + l2 + l + nju1) % 2) ? -1.0 : 1.0) : 1.0;
        double s = 0.0;
        for (int k1p = -j1p; k1p <= j1p; ++k1p) {
          const int k1pp = k1p - nju;
          if (abs(k1pp) > j1pp) continue;
          s += orc_cg(j1pp, l1, j1p, k1pp, nju, k1p) * vp[j1p + k1p] * vpp[j1pp + k1pp];
        }
        m1 += phase * s;
      }
      double m3 = 0.0;
      for (int mp = -j1p; mp <= j1p; ++mp) {
        if (abs(m - mp) > j2p) continue;
        const double cg_p = orc_cg(j1p, j2p, j12p, mp, m - mp, m);
        double m2 = 0.0;
        const int mx = l1 < l2 ? l1 : l2;
        for (int me = -mx; me <= mx; ++me) {
          const int mpp = mp - me;
          if (abs(mpp) > j1pp || abs(m - mpp) > j2pp) continue;
          m2 += orc_cg(l1, l2, l, me, -me, 0) * orc_cg(j1pp, j2pp, j12pp, mpp, m - mpp, m) *
                orc_cg(j1pp, l1, j1p, mpp, me, mp) * orc_cg(j2pp, l2, j2p, m - mpp, -me, m - mp);
        }
        m3 += m2 * cg_p;
      }
      const double a = coef3 * cg_j2 * m1 * m3;
      if (a == 0.0) continue;
      for (int i = 0; i < nR; ++i) out[i] += terms[(size_t)i * n_terms + t] * a;
    }
    for (int i = 0; i < nR; ++i) out[i] *= coef12 * ORC_CM_TO_HARTREE;
  }
  return 0;
}

/* EXPANSION_MATRIX_ELEMENT for a rotor and an atom (SRC/pot_comp.f:6551-6622 SYS_TYPE 1,
 * :6846-6954 SYS_TYPE 3, :6955-7075 SYS_TYPE 4): for the pair (st', st''), j', j'' the
 * rotor levels and m the pair's m12,
 *   M = e_unit sqrt((2j'+1)/(2j''+1)) sum_t T_t(R) sqrt((2l+1)/4pi) <j' m l 0|j'' m> S_t
 * with S_t = <j' 0 l 0|j'' 0> (type 1), the K-sum over the rotor vectors
 * sum_{+-nju} phase (-1)^nju sum_K <j' K l nju|j'' K+nju> c'_K c''_{K+nju} (type 4: phase 1
 * for +nju, (-1)^nju for -nju) or the same over the parity-adapted symmetric-top
 * components with 1/sqrt(2(1+d_k'0) 2(1+d_k''0)) (type 3, whose -nju branch carries the
 * factor (-1)**(-1)**nju = -1 as written there).  Terms nR x n_terms, labels 5 per term
 * (l, nju, ...). */
int orc_expansion_matrix_atom(const orc_system* sys, const int32_t* indx_chann,
                              const int32_t* j12, const int32_t* m12, int64_t P,
                              const int32_t* ind_mat, int n_terms, const int32_t* a_top, int nR,
                              const double* terms, double e_unit, double* mat) {
  const int type = sys->sys_type;
  if (type != 1 && type != 3 && type != 4) return -1;
  if (type == 4 && !sys->vec1) return -1;
  if (type == 3 && (!sys->ka1 || !sys->kc1)) return -1;
  (void)j12;
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < P; ++k) {
    const int sp = ind_mat[2 * k] - 1, spp = ind_mat[2 * k + 1] - 1;
    const int cp = indx_chann[sp] - 1, cpp = indx_chann[spp] - 1;
    const int jp = sys->j1[cp], jpp = sys->j1[cpp], m = m12[sp];
    const double coef1 = sqrt((2.0 * jp + 1.0) / (2.0 * jpp + 1.0));
    double* out = mat + (size_t)k * nR;
    for (int i = 0; i < nR; ++i) out[i] = 0.0;
    for (int t = 0; t < n_terms; ++t) {
      const int l = a_top[5 * t], nju0 = type == 1 ? 0 : a_top[5 * t + 1];
      if (!orc_triangle(jpp, l, jp)) continue;
      const double coef2 = sqrt((2.0 * l + 1.0) / (4.0 * ORC_PI));
      const double cg_m = orc_cg(jp, l, jpp, m, 0, m);
      double S = 0.0;
      if (type == 1) {
        S = orc_cg(jp, l, jpp, 0, 0, 0);
      } else if (type == 4) {
        const double* vp = sys->vec1 + (size_t)cp * sys->ldv;
        const double* vpp = sys->vec1 + (size_t)cpp * sys->ldv;
        for (int planar = 0; planar < (nju0 == 0 ? 1 : 2); ++planar) {
          const double phase = planar ? ((nju0 % 2) ? -1.0 : 1.0) : 1.0;
          const int nju = planar ? -nju0 : nju0;
          const double sg = (abs(nju) % 2) ? -1.0 : 1.0;
          for (int kp = -jp; kp <= jp; ++kp) {
            const int kpp = kp + nju;
            if (abs(kpp) > jpp) continue;
            S += phase * sg * orc_cg(jp, l, jpp, kp, nju, kpp) * vp[jp + kp] * vpp[jpp + kpp];
          }
        }
      } else {  /* type 3: channel (j, k, eps) */
        const int kc_p = sys->ka1[cp], kc_pp = sys->ka1[cpp];
        const int ep = sys->kc1[cp], epp = sys->kc1[cpp];
        const double norm = 1.0 / sqrt(2.0 * (1.0 + (kc_p == 0)) * 2.0 * (1.0 + (kc_pp == 0)));
        for (int planar = 0; planar < (nju0 == 0 ? 1 : 2); ++planar) {
          const double phase = planar ? -1.0 : 1.0;
          const int nju = planar ? -nju0 : nju0;
          const double sg = (abs(nju) % 2) ? -1.0 : 1.0;
          for (int par_p = 0; par_p < 2; ++par_p)
            for (int par_pp = 0; par_pp < 2; ++par_pp) {
              const int kp = par_p ? -kc_p : kc_p, kpp = par_pp ? -kc_pp : kc_pp;
              if (kpp != kp + nju) continue;
              const double sp_ = (par_p && (ep % 2)) ? -1.0 : 1.0;
              const double spp_ = (par_pp && (epp % 2)) ? -1.0 : 1.0;
              S += phase * sg * orc_cg(jp, l, jpp, kp, nju, kpp) * sp_ * spp_;
            }
        }
        S *= norm;
      }
      const double a = coef2 * cg_m * S;
      if (a == 0.0) continue;
      for (int i = 0; i < nR; ++i) out[i] += terms[(size_t)i * n_terms + t] * a;
    }
    for (int i = 0; i < nR; ++i) out[i] *= coef1 * e_unit;
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* SRC/pot_comp.f:8257-8746 (EXPANSION_MATRIX_ELEMENT, SYS_TYPE 0, two asymmetric
 * tops, partners distinguishable: the CG_jk_1 / M_coulp_1 branch).  For the pair
 * (p = stp, pp = stpp) with total m and the term (l1, nju1, l2, nju2, l):
 *   A_t = sqrt((2l1+1)(2l2+1))/(8 pi^2) K_t M3_t,
 *   K_t = sum over (nju1, nju2) and, unless both vanish, (-nju1, -nju2) with the
 *         phase (-1)^(l1+l2+l+nju1+nju2) for the second, of S1 S2 with
 *         S1 = sum_{k1'} <j1'' k1'-nju1 l1 nju1|j1' k1'> c1'_{k1'} c1''_{k1'-nju1},
 *         S2 = sum_{k2'} <j2'' k2'-nju2 l2 nju2|j2' k2'> c2'_{k2'} c2''_{k2'-nju2}
 *         (:8388-8425, triangle rules of :8381-8382),
 *   M3_t as for SYS_TYPE 8 (:8577-8650),
 *   M_k(R) = e_unit sqrt((2j1''+1)/(2j1'+1)) sqrt((2j2''+1)/(2j2'+1)) sum_t T_t(R) A_t
 * (:8653-8672; e_unit = conv_unit_e, SRC/matrix_ini.f:918-921). */
int orc_expansion_matrix_type0(const orc_system* sys, const int32_t* indx_chann,
                               const int32_t* j12, const int32_t* m12, int64_t P,
                               const int32_t* ind_mat, int n_terms, const int32_t* labels,
                               int nR, const double* terms, double e_unit, double* mat) {
  const int t9 = sys->sys_type == 9;
  if ((sys->sys_type != 0 && !t9) || !sys->j2 || !sys->vec1) return -1;
  if (t9 ? (!sys->ka2 || !sys->kc2) : !sys->vec2) return -1;
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < P; ++k) {
    const int sp = ind_mat[2 * k] - 1, spp = ind_mat[2 * k + 1] - 1;
    const int cp = indx_chann[sp] - 1, cpp = indx_chann[spp] - 1;
    const int j1p = sys->j1[cp], j2p = sys->j2[cp], j1pp = sys->j1[cpp], j2pp = sys->j2[cpp];
    const int j12p = j12[sp], j12pp = j12[spp], m = m12[sp];
    /* SYS_TYPE 9: the second rotor is the symmetric top (j2, k2, eps2) of ka2, kc2 */
    const int k2p_ = t9 ? sys->ka2[cp] : 0, k2pp_ = t9 ? sys->ka2[cpp] : 0;
    const int e2p = t9 ? sys->kc2[cp] : 0, e2pp = t9 ? sys->kc2[cpp] : 0;
    const double coef_parity = 1.0 / sqrt(2.0 * (1.0 + (k2p_ == 0)) * 2.0 * (1.0 + (k2pp_ == 0)));
    const double* v1p = sys->vec1 + (size_t)cp * sys->ldv;
    const double* v1pp = sys->vec1 + (size_t)cpp * sys->ldv;
    const double* v2p = t9 ? NULL : sys->vec2 + (size_t)cp * sys->ldv;
    const double* v2pp = t9 ? NULL : sys->vec2 + (size_t)cpp * sys->ldv;
    const double coef12 = sqrt((2.0 * j1pp + 1.0) / (2.0 * j1p + 1.0)) *
                          sqrt((2.0 * j2pp + 1.0) / (2.0 * j2p + 1.0)) * (t9 ? coef_parity : 1.0);
    double* out = mat + (size_t)k * nR;
    for (int i = 0; i < nR; ++i) out[i] = 0.0;
    for (int t = 0; t < n_terms; ++t) {
      const int l1 = labels[5 * t], nju1 = labels[5 * t + 1], l2 = labels[5 * t + 2],
                nju2 = labels[5 * t + 3], l = labels[5 * t + 4];
      if (!orc_triangle(j1pp, l1, j1p) || !orc_triangle(j2pp, l2, j2p) || !orc_triangle(l1, l2, l))
        continue;
      const double coef3 = sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0)) / (8.0 * ORC_PI * ORC_PI);
      double kt = 0.0;
      const int n_planar = (nju1 == 0 && nju2 == 0) ? 1 : 2;
      for (int planar = 0; planar < n_planar; ++planar) {
        const int n1 = planar ? -nju1 : nju1, n2 = planar ? -nju2 : nju2;
        const double phase = planar ? (((l1 + l2 + l + nju1 + nju2) & 1) ? -1.0 : 1.0) : 1.0;
        double s1 = 0.0, s2 = 0.0;
        for (int k1p = -j1p; k1p <= j1p; ++k1p) {
          const int k1pp = k1p - n1;
          if (abs(k1pp) > j1pp) continue;
          s1 += orc_cg(j1pp, l1, j1p, k1pp, n1, k1p) * v1p[j1p + k1p] * v1pp[j1pp + k1pp];
        }
        if (t9) {  /* CG_in_all of case 9, SRC/pot_comp.f:8161-8172 */
          const double sgp = (e2p & 1) ? -1.0 : 1.0, sgpp = (e2pp & 1) ? -1.0 : 1.0;
          s2 = orc_cg(j2pp, l2, j2p, k2pp_, n2, k2p_) +
               orc_cg(j2pp, l2, j2p, k2pp_, n2, -k2p_) * sgp +
               orc_cg(j2pp, l2, j2p, -k2pp_, n2, k2p_) * sgpp +
               orc_cg(j2pp, l2, j2p, -k2pp_, n2, -k2p_) * sgp * sgpp;
        } else {
          for (int k2p = -j2p; k2p <= j2p; ++k2p) {
            const int k2pp = k2p - n2;
            if (abs(k2pp) > j2pp) continue;
            s2 += orc_cg(j2pp, l2, j2p, k2pp, n2, k2p) * v2p[j2p + k2p] * v2pp[j2pp + k2pp];
          }
        }
        kt += phase * s1 * s2;
      }
      double m3 = 0.0;
      for (int mp = -j1p; mp <= j1p; ++mp) {
        if (abs(m - mp) > j2p) continue;
        const double cg_p = orc_cg(j1p, j2p, j12p, mp, m - mp, m);
        double m2 = 0.0;
        const int mx = l1 < l2 ? l1 : l2;
        for (int me = -mx; me <= mx; ++me) {
          const int mpp = mp - me;
          if (abs(mpp) > j1pp || abs(m - mpp) > j2pp) continue;
          m2 += orc_cg(l1, l2, l, me, -me, 0) * orc_cg(j1pp, j2pp, j12pp, mpp, m - mpp, m) *
                orc_cg(j1pp, l1, j1p, mpp, me, mp) * orc_cg(j2pp, l2, j2p, m - mpp, -me, m - mp);
        }
        m3 += m2 * cg_p;
      }
      const double a = coef3 * kt * m3;
      if (a == 0.0) continue;
      for (int i = 0; i < nR; ++i) out[i] += terms[(size_t)i * n_terms + t] * a;
    }
    for (int i = 0; i < nR; ++i) out[i] *= coef12 * e_unit;
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* SRC/pot_comp.f:7593-7824 (EXPANSION_MATRIX_ELEMENT, SYS_TYPE 7: symmetric top
 * (j1, k, eps) + diatom j2, the parity-adapted top |j k eps> =
 * (|j k> + (-1)^eps |j -k>) / sqrt(2 (1 + delta_k0))).  For the pair (p, pp) and the
 * term (l1, nju1, l2, l):
 *   A_t = sqrt((2l1+1)(2l2+1))/(4 pi) coef4 <j2'' 0 l2 0|j2' 0> M1 M3,
 *   coef4 = 1/sqrt(2(1+d_{k'0}) 2(1+d_{k''0})),
 *   M1 = sum over nju = nju1 and (nju1 != 0) -nju1, phase (-1)^(l1+l2+l+nju1) on the
 *        second, of <j1'' k'' l1 nju|j1' k'> + (-1)^eps' <j1'' k'' l1 nju|j1' -k'>
 *        + (-1)^eps'' <j1'' -k'' l1 nju|j1' k'> + (-1)^(eps'+eps'') <j1'' -k'' l1 nju|j1' -k'>
 *        (:7680-7707),
 *   M3 as for SYS_TYPE 8 (:7712-7745),
 *   M_k(R) = e_unit sqrt((2j1''+1)/(2j1'+1)) sqrt((2j2''+1)/(2j2'+1)) sum_t T_t(R) A_t.
 * The channel's k is sys->ka1, its eps sys->kc1; labels 4 per term. */
int orc_expansion_matrix_type7(const orc_system* sys, const int32_t* indx_chann,
                               const int32_t* j12, const int32_t* m12, int64_t P,
                               const int32_t* ind_mat, int n_terms, const int32_t* labels,
                               int nR, const double* terms, double e_unit, double* mat) {
  if (sys->sys_type != 7 || !sys->j2 || !sys->ka1 || !sys->kc1) return -1;
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < P; ++k) {
    const int sp = ind_mat[2 * k] - 1, spp = ind_mat[2 * k + 1] - 1;
    const int cp = indx_chann[sp] - 1, cpp = indx_chann[spp] - 1;
    const int j1p = sys->j1[cp], j2p = sys->j2[cp], j1pp = sys->j1[cpp], j2pp = sys->j2[cpp];
    const int kp = sys->ka1[cp], kpp = sys->ka1[cpp];
    const double sp_eps = (sys->kc1[cp] & 1) ? -1.0 : 1.0, spp_eps = (sys->kc1[cpp] & 1) ? -1.0 : 1.0;
    const int j12p = j12[sp], j12pp = j12[spp], m = m12[sp];
    const double coef12 = sqrt((2.0 * j1pp + 1.0) / (2.0 * j1p + 1.0)) *
                          sqrt((2.0 * j2pp + 1.0) / (2.0 * j2p + 1.0));
    const double coef4 = 1.0 / sqrt(2.0 * (1.0 + (kp == 0)) * 2.0 * (1.0 + (kpp == 0)));
    double* out = mat + (size_t)k * nR;
    for (int i = 0; i < nR; ++i) out[i] = 0.0;
    for (int t = 0; t < n_terms; ++t) {
      const int l1 = labels[4 * t], nju1 = labels[4 * t + 1], l2 = labels[4 * t + 2],
                l = labels[4 * t + 3];
      if (!orc_triangle(j1pp, l1, j1p) || !orc_triangle(l1, l2, l) || !orc_triangle(j2pp, l2, j2p))
        continue;
      const double coef3 = sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0)) / (4.0 * ORC_PI);
      const double cg_j2 = orc_cg(j2pp, l2, j2p, 0, 0, 0);
      double m1 = 0.0;
      for (int planar = 0; planar < (nju1 == 0 ? 1 : 2); ++planar) {
        const int nju = planar ? -nju1 : nju1;
        const double phase = planar ? (((l1 + l2 + l + nju1) % 2) ? -1.0 : 1.0) : 1.0;
        const double cg_all = orc_cg(j1pp, l1, j1p, kpp, nju, kp) +
                              orc_cg(j1pp, l1, j1p, kpp, nju, -kp) * sp_eps +
                              orc_cg(j1pp, l1, j1p, -kpp, nju, kp) * spp_eps +
                              orc_cg(j1pp, l1, j1p, -kpp, nju, -kp) * sp_eps * spp_eps;
        m1 += phase * cg_all;
      }
      double m3 = 0.0;
      for (int mp = -j1p; mp <= j1p; ++mp) {
        if (abs(m - mp) > j2p) continue;
        const double cg_p = orc_cg(j1p, j2p, j12p, mp, m - mp, m);
        double m2 = 0.0;
        const int mx = l1 < l2 ? l1 : l2;
        for (int me = -mx; me <= mx; ++me) {
          const int mpp = mp - me;
          if (abs(mpp) > j1pp || abs(m - mpp) > j2pp) continue;
          m2 += orc_cg(l1, l2, l, me, -me, 0) * orc_cg(j1pp, j2pp, j12pp, mpp, m - mpp, m) *
                orc_cg(j1pp, l1, j1p, mpp, me, mp) * orc_cg(j2pp, l2, j2p, m - mpp, -me, m - mp);
        }
        m3 += m2 * cg_p;
      }
      const double a = coef3 * coef4 * cg_j2 * m1 * m3;
      if (a == 0.0) continue;
      for (int i = 0; i < nR; ++i) out[i] += terms[(size_t)i * n_terms + t] * a;
    }
    for (int i = 0; i < nR; ++i) out[i] *= coef12 * e_unit;
  }
  return 0;
}

/* ---------------------------------------------------------------------- */
/* Identical partners (IDENTICAL = YES with IDENTICAL_PES = YES), SYS_TYPE 0,
 * SRC/pot_comp.f:8257-8746 (EXPANSION_MATRIX_ELEMENT, case 0, all four symmetry
 * branches).  States carry the exchange parity par = parity_state (+-1,
 * SRC/matrix_ini.f:482-530); the channel's inversion parity p_inv = p1 p2 with p_r the
 * sign of c_K c_-K for the first K = -j.. with a non-zero product (SRC/pot_comp.f:
 * 70-110) and kappa = (-1)^(k1 + k2), k_r the parity of Ka_r - Kc_r (SRC/matrix_ini.f:
 * 9147-9190) give parity_state_bk = (-1)^j12 p_inv kappa (SRC/matrix_ini.f:504), except
 * for a diagonal pair of a channel whose two rotors are in the same level, where it is
 * (-1)^j12 (SRC/pot_comp.f:8500-8505).  Per pair and term (l1, nju1, l2, nju2, l):
 *   sym1: (j1'',l1,j1'), (j2'',l2,j2') triangles -- the direct branch;
 *   sym2: unless l1 = l2 and |nju1| = |nju2|, (j1'',l2,j1'), (j2'',l1,j2') -- l1 <-> l2;
 *   sym3: (j1'',l1,j2'), (j2'',l2,j1') -- the molecules exchanged, times par' bk';
 *   sym4: unless l1 = l2 and |nju1| = |nju2|, (j1'',l2,j2'), (j2'',l1,j1'), likewise,
 * each a planar sum of products of rotor sums (K-sums), and a sum over m' (|m'| <= j1'
 * for the direct branches, |m'| <= j2' for the exchanged ones) and m_e of Clebsch-Gordan
 * products (:8577-8650; the source loops m' over -j1'..j1' for all four, but the
 * reference's own output for this case, EXAMPLES_IO/SYS_TYPE_0/H2O_H2O_Identical/MTRX.DAT,
 * has the exchanged branches summed over |m'| <= j2', which this follows); the element is divided by
 * sqrt(1 + d(j1',j2') d_p) sqrt(1 + d(j1'',j2'') d_pp), d_p = 1 when the two rotors of
 * the channel are in the same level (:8674-8684). */
static double orc_ksum(int jpp, int l, int jp, int nju, const double* vp, const double* vpp) {
  double s = 0.0;
  for (int kp = -jp; kp <= jp; ++kp) {
    const int kpp = kp - nju;
    if (abs(kpp) > jpp) continue;
    s += orc_cg(jpp, l, jp, kpp, nju, kp) * vp[jp + kp] * vpp[jpp + kpp];
  }
  return s;
}
int orc_parity_inversion(const double* v1, int j1, const double* v2, int j2) {
  int par[2] = {1, 1};
  const double* v[2] = {v1, v2};
  const int jj[2] = {j1, j2};
  for (int r = 0; r < 2; ++r)
    for (int i = 0; i <= jj[r]; ++i) {  /* K = -j + i and -K */
      const double d = v[r][i] * v[r][2 * jj[r] - i];
      if (d == 0.0) continue;
      par[r] = d > 0.0 ? 1 : -1;
      break;
    }
  return par[0] * par[1];
}
int orc_expansion_matrix_type0_identical(const orc_system* sys, const int32_t* indx_chann,
                                         const int32_t* j12, const int32_t* m12,
                                         const int32_t* parity, int64_t P,
                                         const int32_t* ind_mat, int n_terms,
                                         const int32_t* labels, int nR, const double* terms,
                                         double e_unit, double* mat) {
  if (sys->sys_type != 0 || !sys->j2 || !sys->vec1 || !sys->vec2 || !sys->ka1 || !sys->kc1 ||
      !sys->ka2 || !sys->kc2 || !parity)
    return -1;
  const int nch = sys->n_channels;
  int* pinv = (int*)malloc(sizeof(int) * nch);
  int* kap = (int*)malloc(sizeof(int) * nch);
  int* same = (int*)malloc(sizeof(int) * nch);
  for (int c = 0; c < nch; ++c) {
    pinv[c] = orc_parity_inversion(sys->vec1 + (size_t)c * sys->ldv, sys->j1[c],
                                   sys->vec2 + (size_t)c * sys->ldv, sys->j2[c]);
    const int k1 = abs(sys->ka1[c] - sys->kc1[c]) % 2, k2 = abs(sys->ka2[c] - sys->kc2[c]) % 2;
    kap[c] = ((k1 + k2) % 2) ? -1 : 1;
    same[c] = sys->j1[c] == sys->j2[c] && sys->ka1[c] == sys->ka2[c] && sys->kc1[c] == sys->kc2[c];
  }
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < P; ++k) {
    const int sp = ind_mat[2 * k] - 1, spp = ind_mat[2 * k + 1] - 1;
    const int cp = indx_chann[sp] - 1, cpp = indx_chann[spp] - 1;
    const int j1p = sys->j1[cp], j2p = sys->j2[cp], j1pp = sys->j1[cpp], j2pp = sys->j2[cpp];
    const int j12p = j12[sp], j12pp = j12[spp], m = m12[sp];
    const double* v1p = sys->vec1 + (size_t)cp * sys->ldv;
    const double* v1pp = sys->vec1 + (size_t)cpp * sys->ldv;
    const double* v2p = sys->vec2 + (size_t)cp * sys->ldv;
    const double* v2pp = sys->vec2 + (size_t)cpp * sys->ldv;
    const double par_p = parity[sp];
    double bk_par1 = ((j12p % 2) ? -1.0 : 1.0) * pinv[cp] * kap[cp];
    if (sp == spp && same[cp]) bk_par1 = (j12p % 2) ? -1.0 : 1.0;
    const double coef12 = sqrt((2.0 * j1pp + 1.0) / (2.0 * j1p + 1.0)) *
                          sqrt((2.0 * j2pp + 1.0) / (2.0 * j2p + 1.0));
    double* out = mat + (size_t)k * nR;
    for (int i = 0; i < nR; ++i) out[i] = 0.0;
    for (int t = 0; t < n_terms; ++t) {
      const int l1 = labels[5 * t], nju1 = labels[5 * t + 1], l2 = labels[5 * t + 2],
                nju2 = labels[5 * t + 3], l = labels[5 * t + 4];
      if (!orc_triangle(l1, l2, l)) continue;
      const double coef3 = sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0)) / (8.0 * ORC_PI * ORC_PI);
      const int n_planar = (nju1 == 0 && nju2 == 0) ? 1 : 2;
      const int swap_ok = !(l1 == l2 && abs(nju1) == abs(nju2));
      const int s1 = orc_triangle(j1pp, l1, j1p) && orc_triangle(j2pp, l2, j2p);
      const int s2 = swap_ok && orc_triangle(j1pp, l2, j1p) && orc_triangle(j2pp, l1, j2p);
      const int s3 = orc_triangle(j1pp, l1, j2p) && orc_triangle(j2pp, l2, j1p);
      const int s4 = swap_ok && orc_triangle(j1pp, l2, j2p) && orc_triangle(j2pp, l1, j1p);
      if (!s1 && !s2 && !s3 && !s4) continue;
      double k1 = 0.0, k2 = 0.0, k3 = 0.0, k4 = 0.0;
      for (int planar = 0; planar < n_planar; ++planar) {
        const int n1 = planar ? -nju1 : nju1, n2 = planar ? -nju2 : nju2;
        const double sg = planar ? (((l1 + l2 + l + nju1 + nju2) % 2) ? -1.0 : 1.0) : 1.0;
        const double sx = ((l1 + l2) % 2) ? -1.0 : 1.0;
        if (s1) k1 += orc_ksum(j1pp, l1, j1p, n1, v1p, v1pp) * orc_ksum(j2pp, l2, j2p, n2, v2p, v2pp) * sg;
        if (s2)
          k2 += orc_ksum(j1pp, l2, j1p, n2, v1p, v1pp) * orc_ksum(j2pp, l1, j2p, n1, v2p, v2pp) * (sg * sx);
        if (s3)
          k3 += orc_ksum(j1pp, l1, j2p, n1, v2p, v1pp) * orc_ksum(j2pp, l2, j1p, n2, v1p, v2pp) * sg *
                par_p * bk_par1;
        if (s4)
          k4 += orc_ksum(j1pp, l2, j2p, n2, v2p, v1pp) * orc_ksum(j2pp, l1, j1p, n1, v1p, v2pp) *
                (sg * sx) * par_p * bk_par1;
      }
      double m5 = 0.0;
      const int mx = l1 < l2 ? l1 : l2;
      const int jm = j1p > j2p ? j1p : j2p;  /* direct branches |m'| <= j1', exchanged <= j2' */
      for (int mp = -jm; mp <= jm; ++mp) {
        if (abs(m - mp) > j1p && abs(m - mp) > j2p) continue;
        const double cg_p = orc_cg(j1p, j2p, j12p, mp, m - mp, m);   /* 0 when |m - mp| > j2' */
        const double cg_x = orc_cg(j2p, j1p, j12p, mp, m - mp, m);
        double a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
        for (int me = -mx; me <= mx; ++me) {
          const int mpp = mp - me;
          if (abs(mpp) > j1pp || abs(m - mpp) > j2pp) continue;
          const double c0 = orc_cg(l1, l2, l, me, -me, 0) * orc_cg(j1pp, j2pp, j12pp, mpp, m - mpp, m);
          if (abs(mp) <= j1p) {
            if (s1) a1 += c0 * orc_cg(j1pp, l1, j1p, mpp, me, mp) * orc_cg(j2pp, l2, j2p, m - mpp, -me, m - mp);
            if (s2) a2 += c0 * orc_cg(j1pp, l2, j1p, mpp, me, mp) * orc_cg(j2pp, l1, j2p, m - mpp, -me, m - mp);
          }
          if (abs(mp) <= j2p) {
            if (s3) a3 += c0 * orc_cg(j1pp, l1, j2p, mpp, me, mp) * orc_cg(j2pp, l2, j1p, m - mpp, -me, m - mp);
            if (s4) a4 += c0 * orc_cg(j1pp, l2, j2p, mpp, me, mp) * orc_cg(j2pp, l1, j1p, m - mpp, -me, m - mp);
          }
        }
        if (s1) m5 += a1 * cg_p * k1;
        if (s2) m5 += a2 * cg_p * k2;
        if (s3) m5 += a3 * cg_x * k3;
        if (s4) m5 += a4 * cg_x * k4;
      }
      const double a = coef3 * m5;
      if (a == 0.0) continue;
      for (int i = 0; i < nR; ++i) out[i] += terms[(size_t)i * n_terms + t] * a;
    }
    const double dp = (j1p == j2p && same[cp]) ? 1.0 : 0.0, dpp = (j1pp == j2pp && same[cpp]) ? 1.0 : 0.0;
    const double norm = coef12 / sqrt(1.0 + dp) / sqrt(1.0 + dpp);
    for (int i = 0; i < nR; ++i) out[i] *= norm * e_unit;
  }
  free(pinv); free(kap); free(same);
  return 0;
}

/* ---------------------------------------------------------------------- */
/* EXPANSION_TERM (SRC/pot_comp.f:3739-3896) for SYS_TYPE 7 and 8 (the same function,
 * :3796-3824) and 0 (:3873-3895): the angular function of a PES expansion term at the
 * grid angles (beta1, gamma1) of molecule 1 (alpha1 = 0) and (alpha2, beta2, gamma2) of
 * molecule 2,
 *   7, 8: sqrt((2l1+1)/4pi) sum_{m=-l2..l2, |m|<=l1} <l1 m l2 -m|l 0>
 *         Djkm(l1, nju1, m; 0, beta1, gamma1) WF_DIAT_TOP(l2, -m; beta2, alpha2)
 *   0:    sum_{|m|<=min(l1,l2)} <l1 m l2 -m|l 0> N1 Djkm(l1, nju1, m; 0, beta1, gamma1)
 *         N2 Djkm(l2, nju2, -m; alpha2, beta2, gamma2),  N = sqrt((2l+1)/8pi^2). */
void orc_expansion_term(int sys_type, int l, int l1, int l2, int nju1, int nju2, double beta1,
                        double gamma1, double alpha2, double beta2, double gamma2, double* wfr,
                        double* wfi) {
  double wr = 0.0, wi = 0.0;
  if (sys_type == 0) {
    const int mm = l1 < l2 ? l1 : l2;
    for (int m = -mm; m <= mm; ++m) {
      double dr1, di1, dr2, di2;
      orc_djkm(l1, nju1, m, 0.0, beta1, gamma1, &dr1, &di1);
      const double n1 = sqrt((2.0 * l1 + 1.0) / 8.0 / (ORC_PI * ORC_PI));
      dr1 *= n1;
      di1 *= n1;
      orc_djkm(l2, nju2, -m, alpha2, beta2, gamma2, &dr2, &di2);
      const double n2 = sqrt((2.0 * l2 + 1.0) / 8.0 / (ORC_PI * ORC_PI));
      dr2 *= n2;
      di2 *= n2;
      const double cg = orc_cg(l1, l2, l, m, -m, 0);
      wr += cg * (dr1 * dr2 - di1 * di2);
      wi += cg * (dr1 * di2 + dr2 * di1);
    }
    *wfr = wr;
    *wfi = wi;
    return;
  }
  for (int m = -l2; m <= l2; ++m) {
    if (abs(m) > l1) continue;
    double dr1, di1, dr2, di2;
    orc_djkm(l1, nju1, m, 0.0, beta1, gamma1, &dr1, &di1);
    orc_wf_diat(l2, -m, beta2, alpha2, &dr2, &di2);
    const double cg = orc_cg(l1, l2, l, m, -m, 0);
    wr += cg * (dr1 * dr2 - di1 * di2);
    wi += cg * (dr1 * di2 + dr2 * di1);
  }
  const double f = sqrt((2.0 * l1 + 1.0) / 4.0 / ORC_PI);
  *wfr = wr * f;
  *wfi = wi * f;
}

/* CALC_EXPANSION_TERMS (SRC/pot_comp.f:5174-5417 for SYS_TYPE 7 and 8, :5557-5765 for
 * 0; the grids of INI_POT_STORAGE, :1310-1370 and :1628-1700): the quadrature
 * projection of V on the angular grid onto each term,
 *   terms[t * nR + iR] = sum_g V Re(EXPANSION_TERM) wb wg sin(beta1) waa wbb sin(beta2)
 *                        [wgg] xbl xgl xaal xbbl [xggl 2 pi]   (terms_im: Im)
 * the bracketed factors for SYS_TYPE 0 only; beta1, beta2 Gauss-Legendre on [0, pi];
 * alpha2, gamma1, gamma2 on [0, 2 pi] midpoint-equidistant with weight 2/n (eq_gamma) or
 * Gauss-Legendre.  V[iR][alpha2][beta1][beta2][gamma1][gamma2] (V_3_2 / V_TRANSFER with
 * gamma2, then gamma1, fastest; n_gamma2 = 1 for SYS_TYPE 7 and 8).  a_top: 5 per term,
 * (l1, nju1, l2, l, -) for 7 and 8, (l1, nju1, l2, nju2, l) for 0. */
int orc_project_terms(int sys_type, int n_terms, const int32_t* a_top, int n_alpha2,
                      int n_beta1, int n_beta2, int n_gamma1, int n_gamma2, int eq_gamma, int nR,
                      const double* V, double* terms, double* terms_im) {
  if (sys_type != 0) n_gamma2 = 1;
  double* xb = (double*)malloc(sizeof(double) * n_beta1);
  double* wb = (double*)malloc(sizeof(double) * n_beta1);
  double* xbb = (double*)malloc(sizeof(double) * n_beta2);
  double* wbb = (double*)malloc(sizeof(double) * n_beta2);
  double* xg = (double*)malloc(sizeof(double) * n_gamma1);
  double* wg = (double*)malloc(sizeof(double) * n_gamma1);
  double* xgg = (double*)malloc(sizeof(double) * n_gamma2);
  double* wgg = (double*)malloc(sizeof(double) * n_gamma2);
  double* xaa = (double*)malloc(sizeof(double) * n_alpha2);
  double* waa = (double*)malloc(sizeof(double) * n_alpha2);
  orc_gauleg(n_beta1, xb, wb);
  orc_gauleg(n_beta2, xbb, wbb);
  const double xbm = 0.5 * ORC_PI, xbl = 0.5 * ORC_PI, xgm = ORC_PI, xgl = ORC_PI;
  const int nax[3] = {n_gamma1, n_gamma2, n_alpha2};
  double* ax[3] = {xg, xgg, xaa};
  double* aw[3] = {wg, wgg, waa};
  for (int a = 0; a < 3; ++a) {
    if (eq_gamma) {
      for (int i = 0; i < nax[a]; ++i) {
        ax[a][i] = (i + 0.5) * 2.0 * xgl / nax[a];
        aw[a][i] = 2.0 / nax[a];
      }
    } else {
      orc_gauleg(nax[a], ax[a], aw[a]);
      for (int i = 0; i < nax[a]; ++i) ax[a][i] = xgm + xgl * ax[a][i];
    }
  }
  if (sys_type != 0) {
    xgg[0] = 0.0;
    wgg[0] = 1.0;
  }
  const double tail = sys_type == 0 ? xbl * xgl * xgl * xbl * xgl * 2.0 * ORC_PI
                                    : xbl * xgl * xgl * xbl;
  const size_t G = (size_t)n_alpha2 * n_beta1 * n_beta2 * n_gamma1 * n_gamma2;
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int t = 0; t < n_terms; ++t)
    for (int iR = 0; iR < nR; ++iR) {
      const int32_t* lab = a_top + 5 * t;
      const int l1 = lab[0], nju1 = lab[1], l2 = lab[2];
      const int nju2 = sys_type == 0 ? lab[3] : 0, l = sys_type == 0 ? lab[4] : lab[3];
      const double* v = V + (size_t)iR * G;
      double ir = 0.0, ii = 0.0;
      size_t g = 0;
      for (int i2 = 0; i2 < n_alpha2; ++i2)
        for (int i3 = 0; i3 < n_beta1; ++i3)
          for (int i4 = 0; i4 < n_beta2; ++i4)
            for (int i5 = 0; i5 < n_gamma1; ++i5)
              for (int i6 = 0; i6 < n_gamma2; ++i6, ++g) {
                const double beta = xbm + xbl * xb[i3], bbeta = xbm + xbl * xbb[i4];
                double wfr, wfi;
                orc_expansion_term(sys_type, l, l1, l2, nju1, nju2, beta, xg[i5], xaa[i2], bbeta,
                                   xgg[i6], &wfr, &wfi);
                const double w = wb[i3] * wg[i5] * sin(beta) * waa[i2] * wbb[i4] * wgg[i6] *
                                 sin(bbeta);
                ir += v[g] * wfr * w * tail;
                ii += v[g] * wfi * w * tail;
              }
      terms[(size_t)t * nR + iR] = ir;
      if (terms_im) terms_im[(size_t)t * nR + iR] = ii;
    }
  free(xb); free(wb); free(xbb); free(wbb); free(xg); free(wg); free(xgg); free(wgg);
  free(xaa); free(waa);
  return 0;
}

/* CALC_EXPANSION_TERMS for a rotor and an atom (SRC/pot_comp.f:4973-4999 SYS_TYPE 1,
 * 5054-5104 SYS_TYPE 4, 5000-5053 SYS_TYPE 3 = the loop of 4; EXPANSION_TERM :3756-3780):
 * V[iR][beta] (V_2_1) or V[iR][beta][gamma] (V_3_1), terms[t * nR + iR] the real part as
 * the reference sums it, terms_im the imaginary part. */
int orc_project_terms_atom(int sys_type, int n_terms, const int32_t* a_top, int n_beta,
                           int n_gamma, int eq_gamma, int nR, const double* V, double* terms,
                           double* terms_im) {
  if (sys_type == 3) sys_type = 4;
  if (sys_type != 1 && sys_type != 4) return -1;
  if (sys_type == 1) n_gamma = 1;
  double* xb = (double*)malloc(sizeof(double) * n_beta);
  double* wb = (double*)malloc(sizeof(double) * n_beta);
  double* xg = (double*)malloc(sizeof(double) * n_gamma);
  double* wg = (double*)malloc(sizeof(double) * n_gamma);
  orc_gauleg(n_beta, xb, wb);
  const double xbm = 0.5 * ORC_PI, xbl = 0.5 * ORC_PI, xgm = ORC_PI, xgl = ORC_PI;
  if (eq_gamma) {
    for (int i = 0; i < n_gamma; ++i) { xg[i] = (i + 0.5) * 2.0 * xgl / n_gamma; wg[i] = 2.0 / n_gamma; }
  } else {
    orc_gauleg(n_gamma, xg, wg);
    for (int i = 0; i < n_gamma; ++i) xg[i] = xgm + xgl * xg[i];
  }
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int t = 0; t < n_terms; ++t)
    for (int iR = 0; iR < nR; ++iR) {
      const int l = a_top[5 * t], nju = sys_type == 4 ? a_top[5 * t + 1] : 0;
      double ir = 0.0, ii = 0.0;
      for (int i2 = 0; i2 < n_beta; ++i2) {
        const double beta = xbm + xbl * xb[i2];
        if (sys_type == 1) {
          double wfr, wfi;
          orc_wf_diat(l, 0, beta, 0.0, &wfr, &wfi);
          const double v = V[(size_t)iR * n_beta + i2];
          ir += (wfr * v) * wb[i2] * sin(beta) * xbl * 2.0 * ORC_PI;
          ii += (wfi * v) * wb[i2] * sin(beta) * xbl * 2.0 * ORC_PI;
          continue;
        }
        for (int i3 = 0; i3 < n_gamma; ++i3) {
          double dwr, dwi;
          orc_wf_diat(l, nju, beta, xg[i3], &dwr, &dwi);
          const double sg = (nju % 2) ? -1.0 : 1.0;
          const double v = V[((size_t)iR * n_beta + i2) * n_gamma + i3];
          ir += dwr * sg * v * wb[i2] * wg[i3] * sin(beta) * xbl * xgl;
          ii += dwi * sg * v * wb[i2] * wg[i3] * sin(beta) * xbl * xgl;
        }
      }
      terms[(size_t)t * nR + iR] = ir;
      if (terms_im) terms_im[(size_t)t * nR + iR] = ii;
    }
  free(xb); free(wb); free(xg); free(wg);
  return 0;
}

