// host.cu -- host-side parts of the C ABI: error state, quadrature axes, rigid
// asymmetric-top levels, state/pair enumeration (INI_ARRAYS), the R grid and
// the MTRX_UF.DAT matrix file.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"

namespace mqct {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

void gauss_legendre(int n, double* x, double* w) {
  const double eps = 3.0e-15;
  int m = (n + 1) / 2;
  for (int i = 1; i <= m; ++i) {
    double z = cos(kPi * (i - 0.25) / (n + 0.5)), z1 = 0.0, pp = 0.0;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (fabs(z - z1) > eps);
    x[i - 1] = -z;
    x[n - i] = z;
    w[i - 1] = w[n - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

// Gauss-Legendre axis on [lo, hi]: nodes xm + xl*x, weights as on [-1,1]; the
// half-length xl multiplies the integral (MQCT_SOURCE_CODES/pot_comp.f:376-381).
Axis axis_gl(int n, double lo, double hi) {
  Axis a;
  a.x.resize(n);
  a.w.resize(n);
  gauss_legendre(n, a.x.data(), a.w.data());
  double xm = 0.5 * (hi + lo), xl = 0.5 * (hi - lo);
  for (int i = 0; i < n; ++i) a.x[i] = xm + xl * a.x[i];
  a.half = xl;
  return a;
}
// Midpoint-equidistant axis with weight 2/n (EQ_ANG_GRID,
// MQCT_SOURCE_CODES/pot_comp.f:601-611).
Axis axis_mid(int n, double lo, double hi) {
  Axis a;
  a.x.resize(n);
  a.w.assign(n, 2.0 / n);
  double xl = 0.5 * (hi - lo);
  for (int i = 1; i <= n; ++i) a.x[i - 1] = lo + (i - 0.50) * 2.0 * xl / n;
  a.half = xl;
  return a;
}

// Rigid-rotor Hamiltonian in the symmetric-top basis with z along c
// (MQCT_SOURCE_CODES/asym_top.f:103-137): diagonal (A+B)/2 J(J+1) +
// (C-(A+B)/2) K^2, K+-2 couplings (A-B)/4 sqrt(..)sqrt(..).
static double rotor_h(int j, int k1, int k2, double A, double B, double C) {
  if (k1 == k2) return 0.5 * (A + B) * j * (j + 1.0) + (C - 0.5 * (A + B)) * (double)(k1 * k1);
  if (k1 == k2 - 2 || k1 == k2 + 2) {
    int kav = (k1 + k2) / 2;
    return 0.5 * (A - B) * sqrt((j + 1.0) * j - kav * k1) * sqrt((j + 1.0) * j - kav * k2) / 2.0;
  }
  return 0.0;
}

// Threshold Jacobi diagonalisation of a small symmetric matrix (column-major a).
static void sym_eig(int n, std::vector<double>& a, std::vector<double>& w,
                    std::vector<double>& v) {
  v.assign(n * n, 0.0);
  for (int i = 0; i < n; ++i) v[i * n + i] = 1.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0, scale = 0.0;
    for (int c = 0; c < n; ++c)
      for (int r = 0; r < n; ++r) {
        double x = a[c * n + r] * a[c * n + r];
        if (r == c) scale += x;
        else off += x;
      }
    if (off <= 1e-30 * scale || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[q * n + p];
        if (apq == 0.0) continue;
        double tau = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          double xp = a[p * n + k], xq = a[q * n + k];
          a[p * n + k] = c * xp - s * xq;
          a[q * n + k] = s * xp + c * xq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          double xp = a[k * n + p], xq = a[k * n + q];
          a[k * n + p] = c * xp - s * xq;
          a[k * n + q] = s * xp + c * xq;
        }
        for (int k = 0; k < n; ++k) {
          double xp = v[p * n + k], xq = v[q * n + k];
          v[p * n + k] = c * xp - s * xq;
          v[q * n + k] = s * xp + c * xq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = a[i * n + i];
}

// Level (j, ka, kc) is eigenvalue number j + ka - kc in ascending order, the
// (Ka, Kc) labelling of MQCT_SOURCE_CODES/asym_top.f:139-173.  The eigenvector
// (components K=-j..j) is signed so its first non-negligible component is > 0.
int asym_top_level(double A, double B, double C, int j, int ka, int kc, double* energy,
                   double* vec) {
  if (j < 0 || ka < 0 || kc < 0 || ka > j || kc > j) return MQCT_E_ARG;
  if (ka + kc != j && ka + kc != j + 1) return MQCT_E_ARG;
  int pos = j + ka - kc;  // 0-based rank
  if (pos < 0 || pos > 2 * j || (pos + 1) / 2 != ka) return MQCT_E_ARG;
  int n = 2 * j + 1;
  std::vector<double> a(n * n), w, v;
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) a[c * n + r] = rotor_h(j, r - j, c - j, A, B, C);
  sym_eig(n, a, w, v);
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 1; i < n; ++i)
    for (int k = i; k > 0 && w[ord[k - 1]] > w[ord[k]]; --k) std::swap(ord[k - 1], ord[k]);
  int col = ord[pos];
  *energy = w[col];
  int first = -1;
  for (int k = 0; k < n; ++k) {
    vec[k] = v[col * n + k];
    if (first < 0 && fabs(vec[k]) > 1e-10) first = k;
  }
  if (first >= 0 && vec[first] < 0)
    for (int k = 0; k < n; ++k) vec[k] = -vec[k];
  return MQCT_OK;
}

}  // namespace mqct

using namespace mqct;

extern "C" {

const char* mqct_last_error(void) { return g_err.c_str(); }
int mqct_version(void) { return 10000; }
int mqct_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int mqct_asym_top_level(double A, double B, double C, int32_t j, int32_t ka, int32_t kc,
                        double* energy, double* vec) {
  int rc = asym_top_level(A, B, C, j, ka, kc, energy, vec);
  if (rc) set_error("invalid asymmetric-top level j=%d ka=%d kc=%d", j, ka, kc);
  return rc;
}

// States per channel: m = -j..j (types 1, 4) or j12 = |j1-j2|..j1+j2 with its m
// (types 5, 7, 8, 9, 0), channel-major; type 3 like 1 and 4 (MQCT_SOURCE_CODES/matrix_ini.f:148-173, 261-544).
int mqct_count_states(int32_t sys_type, int32_t n_channels, const int32_t* j1,
                      const int32_t* j2) {
  if (n_channels <= 0 || !j1) return MQCT_E_ARG;
  int st = 0;
  for (int i = 0; i < n_channels; ++i) {
    if (sys_type == 1 || sys_type == 3 || sys_type == 4) st += 2 * j1[i] + 1;
    else if (sys_type == 5 || sys_type == 7 || sys_type == 8 || sys_type == 9 || sys_type == 0) {
      if (!j2) return MQCT_E_ARG;
      for (int js = abs(j1[i] - j2[i]); js <= j1[i] + j2[i]; ++js) st += 2 * js + 1;
    } else {
      set_error("unsupported SYS_TYPE %d", sys_type);
      return MQCT_E_ARG;
    }
  }
  return st;
}

int mqct_enumerate_states(int32_t sys_type, int32_t n_channels, const int32_t* j1,
                          const int32_t* j2, int32_t* indx_chann, int32_t* j12, int32_t* m12) {
  int n = mqct_count_states(sys_type, n_channels, j1, j2);
  if (n < 0) return n;
  int st = 0;
  for (int i = 0; i < n_channels; ++i) {
    const bool one = sys_type == 1 || sys_type == 3 || sys_type == 4;
    int lo = one ? j1[i] : abs(j1[i] - j2[i]);
    int hi = one ? j1[i] : j1[i] + j2[i];
    for (int js = lo; js <= hi; ++js)
      for (int m = -js; m <= js; ++m) {
        indx_chann[st] = i + 1;
        j12[st] = js;
        m12[st] = m;
        ++st;
      }
  }
  return st;
}

// Identical partners: per channel p = 1 and, unless both rotors are in the same level,
// p = 2, each with all (j12, m12); parity (-1)^(p-1), -1 for odd j12 of a same-level
// channel (MQCT_SOURCE_CODES/matrix_ini.f:482-530).
static bool same_level(int c, const int32_t* j1, const int32_t* ka1, const int32_t* kc1,
                       const int32_t* j2, const int32_t* ka2, const int32_t* kc2) {
  return j1[c] == j2[c] && ka1[c] == ka2[c] && kc1[c] == kc2[c];
}
int mqct_count_states_identical(int32_t n_channels, const int32_t* j1, const int32_t* ka1,
                                const int32_t* kc1, const int32_t* j2, const int32_t* ka2,
                                const int32_t* kc2) {
  if (n_channels <= 0 || !j1 || !ka1 || !kc1 || !j2 || !ka2 || !kc2) return MQCT_E_ARG;
  int st = 0;
  for (int c = 0; c < n_channels; ++c) {
    const int np = same_level(c, j1, ka1, kc1, j2, ka2, kc2) ? 1 : 2;
    for (int js = abs(j1[c] - j2[c]); js <= j1[c] + j2[c]; ++js) st += np * (2 * js + 1);
  }
  return st;
}
int mqct_enumerate_states_identical(int32_t n_channels, const int32_t* j1, const int32_t* ka1,
                                    const int32_t* kc1, const int32_t* j2, const int32_t* ka2,
                                    const int32_t* kc2, int32_t* indx_chann, int32_t* j12,
                                    int32_t* m12, int32_t* parity) {
  const int n = mqct_count_states_identical(n_channels, j1, ka1, kc1, j2, ka2, kc2);
  if (n < 0) return n;
  if (!indx_chann || !j12 || !m12 || !parity) return MQCT_E_ARG;
  int st = 0;
  for (int c = 0; c < n_channels; ++c) {
    const bool same = same_level(c, j1, ka1, kc1, j2, ka2, kc2);
    for (int p = 1; p <= (same ? 1 : 2); ++p)
      for (int js = abs(j1[c] - j2[c]); js <= j1[c] + j2[c]; ++js)
        for (int m = -js; m <= js; ++m) {
          indx_chann[st] = c + 1;
          j12[st] = js;
          m12[st] = m;
          parity[st] = (same && (js & 1)) ? -1 : (p == 1 ? 1 : -1);
          ++st;
        }
  }
  return st;
}
int64_t mqct_count_pairs_identical(int32_t n, const int32_t* m12, const int32_t* parity) {
  if (n <= 0 || !m12 || !parity) return MQCT_E_ARG;
  int64_t p = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b <= a; ++b)
      if (m12[a] == m12[b] && parity[a] == parity[b]) ++p;
  return p;
}
int64_t mqct_fill_ind_mat_identical(int32_t n, const int32_t* m12, const int32_t* parity,
                                    int32_t* ind) {
  if (n <= 0 || !m12 || !parity || !ind) return MQCT_E_ARG;
  int64_t p = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b <= a; ++b)
      if (m12[a] == m12[b] && parity[a] == parity[b]) {
        ind[2 * p] = a + 1;
        ind[2 * p + 1] = b + 1;
        ++p;
      }
  return p;
}

// ind_mat: st1 outer, st2 <= st1, equal m12 (MQCT_SOURCE_CODES/matrix_ini.f:553-627).
int64_t mqct_count_pairs(int32_t n, const int32_t* m12) {
  if (n <= 0 || !m12) return MQCT_E_ARG;
  int mmax = 0;
  for (int s = 0; s < n; ++s) mmax = std::max(mmax, abs(m12[s]));
  std::vector<int64_t> cnt(2 * mmax + 1, 0);
  int64_t p = 0;
  for (int s = 0; s < n; ++s) p += ++cnt[m12[s] + mmax];
  return p;
}
int64_t mqct_fill_ind_mat(int32_t n, const int32_t* m12, int32_t* ind) {
  if (n <= 0 || !m12 || !ind) return MQCT_E_ARG;
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

// R grid: equidistant or the 3-segment "optimized" grid
// (MQCT_SOURCE_CODES/matrix_ini.f:954-981).
int mqct_r_grid(int32_t n, double rmin, double rmax, int32_t equidistant, double* R) {
  if (n < 2 || !(rmax > rmin) || !R) return MQCT_E_ARG;
  double dr = (rmax - rmin) / (n - 1.0);
  if (equidistant) {
    for (int i = 1; i <= n; ++i) R[i - 1] = rmin + dr * (i - 1.0);
    return MQCT_OK;
  }
  if (n < 3) {  // the third segment would divide by n - n2 = 0
    set_error("the optimized R grid needs at least 3 points");
    return MQCT_E_ARG;
  }
  int n1 = n / 3, n2 = n / 2 + 1;
  R[0] = rmin;
  R[n - 1] = rmax;
  for (int i = 1; i <= n1; ++i) R[i - 1] = rmin + dr * (i - 1.0) / 3.0;
  for (int i = n1 + 1; i <= n2; ++i) R[i - 1] = R[n1 - 1] + dr * (i - n1);
  dr = (rmax - R[n2 - 1]) / (n - n2);
  for (int i = n2; i <= n; ++i) R[i - 1] = R[n2 - 1] + dr * (i - n2);
  return MQCT_OK;
}

// ---------------------------------------------------------------- MTRX_UF.DAT
static bool put_rec(FILE* f, const void* d, int32_t nb) {
  return fwrite(&nb, 4, 1, f) == 1 && fwrite(d, 1, (size_t)nb, f) == (size_t)nb &&
         fwrite(&nb, 4, 1, f) == 1;
}
static bool get_rec(FILE* f, void* d, int32_t expect, int32_t* got = nullptr) {
  int32_t a = 0, b = 0;
  if (fread(&a, 4, 1, f) != 1) return false;
  if (got) *got = a;
  if (expect >= 0 && a != expect) return false;
  if (a < 0 || a > (1 << 30)) return false;
  if (d && fread(d, 1, (size_t)a, f) != (size_t)a) return false;
  if (!d && fseek(f, a, SEEK_CUR) != 0) return false;
  if (fread(&b, 4, 1, f) != 1 || b != a) return false;
  return true;
}

int mqct_write_mtrx_uf(const char* path, int32_t coll_type, int32_t n_channels,
                       int32_t n_states, const int32_t* state_rec, int32_t state_rec_len,
                       int64_t P, const int32_t* ind_mat, int32_t nR, const double* R,
                       const double* mat) {
  MQCT_ARG_CHECK(path && state_rec && ind_mat && R && mat && P > 0 && nR > 1 &&
                     P < (int64_t)1 << 31 && state_rec_len > 0,
                 "mqct_write_mtrx_uf: bad arguments");
  FILE* f = fopen(path, "wb");
  if (!f) {
    set_error("cannot open %s for writing", path);
    return MQCT_E_IO;
  }
  bool ok = true;
  int32_t hdr[5] = {coll_type, n_channels, n_states, (int32_t)P, nR};
  for (int i = 0; i < 5 && ok; ++i) ok = put_rec(f, &hdr[i], 4);
  for (int s = 0; s < n_states && ok; ++s)
    ok = put_rec(f, state_rec + (size_t)s * state_rec_len, 4 * state_rec_len);
  for (int64_t k = 0; k < P && ok; ++k) {
    int32_t t[3] = {(int32_t)(k + 1), ind_mat[2 * k], ind_mat[2 * k + 1]};
    ok = put_rec(f, t, 12);
  }
  for (int i = 0; i < nR && ok; ++i) {
    unsigned char b[12];
    int32_t ii = i + 1;
    memcpy(b, &ii, 4);
    memcpy(b + 4, &R[i], 8);
    ok = put_rec(f, b, 12);
  }
  for (int64_t k = 0; k < P && ok; ++k) {
    int32_t kk = (int32_t)(k + 1);
    ok = put_rec(f, &kk, 4) && put_rec(f, mat + (size_t)k * nR, 8 * nR);
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) {
    set_error("write error on %s", path);
    return MQCT_E_IO;
  }
  return MQCT_OK;
}

int mqct_read_mtrx_uf_header(const char* path, int32_t* coll_type, int32_t* n_channels,
                             int32_t* n_states, int64_t* P, int32_t* nR,
                             int32_t* state_rec_len) {
  MQCT_ARG_CHECK(path, "null path");
  FILE* f = fopen(path, "rb");
  if (!f) {
    set_error("cannot open %s", path);
    return MQCT_E_IO;
  }
  int32_t h[5];
  bool ok = true;
  for (int i = 0; i < 5 && ok; ++i) ok = get_rec(f, &h[i], 4);
  int32_t len = 0;
  if (ok && h[2] > 0) ok = get_rec(f, nullptr, -1, &len);
  fclose(f);
  if (!ok || h[2] <= 0 || h[3] <= 0 || h[4] <= 1 || len <= 0 || len % 4) {
    set_error("malformed MTRX_UF header in %s", path);
    return MQCT_E_IO;
  }
  *coll_type = h[0];
  *n_channels = h[1];
  *n_states = h[2];
  *P = h[3];
  *nR = h[4];
  *state_rec_len = len / 4;
  return MQCT_OK;
}

int mqct_read_mtrx_uf(const char* path, int32_t state_rec_len, int32_t* state_rec,
                      int32_t* ind_mat, double* R, double* mat) {
  int32_t ct, nch, ns, nR, srl;
  int64_t P;
  int rc = mqct_read_mtrx_uf_header(path, &ct, &nch, &ns, &P, &nR, &srl);
  if (rc) return rc;
  MQCT_ARG_CHECK(srl == state_rec_len && state_rec && ind_mat && R && mat,
                 "state record length %d != %d", srl, state_rec_len);
  FILE* f = fopen(path, "rb");
  if (!f) return MQCT_E_IO;
  bool ok = true;
  for (int i = 0; i < 5 && ok; ++i) ok = get_rec(f, nullptr, 4);
  for (int s = 0; s < ns && ok; ++s) ok = get_rec(f, state_rec + (size_t)s * srl, 4 * srl);
  for (int64_t k = 0; k < P && ok; ++k) {
    int32_t t[3];
    ok = get_rec(f, t, 12) && t[0] == k + 1 && t[1] >= 1 && t[1] <= ns && t[2] >= 1 &&
         t[2] <= ns;
    ind_mat[2 * k] = t[1];
    ind_mat[2 * k + 1] = t[2];
  }
  for (int i = 0; i < nR && ok; ++i) {
    unsigned char b[12];
    int32_t ii;
    ok = get_rec(f, b, 12);
    memcpy(&ii, b, 4);
    memcpy(&R[i], b + 4, 8);
    ok = ok && ii == i + 1;
  }
  for (int64_t k = 0; k < P && ok; ++k) {
    int32_t kk;
    ok = get_rec(f, &kk, 4) && kk == k + 1 && get_rec(f, mat + (size_t)k * nR, 8 * nR);
  }
  fclose(f);
  if (!ok) {
    set_error("malformed MTRX_UF body in %s", path);
    return MQCT_E_IO;
  }
  return MQCT_OK;
}

// ---------------------------------------------------------------- MTRX.DAT (formatted)
// The formatted matrix file of SAVE_MTRX / READ_MTRX with UNFORMAT = NO: PRINT_MIJ
// (MQCT_SOURCE_CODES/matrix_ini.f:4692-4877) writes five header counts, the state
// table, ind_mat, the R grid and one line (k, iR, Mij) per element; READ_MIJ reads it.

// Fortran Ew.d output (0.ddd...E+ee, or 0.ddd...+eee for |exponent| > 99), right
// justified in w columns; d significant digits, rounded to nearest.
static std::string fortran_e(double v, int w, int d) {
  char buf[64];
  std::string body;
  if (v == 0.0 || !std::isfinite(v)) {
    if (!std::isfinite(v)) {
      body = std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity");
    } else {
      body = "0.";
      body.append(d, '0');
      body += "E+00";
    }
  } else {
    // d significant digits in C's d.ddd form, then shifted into 0.dddd form
    snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(v));
    const char* e = strchr(buf, 'e');
    std::string digits;
    for (const char* c = buf; c < e; ++c)
      if (*c >= '0' && *c <= '9') digits += *c;
    const int ex = atoi(e + 1) + 1;
    body = std::string(v < 0 ? "-" : "") + "0." + digits;
    const int ax = ex < 0 ? -ex : ex;
    if (ax <= 99) snprintf(buf, sizeof buf, "E%c%02d", ex < 0 ? '-' : '+', ax);
    else snprintf(buf, sizeof buf, "%c%03d", ex < 0 ? '-' : '+', ax);
    body += buf;
  }
  if ((int)body.size() >= w) return body;
  return std::string(w - body.size(), ' ') + body;
}

// A Fortran real: also accepts the exponent form without the letter (0.1-100).
static bool parse_fortran_real(const char*& p, double* out) {
  while (*p == ' ' || *p == '\t') ++p;
  if (!*p || *p == '\n' || *p == '\r') return false;
  const char* start = p;
  while (*p && *p != ' ' && *p != '\t' && *p != '\n' && *p != '\r') ++p;
  std::string tok(start, p - start);
  for (auto& c : tok)
    if (c == 'D' || c == 'd') c = 'E';
  // a sign after the first digit without an exponent letter starts the exponent
  for (size_t i = 1; i < tok.size(); ++i)
    if ((tok[i] == '-' || tok[i] == '+') && tok[i - 1] != 'E' && tok[i - 1] != 'e') {
      tok.insert(i, "E");
      break;
    }
  char* end = nullptr;
  *out = strtod(tok.c_str(), &end);
  return end && *end == '\0';
}

static const char* const* mtrx_dat_columns(int coll_type, int* n) {
  static const char* c1[] = {"#STATE", "#CHANNEL", "J12", "M12", "J"};
  static const char* c3[] = {"#STATE", "#CHANNEL", "J12", "M12", "J", "K", "EPS"};
  static const char* c4[] = {"#STATE", "#CHANNEL", "J12", "M12", "J", "KA", "KC"};
  static const char* c5[] = {"#STATE", "#CHANNEL", "J12", "M12", "J1", "J2"};
  static const char* c7[] = {"#STATE", "#CHANNEL", "J12", "M12", "J1", "K", "EPS", "J2"};
  static const char* c8[] = {"#STATE", "#CHANNEL", "J12", "M12", "J1", "K1A", "K1C", "J2"};
  static const char* c9[] = {"#STATE", "#CHANNEL", "J12", "M12", "J1", "K1A", "K1C",
                             "J2", "K2", "EPS"};
  static const char* c0[] = {"#STATE", "#CHANNEL", "J12", "M12", "J1", "KA1", "KC1",
                             "J2", "KA2", "KC2", "P"};
  switch (coll_type) {
    case 1: *n = 5; return c1;
    case 3: *n = 7; return c3;
    case 4: *n = 7; return c4;
    case 5: *n = 6; return c5;
    case 7: *n = 8; return c7;
    case 8: *n = 8; return c8;
    case 9: *n = 10; return c9;
    case 0: *n = 10; return c0;  // 11 with the exchange parity of identical partners
    default: *n = 0; return nullptr;
  }
}

int mqct_write_mtrx_dat(const char* path, int32_t coll_type, int32_t n_channels,
                        int32_t n_states, const int32_t* state_rec, int32_t state_rec_len,
                        int64_t P, const int32_t* ind_mat, int32_t nR, const double* R,
                        const double* mat) {
  int ncol = 0;
  const char* const* cols = mtrx_dat_columns(coll_type, &ncol);
  MQCT_ARG_CHECK(cols, "mqct_write_mtrx_dat: SYS_TYPE %d not supported (1, 3, 4, 5, 7, 8, 9, 0)",
                 coll_type);
  MQCT_ARG_CHECK(path && state_rec && ind_mat && R && mat && P > 0 && nR > 1 && n_states > 0,
                 "mqct_write_mtrx_dat: bad arguments");
  if (coll_type == 0 && state_rec_len == 11) ncol = 11;  // identical partners: P column
  MQCT_ARG_CHECK(state_rec_len == ncol, "SYS_TYPE %d state records have %d columns (got %d)",
                 coll_type, ncol, state_rec_len);
  FILE* f = fopen(path, "w");
  if (!f) {
    set_error("cannot open %s for writing", path);
    return MQCT_E_IO;
  }
  fprintf(f, "COLLISION_TYPE= %1d\n", coll_type);
  fprintf(f, "NUMBER_OF_CHANLS=%5d\n", n_channels);
  fprintf(f, "NUMBER_OF_STATES= %6d\n", n_states);
  fprintf(f, "MATRIX_SIZE= %9lld\n", (long long)P);
  fprintf(f, "R_GRID_SIZE= %4d\n", nR);
  // the P column of identical partners is a2 / i2 (matrix_ini.f:4846-4857); SYS_TYPE 9
  // writes the columns after #CHANNEL as a3 / i3 (:4821-4832)
  auto width = [&](int c) { return c == 0 || c == 1 ? 8 : (c == 10 ? 2 : (coll_type == 9 ? 3 : 8)); };
  for (int c = 0; c < ncol; ++c) fprintf(f, c == 0 ? "%*s" : " %*s", width(c), cols[c]);
  fputc('\n', f);
  for (int st = 0; st < n_states; ++st) {
    for (int c = 0; c < ncol; ++c)
      fprintf(f, c == 0 ? "%*d" : " %*d", width(c), state_rec[(size_t)st * ncol + c]);
    fputc('\n', f);
  }
  fprintf(f, "%16s %8s %8s\n", "MIJ_INDEX", "ST_1", "ST_2");
  for (int64_t k = 0; k < P; ++k)
    fprintf(f, "%16lld %8d %8d\n", (long long)k + 1, ind_mat[2 * k], ind_mat[2 * k + 1]);
  fprintf(f, "%5s %19s\n", "#iR", "R_COM(iR)");
  for (int i = 0; i < nR; ++i) fprintf(f, "%5d %s\n", i + 1, fortran_e(R[i], 19, 12).c_str());
  fprintf(f, "%16s %8s %19s\n", "#k_matel", "#iR", "Mij(iR,k_matel)");
  for (int64_t k = 0; k < P; ++k)
    for (int i = 0; i < nR; ++i)
      fprintf(f, "%16lld %8d %s\n", (long long)k + 1, i + 1,
              fortran_e(mat[(size_t)k * nR + i], 19, 12).c_str());
  if (fclose(f) != 0) {
    set_error("write error on %s", path);
    return MQCT_E_IO;
  }
  return MQCT_OK;
}

static bool read_line(FILE* f, std::string& line) {
  line.clear();
  int c;
  while ((c = fgetc(f)) != EOF && c != '\n') line += (char)c;
  return !(c == EOF && line.empty());
}

static bool header_count(const std::string& line, const char* key, long long* v) {
  const size_t n = strlen(key);
  if (line.compare(0, n, key) != 0) return false;
  char* end = nullptr;
  *v = strtoll(line.c_str() + n, &end, 10);
  return end != line.c_str() + n;
}

int mqct_read_mtrx_dat_header(const char* path, int32_t* coll_type, int32_t* n_channels,
                              int32_t* n_states, int64_t* P, int32_t* nR,
                              int32_t* state_rec_len) {
  MQCT_ARG_CHECK(path && coll_type && n_channels && n_states && P && nR && state_rec_len,
                 "null argument");
  FILE* f = fopen(path, "r");
  if (!f) {
    set_error("cannot open %s", path);
    return MQCT_E_IO;
  }
  static const char* keys[5] = {"COLLISION_TYPE=", "NUMBER_OF_CHANLS=", "NUMBER_OF_STATES=",
                                "MATRIX_SIZE=", "R_GRID_SIZE="};
  long long h[5] = {0, 0, 0, 0, 0};
  std::string line;
  bool ok = true;
  for (int i = 0; i < 5 && ok; ++i) ok = read_line(f, line) && header_count(line, keys[i], &h[i]);
  int ncol = 0;
  if (ok && read_line(f, line)) {
    const char* p = line.c_str();
    while (*p) {
      while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
      if (!*p) break;
      ++ncol;
      while (*p && *p != ' ' && *p != '\t' && *p != '\r') ++p;
    }
  }
  fclose(f);
  if (!ok || h[2] <= 0 || h[3] <= 0 || h[3] >= ((long long)1 << 31) || h[4] <= 1 || ncol < 5) {
    set_error("malformed MTRX.DAT header in %s", path);
    return MQCT_E_IO;
  }
  *coll_type = (int32_t)h[0];
  *n_channels = (int32_t)h[1];
  *n_states = (int32_t)h[2];
  *P = h[3];
  *nR = (int32_t)h[4];
  *state_rec_len = ncol;
  return MQCT_OK;
}

int mqct_read_mtrx_dat(const char* path, int32_t state_rec_len, int32_t* state_rec,
                       int32_t* ind_mat, double* R, double* mat) {
  int32_t ct, nch, ns, nR, ncol;
  int64_t P;
  int rc = mqct_read_mtrx_dat_header(path, &ct, &nch, &ns, &P, &nR, &ncol);
  if (rc) return rc;
  MQCT_ARG_CHECK(state_rec && ind_mat && R && mat, "null argument");
  MQCT_ARG_CHECK(state_rec_len == ncol, "%s has %d state columns (caller expects %d)", path, ncol,
                 state_rec_len);
  FILE* f = fopen(path, "r");
  if (!f) {
    set_error("cannot open %s", path);
    return MQCT_E_IO;
  }
  std::string line;
  auto fail = [&](const char* what, long long at) {
    fclose(f);
    set_error("malformed MTRX.DAT %s (%s, entry %lld)", path, what, at);
    return MQCT_E_IO;
  };
  for (int i = 0; i < 6; ++i)
    if (!read_line(f, line)) return fail("header", i + 1);
  for (int s = 0; s < ns; ++s) {
    if (!read_line(f, line)) return fail("state table", s + 1);
    const char* p = line.c_str();
    for (int c = 0; c < ncol; ++c) {
      char* end = nullptr;
      const long v = strtol(p, &end, 10);
      if (end == p) return fail("state table", s + 1);
      state_rec[(size_t)s * ncol + c] = (int32_t)v;
      p = end;
    }
  }
  if (!read_line(f, line)) return fail("pair header", 0);
  for (int64_t k = 0; k < P; ++k) {
    long long kk;
    int a, b;
    if (!read_line(f, line) || sscanf(line.c_str(), "%lld %d %d", &kk, &a, &b) != 3 || kk != k + 1 ||
        a < 1 || a > ns || b < 1 || b > ns)
      return fail("ind_mat", k + 1);
    ind_mat[2 * k] = a;
    ind_mat[2 * k + 1] = b;
  }
  if (!read_line(f, line)) return fail("R header", 0);
  for (int i = 0; i < nR; ++i) {
    int ii;
    char* end = nullptr;
    if (!read_line(f, line)) return fail("R grid", i + 1);
    ii = (int)strtol(line.c_str(), &end, 10);
    const char* p = end;
    if (ii != i + 1 || !parse_fortran_real(p, &R[i])) return fail("R grid", i + 1);
  }
  if (!read_line(f, line)) return fail("element header", 0);
  std::vector<char> seen((size_t)P * nR, 0);
  for (int64_t q = 0; q < P * (int64_t)nR; ++q) {
    if (!read_line(f, line)) return fail("elements", q + 1);
    char* end = nullptr;
    const long long kk = strtoll(line.c_str(), &end, 10);
    const char* p = end;
    const long ii = strtol(p, &end, 10);
    p = end;
    double v;
    if (kk < 1 || kk > P || ii < 1 || ii > nR || !parse_fortran_real(p, &v))
      return fail("elements", q + 1);
    const size_t at = (size_t)(kk - 1) * nR + (ii - 1);
    if (seen[at]) return fail("repeated element", q + 1);
    seen[at] = 1;
    mat[at] = v;
  }
  fclose(f);
  return MQCT_OK;
}

// ---------------------------------------------------------------- PES_EXPAN_TERMS.DAT
// READ_EXPANSION_TERMS (MQCT_SOURCE_CODES/pot_comp.f:6344-6388): one header line, then
// per R point the value of R and the nterms expansion coefficients.  Output in the
// reference's layout: R[iR], terms[t * nR + iR] (expansion_terms(n_r_coll, nterms)).
int mqct_read_expansion_terms(const char* path, int32_t nR, int32_t n_terms, double* R,
                              double* terms) {
  MQCT_ARG_CHECK(path && R && terms && nR > 0 && n_terms > 0, "bad arguments");
  FILE* f = fopen(path, "r");
  if (!f) {
    set_error("cannot open %s", path);
    return MQCT_E_IO;
  }
  std::string line;
  if (!read_line(f, line)) {  // header
    fclose(f);
    set_error("%s is empty", path);
    return MQCT_E_IO;
  }
  for (int i = 0; i < nR; ++i) {
    bool ok = read_line(f, line);
    const char* p = line.c_str();
    ok = ok && parse_fortran_real(p, &R[i]);
    for (int t = 0; t < n_terms && ok; ++t) ok = parse_fortran_real(p, &terms[(size_t)t * nR + i]);
    if (!ok) {
      fclose(f);
      set_error("%s: R point %d has fewer than %d terms (or is missing)", path, i + 1, n_terms);
      return MQCT_E_IO;
    }
  }
  fclose(f);
  return MQCT_OK;
}

// The writer of CALC_EXPANSION_TERMS (MQCT_SOURCE_CODES/pot_comp.f:5918-6270): appends
// to the file; the header line ("R_Bohr" then one a19 label v_l1_nju1_l2_l, or
// v_l1_nju1_l2_nju2_l for SYS_TYPE 0 and 9, per term, 3 blanks after each) only when the file
// holds at most one line, then per R point f6.2, 1x and e19.12 with 3 blanks per term.
int mqct_write_expansion_terms(const char* path, int32_t sys_type, int32_t n_terms,
                               const int32_t* a_top, int32_t nR, const double* R,
                               const double* terms) {
  MQCT_ARG_CHECK(path && a_top && R && terms && nR > 0 && n_terms > 0, "bad arguments");
  MQCT_ARG_CHECK(sys_type == 7 || sys_type == 8 || sys_type == 9 || sys_type == 0,
                 "PES_EXPAN_TERMS.DAT is written here for SYS_TYPE 7, 8, 9 and 0");
  int lines = 0;
  if (FILE* in = fopen(path, "r")) {
    std::string line;
    while (read_line(in, line)) ++lines;
    fclose(in);
  }
  FILE* f = fopen(path, "a");
  if (!f) {
    set_error("cannot open %s", path);
    return MQCT_E_IO;
  }
  if (lines <= 1) {
    for (int t = 0; t < n_terms; ++t) {
      const int32_t* q = a_top + 5 * t;
      char lab[96];
      if (sys_type == 0 || sys_type == 9)  // :6191-6214 as case 0
        snprintf(lab, sizeof lab, "v_%d_%d_%d_%d_%d", q[0], q[1], q[2], q[3], q[4]);
      else snprintf(lab, sizeof lab, "v_%d_%d_%d_%d", q[0], q[1], q[2], q[3]);
      lab[19] = 0;  // a19 keeps the leftmost 19 characters
      if (t == 0) fprintf(f, "%-6s ", "R_Bohr");
      fprintf(f, "%19s   ", lab);
    }
    fprintf(f, "\n");
  }
  for (int i = 0; i < nR; ++i) {
    fprintf(f, "%6.2f ", R[i]);
    for (int t = 0; t < n_terms; ++t)
      fprintf(f, "%s   ", fortran_e(terms[(size_t)t * nR + i], 19, 12).c_str());
    fprintf(f, "\n");
  }
  if (fclose(f) != 0) {
    set_error("write to %s failed", path);
    return MQCT_E_IO;
  }
  return MQCT_OK;
}

// ---------------------------------------------------------------- result files
// The reference's per-energy output files (MQCT_SOURCE_CODES/propagator.f:4843-4880,
// 5830-5896; print_output.f:46-101), appended block by block as the reference appends.
static FILE* open_append(const char* path) {
  FILE* f = fopen(path, "a");
  if (!f) set_error("cannot open %s", path);
  return f;
}

static int close_checked(FILE* f, const char* path) {
  if (fclose(f) != 0) {
    set_error("write to %s failed", path);
    return MQCT_E_IO;
  }
  return MQCT_OK;
}

// Fortran F0.3 of a value >= 0 as gfortran writes it.
static std::string fortran_f0_3(double v) {
  char buf[64];
  snprintf(buf, sizeof buf, "%.3f", v);
  return buf;
}

static void state_header(FILE* f, int32_t s_st, int32_t j12, int32_t m12, int32_t i_ener,
                         double U_cm) {
  fprintf(f, "STATE= %d\nj12= %d\nm12= %d\nENERGY#%d, U(i)= %s cm^-1\n", s_st, j12, m12, i_ener,
          fortran_f0_3(U_cm).c_str());
}

// OPACITY_FUNCTIONS_L.out and TOTAL_PROBABILITIES_L.out (propagator.f:5837-5896): per
// trajectory l / k, l and the channel probabilities; the totals file (path_total may be
// NULL) the sum and the sum without the initial channel (chann_ini, 1-based).
int mqct_write_opacity(const char* path, const char* path_total, int32_t s_st, int32_t j12,
                       int32_t m12, int32_t i_ener, double U_cm, int32_t n_traj, const int32_t* l,
                       double k_vec, int32_t n_ch, const double* prob, int32_t chann_ini) {
  MQCT_ARG_CHECK(path && l && prob && n_traj > 0 && n_ch > 0 && k_vec > 0.0, "bad arguments");
  MQCT_ARG_CHECK(!path_total || (chann_ini >= 1 && chann_ini <= n_ch), "chann_ini out of range");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  state_header(f, s_st, j12, m12, i_ener, U_cm);
  for (int c = 1; c <= n_ch; ++c) {
    if (c == 1) fprintf(f, "    %-8s   %-7s  ", "B_IMPACT", "     L ");
    fprintf(f, "CHANNEL=%6d  ", c);
  }
  fprintf(f, "\n");
  for (int t = 0; t < n_traj; ++t) {
    fprintf(f, "%s %6d ", fortran_e(l[t] / k_vec, 15, 8).c_str(), l[t]);
    for (int c = 0; c < n_ch; ++c)
      fprintf(f, "%s ", fortran_e(prob[(size_t)t * n_ch + c], 15, 8).c_str());
    fprintf(f, "\n");
  }
  fprintf(f, " \n");
  int rc = close_checked(f, path);
  if (rc || !path_total) return rc;
  f = open_append(path_total);
  if (!f) return MQCT_E_IO;
  state_header(f, s_st, j12, m12, i_ener, U_cm);
  fprintf(f, "B_IMPACT       %-7s %15s %16s\n", "     L ", "TOT_ELAST_PROB", "TOT_INELAST_PROB");
  for (int t = 0; t < n_traj; ++t) {
    double sum = 0.0;
    for (int c = 0; c < n_ch; ++c) sum += prob[(size_t)t * n_ch + c];
    fprintf(f, "%s %6d %s %s\n", fortran_e(l[t] / k_vec, 15, 8).c_str(), l[t],
            fortran_e(sum, 15, 8).c_str(),
            fortran_e(sum - prob[(size_t)t * n_ch + chann_ini - 1], 15, 8).c_str());
  }
  fprintf(f, " \n");
  return close_checked(f, path_total);
}

// DEFLECTION_FUNCTION.out (ELAST_CALC, propagator.f:5897-5928): per trajectory l, l / k,
// the deflection angle and scattering phase (rad), the finish time (a.u.), the energy and
// norm errors (percent), the orbiting periods and the oscillations of R.
int mqct_write_deflection(const char* path, int32_t s_st, int32_t j12, int32_t m12,
                          int32_t i_ener, double U_cm, int32_t n_traj, const int32_t* l,
                          double k_vec, const double* deflection, const double* phase,
                          const double* finish_time, const double* e_err_pct,
                          const double* p_err_pct, const int32_t* periods,
                          const int32_t* oscillations) {
  MQCT_ARG_CHECK(path && l && deflection && phase && finish_time && e_err_pct && p_err_pct &&
                     periods && oscillations && n_traj > 0 && k_vec > 0.0,
                 "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  fprintf(f, "energy#%d, (U= %s cm^-1)\nstate= %d\nj12= %d\nm12= %d\n", i_ener,
          fortran_f0_3(U_cm).c_str(), s_st, j12, m12);
  fprintf(f, "%5s  %14s     %17s    %15s       %17s    %15s      %13s    %5s   %5s\n", "L_ORB",
          "B_IMPACT(a.u.)", "DEFLCT_ANGLE(rad)", "SCAT_PHASE(rad)", "FINISH_TIME(a.u.)",
          "ENERGY_ERROR(%)", "NORM_ERROR(%)", "LOOPS", "OSCIL");
  for (int t = 0; t < n_traj; ++t)
    fprintf(f, "%4d  %s %s  %s   %s %s %s   %5d   %5d\n", l[t],
            fortran_e(l[t] / k_vec, 15, 8).c_str(), fortran_e(deflection[t], 19, 8).c_str(),
            fortran_e(phase[t], 19, 8).c_str(), fortran_e(finish_time[t], 19, 8).c_str(),
            fortran_e(e_err_pct[t], 19, 8).c_str(), fortran_e(p_err_pct[t], 19, 8).c_str(),
            periods[t], oscillations[t]);
  fprintf(f, " \n");
  return close_checked(f, path);
}

// DIFF_CROSS.out (ELAST_CALC with DIFF_CROSS = YES, propagator.f:5931-5943): the angle
// in degrees and the elastic differential cross section in Angstrom^2 (list-directed
// header records as gfortran writes them).
int mqct_write_diff_cross(const char* path, int32_t i_ener, int32_t s_st, int32_t j12,
                          int32_t m12, int32_t n_angles, const double* theta_rad,
                          const double* dcs) {
  MQCT_ARG_CHECK(path && theta_rad && dcs && n_angles > 0, "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  fprintf(f, " energy %11d\n state =  %11d\n j12= %11d\n m12= %11d\n", i_ener, s_st, j12, m12);
  fprintf(f, "%19s %19s\n", "ANGLE,deg", "DIFF. CROSS.,angs^2");
  for (int k = 0; k < n_angles; ++k)
    fprintf(f, "%s %s\n", fortran_e(theta_rad[k] * 180.0 / kPi, 19, 7).c_str(),
            fortran_e(dcs[k], 19, 7).c_str());
  fprintf(f, " \n");
  return close_checked(f, path);
}

// SPLINED_DEFLECTION_OPACITY_L.out (ELAST_CALC with PROB_SPLINE, propagator.f:6063-6110):
// per integer l the impact parameter l / k, l, the splined deflection function and the
// splined channel probabilities.
int mqct_write_splined_opacity(const char* path, int32_t n_l, const int32_t* l, double k_vec,
                               const double* deflection, int32_t n_ch, const double* prob) {
  MQCT_ARG_CHECK(path && l && deflection && prob && n_l > 0 && n_ch > 0 && k_vec > 0.0,
                 "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  for (int c = 1; c <= n_ch; ++c) {
    if (c == 1) fprintf(f, "%-8s       %-7s     %-12s  ", "B_IMPACT", "     L ", "DEF_FUNCTION");
    fprintf(f, "CHANNEL=%6d  ", c);
  }
  fprintf(f, "\n");
  for (int i = 0; i < n_l; ++i) {
    fprintf(f, "%s %6d %12.4f     ", fortran_e(l[i] / k_vec, 15, 8).c_str(), l[i], deflection[i]);
    for (int c = 0; c < n_ch; ++c)
      fprintf(f, "%s ", fortran_e(prob[(size_t)i * n_ch + c], 15, 8).c_str());
    fprintf(f, "\n");
  }
  fprintf(f, " \n");
  return close_checked(f, path);
}

// PARTIAL_CROSS_SECTIONS_J.out (propagator.f:4845-4868): per total J the J-resolved
// cross sections of every channel, Angstrom^2.
int mqct_write_partial_j(const char* path, int32_t s_st, int32_t j12, int32_t m12,
                         int32_t i_ener, double U_cm, int32_t n_J, const int32_t* J, int32_t n_ch,
                         const double* partial) {
  MQCT_ARG_CHECK(path && J && partial && n_J > 0 && n_ch > 0, "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  state_header(f, s_st, j12, m12, i_ener, U_cm);
  for (int c = 1; c <= n_ch; ++c) {
    if (c == 1) fprintf(f, "%-7s  ", "J_TOTAL");
    fprintf(f, "CHANNEL=%6d  ", c);
  }
  fprintf(f, "\n");
  for (int i = 0; i < n_J; ++i) {
    fprintf(f, "%5d   ", J[i]);
    for (int c = 0; c < n_ch; ++c)
      fprintf(f, "%s ", fortran_e(partial[(size_t)i * n_ch + c], 15, 8).c_str());
    fprintf(f, "\n");
  }
  return close_checked(f, path);
}

// M_PROJ_CROSSECTIONS.out (propagator.f:4870-4880): the cross sections of one initial
// state without the Billing correction, Angstrom^2.
int mqct_write_m_proj(const char* path, int32_t s_st, int32_t i_ener, int32_t j12, int32_t m12,
                      int32_t n_ch, const double* sigma) {
  MQCT_ARG_CHECK(path && sigma && n_ch > 0, "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  fprintf(f, " M RESOLVED CROSSECTIONS WITHOUT BILLING CORRECTION\n");
  fprintf(f, "%10s %4d\n%10s %4d\n", "INI_STATE#", s_st, "ENERGY#", i_ener);
  fprintf(f, " j12=%12d\n m12=%12d\n", j12, m12);
  fprintf(f, "%-8s %19s\n", "CHANNEL#", "CROSSSECTIONS,ANG^2");
  for (int c = 0; c < n_ch; ++c) fprintf(f, "%4d      %s\n", c + 1, fortran_e(sigma[c], 18, 11).c_str());
  return close_checked(f, path);
}

// One energy block of CROSS_SECTIONS.out (print_output.f:46-101): per final channel with
// a Billing energy (exists[c] != 0, or every channel when exists is NULL) the initial and
// final channel, sigma(U) = sigma_f / U * E_bill, E_bill and sigma_f (Angstrom^2, cm^-1);
// then the probability conservation error and, when with_e_err, the energy conservation
// error (percent), and a blank record.  mqct_write_cross_sections_footer appends the
// closing trajectory count.
int mqct_write_cross_sections(const char* path, double U_cm, int32_t chann_ini, int32_t n_ch,
                              const int32_t* exists, const double* sigma_f, const double* E_bill,
                              double p_err_pct, int32_t with_e_err, double e_err_pct) {
  MQCT_ARG_CHECK(path && sigma_f && E_bill && n_ch > 0 && U_cm > 0.0, "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  fprintf(f, "U= %14.6f cm^-1\n", U_cm);
  fprintf(f, "%6s  %6s  %19s  %14s  %19s\n", "ilv", "flv", "sigma(U),ANG^2", "E_coll,cm^-1",
          "sigma(E_coll),ANG^2");
  for (int c = 0; c < n_ch; ++c) {
    if (exists && !exists[c]) continue;
    fprintf(f, "%6d  %6d  %s  %14.6f  %s\n", chann_ini, c + 1,
            fortran_e(sigma_f[c] / U_cm * E_bill[c], 19, 10).c_str(), E_bill[c],
            fortran_e(sigma_f[c], 19, 10).c_str());
  }
  fprintf(f, "%-28s %s\n", "TOTAL P CONSERVATION ERROR,%", fortran_e(p_err_pct, 12, 5).c_str());
  if (with_e_err)
    fprintf(f, "%-28s %s\n", "TOTAL E CONSERVATION ERROR,%", fortran_e(e_err_pct, 12, 5).c_str());
  fprintf(f, " \n");
  return close_checked(f, path);
}

int mqct_write_cross_sections_footer(const char* path, int32_t n_traj_total) {
  MQCT_ARG_CHECK(path, "bad arguments");
  FILE* f = open_append(path);
  if (!f) return MQCT_E_IO;
  fprintf(f, "TOTAL NUMBER OF TRAJECTORIES = %3d\n", n_traj_total);
  return close_checked(f, path);
}

}  // extern "C"
