// pes.cuh -- device evaluation of the built-in potential energy surfaces (the
// stand-ins for the USER_DEFINED_PES plugin the reference links from
// PES_DIRECTORIES, called through MQCT_SOURCE_CODES/pes_sys_type.f:2-97), shared by
// the matrix build and the surrogate.  Values in cm^-1, R in bohr.
#pragma once
#include "common.cuh"

namespace mqct {

struct PesDev {
  int kind, n_terms, n_sites1, n_sites2;
  const double* p;
  const double* s1;
  const double* s2;
  const double* table;
};

__device__ inline double site_term(double r, const double* t) {
  double D = t[0], a = t[1], re = t[2], c6 = t[3], rd = t[4];
  double e = exp(-a * (r - re));
  double r2 = r * r, r6 = r2 * r2 * r2;
  double x = r / rd, x2 = x * x, x6 = x2 * x2 * x2;
  return D * (e * e - 2.0 * e) - c6 * (1.0 - exp(-x6)) / r6;
}

// Rotation Rz(a) Ry(b) Rz(g) applied to a site position.
__device__ inline void euler_apply(double a, double b, double g, const double* s, double* x) {
  double ca, sa, cb, sb, cg, sg;
  sincos(a, &sa, &ca);
  sincos(b, &sb, &cb);
  sincos(g, &sg, &cg);
  const double m00 = ca * cb * cg - sa * sg, m01 = -ca * cb * sg - sa * cg, m02 = ca * sb;
  const double m10 = sa * cb * cg + ca * sg, m11 = -sa * cb * sg + ca * cg, m12 = sa * sb;
  const double m20 = -sb * cg, m21 = sb * sg, m22 = cb;
  x[0] = m00 * s[0] + m01 * s[1] + m02 * s[2];
  x[1] = m10 * s[0] + m11 * s[1] + m12 * s[2];
  x[2] = m20 * s[0] + m21 * s[1] + m22 * s[2];
}

// SITES2 family for two rigid rotors: rotor 1 at the origin with Euler angles
// (alpha, beta, gamma), rotor 2 at R z with (aalpha, bbeta, ggamma); per term
// [site1, site2, D, a, re, C6, rd].
__device__ inline double pes_eval_sites2(const PesDev& P, double R, double alpha, double beta,
                                         double gamma, double aalpha, double bbeta, double ggamma) {
  double v = 0.0;
  for (int t = 0; t < P.n_terms; ++t) {
    const double* q = P.p + 7 * t;
    double x1[3], x2[3];
    euler_apply(alpha, beta, gamma, P.s1 + 3 * (int)q[0], x1);
    euler_apply(aalpha, bbeta, ggamma, P.s2 + 3 * (int)q[1], x2);
    x2[2] += R;
    const double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
    v += site_term(sqrt(dx * dx + dy * dy + dz * dz), q + 2);
  }
  return v;
}

// USER_DEFINED_PES(V,R,..,alpha,beta,gamma,..) for the built-in families.
__device__ inline double pes_eval(const PesDev& P, double R, double beta, double gamma) {
  if (P.kind == MQCT_PES_LEGENDRE) {
    double x = cos(beta), v = 0.0;
    double r2 = R * R, r6 = r2 * r2 * r2;
    int n = P.n_terms;
    // P_l(x) by Bonnet's recurrence
    double pm = 1.0, pc = x;
    for (int l = 0; l < n; ++l) {
      double pl;
      if (l == 0) pl = 1.0;
      else if (l == 1) pl = x;
      else {
        pl = ((2.0 * l - 1.0) * x * pc - (l - 1.0) * pm) / l;
        pm = pc;
        pc = pl;
      }
      v += (P.p[l] * exp(-P.p[n + l] * R) - P.p[2 * n + l] / r6) * pl;
    }
    return v;
  }
  if (P.kind == MQCT_PES_SITES1) {
    double sb, cb, sg, cg;
    sincos(beta, &sb, &cb);
    sincos(gamma, &sg, &cg);
    double ax = R * sb * cg, ay = R * sb * sg, az = R * cb, v = 0.0;
    for (int t = 0; t < P.n_terms; ++t) {
      const double* q = P.p + 6 * t;
      const double* s = P.s1 + 3 * (int)q[0];
      double dx = ax - s[0], dy = ay - s[1], dz = az - s[2];
      v += site_term(sqrt(dx * dx + dy * dy + dz * dz), q + 1);
    }
    return v;
  }
  return nan("");
}

}  // namespace mqct

namespace mqct {

// V at the reference's PES arguments of each system type
// (MQCT_SOURCE_CODES/pes_sys_type.f): type 1 (R, beta) :2-9, type 4 (R, -beta,
// -gamma) :32-37, type 0 (R, 0, beta1, gamma1, alpha2, beta2, gamma2) :90-97.
// ang = (beta1, gamma1, alpha2, beta2, gamma2); TABLE surfaces are not evaluable here.
__device__ inline double pes_at(int sys_type, const PesDev& P, double R, const double* ang) {
  if (sys_type == 1) return pes_eval(P, R, ang[0], 0.0);
  if (sys_type == 4) return pes_eval(P, R, -ang[0], -ang[1]);
  return pes_eval_sites2(P, R, 0.0, ang[0], ang[1], ang[2], ang[3], ang[4]);
}

}  // namespace mqct
