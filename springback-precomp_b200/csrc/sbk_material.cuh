// Device material point: the J2 radial return, the general (Hill48 /
// Chaboche) closest-point return with its consistent tangent, and the
// logarithmic strain with its first and second derivatives, written for one
// thread per integration point with every small matrix in registers.
//
// Algorithms (the reference's, restated for the GPU):
//   return_3d           src/material/Plasticity.cpp:66-171
//   return_general_3d   src/material/Plasticity.cpp:178-471
//   hardening           src/material/Material.cpp:73-90
//   logarithmic strain  src/material/LogarithmicStrain.cpp:24-197
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "sbk_params.h"

namespace sbk {

constexpr double kEps = 2.220446049250313e-16;

// How the closest-point return's helpers (the residual evaluation, the
// consistent tangent, the backstress decay) are compiled: as calls (one
// copy of their code for every caller) unless a translation unit asks for
// them inlined.
#ifndef SBK_RETURN_HELPER
#define SBK_RETURN_HELPER __noinline__
#endif

// Point-failure codes (sbk_element_code).
constexpr int kFailInverted = SBK_EL_INVERTED_POINT;
constexpr int kFailReturn = SBK_EL_RETURN_NO_CONVERGE;
constexpr int kFailNonFinite = SBK_EL_NONFINITE;
constexpr int kFailDegenerate = SBK_EL_DEGENERATE;

__device__ __forceinline__ double yield_of(const Params& p, double a) {
  return p.sy0 + p.H * a + p.Q * -expm1(-p.delta * a);
}
__device__ __forceinline__ double yield_slope_of(const Params& p, double a) {
  return p.H + p.Q * p.delta * exp(-p.delta * a);
}
__device__ __forceinline__ double isotropic_energy_of(const Params& p, double a) {
  double out = 0.5 * p.H * a * a;
  if (p.Q != 0.0) out += p.Q * (a + expm1(-p.delta * a) / p.delta);
  return out;
}

__device__ __forceinline__ double tnorm(const double v[6]) {
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + 2.0 * (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]));
}
__device__ __forceinline__ double dev_norm2(const double e[6]) {
  const double mean = (e[0] + e[1] + e[2]) / 3.0;
  double out = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) out += (e[i] - mean) * (e[i] - mean);
#pragma unroll
  for (int i = 3; i < 6; ++i) out += 0.5 * e[i] * e[i];
  return out;
}

// Accessor of one point's state: field f at base[f * stride].
struct PointState {
  const double* in;
  double* out;
  int64_t stride;
  __device__ __forceinline__ double get(int f) const { return in[f * stride]; }
  __device__ __forceinline__ void put(int f, double v) const { out[f * stride] = v; }
};

struct Response {
  double stress[6];
  double C[36];  // d sigma / d eps, row-major
  double energy;
  bool yielding;
};

__device__ __forceinline__ void elastic_C(const Params& p, double C[36]) {
#pragma unroll
  for (int i = 0; i < 36; ++i) C[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) C[i * 6 + j] = p.K - 2.0 * p.G / 3.0;
    C[i * 6 + i] = p.K + 4.0 * p.G / 3.0;
    C[(3 + i) * 6 + 3 + i] = p.G;
  }
}

// ---------------------------------------------------------------------------
// J2 radial return (Plasticity.cpp:66-171). Returns 0 or a failure code;
// writes the updated state through `st`.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int radial_return(const Params& p, const double strain[6], const PointState& st,
                                          Response& out) {
  const double g = p.G, k = p.K, hk = p.Hkin;
  double ep[6], el[6], s[6], xi[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    ep[i] = st.get(kFieldEp + i);
    el[i] = strain[i] - ep[i];
  }
  const double vol = el[0] + el[1] + el[2];
  {
    const double mean = vol / 3.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] = 2.0 * g * (el[i] - mean);
#pragma unroll
    for (int i = 3; i < 6; ++i) s[i] = g * el[i];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) xi[i] = s[i] - st.get(kFieldBeta + i);
  const double xi_norm = tnorm(xi);
  const double a_n = st.get(field_eqps(0));
  const bool loading_n = st.get(field_loading(0)) != 0.0;
  const double sq23 = 0.816496580927726;  // sqrt(2/3)
  const double radius_n = sq23 * yield_of(p, a_n);
  const double f_trial = xi_norm - radius_n;
  // Prager energy of the committed plastic strain.
  auto prager = [&](const double* e) {
    double o = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) o += e[i] * e[i];
#pragma unroll
    for (int i = 3; i < 6; ++i) o += 0.5 * e[i] * e[i];
    return hk / 3.0 * o;
  };
  if (!p.enabled || f_trial <= 1.0e-12 * radius_n) {
#pragma unroll
    for (int i = 0; i < 6; ++i) out.stress[i] = s[i] + (i < 3 ? k * vol : 0.0);
    elastic_C(p, out.C);
    out.energy = 0.5 * k * vol * vol + g * dev_norm2(el) + isotropic_energy_of(p, a_n) + prager(ep);
    out.yielding = false;
    bool loading = false;
    if (p.enabled && loading_n && f_trial > -1.0e-10 * radius_n && xi_norm > 0.0) {
      const double f = 2.0 * g / (1.0 + (yield_slope_of(p, a_n) + hk) / (3.0 * g));
      double n[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) n[i] = xi[i] / xi_norm;
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) out.C[i * 6 + j] -= f * (n[i] * n[j]);
      loading = true;
    }
    // The state is the committed one, with the loading flag.
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      st.put(kFieldEp + i, ep[i]);
      st.put(kFieldBeta + i, st.get(kFieldBeta + i));
    }
    st.put(field_eqps(0), a_n);
    st.put(field_loading(0), loading ? 1.0 : 0.0);
    return 0;
  }
  const double stiff = 2.0 * g + 2.0 / 3.0 * hk;
  double dgamma = f_trial / (stiff + 2.0 / 3.0 * yield_slope_of(p, a_n));
  if (p.Q != 0.0) {
    dgamma = 0.0;
    bool converged = false;
    for (int it = 0; it < 60; ++it) {
      const double a = a_n + sq23 * dgamma;
      const double res = xi_norm - stiff * dgamma - sq23 * yield_of(p, a);
      if (fabs(res) <= 1.0e-13 * radius_n) {
        converged = true;
        break;
      }
      dgamma += res / (stiff + 2.0 / 3.0 * yield_slope_of(p, a));
    }
    if (!converged) {
      const double a = a_n + sq23 * dgamma;
      const double res = xi_norm - stiff * dgamma - sq23 * yield_of(p, a);
      converged = fabs(res) <= 8.0 * kEps * xi_norm;
    }
    if (!converged) return kFailReturn;
  }
  const double a = a_n + sq23 * dgamma;
  double n[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) n[i] = xi[i] / xi_norm;
  out.yielding = true;
#pragma unroll
  for (int i = 0; i < 6; ++i) out.stress[i] = s[i] - 2.0 * g * dgamma * n[i] + (i < 3 ? k * vol : 0.0);
  const double theta = 1.0 - 2.0 * g * dgamma / xi_norm;
  const double theta_bar = 1.0 / (1.0 + (yield_slope_of(p, a) + hk) / (3.0 * g)) - (1.0 - theta);
#pragma unroll
  for (int i = 0; i < 36; ++i) out.C[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) out.C[i * 6 + j] = k - 2.0 * g * theta / 3.0;
    out.C[i * 6 + i] = k + 4.0 * g * theta / 3.0;
    out.C[(3 + i) * 6 + 3 + i] = g * theta;
  }
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) out.C[i * 6 + j] -= 2.0 * g * theta_bar * (n[i] * n[j]);
  double ep_new[6], el_new[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double f = i < 3 ? 1.0 : 2.0;  // engineering shear
    ep_new[i] = ep[i] + f * dgamma * n[i];
    el_new[i] = el[i] - f * dgamma * n[i];
  }
  out.energy = 0.5 * k * vol * vol + g * dev_norm2(el_new) + isotropic_energy_of(p, a) + prager(ep_new);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    st.put(kFieldEp + i, ep_new[i]);
    st.put(kFieldBeta + i, st.get(kFieldBeta + i) + 2.0 / 3.0 * hk * dgamma * n[i]);
  }
  st.put(field_eqps(0), a);
  st.put(field_loading(0), 1.0);
  return 0;
}

// ---------------------------------------------------------------------------
// General return (Plasticity.cpp:178-471).
// ---------------------------------------------------------------------------
struct Decay {
  double theta, chi, dtheta, dchi;
};
static __device__ SBK_RETURN_HELPER Decay decay_of(double gamma, double dl, int integration) {
  Decay d{1.0, 0.0, 0.0, 1.0};
  if (gamma == 0.0) {
    d.chi = dl;
    return d;
  }
  if (integration == 0) {
    d.theta = exp(-gamma * dl);
    d.chi = -expm1(-gamma * dl) / gamma;
    d.dtheta = -gamma * d.theta;
    d.dchi = d.theta;
  } else {
    d.theta = 1.0 / (1.0 + gamma * dl);
    d.chi = d.theta * dl;
    d.dtheta = -gamma * d.theta * d.theta;
    d.dchi = d.theta * d.theta;
  }
  return d;
}

// The closest-point residual at (xi, dl) and what the Jacobian needs.
struct GPoint {
  double eq;        // sigma_bar(xi)
  double m[6];      // P xi / sigma_bar (engineering)
  double b, db;     // 2G dl + 2/3 sum C chi, and d/d dl
  double back_rate[6];
  double res[7];
};

// Committed kinematic terms of the point, read once per return.
struct Terms {
  double a[SBK_MAX_BACKSTRESSES][6];
};

static __device__ SBK_RETURN_HELPER bool gr_evaluate(const Params& p, const double s_trial[6], const Terms& tn,
                                            double a_n, const double xi[6], double dl, GPoint& e) {
  double pxi[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) s += p.P[i * 6 + j] * xi[j];
    pxi[i] = s;
  }
  double q = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) q += xi[i] * pxi[i];
  if (!(q > 0.0) || !isfinite(q)) return false;
  e.eq = sqrt(q);
  const double inv = 1.0 / e.eq;
#pragma unroll
  for (int i = 0; i < 6; ++i) e.m[i] = pxi[i] * inv;
  double xt[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    xt[i] = s_trial[i];
    e.back_rate[i] = 0.0;
  }
  e.b = 2.0 * p.G * dl;
  e.db = 2.0 * p.G;
#pragma unroll 1
  for (int t = 0; t < p.nterms; ++t) {
    {
      const Decay d = decay_of(p.termG[t], dl, p.integration);
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        xt[i] -= d.theta * tn.a[t][i];
        e.back_rate[i] += d.dtheta * tn.a[t][i];
      }
      e.b += 2.0 / 3.0 * p.termC[t] * d.chi;
      e.db += 2.0 / 3.0 * p.termC[t] * d.dchi;
    }
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double mt = i < 3 ? e.m[i] : 0.5 * e.m[i];
    e.res[i] = xi[i] - xt[i] + e.b * mt;
  }
  e.res[6] = e.eq - yield_of(p, a_n + dl);
  return true;
}

// The closest-point Jacobian (Plasticity.cpp:246-311) has the block form
//   J = [[A, j], [m^T, -h]],  A = I + f S (P - m m^T),  f = b / sigma_bar,
//   j = back_rate + db S m,  h = sigma_y'(a_n + dl),
// S = diag(1, 1, 1, 1/2, 1/2, 1/2). Writing A = S (B - f m m^T) with
// B = S^-1 + f P, and P = S^-1 V L V^T S^-1 with V^T S^-1 V = I (the
// generalised eigenvectors of the material's constant yield matrix, found
// once on the host), B^-1 = V (I + f L)^-1 V^T: two 6x6 products. The rank
// one term by Sherman-Morrison and the bordered row by its Schur complement
// then solve J [x; y] = [r; s] without pivoting or branches. This is the
// solution the reference's partial-pivoting LU of J gives, reached by a
// factorisation that suits the GPU (no row exchanges, 3 small products per
// Newton step); both agree to the round-off of J's conditioning.
struct JFactor {
  double f;      // b / sigma_bar
  double d[6];   // 1 / (1 + f L_k)
  double bm[6];  // B^-1 m
  double c;      // f / (1 - f m^T B^-1 m)
  double aj[6];  // A^-1 j
  double s;      // m^T A^-1 j + h
};

// out = B^-1 w = PV diag(d) PV^T w.
__device__ __forceinline__ void b_apply(const Params& p, const JFactor& jf, const double w[6], double out[6]) {
  double t[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double a = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) a += p.PV[i * 6 + k] * w[i];
    t[k] = a * jf.d[k];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double a = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) a += p.PV[i * 6 + k] * t[k];
    out[i] = a;
  }
}

// out = A^-1 z = (B - f m m^T)^-1 w with w = S^-1 z (Sherman-Morrison).
__device__ __forceinline__ void a_solve(const Params& p, const JFactor& jf, const double z[6], double out[6]) {
  double w[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) w[i] = i < 3 ? z[i] : 2.0 * z[i];
  b_apply(p, jf, w, out);
  double bw = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) bw += jf.bm[i] * w[i];
  const double g = jf.c * bw;
#pragma unroll
  for (int i = 0; i < 6; ++i) out[i] += g * jf.bm[i];
}

__device__ __forceinline__ void j_factor(const Params& p, const GPoint& e, double a_n, double dl, JFactor& jf) {
  jf.f = e.b / e.eq;
#pragma unroll
  for (int k = 0; k < 6; ++k) jf.d[k] = 1.0 / (1.0 + jf.f * p.PL[k]);
  b_apply(p, jf, e.m, jf.bm);
  double mbm = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) mbm += e.m[i] * jf.bm[i];
  jf.c = jf.f / (1.0 - jf.f * mbm);
  double jv[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) jv[i] = e.back_rate[i] + e.db * (i < 3 ? e.m[i] : 0.5 * e.m[i]);
  a_solve(p, jf, jv, jf.aj);
  double maj = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) maj += e.m[i] * jf.aj[i];
  jf.s = maj + yield_slope_of(p, a_n + dl);
}

// J [x; y] = [r; rs]: y = (m^T A^-1 r - rs) / s, x = A^-1 r - A^-1 j y.
__device__ __forceinline__ void j_solve(const Params& p, const GPoint& e, const JFactor& jf, const double r[6], double rs,
                                        double x[7]) {
  double ar[6];
  a_solve(p, jf, r, ar);
  double mar = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) mar += e.m[i] * ar[i];
  const double y = (mar - rs) / jf.s;
#pragma unroll
  for (int i = 0; i < 6; ++i) x[i] = ar[i] - jf.aj[i] * y;
  x[6] = y;
}

// C_alg = C^e - 2G [m_t a^T + (dl / sigma_bar) S (P - m m^T) A] with
// [A; a^T] = J^-1 [D_dev; 0] (Plasticity.cpp:299-311).
static __device__ SBK_RETURN_HELPER void gr_tangent(const Params& p, const GPoint& e, double a_n, double dl, double C[36]) {
  JFactor jf;
  j_factor(p, e, a_n, dl, jf);
  const double g = p.G;
  elastic_C(p, C);
  const double f = (dl > 0.0) ? 2.0 * g * dl / e.eq : 0.0;
#pragma unroll 1
  for (int col = 0; col < 6; ++col) {
    double r[6], x[7];
#pragma unroll
    for (int i = 0; i < 3; ++i) r[i] = col < 3 ? (i == col ? 4.0 * g / 3.0 : -2.0 * g / 3.0) : 0.0;
#pragma unroll
    for (int i = 3; i < 6; ++i) r[i] = (i == col) ? g : 0.0;
    j_solve(p, e, jf, r, 0.0, x);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const double mt = i < 3 ? e.m[i] : 0.5 * e.m[i];
      double v = 2.0 * g * (mt * x[6]);
      if (dl > 0.0) {
        const double sc = i < 3 ? 1.0 : 0.5;
        double sum = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) sum += sc * (p.P[i * 6 + k] - e.m[i] * e.m[k]) * x[k];
        v += f * sum;
      }
      C[i * 6 + col] -= v;
    }
  }
}

// The Newton step of the closest-point equations: J step = -R.
__device__ __forceinline__ void gr_newton_step(const Params& p, const GPoint& e, double a_n, double dl, double step[7]) {
  JFactor jf;
  j_factor(p, e, a_n, dl, jf);
  double r[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) r[i] = -e.res[i];
  j_solve(p, e, jf, r, -e.res[6], step);
}

// The trial state of the general return (Plasticity.cpp:337-352): the
// elastic strain, the trial deviator and relative stress, the committed
// terms, the yield stress and the overstress f_trial.
struct GTrial {
  double ep[6], el[6], s_trial[6], xi_tr[6];
  Terms tn;
  double vol, a_n, sy_n, eq_trial, f_trial;
  bool loading_n;
};

__device__ __forceinline__ void general_trial(const Params& p, const double strain[6], const PointState& st,
                                              GTrial& T) {
  const double g = p.G;
  const int nt = p.nterms;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    T.ep[i] = st.get(kFieldEp + i);
    T.el[i] = strain[i] - T.ep[i];
  }
  T.vol = T.el[0] + T.el[1] + T.el[2];
  {
    const double mean = T.vol / 3.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) T.s_trial[i] = 2.0 * g * (T.el[i] - mean);
#pragma unroll
    for (int i = 3; i < 6; ++i) T.s_trial[i] = g * T.el[i];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) T.xi_tr[i] = T.s_trial[i];
#pragma unroll
  for (int t = 0; t < SBK_MAX_BACKSTRESSES; ++t) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      T.tn.a[t][i] = t < nt ? st.get(kFieldAlpha + 6 * t + i) : 0.0;
      T.xi_tr[i] -= T.tn.a[t][i];
    }
  }
  T.a_n = st.get(field_eqps(nt));
  T.loading_n = st.get(field_loading(nt)) != 0.0;
  T.sy_n = yield_of(p, T.a_n);
  double q = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) s += p.P[i * 6 + j] * T.xi_tr[j];
    q += T.xi_tr[i] * s;
  }
  T.eq_trial = sqrt(fmax(q, 0.0));
  T.f_trial = T.eq_trial - T.sy_n;
}

// Whether the return takes its elastic branch at this trial state.
__device__ __forceinline__ bool general_is_elastic(const Params& p, const GTrial& T) {
  return !p.enabled || T.f_trial <= 1.0e-12 * T.sy_n;
}

__device__ __forceinline__ double kinematic_energy(const Params& p, const double (*a)[6]) {
  double o = 0.0;
#pragma unroll
  for (int t = 0; t < SBK_MAX_BACKSTRESSES; ++t) {
    if (t < p.nterms) {
      const double n = tnorm(a[t]);
      o += 0.75 * n * n / p.termC[t];
    }
  }
  return o;
}

// The loading window of the elastic branch (Plasticity.cpp:373): a point
// loading at the last commit and within 1e-10 sigma_y of the surface keeps
// loading, with the general tangent at dl = 0.
__device__ __forceinline__ bool general_loading_window(const Params& p, const GTrial& T) {
  return p.enabled && T.loading_n && T.f_trial > -1.0e-10 * T.sy_n && T.eq_trial > 0.0;
}

// The elastic branch: the trial stress, the elastic tangent (the general
// tangent at dl = 0 inside the loading window), the committed state with
// the loading flag. WINDOW = false: for a point known to be outside the
// window (the same result, without the window's code).
template <bool WINDOW = true>
__device__ __forceinline__ int general_elastic(const Params& p, const GTrial& T, const PointState& st, Response& out) {
  const double g = p.G, k = p.K;
  const int nt = p.nterms;
#pragma unroll
  for (int i = 0; i < 6; ++i) out.stress[i] = T.s_trial[i] + (i < 3 ? k * T.vol : 0.0);
  elastic_C(p, out.C);
  out.energy = 0.5 * k * T.vol * T.vol + g * dev_norm2(T.el) + isotropic_energy_of(p, T.a_n) + kinematic_energy(p, T.tn.a);
  out.yielding = false;
  bool loading = false;
  if (WINDOW && general_loading_window(p, T)) {
    loading = true;
    GPoint e;
    if (gr_evaluate(p, T.s_trial, T.tn, T.a_n, T.xi_tr, 0.0, e)) gr_tangent(p, e, T.a_n, 0.0, out.C);
  }
  // The committed state with the loading flag.
  const int nf = state_fields(nt);
  for (int f = 0; f < nf - 1; ++f) st.put(f, st.get(f));
  st.put(field_loading(nt), loading ? 1.0 : 0.0);
  return 0;
}

// warm: the point's last converged closest point (xi 6, dl, valid flag) in
// this element's local iteration, or NULL. The Newton iteration starts from
// whichever of it and the trial state has the smaller residual; the converged
// point is the same either way (to the return's tolerance), and from within
// one local iteration the warm start takes fewer steps. If a warm start does
// not converge, the return runs again from the trial state, as the
// reference's always does.
__device__ __forceinline__ int general_plastic(const Params& p, const GTrial& T, const PointState& st, Response& out,
                                               double* warm) {
  const double g = p.G, k = p.K;
  const int nt = p.nterms;
  const double* ep = T.ep;
  const double* el = T.el;
  const double* s_trial = T.s_trial;
  const double* xi_tr = T.xi_tr;
  const Terms& tn = T.tn;
  const double vol = T.vol, a_n = T.a_n, sy_n = T.sy_n;
  double scale = sy_n;
#pragma unroll
  for (int i = 0; i < 6; ++i) scale = fmax(scale, fmax(fabs(s_trial[i]), fabs(xi_tr[i])));
  const double eps_scale = kEps * scale;
  const double tol = fmax(1.0e-13 * sy_n, 32.0 * eps_scale);
  auto rinf = [](const GPoint& x) {
    double m = fabs(x.res[0]);
#pragma unroll
    for (int i = 1; i < 7; ++i) m = fmax(m, fabs(x.res[i]));
    return m;
  };
  auto rnorm = [](const GPoint& x) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 7; ++i) s += x.res[i] * x.res[i];
    return sqrt(s);
  };
  double xi[6], dl = 0.0;
  GPoint e;
  bool converged = false;
  // Attempt 0 starts warm (when that start has the smaller residual),
  // attempt 1 from the trial state (Plasticity.cpp:353-430).
  for (int attempt = (warm != nullptr && warm[7] != 0.0) ? 0 : 1; attempt < 2 && !converged; ++attempt) {
#pragma unroll
    for (int i = 0; i < 6; ++i) xi[i] = xi_tr[i];
    dl = 0.0;
    gr_evaluate(p, s_trial, tn, a_n, xi, dl, e);
    if (attempt == 0) {
      double xw[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) xw[i] = warm[i];
      GPoint ew;
      if (!gr_evaluate(p, s_trial, tn, a_n, xw, warm[6], ew) || !(rnorm(ew) < rnorm(e))) continue;
#pragma unroll
      for (int i = 0; i < 6; ++i) xi[i] = xw[i];
      dl = warm[6];
      e = ew;
    }
    for (int it = 0; it < 50; ++it) {
      const double r_inf = rinf(e);
      if (r_inf <= tol) {
        converged = true;
        break;
      }
      double step[7];
      gr_newton_step(p, e, a_n, dl, step);
      const double r0 = rnorm(e);
      double t = 1.0;
      bool accepted = false;
      for (int ls = 0; ls < 40; ++ls) {
        double xt[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) xt[i] = xi[i] + t * step[i];
        const double dlt = fmax(dl + t * step[6], 0.0);
        GPoint tr;
        if (gr_evaluate(p, s_trial, tn, a_n, xt, dlt, tr) && rnorm(tr) <= (1.0 - 1.0e-4 * t) * r0) {
#pragma unroll
          for (int i = 0; i < 6; ++i) xi[i] = xt[i];
          dl = dlt;
          e = tr;
          accepted = true;
          break;
        }
        t *= 0.5;
      }
      if (!accepted) {
        converged = r_inf <= 4.0 * tol;
        break;
      }
    }
  }
  if (!converged) return kFailReturn;
  if (rinf(e) > 4.0 * eps_scale) {
    // One more full Newton step (Plasticity.cpp:431-448).
    double step[7];
    gr_newton_step(p, e, a_n, dl, step);
    double xp[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) xp[i] = xi[i] + step[i];
    const double dlp = fmax(dl + step[6], 0.0);
    GPoint po;
    if (gr_evaluate(p, s_trial, tn, a_n, xp, dlp, po) && rinf(po) < rinf(e)) {
#pragma unroll
      for (int i = 0; i < 6; ++i) xi[i] = xp[i];
      dl = dlp;
      e = po;
    }
  }
  if (warm != nullptr) {
#pragma unroll
    for (int i = 0; i < 6; ++i) warm[i] = xi[i];
    warm[6] = dl;
    warm[7] = 1.0;
  }
  out.yielding = true;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const double mt = i < 3 ? e.m[i] : 0.5 * e.m[i];
    out.stress[i] = s_trial[i] - 2.0 * g * dl * mt + (i < 3 ? k * vol : 0.0);
  }
  // The updated state: plastic strain, the terms, their sum.
  double beta[6] = {0, 0, 0, 0, 0, 0};
  double anew[SBK_MAX_BACKSTRESSES][6];
#pragma unroll
  for (int t = 0; t < SBK_MAX_BACKSTRESSES; ++t) {
    if (t < nt) {
      const Decay d = decay_of(p.termG[t], dl, p.integration);
      const double f = 2.0 / 3.0 * p.termC[t] * d.chi;
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        const double mt = i < 3 ? e.m[i] : 0.5 * e.m[i];
        anew[t][i] = d.theta * tn.a[t][i] + f * mt;
        beta[i] += anew[t][i];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i) anew[t][i] = 0.0;
    }
  }
  double el_new[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    st.put(kFieldEp + i, ep[i] + dl * e.m[i]);
    st.put(kFieldBeta + i, beta[i]);
    el_new[i] = el[i] - dl * e.m[i];
  }
#pragma unroll
  for (int t = 0; t < SBK_MAX_BACKSTRESSES; ++t)
    if (t < nt)
#pragma unroll
      for (int i = 0; i < 6; ++i) st.put(kFieldAlpha + 6 * t + i, anew[t][i]);
  st.put(field_eqps(nt), a_n + dl);
  st.put(field_loading(nt), 1.0);
  out.energy = 0.5 * k * vol * vol + g * dev_norm2(el_new) + isotropic_energy_of(p, a_n + dl) + kinematic_energy(p, anew);
  gr_tangent(p, e, a_n, dl, out.C);
  return 0;
}


__device__ __forceinline__ int general_return(const Params& p, const double strain[6], const PointState& st,
                                              Response& out, double* warm = nullptr) {
  GTrial T;
  general_trial(p, strain, st, T);
  if (!isfinite(T.f_trial)) return kFailReturn;
  if (general_is_elastic(p, T)) return general_elastic(p, T, st, out);
  return general_plastic(p, T, st, out, warm);
}

// ---------------------------------------------------------------------------
// Logarithmic strain (LogarithmicStrain.cpp): eigen-decomposition of the
// Green-Lagrange strain by cyclic Jacobi, E_log = 1/2 log1p(2 mu), the first
// and second divided differences of ln, and the maps to the second
// Piola-Kirchhoff stress and the material tangent.
// ---------------------------------------------------------------------------
struct LogKin {
  double q[9];      // principal axes, columns (row-major q[3 i + a] = Q(i, a))
  double mu[3];     // principal Green-Lagrange strains, ascending
  double first[6];  // l[a, b]: (00, 11, 22, 01, 12, 20)
};

__device__ __forceinline__ void jacobi_rotate(double a[9], double v[9], int p, int q) {
  const double apq = a[p * 3 + q];
  if (apq == 0.0) return;
  const double theta = (a[q * 3 + q] - a[p * 3 + p]) / (2.0 * apq);
  const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
  const double c = 1.0 / sqrt(t * t + 1.0);
  const double s = t * c;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double akp = a[k * 3 + p], akq = a[k * 3 + q];
    a[k * 3 + p] = c * akp - s * akq;
    a[k * 3 + q] = s * akp + c * akq;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double apk = a[p * 3 + k], aqk = a[q * 3 + k];
    a[p * 3 + k] = c * apk - s * aqk;
    a[q * 3 + k] = s * apk + c * aqk;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double vkp = v[k * 3 + p], vkq = v[k * 3 + q];
    v[k * 3 + p] = c * vkp - s * vkq;
    v[k * 3 + q] = s * vkp + c * vkq;
  }
}

static __device__ __noinline__ double log_div(double mx, double my) {
  if (mx > my) {
    const double t = mx;
    mx = my;
    my = t;
  }
  const double y = 1.0 + 2.0 * my;
  const double d = 2.0 * (mx - my);
  if (d == 0.0) return 1.0 / y;
  return log1p(d / y) / d;
}

// first(a, b) from the packed layout.
__device__ __forceinline__ double first_of(const double f[6], int a, int b) {
  if (a == b) return f[a];
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return (lo == 0 && hi == 1) ? f[3] : ((lo == 1 && hi == 2) ? f[4] : f[5]);
}

static __device__ __noinline__ double log_div2(const LogKin& L, int a, int b, int c) {
  int i = a, j = b, k = c;
  if (L.mu[i] < L.mu[j]) { const int t = i; i = j; j = t; }
  if (L.mu[j] < L.mu[k]) { const int t = j; j = k; k = t; }
  if (L.mu[i] < L.mu[j]) { const int t = i; i = j; j = t; }
  const double y = 1.0 + 2.0 * L.mu[j];
  const double spread = 2.0 * (L.mu[i] - L.mu[k]);
  if (spread > 5.0e-3 * y) return (first_of(L.first, i, j) - first_of(L.first, j, k)) / spread;
  const double u = 2.0 * (L.mu[i] - L.mu[j]) / y;
  const double w = 2.0 * (L.mu[k] - L.mu[j]) / y;
  double h = 1.0, wn = 1.0, sum = -0.5;
#pragma unroll
  for (int n = 1; n <= 5; ++n) {
    wn *= w;
    h = u * h + wn;
    sum += (n % 2 == 1 ? 1.0 : -1.0) * h / (double)(n + 2);
  }
  return sum / (y * y);
}

// E_log of an engineering Green-Lagrange strain; 0 or a failure code.
__device__ __forceinline__ int log_strain(const double green[6], LogKin& L, double elog[6]) {
#pragma unroll
  for (int i = 0; i < 6; ++i)
    if (!isfinite(green[i])) return kFailNonFinite;
  double a[9] = {green[0], 0.5 * green[3], 0.5 * green[5], 0.5 * green[3], green[1],
                 0.5 * green[4], 0.5 * green[5], 0.5 * green[4], green[2]};
  double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int sweep = 0; sweep < 60; ++sweep) {
    const double off = a[1] * a[1] + a[2] * a[2] + a[5] * a[5];
    const double diag = a[0] * a[0] + a[4] * a[4] + a[8] * a[8];
    if (off == 0.0 || off <= 1.0e-36 * diag) break;
    jacobi_rotate(a, v, 0, 1);
    jacobi_rotate(a, v, 0, 2);
    jacobi_rotate(a, v, 1, 2);
  }
  double w[3] = {a[0], a[4], a[8]};
  // Sort ascending (selection), columns of v follow.
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    int m = i;
#pragma unroll
    for (int j = i + 1; j < 3; ++j)
      if (w[j] < w[m]) m = j;
#pragma unroll
    for (int j = i + 1; j < 3; ++j) {
      if (j == m) {
        const double t = w[i];
        w[i] = w[j];
        w[j] = t;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
          const double tv = v[r * 3 + i];
          v[r * 3 + i] = v[r * 3 + j];
          v[r * 3 + j] = tv;
        }
      }
    }
  }
  double pr[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double s2 = 1.0 + 2.0 * w[c];
    if (!(s2 > 0.0) || !isfinite(s2)) return kFailDegenerate;
    pr[c] = 0.5 * log1p(2.0 * w[c]);
    L.mu[c] = w[c];
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) L.q[i] = v[i];
  // E_log = Q diag(pr) Q^T, engineering Voigt.
  double e3[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) s += v[i * 3 + c] * pr[c] * v[j * 3 + c];
      e3[i * 3 + j] = s;
    }
  elog[0] = e3[0];
  elog[1] = e3[4];
  elog[2] = e3[8];
  elog[3] = 2.0 * e3[1];
  elog[4] = 2.0 * e3[5];
  elog[5] = 2.0 * e3[6];
  L.first[0] = log_div(w[0], w[0]);
  L.first[1] = log_div(w[1], w[1]);
  L.first[2] = log_div(w[2], w[2]);
  L.first[3] = log_div(w[0], w[1]);
  L.first[4] = log_div(w[1], w[2]);
  L.first[5] = log_div(w[2], w[0]);
  return 0;
}

// The Voigt principal rotation M (6x6): t(Q^T A Q) = M t(A) for tensorial t.
__device__ __forceinline__ double rot_m(const double q[9], int r, int c) {
  const int kr[6] = {0, 1, 2, 0, 1, 2};
  const int kc[6] = {0, 1, 2, 1, 2, 0};
  const int a = kr[r], b = kc[r], i = kr[c], j = kc[c];
  return i == j ? q[i * 3 + a] * q[i * 3 + b] : q[i * 3 + a] * q[j * 3 + b] + q[j * 3 + a] * q[i * 3 + b];
}

// S = P^T T alone (LogarithmicStrain.cpp:144-149): the second
// Piola-Kirchhoff stress of the Kirchhoff-like stress T work-conjugate to
// E_log, for stress recovery.
static __device__ __noinline__ void log_stress(const LogKin& L, const double t[6], double s_out[6]) {
  const int kr[6] = {0, 1, 2, 0, 1, 2};
  const int kc[6] = {0, 1, 2, 1, 2, 0};
  double tpv[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double v = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) v += rot_m(L.q, r, c) * t[c];
    tpv[r] = v;
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) v += rot_m(L.q, k, i) * ((k < 3 ? 1.0 : 2.0) * first_of(L.first, kr[k], kc[k])) * tpv[k];
    s_out[i] = i < 3 ? v : 0.5 * v;
  }
}

// S = P^T T, and material = P^T C P + T : L in global axes (engineering
// strain columns, tensorial stress rows). C is overwritten by the material.
__device__ __forceinline__ void log_transform(const LogKin& L, const double t[6], double s_out[6], double C[36]) {
  const int kr[6] = {0, 1, 2, 0, 1, 2};
  const int kc[6] = {0, 1, 2, 1, 2, 0};
  double M[36];
#pragma unroll
  for (int r = 0; r < 6; ++r)
#pragma unroll
    for (int c = 0; c < 6; ++c) M[r * 6 + c] = rot_m(L.q, r, c);
  // tp = Q^T T Q (principal components of T), tensorial Voigt.
  double tpv[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) s += M[r * 6 + c] * t[c];
    tpv[r] = s;
  }
  // S = M^-1 (first o tp) = S^-1 M^T S (first o tp).
  double sd[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) sd[k] = (k < 3 ? 1.0 : 2.0) * first_of(L.first, kr[k], kc[k]);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s += M[k * 6 + i] * sd[k] * tpv[k];
    s_out[i] = i < 3 ? s : 0.5 * s;
  }
  // Second divided differences, symmetric in their indices.
  double second[27];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c) {
        const double v = log_div2(L, a, b, c);
        second[a + 3 * b + 9 * c] = v;
        second[a + 3 * c + 9 * b] = v;
        second[b + 3 * a + 9 * c] = v;
        second[b + 3 * c + 9 * a] = v;
        second[c + 3 * a + 9 * b] = v;
        second[c + 3 * b + 9 * a] = v;
      }
  double tp[9];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    tp[kr[k] * 3 + kc[k]] = tpv[k];
    tp[kc[k] * 3 + kr[k]] = tpv[k];
  }
  // inner = diag(sd) (M C M^T) diag(sd) + hp, all in the principal frame.
  double X[36];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += C[i * 6 + k] * M[j * 6 + k];
      X[i * 6 + j] = s;  // C M^T
    }
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += M[i * 6 + k] * X[k * 6 + j];
      C[i * 6 + j] = sd[i] * s * sd[j];  // diag(sd) M C M^T diag(sd)
    }
  // + hp: 2 (half(k, l) + half(l, k)) over the principal unit tensors.
#pragma unroll
  for (int k = 0; k < 6; ++k)
#pragma unroll
    for (int l = k; l < 6; ++l) {
      double h = 0.0;
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        const int kx = pass == 0 ? k : l;
        const int ky = pass == 0 ? l : k;
        const int nx = kx < 3 ? 1 : 2, ny = ky < 3 ? 1 : 2;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          if (s < nx) {
            const int a = s == 0 ? kr[kx] : kc[kx];
            const int c = s == 0 ? kc[kx] : kr[kx];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
              if (r < ny) {
                const int yr = r == 0 ? kr[ky] : kc[ky];
                const int b = r == 0 ? kc[ky] : kr[ky];
                if (yr == c) h += tp[a * 3 + b] * second[a + 3 * b + 9 * c];
              }
            }
          }
        }
      }
      C[k * 6 + l] += 2.0 * h;
      if (l != k) C[l * 6 + k] += 2.0 * h;
    }
  // material = S^-1 M^T inner M S^-1.
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += C[i * 6 + k] * M[k * 6 + j];
      X[i * 6 + j] = s;  // inner M
    }
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) s += M[k * 6 + i] * X[k * 6 + j];
      C[i * 6 + j] = (i < 3 ? 1.0 : 0.5) * s * (j < 3 ? 1.0 : 0.5);
    }
}

}  // namespace sbk
