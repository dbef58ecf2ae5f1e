// ORACLE — test infrastructure only (see oracle_core.hpp).
//
// The incompatible-mode Hex8 element of the reference, restated:
// Gauss-Legendre rules (src/elements/Quadrature.cpp:16-219), Hex8 shape
// gradients (src/elements/Hex8.cpp:52-64), the Taylor-corrected mode
// gradients (src/elements/Hex8Incompatible.cpp:73-83), and the local Newton
// iteration with its condensation (src/fem/IncompatibleModes.cpp:134-600,
// constants src/fem/IncompatibleModes.hpp:98-127).
#pragma once

#include "oracle_core.hpp"

#include <vector>

namespace orc {

struct QPoint {
  double xi, eta, zeta, weight;
};

/// The 1-D Gauss-Legendre rule of n <= 7 points (Quadrature.cpp:16-163).
inline std::vector<std::pair<double, double>> line_rule(int n) {
  std::vector<std::pair<double, double>> r;
  if (n == 1) { r = {{0.0, 2.0}}; return r; }
  if (n == 2) { const double a = 1.0 / std::sqrt(3.0); r = {{-a, 1.0}, {a, 1.0}}; return r; }
  if (n == 3) {
    const double a = std::sqrt(3.0 / 5.0);
    r = {{-a, 5.0 / 9.0}, {0.0, 8.0 / 9.0}, {a, 5.0 / 9.0}};
    return r;
  }
  if (n == 4) {
    const double s6 = std::sqrt(6.0 / 5.0);
    const double x1 = std::sqrt((3.0 - 2.0 * s6) / 7.0);
    const double x2 = std::sqrt((3.0 + 2.0 * s6) / 7.0);
    const double s = std::sqrt(30.0);
    const double w1 = (18.0 + s) / 36.0, w2 = (18.0 - s) / 36.0;
    r = {{-x2, w2}, {-x1, w1}, {x1, w1}, {x2, w2}};
    return r;
  }
  // Newton on P_n from Tricomi's guesses (Quadrature.cpp:100-139).
  r.assign(static_cast<std::size_t>(n), {0.0, 0.0});
  const double pi = std::acos(-1.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double x = std::cos(pi * (i + 0.75) / (n + 0.5));
    double derivative = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      derivative = n * (x * p1 - p0) / (x * x - 1.0);
      const double step = p1 / derivative;
      x -= step;
      if (std::fabs(step) <= 1.0e-16) break;
    }
    if (2 * i + 1 == n) x = 0.0;
    double p0 = 1.0, p1 = x;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    derivative = n * (x * p1 - p0) / (x * x - 1.0);
    const double weight = 2.0 / ((1.0 - x * x) * derivative * derivative);
    r[static_cast<std::size_t>(i)] = {-x, weight};
    r[static_cast<std::size_t>(n - 1 - i)] = {x, weight};
  }
  return r;
}

/// The Hex8 stiffness rule (Hex8Kernels.hpp:125-130, Quadrature.cpp:72-93,
/// 165-219): the cube rule, or the box rule with thickness points; xi
/// fastest, weights multiplied x * y * z.
inline std::vector<QPoint> hex8_rule(int in_plane, int thickness, int axis) {
  if (thickness <= 0 || thickness == in_plane) thickness = in_plane, axis = 2;
  const auto plane = line_rule(in_plane);
  const auto through = line_rule(thickness);
  const auto& rx = axis == 0 ? through : plane;
  const auto& ry = axis == 1 ? through : plane;
  const auto& rz = axis == 2 ? through : plane;
  std::vector<QPoint> out;
  for (const auto& gk : rz)
    for (const auto& gj : ry)
      for (const auto& gi : rx) out.push_back({gi.first, gj.first, gk.first, gi.second * gj.second * gk.second});
  return out;
}

constexpr double kCorner[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

/// dN/dxi, 8 x 3 (Hex8.cpp:52-64).
inline Mat<double, 8, 3> shape_gradients(double xi, double eta, double zeta) {
  Mat<double, 8, 3> g;
  for (int a = 0; a < 8; ++a) {
    const double fx = 1.0 + xi * kCorner[a][0];
    const double fy = 1.0 + eta * kCorner[a][1];
    const double fz = 1.0 + zeta * kCorner[a][2];
    g(a, 0) = 0.125 * kCorner[a][0] * fy * fz;
    g(a, 1) = 0.125 * kCorner[a][1] * fx * fz;
    g(a, 2) = 0.125 * kCorner[a][2] * fx * fy;
  }
  return g;
}

enum Kinematics { kSmall = 0, kFinite = 1, kLogarithmic = 2 };

constexpr int kMaxLocal = 25;
constexpr double kFullStepReduction = 1.0 - 1.0e-4;
constexpr int kMaxLineSearch = 8;
constexpr double kLineSearchRatio = 0.5;
constexpr double kLocalShift = 1.0e-3;
constexpr double kLocalMarquardt = 1.0e-6;
constexpr double kLocalTolerance = 1.0e-8;
constexpr double kLocalRoundOff = 1.0e-13;

template <class T>
struct PointWork {
  Mat<T, 3, 11> g;  // [G | G~]
  Mat<T, 3, 3> hu;
  T weight = T(0.0);
  Mat<T, 3, 3> h;
  Mat<T, 6, 33> mb;
  Vec<T, 6> strain;
  LogStrain<T> log;
  Vec<T, 6> s;
  Mat<T, 6, 6> material;
  T energy = T(0.0);
  State<T> state;
  bool yielding = false;
};

template <class T>
struct Sums {
  Vec<T, 33> r;
  Vec<T, 9> scale, floor;
  Mat<T, 9, 9> kaa;
  Mat<T, 24, 9> kua;
  Mat<T, 9, 24> kau;
  Mat<T, 24, 24> kuu;
  T energy = T(0.0);
};

template <class T>
Mat<T, 3, 3> tensor3(const Vec<T, 6>& v) {
  Mat<T, 3, 3> t;
  t(0, 0) = v[0]; t(0, 1) = v[3]; t(0, 2) = v[5];
  t(1, 0) = v[3]; t(1, 1) = v[1]; t(1, 2) = v[4];
  t(2, 0) = v[5]; t(2, 1) = v[4]; t(2, 2) = v[2];
  return t;
}

template <class T>
Vec<T, 6> green_lagrange_6(const Mat<T, 3, 3>& h) {
  Mat<T, 3, 3> e;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T s = T(0.0);
      for (int k = 0; k < 3; ++k) s += h(k, i) * h(k, j);
      e(i, j) = T(0.5) * (h(i, j) + h(j, i) + s);
    }
  Vec<T, 6> v;
  v[0] = e(0, 0); v[1] = e(1, 1); v[2] = e(2, 2);
  v[3] = T(2.0) * e(0, 1); v[4] = T(2.0) * e(1, 2); v[5] = T(2.0) * e(2, 0);
  return v;
}

template <class T>
void green_lagrange_operator_11(const Mat<T, 3, 3>& f, const Mat<T, 3, 11>& g, Mat<T, 6, 33>& b) {
  static constexpr int kPair[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 2}, {2, 0}};
  for (int c = 0; c < 6; ++c) {
    const int i = kPair[c][0], j = kPair[c][1];
    for (int a = 0; a < 11; ++a)
      for (int k = 0; k < 3; ++k)
        b(c, 3 * a + k) = i == j ? f(k, i) * g(i, a) : f(k, i) * g(j, a) + f(k, j) * g(i, a);
  }
}

/// One element's result (ElastoplasticElement, Elastoplastic.hpp:171-186).
template <class T>
struct ElementOut {
  Vec<T, 24> force;
  Mat<T, 24, 24> tangent;
  T energy = T(0.0);
  Vec<T, 9> alpha;
  int iterations = 0;
  int yielding = 0;
  std::vector<State<T>> states;
  std::vector<char> point_yield;
  bool symmetric = true;
};

/// ElastoplasticStress (include/sparlab/fem/Elastoplastic.hpp:206-221):
/// point averages of the Cauchy, second Piola-Kirchhoff and (logarithmic)
/// Kirchhoff stresses and log strain, the von Mises stress of the average
/// Cauchy stress, the largest accumulated plastic strain and strain
/// component, the smallest det F.
struct ElementStress {
  double cauchy[6] = {}, piola_kirchhoff[6] = {}, kirchhoff[6] = {}, log_strain[6] = {};
  double von_mises = 0.0, max_eqps = 0.0, max_strain = 0.0, min_jacobian = 1.0;
};

template <class T>
class IMElement {
 public:
  /// incompatible_elastoplastic_stress (IncompatibleModes.cpp:602-664): the
  /// measures at the converged state, the modes at their committed values
  /// (no local iteration), every point's return an elastic check from its
  /// committed state.
  ElementStress stress(const double* x, const T* ue, const std::vector<State<T>>& committed, const T* alpha) {
    set_up(x, ue);
    Vec<T, 9> a;
    for (int i = 0; i < 9; ++i) a[i] = alpha ? alpha[i] : T(0.0);
    kinematics_at(a);
    ElementStress out;
    out.min_jacobian = std::numeric_limits<double>::infinity();
    const bool finite = kin_ == kFinite, logarithmic = kin_ == kLogarithmic;
    for (std::size_t q = 0; q < points_.size(); ++q) {
      const PointWork<T>& p = points_[q];
      const Response<T> r = plastic_return(mat_, p.strain, committed[q], false);
      Vec<T, 6> cauchy = r.stress, pk = r.stress;
      Mat<T, 3, 3> f = p.h, sym;
      for (int i = 0; i < 3; ++i) f(i, i) += T(1.0);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sym(i, j) = T(0.5) * (p.h(i, j) + p.h(j, i));
      auto absmax = [](const Mat<T, 3, 3>& m) {
        double v = 0.0;
        for (int i = 0; i < 9; ++i) v = std::max(v, std::fabs(val(m[i])));
        return v;
      };
      if (logarithmic) {
        pk = logarithmic_stress(p.log, r.stress);
        const Vec<T, 6> tau = voigt_of(mul(mul(f, tensor3(pk)), tr(f)), 1.0);
        Vec<T, 6> strain = p.strain;
        for (int i = 3; i < 6; ++i) strain[i] = T(0.5) * strain[i];
        const T j = exp(strain[0] + strain[1] + strain[2]);
        for (int i = 0; i < 6; ++i) {
          cauchy[i] = tau[i] / j;
          out.kirchhoff[i] += val(tau[i]);
          out.log_strain[i] += val(strain[i]);
          out.max_strain = std::max(out.max_strain, std::fabs(val(strain[i])));
        }
        out.min_jacobian = std::min(out.min_jacobian, val(det3(f)));
      } else if (finite) {
        const T j = det3(f);
        const Vec<T, 6> c = voigt_of(mul(mul(f, tensor3(r.stress)), tr(f)), 1.0);
        for (int i = 0; i < 6; ++i) cauchy[i] = c[i] / j;
        Mat<T, 3, 3> green = sym;
        const Mat<T, 3, 3> hth = mul(tr(p.h), p.h);
        for (int i = 0; i < 9; ++i) green[i] += T(0.5) * hth[i];
        out.max_strain = std::max(out.max_strain, absmax(green));
        out.min_jacobian = std::min(out.min_jacobian, val(j));
      } else {
        out.max_strain = std::max(out.max_strain, absmax(sym));
      }
      for (int i = 0; i < 6; ++i) {
        out.cauchy[i] += val(cauchy[i]);
        out.piola_kirchhoff[i] += val(pk[i]);
      }
      out.max_eqps = std::max(out.max_eqps, val(r.state.eqps));
    }
    const double count = static_cast<double>(points_.size());
    for (int i = 0; i < 6; ++i) {
      out.cauchy[i] /= count;
      out.piola_kirchhoff[i] /= count;
      out.kirchhoff[i] /= count;
      out.log_strain[i] /= count;
    }
    const double* c = out.cauchy;
    out.von_mises = std::sqrt(0.5 * ((c[0] - c[1]) * (c[0] - c[1]) + (c[1] - c[2]) * (c[1] - c[2]) +
                                     (c[2] - c[0]) * (c[2] - c[0])) +
                              3.0 * (c[3] * c[3] + c[4] * c[4] + c[5] * c[5]));
    if (!finite && !logarithmic) out.min_jacobian = 1.0;
    return out;
  }

  IMElement(const Material& mat, const std::vector<QPoint>& rule, int kinematics)
      : mat_(mat), rule_(rule), kin_(kinematics) {}

  /// The vector-Jacobian product of the condensed residual with respect to
  /// the element's reference coordinates, out[3a+i] = lambda . d f* / d X_ia,
  /// at fixed displacements and committed history (finite or logarithmic
  /// kinematics), the modes following through their local equilibrium:
  ///   d f*/dX = d r_u/dX + K_ua d alpha/dX,  K_aa d alpha/dX = -d r_a/dX,
  /// so lambda^T d f*/dX = [lambda; mu]^T d r/dX|_alpha with
  /// mu = -K_aa^-T K_ua^T lambda and r = (r_u, r_a) = sum_q w F S [G | G~].
  /// Per point the chain runs r -> (F, S, [G | G~], w); S -> E (the point's
  /// material tangent dS/dE) -> F; F = I + U [G | G~]^T -> [G | G~];
  /// G = dN J^-1, G~ = (det0/det)(-2 xi) J0^-1, w = w_q det J -> (J, J0) -> X.
  /// Throws Failure where evaluate does.
  void vjp_x(const double* x, const T* ue, const std::vector<State<T>>& committed, const T* alpha_n,
             const double* lambda, double* out) {
    ElementOut<T> eo = evaluate(x, ue, committed, alpha_n, true);
    Vec<T, 9> a;
    for (int i = 0; i < 9; ++i) a[i] = eo.alpha[i];
    kinematics_at(a);
    respond(committed);
    Sums<T> sums;
    accumulate_local(sums);
    accumulate_coupling(false, sums);
    // mu = -K_aa^-T K_ua^T lambda.
    Vec<T, 9> b;
    for (int j = 0; j < 9; ++j) {
      T acc = T(0.0);
      for (int i = 0; i < 24; ++i) acc += sums.kua(i, j) * T(lambda[i]);
      b[j] = acc;
    }
    FullPivLU<T, 9> lut;
    lut.compute(tr(sums.kaa));
    const Vec<T, 9> y = lut.solve(b);
    // Lambda (3 x 11): nodes, then modes (residual index 3 m + k).
    double L[3][11], Uu[3][11];
    for (int k = 0; k < 3; ++k) {
      for (int n = 0; n < 8; ++n) {
        L[k][n] = lambda[3 * n + k];
        Uu[k][n] = val(ue[3 * n + k]);
      }
      for (int m = 0; m < 3; ++m) {
        L[k][8 + m] = -val(y[3 * m + k]);
        Uu[k][8 + m] = val(a[3 * m + k]);
      }
    }
    for (int i = 0; i < 24; ++i) out[i] = 0.0;
    // Reference Jacobians (set_up's).
    auto jac_at = [&](const Mat<double, 8, 3>& dn, double J[3][3]) {
      for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) {
          double acc = 0.0;
          for (int n = 0; n < 8; ++n) acc += x[3 * n + i] * dn(n, c);
          J[i][c] = acc;
        }
    };
    auto inv_det = [](const double J[3][3], double Ji[3][3]) {
      const double d = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) -
                       J[1][0] * (J[0][1] * J[2][2] - J[2][1] * J[0][2]) +
                       J[2][0] * (J[0][1] * J[1][2] - J[1][1] * J[0][2]);
      Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / d;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / d;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / d;
      Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / d;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / d;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / d;
      Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / d;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / d;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / d;
      return d;
    };
    const Mat<double, 8, 3> dn0 = shape_gradients(0.0, 0.0, 0.0);
    double J0[3][3], J0i[3][3];
    jac_at(dn0, J0);
    inv_det(J0, J0i);
    double J0bar[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (std::size_t q = 0; q < rule_.size(); ++q) {
      const PointWork<T>& p = points_[q];
      const QPoint& xi = rule_[q];
      const Mat<double, 8, 3> dn = shape_gradients(xi.xi, xi.eta, xi.zeta);
      double J[3][3], Ji[3][3];
      jac_at(dn, J);
      inv_det(J, Ji);
      const double w = val(p.weight);
      double F[3][3], S[3][3], G[3][11];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = val(p.h(i, j)) + (i == j ? 1.0 : 0.0);
      const double s6[6] = {val(p.s[0]), val(p.s[1]), val(p.s[2]), val(p.s[3]), val(p.s[4]), val(p.s[5])};
      S[0][0] = s6[0]; S[1][1] = s6[1]; S[2][2] = s6[2];
      S[0][1] = S[1][0] = s6[3]; S[1][2] = S[2][1] = s6[4]; S[2][0] = S[0][2] = s6[5];
      for (int j = 0; j < 3; ++j)
        for (int n = 0; n < 11; ++n) G[j][n] = val(p.g(j, n));
      // phi_q = w sum_{k,n} L_kn (F S G)_kn; Q = L G^T.
      double FS[3][3], Q[3][3];
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0, acq = 0.0;
          for (int i = 0; i < 3; ++i) acc += F[k][i] * S[i][j];
          for (int n = 0; n < 11; ++n) acq += L[k][n] * G[j][n];
          FS[k][j] = acc;
          Q[k][j] = acq;
        }
      double phi = 0.0;
      for (int k = 0; k < 3; ++k)
        for (int n = 0; n < 11; ++n) {
          double acc = 0.0;
          for (int j = 0; j < 3; ++j) acc += FS[k][j] * G[j][n];
          phi += L[k][n] * acc;
        }
      phi *= w;
      // Gbar = w S F^T L (direct), Fbar = w Q S + F Ebar.
      double Gb[3][11];
      for (int j = 0; j < 3; ++j)
        for (int n = 0; n < 11; ++n) {
          double acc = 0.0;
          for (int k = 0; k < 3; ++k) acc += FS[k][j] * L[k][n];  // (S F^T L)_jn = sum_k (F S)_kj L_kn
          Gb[j][n] = w * acc;
        }
      // Sbar = w sym(F^T Q); sbar (Voigt: normal, 2 x shear) -> ebar = M^T sbar.
      double FtQ[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0;
          for (int k = 0; k < 3; ++k) acc += F[k][i] * Q[k][j];
          FtQ[i][j] = w * acc;
        }
      const int vi[6] = {0, 1, 2, 0, 1, 2}, vj[6] = {0, 1, 2, 1, 2, 0};
      double sb[6];
      for (int c = 0; c < 6; ++c) {
        const double sym = 0.5 * (FtQ[vi[c]][vj[c]] + FtQ[vj[c]][vi[c]]);
        sb[c] = c < 3 ? sym : 2.0 * sym;
      }
      double eb[6];
      for (int d = 0; d < 6; ++d) {
        double acc = 0.0;
        for (int c = 0; c < 6; ++c) acc += val(p.material(c, d)) * sb[c];
        eb[d] = acc;
      }
      double Eb[3][3];
      for (int c = 0; c < 6; ++c) {
        Eb[vi[c]][vj[c]] = eb[c];
        Eb[vj[c]][vi[c]] = eb[c];
      }
      double Fb[3][3];
      for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0, acf = 0.0;
          for (int i = 0; i < 3; ++i) {
            acc += Q[k][i] * S[i][j];
            acf += F[k][i] * Eb[i][j];
          }
          Fb[k][j] = w * acc + acf;
        }
      // F = I + U G^T: Gbar += Fbar^T U.
      for (int j = 0; j < 3; ++j)
        for (int n = 0; n < 11; ++n) {
          double acc = 0.0;
          for (int i = 0; i < 3; ++i) acc += Fb[i][j] * Uu[i][n];
          Gb[j][n] += acc;
        }
      // w = w_q det J: Jbar = phi J^-T.
      double Jb[3][3];
      for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) Jb[i][c] = phi * Ji[c][i];
      // G = (dN J^-1)^T: Jbar -= J^-T K1 J^-T with K1_cj = sum_n dN_nc Gbar_jn.
      double K1[3][3];
      for (int c = 0; c < 3; ++c)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0;
          for (int n = 0; n < 8; ++n) acc += dn(n, c) * Gb[j][n];
          K1[c][j] = acc;
        }
      for (int pp = 0; pp < 3; ++pp)
        for (int r = 0; r < 3; ++r) {
          double acc = 0.0;
          for (int c = 0; c < 3; ++c)
            for (int j = 0; j < 3; ++j) acc += Ji[c][pp] * K1[c][j] * Ji[r][j];
          Jb[pp][r] -= acc;
        }
      // G~_im = ratio c_m J0^-1_mi, ratio = det0 / det, c_m = -2 xi_m.
      const double det = J[0][0] * (J[1][1] * J[2][2] - J[2][1] * J[1][2]) -
                         J[1][0] * (J[0][1] * J[2][2] - J[2][1] * J[0][2]) +
                         J[2][0] * (J[0][1] * J[1][2] - J[1][1] * J[0][2]);
      const double det0 = J0[0][0] * (J0[1][1] * J0[2][2] - J0[2][1] * J0[1][2]) -
                          J0[1][0] * (J0[0][1] * J0[2][2] - J0[2][1] * J0[0][2]) +
                          J0[2][0] * (J0[0][1] * J0[1][2] - J0[1][1] * J0[0][2]);
      const double ratio = det0 / det;
      const double cm[3] = {-2.0 * xi.xi, -2.0 * xi.eta, -2.0 * xi.zeta};
      double R = 0.0, K2[3][3];
      for (int m = 0; m < 3; ++m)
        for (int i = 0; i < 3; ++i) {
          R += Gb[i][8 + m] * cm[m] * J0i[m][i];
          K2[m][i] = cm[m] * Gb[i][8 + m];
        }
      for (int pp = 0; pp < 3; ++pp)
        for (int r = 0; r < 3; ++r) {
          J0bar[pp][r] += ratio * R * J0i[r][pp];
          Jb[pp][r] -= ratio * R * Ji[r][pp];
          double acc = 0.0;
          for (int m = 0; m < 3; ++m)
            for (int i = 0; i < 3; ++i) acc += J0i[m][pp] * K2[m][i] * J0i[r][i];
          J0bar[pp][r] -= ratio * acc;
        }
      // J = X dN: Xbar_in += sum_c Jbar_ic dN_nc.
      for (int n = 0; n < 8; ++n)
        for (int i = 0; i < 3; ++i) {
          double acc = 0.0;
          for (int c = 0; c < 3; ++c) acc += Jb[i][c] * dn(n, c);
          out[3 * n + i] += acc;
        }
    }
    for (int n = 0; n < 8; ++n)
      for (int i = 0; i < 3; ++i) {
        double acc = 0.0;
        for (int c = 0; c < 3; ++c) acc += J0bar[i][c] * dn0(n, c);
        out[3 * n + i] += acc;
      }
  }

  /// incompatible_elastoplastic_element (IncompatibleModes.cpp:577-600).
  /// Throws Failure.
  ElementOut<T> evaluate(const double* x /*3x8 node-major: x[3a+i]*/, const T* ue,
                         const std::vector<State<T>>& committed, const T* alpha_n,
                         bool want_tangent) {
    set_up(x, ue);
    ElementOut<T> out;
    solve_and_condense(committed, alpha_n, want_tangent, out);
    out.symmetric = symmetric_;
    out.states.reserve(points_.size());
    for (const PointWork<T>& p : points_) {
      out.states.push_back(p.state);
      out.point_yield.push_back(p.yielding ? 1 : 0);
      if (p.yielding) ++out.yielding;
    }
    return out;
  }

 private:
  void set_up(const double* x, const T* ue) {
    symmetric_ = mat_.symmetric();
    for (int a = 0; a < 8; ++a)
      for (int k = 0; k < 3; ++k) u_(k, a) = ue[3 * a + k];
    for (int i = 0; i < 24; ++i) ue_[i] = ue[i];
    Mat<T, 3, 8> x0;
    for (int a = 0; a < 8; ++a)
      for (int k = 0; k < 3; ++k) x0(k, a) = T(x[3 * a + k]);
    auto jacobian_at = [&](const Mat<double, 8, 3>& dn) {
      Mat<T, 3, 3> j;
      for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) {
          T s = T(0.0);
          for (int a = 0; a < 8; ++a) s += x0(i, a) * T(dn(a, c));
          j(i, c) = s;
        }
      return j;
    };
    const Mat<T, 3, 3> jac0 = jacobian_at(shape_gradients(0.0, 0.0, 0.0));
    const T det0 = det3(jac0);
    if (!(det0 > T(0.0))) throw Failure{kMeshInverted};
    const Mat<T, 3, 3> jinv0 = inv3(jac0);
    points_.assign(rule_.size(), PointWork<T>());
    for (std::size_t q = 0; q < rule_.size(); ++q) {
      const QPoint& xi = rule_[q];
      PointWork<T>& p = points_[q];
      const Mat<double, 8, 3> dn = shape_gradients(xi.xi, xi.eta, xi.zeta);
      const Mat<T, 3, 3> jac = jacobian_at(dn);
      const T det = det3(jac);
      if (!(det > T(0.0))) throw Failure{kMeshInverted};
      const Mat<T, 3, 3> jinv = inv3(jac);
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
          T s = T(0.0);
          for (int c = 0; c < 3; ++c) s += T(dn(a, c)) * jinv(c, i);
          p.g(i, a) = s;
        }
      // hex8_incompatible_gradients: column k = (det0/det)(-2 xi_k) row k of J0^-1.
      const T ratio = det0 / det;
      const double nat[3] = {xi.xi, xi.eta, xi.zeta};
      for (int k = 0; k < 3; ++k) {
        const T f = ratio * T(-2.0 * nat[k]);
        for (int i = 0; i < 3; ++i) p.g(i, 8 + k) = f * jinv0(k, i);
      }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          T s = T(0.0);
          for (int a = 0; a < 8; ++a) s += u_(i, a) * p.g(j, a);
          p.hu(i, j) = s;
        }
      p.weight = T(xi.weight) * det;
      if (kin_ == kSmall) {
        Mat<T, 3, 3> id;
        for (int i = 0; i < 3; ++i) id(i, i) = T(1.0);
        green_lagrange_operator_11(id, p.g, p.mb);
      }
    }
  }

  void kinematics_at(const Vec<T, 9>& alpha) {
    Mat<T, 3, 3> a;
    for (int m = 0; m < 3; ++m)
      for (int k = 0; k < 3; ++k) a(k, m) = alpha[3 * m + k];
    for (PointWork<T>& p : points_) {
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          T s = T(0.0);
          for (int m = 0; m < 3; ++m) s += a(i, m) * p.g(j, 8 + m);
          p.h(i, j) = p.hu(i, j) + s;
        }
      if (kin_ == kSmall) {
        for (int c = 0; c < 6; ++c) {
          T s = T(0.0);
          for (int j = 0; j < 24; ++j) s += p.mb(c, j) * ue_[j];
          T t = T(0.0);
          for (int j = 0; j < 9; ++j) t += p.mb(c, 24 + j) * alpha[j];
          p.strain[c] = s + t;
        }
      } else {
        Mat<T, 3, 3> f = p.h;
        for (int i = 0; i < 3; ++i) f(i, i) += T(1.0);
        if (kin_ == kLogarithmic && !(det3(f) > T(0.0))) throw Failure{kInverted};
        green_lagrange_operator_11(f, p.g, p.mb);
        if (kin_ == kFinite) {
          p.strain = green_lagrange_6(p.h);
        } else {
          p.log = logarithmic_strain(green_lagrange_6(p.h));
          p.strain = p.log.strain;
        }
      }
    }
  }

  void respond(const std::vector<State<T>>& committed) {
    for (std::size_t q = 0; q < points_.size(); ++q) {
      PointWork<T>& p = points_[q];
      const Response<T> r = plastic_return(mat_, p.strain, committed[q], true);
      p.energy = r.energy;
      p.state = r.state;
      p.yielding = r.yielding;
      if (kin_ == kLogarithmic) {
        p.s = logarithmic_stress(p.log, r.stress);
        const Mat<T, 6, 6> pcp = mul(mul(tr(p.log.projection), r.tangent), p.log.projection);
        const Mat<T, 6, 6> curv = logarithmic_curvature(p.log, r.stress);
        for (int i = 0; i < 36; ++i) p.material[i] = pcp[i] + curv[i];
      } else {
        p.s = r.stress;
        p.material = r.tangent;
      }
    }
  }

  void accumulate_local(Sums<T>& sums) {
    const bool geometric = kin_ != kSmall;
    for (const PointWork<T>& p : points_) {
      const T w = p.weight;
      for (int j = 0; j < 33; ++j) {
        T s = T(0.0);
        for (int c = 0; c < 6; ++c) s += p.mb(c, j) * p.s[c];
        sums.r[j] += w * s;
      }
      for (int j = 0; j < 9; ++j) {
        T s = T(0.0);
        for (int c = 0; c < 6; ++c) s += abs(p.mb(c, 24 + j)) * abs(p.s[c]);
        sums.scale[j] += w * s;
      }
      const T h = maxabs(p.h);
      const T f = w * maxabs(p.material) * h * (T(1.0) + h);
      for (int j = 0; j < 9; ++j) {
        T s = T(0.0);
        for (int c = 0; c < 6; ++c) s += abs(p.mb(c, 24 + j));
        sums.floor[j] += f * s;
      }
      sums.energy += w * p.energy;
      Mat<T, 6, 9> mba;
      for (int c = 0; c < 6; ++c)
        for (int j = 0; j < 9; ++j) {
          T s = T(0.0);
          for (int d = 0; d < 6; ++d) s += p.material(c, d) * p.mb(d, 24 + j);
          mba(c, j) = s;
        }
      for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) {
          T s = T(0.0);
          for (int c = 0; c < 6; ++c) s += p.mb(c, 24 + i) * mba(c, j);
          sums.kaa(i, j) += w * s;
        }
      if (geometric) {
        const Mat<T, 3, 3> st = tensor3(p.s);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            T s = T(0.0);
            for (int i = 0; i < 3; ++i)
              for (int j = 0; j < 3; ++j) s += p.g(i, 8 + a) * st(i, j) * p.g(j, 8 + b);
            for (int k = 0; k < 3; ++k) sums.kaa(3 * a + k, 3 * b + k) += w * s;
          }
      }
    }
  }

  void accumulate_coupling(bool full, Sums<T>& sums) {
    const bool geometric = kin_ != kSmall;
    for (const PointWork<T>& p : points_) {
      const T w = p.weight;
      // material * mb (6 x 33)
      Mat<T, 6, 33> mb2;
      for (int c = 0; c < 6; ++c)
        for (int j = 0; j < 33; ++j) {
          T s = T(0.0);
          for (int d = 0; d < 6; ++d) s += p.material(c, d) * p.mb(d, j);
          mb2(c, j) = s;
        }
      for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 9; ++j) {
          T s = T(0.0);
          for (int c = 0; c < 6; ++c) s += p.mb(c, i) * mb2(c, 24 + j);
          sums.kua(i, j) += w * s;
        }
      if (!symmetric_) {
        for (int i = 0; i < 9; ++i)
          for (int j = 0; j < 24; ++j) {
            T s = T(0.0);
            for (int c = 0; c < 6; ++c) s += p.mb(c, 24 + i) * mb2(c, j);
            sums.kau(i, j) += w * s;
          }
      }
      if (full) {
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            T s = T(0.0);
            for (int c = 0; c < 6; ++c) s += p.mb(c, i) * mb2(c, j);
            sums.kuu(i, j) += w * s;
          }
      }
      if (geometric) {
        const Mat<T, 3, 3> st = tensor3(p.s);
        for (int a = 0; a < 8; ++a)
          for (int b = 0; b < 11; ++b) {
            T s = T(0.0);
            for (int i = 0; i < 3; ++i)
              for (int j = 0; j < 3; ++j) s += p.g(i, a) * st(i, j) * p.g(j, b);
            const T v = w * s;
            for (int k = 0; k < 3; ++k) {
              if (b < 8) {
                if (full) sums.kuu(3 * a + k, 3 * b + k) += v;
              } else {
                sums.kua(3 * a + k, 3 * (b - 8) + k) += v;
                if (!symmetric_) sums.kau(3 * (b - 8) + k, 3 * a + k) += v;
              }
            }
          }
      }
    }
  }

  static Vec<T, 9> tail9(const Vec<T, 33>& r) {
    Vec<T, 9> t;
    for (int i = 0; i < 9; ++i) t[i] = r[24 + i];
    return t;
  }

  void solve_and_condense(const std::vector<State<T>>& committed, const T* start,
                          bool want_tangent, ElementOut<T>& out) {
    Vec<T, 9> alpha;
    if (start != nullptr)
      for (int i = 0; i < 9; ++i) alpha[i] = start[i];
    Sums<T> sums;
    FullPivLU<T, 9> lu;
    auto pass = [&](const Vec<T, 9>& at) {
      kinematics_at(at);
      respond(committed);
      sums = Sums<T>();
      accumulate_local(sums);
    };
    auto try_pass = [&](const Vec<T, 9>& at) {
      try {
        pass(at);
        return true;
      } catch (const Failure&) {
        return false;
      }
    };
    auto axpy = [](const Vec<T, 9>& a, T s, const Vec<T, 9>& d) {
      Vec<T, 9> o;
      for (int i = 0; i < 9; ++i) o[i] = a[i] + s * d[i];
      return o;
    };
    pass(alpha);
    T residual = norm(tail9(sums.r));
    auto search_norm = [&](const Vec<T, 9>& d, T reach) {
      T best_step = T(0.0);
      T best = residual;
      bool last_is_best = false;
      T trial_step = reach;
      for (int search = 0; search < kMaxLineSearch; ++search, trial_step = trial_step * T(0.5)) {
        if (!try_pass(axpy(alpha, trial_step, d))) { last_is_best = false; continue; }
        const T n = norm(tail9(sums.r));
        last_is_best = n < best;
        if (last_is_best) { best = n; best_step = trial_step; }
        if (n <= T(kFullStepReduction) * residual) break;
      }
      if (best_step == T(0.0)) return false;
      if (!last_is_best) pass(axpy(alpha, best_step, d));
      alpha = axpy(alpha, best_step, d);
      residual = best;
      return true;
    };
    auto line_search = [&](const Vec<T, 9>& d, const Vec<T, 9>& r0) {
      const T phi0 = dot(d, r0);
      T reach = T(1.0);
      bool evaluated = try_pass(axpy(alpha, T(1.0), d));
      for (int halving = 0; !evaluated && halving < kMaxLineSearch; ++halving) {
        reach = reach * T(0.5);
        evaluated = try_pass(axpy(alpha, reach, d));
      }
      if (!evaluated) return false;
      const T full = norm(tail9(sums.r));
      if (full <= T(kFullStepReduction) * residual ||
          maxabs(tail9(sums.r)) <= T(kLocalTolerance) * maxabs(sums.scale) + T(kLocalRoundOff) * maxabs(sums.floor)) {
        alpha = axpy(alpha, reach, d);
        residual = full;
        return true;
      }
      const T phi1 = dot(d, tail9(sums.r));
      if (!(phi0 < T(0.0)) || !(phi1 > T(0.0)) || !isfinite(phi1)) return search_norm(d, T(0.5) * reach);
      T s0 = T(0.0), f0 = phi0, s1 = reach, f1 = phi1, step = reach;
      int side = 0;
      for (int search = 0; search < kMaxLineSearch; ++search) {
        const T width = s1 - s0;
        step = tclamp((s0 * f1 - s1 * f0) / (f1 - f0), s0 + T(0.1) * width, s1 - T(0.1) * width);
        evaluated = try_pass(axpy(alpha, step, d));
        const T f = evaluated ? dot(d, tail9(sums.r)) : T(std::numeric_limits<double>::infinity());
        if (evaluated && abs(f) <= T(kLineSearchRatio) * abs(phi0)) break;
        if (!evaluated || f > T(0.0)) {
          s1 = step;
          f1 = evaluated ? f : T(0.5) * f1;
          if (side == 1) f0 = f0 * T(0.5);
          side = 1;
        } else {
          s0 = step;
          f0 = f;
          if (side == -1) f1 = f1 * T(0.5);
          side = -1;
        }
      }
      if (!evaluated) {
        if (s0 == T(0.0)) return false;
        step = s0;
        pass(axpy(alpha, step, d));
      }
      alpha = axpy(alpha, step, d);
      residual = norm(tail9(sums.r));
      return true;
    };
    for (;;) {
      const Vec<T, 9> ra = tail9(sums.r);
      const T largest = maxabs(ra);
      const T scale = maxabs(sums.scale);
      const T floor = T(kLocalRoundOff) * maxabs(sums.floor);
      lu.compute(sums.kaa);
      if (!lu.invertible()) throw Failure{kLocalSingular};
      if (largest <= T(kLocalTolerance) * scale + floor || largest == T(0.0)) break;
      if (out.iterations == kMaxLocal || !isfinite(largest)) throw Failure{kLocalNoConverge};
      ++out.iterations;
      const Vec<T, 9> r0 = ra;
      const Mat<T, 9, 9> k0 = sums.kaa;
      Vec<T, 9> newton = lu.solve(r0);
      for (int i = 0; i < 9; ++i) newton[i] = -newton[i];
      Mat<T, 9, 9> sym;
      for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) sym(i, j) = T(0.5) * (k0(i, j) + k0(j, i));
      Mat<T, 9, 9> chol = sym;
      if (llt<T, 9>(chol)) {
        if (line_search(newton, r0)) continue;
      } else {
        if (try_pass(axpy(alpha, T(1.0), newton))) {
          const T full = norm(tail9(sums.r));
          if (full <= T(kFullStepReduction) * residual) {
            alpha = axpy(alpha, T(1.0), newton);
            residual = full;
            continue;
          }
        }
        Vec<T, 9> ev;
        Mat<T, 9, 9> evec;
        sym_eigen<T, 9>(sym, ev, evec);
        const T top = maxabs(ev);
        const T mu = T(kLocalShift) * top - ev[0];
        Mat<T, 9, 9> shifted_m = k0;
        for (int i = 0; i < 9; ++i) shifted_m(i, i) += mu;
        int perm[9];
        lu_partial(shifted_m, perm);
        Vec<T, 9> shifted = lu_partial_solve(shifted_m, perm, r0);
        for (int i = 0; i < 9; ++i) shifted[i] = -shifted[i];
        if (line_search(shifted, r0) || search_norm(newton, T(0.5))) continue;
      }
      // Levenberg-Marquardt fallback (IncompatibleModes.cpp:522-545).
      const Mat<T, 9, 9> normal = mul(tr(k0), k0);
      Vec<T, 9> gradient;
      for (int i = 0; i < 9; ++i) {
        T s = T(0.0);
        for (int j = 0; j < 9; ++j) s += k0(j, i) * r0[j];
        gradient[i] = s;
      }
      T dmax = normal(0, 0);
      for (int i = 1; i < 9; ++i) dmax = tmax(dmax, normal(i, i));
      T mu = T(kLocalMarquardt) * dmax;
      bool moved = false;
      for (int search = 0; search < kMaxLineSearch && !moved; ++search, mu = mu * T(10.0)) {
        Mat<T, 9, 9> a = normal;
        for (int i = 0; i < 9; ++i) a(i, i) += mu;
        if (!llt<T, 9>(a)) continue;  // (normal + mu I) is positive definite for mu > 0
        Vec<T, 9> d = llt_solve(a, gradient);
        for (int i = 0; i < 9; ++i) d[i] = -d[i];
        if (!try_pass(axpy(alpha, T(1.0), d))) continue;
        const T n = norm(tail9(sums.r));
        if (n < residual) {
          alpha = axpy(alpha, T(1.0), d);
          residual = n;
          moved = true;
        }
      }
      if (!moved) throw Failure{kLocalNoDescent};
    }
    accumulate_coupling(want_tangent, sums);
    const Vec<T, 9> correction = lu.solve(tail9(sums.r));
    for (int i = 0; i < 24; ++i) {
      T s = T(0.0);
      for (int j = 0; j < 9; ++j) s += sums.kua(i, j) * correction[j];
      out.force[i] = sums.r[i] - s;
    }
    out.energy = sums.energy;
    if (want_tangent) {
      Mat<T, 9, 24> coupling;
      for (int col = 0; col < 24; ++col) {
        Vec<T, 9> b;
        for (int i = 0; i < 9; ++i) b[i] = symmetric_ ? sums.kua(col, i) : sums.kau(i, col);
        const Vec<T, 9> x = lu.solve(b);
        for (int i = 0; i < 9; ++i) coupling(i, col) = x[i];
      }
      Mat<T, 24, 24> k;
      for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
          T s = T(0.0);
          for (int m = 0; m < 9; ++m) s += sums.kua(i, m) * coupling(m, j);
          k(i, j) = sums.kuu(i, j) - s;
        }
      if (symmetric_) {
        Mat<T, 24, 24> ks;
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) ks(i, j) = T(0.5) * (k(i, j) + k(j, i));
        k = ks;
      }
      out.tangent = k;
    }
    out.alpha = alpha;
  }

  const Material& mat_;
  const std::vector<QPoint>& rule_;
  int kin_;
  bool symmetric_ = true;
  Mat<T, 3, 8> u_;
  Vec<T, 24> ue_;
  std::vector<PointWork<T>> points_;
};

/// elastoplastic_element for the standard Hex8 (src/fem/Elastoplastic.cpp:226-340)
/// with its kinematics (kinematics_of, :104-168): B, B_NL or P B_NL per point,
/// the mean dilatation (B-bar) when `averaged` (the NonlinearSystem's choice,
/// NonlinearSystem.hpp:302-309), the returns, f = sum w b^T sigma and the
/// tangent; logarithmic kinematics assembles its tangent after every return,
/// with the element's mean Kirchhoff pressure and the cross terms of the
/// averaged ln J. Throws Failure.
template <class T>
class StdElement {
 public:
  StdElement(const Material& mat, const std::vector<QPoint>& rule, int kinematics, bool averaged)
      : mat_(mat), rule_(rule), kin_(kinematics), averaged_(averaged && rule.size() > 1) {}

  /// elastoplastic_stress for the standard Hex8 (Elastoplastic.cpp:342-430):
  /// the returns (elastic checks from the committed states) at the strain
  /// the element takes - with mean dilatation the averaged one, which the
  /// Cauchy stress (J-bar) and the averaged log strain follow - and the
  /// point's own deformation for the largest strain and the smallest det F.
  ElementStress stress(const double* x, const T* ue, const std::vector<State<T>>& committed) {
    kinematics_of(x, ue);
    ElementStress out;
    out.min_jacobian = std::numeric_limits<double>::infinity();
    const bool finite = kin_ == kFinite, logarithmic = kin_ == kLogarithmic;
    auto absmax = [](const Mat<T, 3, 3>& m) {
      double v = 0.0;
      for (int i = 0; i < 9; ++i) v = std::max(v, std::fabs(val(m[i])));
      return v;
    };
    for (std::size_t q = 0; q < pts_.size(); ++q) {
      const Pt& p = pts_[q];
      const Response<T> r = plastic_return(mat_, p.strain, committed[q], false);
      Vec<T, 6> cauchy = r.stress, pk = r.stress;
      Mat<T, 3, 3> f = p.h, sym;
      for (int i = 0; i < 3; ++i) f(i, i) += T(1.0);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sym(i, j) = T(0.5) * (p.h(i, j) + p.h(j, i));
      if (logarithmic) {
        pk = logarithmic_stress(p.log, r.stress);
        const Vec<T, 6> tau = voigt_of(mul(mul(f, tensor3(pk)), tr(f)), 1.0);
        Vec<T, 6> strain = p.strain;
        for (int i = 3; i < 6; ++i) strain[i] = T(0.5) * strain[i];
        const T j = exp(strain[0] + strain[1] + strain[2]);
        for (int i = 0; i < 6; ++i) {
          cauchy[i] = tau[i] / j;
          out.kirchhoff[i] += val(tau[i]);
          out.log_strain[i] += val(strain[i]);
          const T own = i < 3 ? p.log.strain[i] : T(0.5) * p.log.strain[i];
          out.max_strain = std::max(out.max_strain, std::fabs(val(own)));
        }
        out.min_jacobian = std::min(out.min_jacobian, val(det3(f)));
      } else if (finite) {
        const T j = det3(f);
        const Vec<T, 6> c = voigt_of(mul(mul(f, tensor3(r.stress)), tr(f)), 1.0);
        for (int i = 0; i < 6; ++i) cauchy[i] = c[i] / j;
        Mat<T, 3, 3> green = sym;
        const Mat<T, 3, 3> hth = mul(tr(p.h), p.h);
        for (int i = 0; i < 9; ++i) green[i] += T(0.5) * hth[i];
        out.max_strain = std::max(out.max_strain, absmax(green));
        out.min_jacobian = std::min(out.min_jacobian, val(j));
      } else {
        out.max_strain = std::max(out.max_strain, absmax(sym));
      }
      for (int i = 0; i < 6; ++i) {
        out.cauchy[i] += val(cauchy[i]);
        out.piola_kirchhoff[i] += val(pk[i]);
      }
      out.max_eqps = std::max(out.max_eqps, val(r.state.eqps));
    }
    const double count = static_cast<double>(pts_.size());
    for (int i = 0; i < 6; ++i) {
      out.cauchy[i] /= count;
      out.piola_kirchhoff[i] /= count;
      out.kirchhoff[i] /= count;
      out.log_strain[i] /= count;
    }
    const double* c = out.cauchy;
    out.von_mises = std::sqrt(0.5 * ((c[0] - c[1]) * (c[0] - c[1]) + (c[1] - c[2]) * (c[1] - c[2]) +
                                     (c[2] - c[0]) * (c[2] - c[0])) +
                              3.0 * (c[3] * c[3] + c[4] * c[4] + c[5] * c[5]));
    if (!finite && !logarithmic) out.min_jacobian = 1.0;
    return out;
  }

  ElementOut<T> evaluate(const double* x, const T* ue, const std::vector<State<T>>& committed,
                         bool want_tangent) {
    kinematics_of(x, ue);
    const bool finite = kin_ == kFinite, logarithmic = kin_ == kLogarithmic;
    ElementOut<T> out;
    for (std::size_t q = 0; q < pts_.size(); ++q) {
      Pt& p = pts_[q];
      const Response<T> r = plastic_return(mat_, p.strain, committed[q], want_tangent);
      const T w = p.weight;
      for (int j = 0; j < 24; ++j) {
        T s = T(0.0);
        for (int c = 0; c < 6; ++c) s += p.b(c, j) * r.stress[c];
        out.force[j] += w * s;
      }
      out.energy += w * r.energy;
      if (logarithmic && want_tangent) {
        p.stress = r.stress;
        p.tangent = r.tangent;
      }
      if (want_tangent && !logarithmic) {
        const Mat<T, 6, 24> cb = mul(r.tangent, p.b);
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            T s = T(0.0);
            for (int c = 0; c < 6; ++c) s += p.b(c, i) * cb(c, j);
            out.tangent(i, j) += w * s;
          }
        if (finite) {
          // S : Delta delta E, with the averaged dilatation
          // (tr S / 3) (Delta delta tr-bar E - Delta delta tr E).
          const Mat<T, 3, 3> st = tensor3(r.stress);
          Mat<T, 8, 8> geo = mul(mul(tr(p.g), st), p.g);
          if (averaged_) {
            const T third = (r.stress[0] + r.stress[1] + r.stress[2]) / T(3.0);
            const Mat<T, 8, 8> gg = mul(tr(p.g), p.g);
            for (int i = 0; i < 64; ++i) geo[i] += third * (gbar_[i] - gg[i]);
          }
          for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b)
              for (int k = 0; k < 3; ++k) out.tangent(3 * a + k, 3 * b + k) += w * geo(a, b);
        }
      }
      if (r.yielding) ++out.yielding;
      out.point_yield.push_back(r.yielding ? 1 : 0);
      out.states.push_back(r.state);
    }
    if (logarithmic && want_tangent) {
      T mean_pressure = T(0.0);
      if (averaged_) {
        T volume = T(0.0);
        for (const Pt& p : pts_) {
          mean_pressure += p.weight * (p.stress[0] + p.stress[1] + p.stress[2]) / T(3.0);
          volume += p.weight;
        }
        mean_pressure /= volume;
      }
      Vec<T, 6> m;
      m[0] = m[1] = m[2] = T(1.0);
      for (const Pt& p : pts_) {
        const T w = p.weight;
        const Mat<T, 6, 6>& proj = p.log.projection;
        Vec<T, 6> t = p.stress;
        if (averaged_) {
          const T shift = mean_pressure - (t[0] + t[1] + t[2]) / T(3.0);
          for (int i = 0; i < 3; ++i) t[i] += shift;
        }
        const Mat<T, 6, 6> pcp = mul(mul(tr(proj), p.tangent), proj);
        const Mat<T, 6, 6> curv = logarithmic_curvature(p.log, t);
        Mat<T, 6, 6> inner;
        for (int i = 0; i < 36; ++i) inner[i] = pcp[i] + curv[i];
        const Mat<T, 6, 24> ib = mul(inner, p.bnl);
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            T s = T(0.0);
            for (int c = 0; c < 6; ++c) s += p.bnl(c, i) * ib(c, j);
            out.tangent(i, j) += w * s;
          }
        if (averaged_) {
          // (A + m s^T/3)^T C (A + m s^T/3) - A^T C A with A = P B_NL.
          const Vec<T, 6> cm = mul(p.tangent, m);
          const Vec<T, 6> mc = mul(tr(p.tangent), m);
          const Vec<T, 24> a_cm = mul(tr(p.bnl), mul(tr(proj), cm));
          const Vec<T, 24> a_mc = mul(tr(p.bnl), mul(tr(proj), mc));
          const T mcm = dot(m, cm) / T(3.0);
          for (int i = 0; i < 24; ++i) {
            const T left = a_cm[i] + mcm * p.shift[i];
            for (int j = 0; j < 24; ++j) out.tangent(i, j) += (w / T(3.0)) * (left * p.shift[j]);
          }
          for (int i = 0; i < 24; ++i)
            for (int j = 0; j < 24; ++j) out.tangent(i, j) += (w / T(3.0)) * (p.shift[i] * a_mc[j]);
        }
        // add_geometric (:60-76) with S' = P^T T'.
        const Mat<T, 3, 3> sd = tensor3(logarithmic_stress(p.log, t));
        const Mat<T, 8, 8> geo = mul(mul(tr(p.g), sd), p.g);
        for (int a = 0; a < 8; ++a)
          for (int b = 0; b < 8; ++b)
            for (int k = 0; k < 3; ++k) out.tangent(3 * a + k, 3 * b + k) += w * geo(a, b);
      }
    }
    out.symmetric = mat_.symmetric();
    if (want_tangent && out.symmetric) {
      for (int i = 0; i < 24; ++i)
        for (int j = i + 1; j < 24; ++j) {
          const T v = T(0.5) * (out.tangent(i, j) + out.tangent(j, i));
          out.tangent(i, j) = v;
          out.tangent(j, i) = v;
        }
    }
    return out;
  }

 private:
  struct Pt {
    Mat<T, 6, 24> b, bnl;
    Vec<T, 6> strain, stress;
    Mat<T, 3, 8> g;
    Mat<T, 3, 3> h;
    T weight = T(0.0);
    LogStrain<T> log;
    Vec<T, 24> shift;
    Mat<T, 6, 6> tangent;
  };

  static Vec<T, 24> dilatation_row(const Mat<T, 6, 24>& b) {
    Vec<T, 24> r;
    for (int j = 0; j < 24; ++j) r[j] = b(0, j) + b(1, j) + b(2, j);
    return r;
  }

  static Mat<T, 6, 24> gl_operator(const Mat<T, 3, 3>& f, const Mat<T, 3, 8>& g) {
    static constexpr int kPair[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {1, 2}, {2, 0}};
    Mat<T, 6, 24> b;
    for (int c = 0; c < 6; ++c) {
      const int i = kPair[c][0], j = kPair[c][1];
      for (int a = 0; a < 8; ++a)
        for (int k = 0; k < 3; ++k)
          b(c, 3 * a + k) = i == j ? f(k, i) * g(i, a) : f(k, i) * g(j, a) + f(k, j) * g(i, a);
    }
    return b;
  }

  // kinematics_of (Elastoplastic.cpp:104-168).
  void kinematics_of(const double* x, const T* ue) {
    Mat<T, 3, 8> u;
    for (int a = 0; a < 8; ++a)
      for (int k = 0; k < 3; ++k) u(k, a) = ue[3 * a + k];
    pts_.assign(rule_.size(), Pt());
    for (std::size_t q = 0; q < rule_.size(); ++q) {
      const QPoint& xi = rule_[q];
      Pt& p = pts_[q];
      const Mat<double, 8, 3> dn = shape_gradients(xi.xi, xi.eta, xi.zeta);
      Mat<T, 3, 3> jac;
      for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) {
          T s = T(0.0);
          for (int a = 0; a < 8; ++a) s += T(x[3 * a + i]) * T(dn(a, c));
          jac(i, c) = s;
        }
      const T det = det3(jac);
      if (!(det > T(0.0))) throw Failure{kMeshInverted};
      const Mat<T, 3, 3> jinv = inv3(jac);
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i) {
          T s = T(0.0);
          for (int c = 0; c < 3; ++c) s += T(dn(a, c)) * jinv(c, i);
          p.g(i, a) = s;
        }
      p.h = mul(u, tr(p.g));
      Mat<T, 3, 3> f = p.h;
      for (int i = 0; i < 3; ++i) f(i, i) += T(1.0);
      if (kin_ == kFinite) {
        p.b = gl_operator(f, p.g);
        p.strain = green_lagrange_6(p.h);
      } else if (kin_ == kLogarithmic) {
        if (!(det3(f) > T(0.0))) throw Failure{kInverted};
        p.bnl = gl_operator(f, p.g);
        p.log = logarithmic_strain(green_lagrange_6(p.h));
        p.strain = p.log.strain;
        p.b = mul(p.log.projection, p.bnl);
      } else {
        Mat<T, 3, 3> id;
        for (int i = 0; i < 3; ++i) id(i, i) = T(1.0);
        p.b = gl_operator(id, p.g);
        for (int c = 0; c < 6; ++c) {
          T s = T(0.0);
          for (int j = 0; j < 24; ++j) s += p.b(c, j) * ue[j];
          p.strain[c] = s;
        }
      }
      p.weight = T(xi.weight) * det;
    }
    if (!averaged_) return;
    Vec<T, 24> mean_row;
    T mean_trace = T(0.0), volume = T(0.0);
    gbar_ = Mat<T, 8, 8>();
    for (const Pt& p : pts_) {
      const Vec<T, 24> d = dilatation_row(p.b);
      for (int j = 0; j < 24; ++j) mean_row[j] += p.weight * d[j];
      mean_trace += p.weight * (p.strain[0] + p.strain[1] + p.strain[2]);
      volume += p.weight;
      if (kin_ == kFinite) {
        const Mat<T, 8, 8> gg = mul(tr(p.g), p.g);
        for (int i = 0; i < 64; ++i) gbar_[i] += p.weight * gg[i];
      }
    }
    for (int j = 0; j < 24; ++j) mean_row[j] /= volume;
    mean_trace /= volume;
    if (kin_ == kFinite)
      for (int i = 0; i < 64; ++i) gbar_[i] /= volume;
    for (Pt& p : pts_) {
      const Vec<T, 24> d = dilatation_row(p.b);
      if (kin_ == kLogarithmic)
        for (int j = 0; j < 24; ++j) p.shift[j] = mean_row[j] - d[j];
      const T shift = (mean_trace - (p.strain[0] + p.strain[1] + p.strain[2])) / T(3.0);
      for (int r = 0; r < 3; ++r) {
        for (int j = 0; j < 24; ++j) p.b(r, j) += (mean_row[j] - d[j]) / T(3.0);
        p.strain[r] += shift;
      }
    }
  }

  const Material& mat_;
  const std::vector<QPoint>& rule_;
  int kin_;
  bool averaged_;
  std::vector<Pt> pts_;
  Mat<T, 8, 8> gbar_;
};

}  // namespace orc
