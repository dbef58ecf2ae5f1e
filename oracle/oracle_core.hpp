// ORACLE — test infrastructure only. A plain CPU restatement of the
// reference's element-level algorithms (sparlab, C++17/Eigen), used by the
// tests, the smoke check and the CPU-baseline leg of bench.py to check the
// results of the CUDA path. Nothing in the product links, includes or calls it.
//
// This header: the material point - hardening laws, the Hill48 yield
// matrix, the J2 radial return, the general (Hill48 / Chaboche)
// closest-point return with its consistent tangent, and the logarithmic
// strain with its first and second derivatives.
//
// Every routine is templated on the scalar so that the same code runs in
// double (the oracle proper) and in a counting scalar (the algorithmic flop
// count reported by bench.py's roofline).
//
// Third-party arithmetic: the reference uses Eigen 3.4.0 (not vendored in
// the reference tree) for its small dense linear algebra. The restatement
// writes the published algorithms by hand: complete-pivoting LU
// (Eigen::FullPivLU: pivot = largest remaining entry, scanned column by
// column, first maximum kept; invertible iff every pivot exceeds n*eps
// times the largest one), partial-pivoting LU (Eigen::PartialPivLU: largest
// entry of the column, first maximum kept), Cholesky (Eigen::LLT: fails at
// the first non-positive pivot), and the symmetric eigenproblem, which here
// is cyclic Jacobi rather than Eigen's tridiagonal QR: eigenvalues agree to
// round-off and every quantity the path uses is invariant under the choice
// of eigenvectors.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace orc {

// ---------------------------------------------------------------------------
// Counting scalar: every +, -, *, / and transcendental counts one flop.
// ---------------------------------------------------------------------------
extern thread_local long long g_flops;

struct CD {
  double v = 0.0;
  CD() = default;
  CD(double x) : v(x) {}  // NOLINT: implicit on purpose (mixed arithmetic)
  explicit operator double() const { return v; }
};
inline CD operator+(CD a, CD b) { ++g_flops; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { ++g_flops; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { ++g_flops; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { ++g_flops; return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }
inline CD& operator+=(CD& a, CD b) { ++g_flops; a.v += b.v; return a; }
inline CD& operator-=(CD& a, CD b) { ++g_flops; a.v -= b.v; return a; }
inline CD& operator*=(CD& a, CD b) { ++g_flops; a.v *= b.v; return a; }
inline CD& operator/=(CD& a, CD b) { ++g_flops; a.v /= b.v; return a; }
inline bool operator<(CD a, CD b) { return a.v < b.v; }
inline bool operator>(CD a, CD b) { return a.v > b.v; }
inline bool operator<=(CD a, CD b) { return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { return a.v >= b.v; }
inline bool operator==(CD a, CD b) { return a.v == b.v; }
inline bool operator!=(CD a, CD b) { return a.v != b.v; }
inline CD sqrt(CD a) { ++g_flops; return CD(std::sqrt(a.v)); }
inline CD log1p(CD a) { ++g_flops; return CD(std::log1p(a.v)); }
inline CD exp(CD a) { ++g_flops; return CD(std::exp(a.v)); }
inline CD expm1(CD a) { ++g_flops; return CD(std::expm1(a.v)); }
inline CD abs(CD a) { return CD(std::fabs(a.v)); }
inline bool isfinite(CD a) { return std::isfinite(a.v); }
inline double val(CD a) { return a.v; }
inline double val(double a) { return a; }

using std::abs;
using std::exp;
using std::expm1;
using std::isfinite;
using std::log1p;
using std::sqrt;

template <class T> inline T tmax(T a, T b) { return a < b ? b : a; }
template <class T> inline T tmin(T a, T b) { return b < a ? b : a; }
template <class T> inline T tclamp(T v, T lo, T hi) { return v < lo ? lo : (hi < v ? hi : v); }

constexpr double kEps = std::numeric_limits<double>::epsilon();
constexpr int kMaxBack = 4;

// ---------------------------------------------------------------------------
// Small fixed-size matrices (row-major).
// ---------------------------------------------------------------------------
template <class T, int R, int C>
struct Mat {
  T a[R * C];
  Mat() { for (int i = 0; i < R * C; ++i) a[i] = T(0.0); }
  T& operator()(int i, int j) { return a[i * C + j]; }
  const T& operator()(int i, int j) const { return a[i * C + j]; }
  T& operator[](int i) { return a[i]; }
  const T& operator[](int i) const { return a[i]; }
};
template <class T, int N> using Vec = Mat<T, N, 1>;

template <class T, int R, int K, int C>
Mat<T, R, C> mul(const Mat<T, R, K>& x, const Mat<T, K, C>& y) {
  Mat<T, R, C> out;
  for (int i = 0; i < R; ++i)
    for (int j = 0; j < C; ++j) {
      T s = T(0.0);
      for (int k = 0; k < K; ++k) s += x(i, k) * y(k, j);
      out(i, j) = s;
    }
  return out;
}
template <class T, int R, int C>
Mat<T, C, R> tr(const Mat<T, R, C>& x) {
  Mat<T, C, R> out;
  for (int i = 0; i < R; ++i)
    for (int j = 0; j < C; ++j) out(j, i) = x(i, j);
  return out;
}
template <class T, int R, int C>
T maxabs(const Mat<T, R, C>& x) {
  T m = abs(x[0]);
  for (int i = 1; i < R * C; ++i) m = tmax(m, abs(x[i]));
  return m;
}
template <class T, int N>
T norm(const Vec<T, N>& v) {
  T s = T(0.0);
  for (int i = 0; i < N; ++i) s += v[i] * v[i];
  return sqrt(s);
}
template <class T, int N>
T dot(const Vec<T, N>& a, const Vec<T, N>& b) {
  T s = T(0.0);
  for (int i = 0; i < N; ++i) s += a[i] * b[i];
  return s;
}
template <class T>
T det3(const Mat<T, 3, 3>& m) {
  // Eigen's 3x3 determinant: cofactor expansion along the first column.
  return m(0, 0) * (m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2)) -
         m(1, 0) * (m(0, 1) * m(2, 2) - m(2, 1) * m(0, 2)) +
         m(2, 0) * (m(0, 1) * m(1, 2) - m(1, 1) * m(0, 2));
}
template <class T>
Mat<T, 3, 3> inv3(const Mat<T, 3, 3>& m) {
  Mat<T, 3, 3> c;  // cofactor matrix transposed (the adjugate)
  c(0, 0) = m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1);
  c(1, 0) = m(1, 2) * m(2, 0) - m(1, 0) * m(2, 2);
  c(2, 0) = m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0);
  const T det = m(0, 0) * c(0, 0) + m(0, 1) * c(1, 0) + m(0, 2) * c(2, 0);
  const T inv = T(1.0) / det;
  c(0, 1) = m(0, 2) * m(2, 1) - m(0, 1) * m(2, 2);
  c(1, 1) = m(0, 0) * m(2, 2) - m(0, 2) * m(2, 0);
  c(2, 1) = m(0, 1) * m(2, 0) - m(0, 0) * m(2, 1);
  c(0, 2) = m(0, 1) * m(1, 2) - m(0, 2) * m(1, 1);
  c(1, 2) = m(0, 2) * m(1, 0) - m(0, 0) * m(1, 2);
  c(2, 2) = m(0, 0) * m(1, 1) - m(0, 1) * m(1, 0);
  for (int i = 0; i < 9; ++i) c[i] = c[i] * inv;
  return c;
}

// ---------------------------------------------------------------------------
// Dense solvers (restated Eigen 3.4.0 algorithms, see the file comment).
// ---------------------------------------------------------------------------

/// Eigen::PartialPivLU, unblocked: in place, row transpositions in `perm`.
template <class T, int N>
void lu_partial(Mat<T, N, N>& a, int (&perm)[N]) {
  for (int k = 0; k < N; ++k) {
    int p = k;
    T big = abs(a(k, k));
    for (int i = k + 1; i < N; ++i)
      if (abs(a(i, k)) > big) { big = abs(a(i, k)); p = i; }
    perm[k] = p;
    if (big != T(0.0)) {
      if (p != k)
        for (int j = 0; j < N; ++j) std::swap(a(k, j), a(p, j));
      for (int i = k + 1; i < N; ++i) a(i, k) = a(i, k) / a(k, k);
    }
    for (int i = k + 1; i < N; ++i)
      for (int j = k + 1; j < N; ++j) a(i, j) -= a(i, k) * a(k, j);
  }
}
template <class T, int N>
Vec<T, N> lu_partial_solve(const Mat<T, N, N>& lu, const int (&perm)[N], Vec<T, N> b) {
  for (int k = 0; k < N; ++k)
    if (perm[k] != k) std::swap(b[k], b[perm[k]]);
  for (int i = 1; i < N; ++i)
    for (int j = 0; j < i; ++j) b[i] -= lu(i, j) * b[j];
  for (int i = N - 1; i >= 0; --i) {
    for (int j = i + 1; j < N; ++j) b[i] -= lu(i, j) * b[j];
    b[i] = b[i] / lu(i, i);
  }
  return b;
}

/// Eigen::FullPivLU: P A Q = L U with complete pivoting.
template <class T, int N>
struct FullPivLU {
  Mat<T, N, N> lu;
  int rowp[N];  // row transpositions
  int colp[N];  // column transpositions
  T maxpivot = T(0.0);
  int nonzero = N;
  void compute(const Mat<T, N, N>& a) {
    lu = a;
    nonzero = N;
    maxpivot = T(0.0);
    for (int k = 0; k < N; ++k) {
      // Largest |entry| of the remaining corner, scanned column-major, the
      // first maximum kept.
      int pr = k, pc = k;
      T big = T(-1.0);
      for (int j = k; j < N; ++j)
        for (int i = k; i < N; ++i)
          if (abs(lu(i, j)) > big) { big = abs(lu(i, j)); pr = i; pc = j; }
      if (big == T(0.0)) {
        nonzero = k;
        for (int i = k; i < N; ++i) { rowp[i] = i; colp[i] = i; }
        break;
      }
      if (big > maxpivot) maxpivot = big;
      rowp[k] = pr;
      colp[k] = pc;
      if (pr != k)
        for (int j = 0; j < N; ++j) std::swap(lu(k, j), lu(pr, j));
      if (pc != k)
        for (int i = 0; i < N; ++i) std::swap(lu(i, k), lu(i, pc));
      for (int i = k + 1; i < N; ++i) lu(i, k) = lu(i, k) / lu(k, k);
      for (int i = k + 1; i < N; ++i)
        for (int j = k + 1; j < N; ++j) lu(i, j) -= lu(i, k) * lu(k, j);
    }
  }
  bool invertible() const {
    if (nonzero < N) return false;
    const T threshold = T(kEps * N) * maxpivot;
    for (int i = 0; i < N; ++i)
      if (!(abs(lu(i, i)) > threshold)) return false;
    return true;
  }
  Vec<T, N> solve(Vec<T, N> b) const {
    for (int k = 0; k < N; ++k)
      if (rowp[k] != k) std::swap(b[k], b[rowp[k]]);
    for (int i = 1; i < N; ++i)
      for (int j = 0; j < i; ++j) b[i] -= lu(i, j) * b[j];
    for (int i = N - 1; i >= 0; --i) {
      for (int j = i + 1; j < N; ++j) b[i] -= lu(i, j) * b[j];
      b[i] = b[i] / lu(i, i);
    }
    for (int k = N - 1; k >= 0; --k)
      if (colp[k] != k) std::swap(b[k], b[colp[k]]);
    return b;
  }
};

/// Eigen::LLT (lower, unblocked): false at the first non-positive pivot.
template <class T, int N>
bool llt(Mat<T, N, N>& a) {
  for (int k = 0; k < N; ++k) {
    T x = a(k, k);
    for (int j = 0; j < k; ++j) x -= a(k, j) * a(k, j);
    if (x <= T(0.0)) return false;
    a(k, k) = sqrt(x);
    for (int i = k + 1; i < N; ++i) {
      T s = a(i, k);
      for (int j = 0; j < k; ++j) s -= a(i, j) * a(k, j);
      a(i, k) = s / a(k, k);
    }
  }
  return true;
}
template <class T, int N>
Vec<T, N> llt_solve(const Mat<T, N, N>& l, Vec<T, N> b) {
  for (int i = 0; i < N; ++i) {
    for (int j = 0; j < i; ++j) b[i] -= l(i, j) * b[j];
    b[i] = b[i] / l(i, i);
  }
  for (int i = N - 1; i >= 0; --i) {
    for (int j = i + 1; j < N; ++j) b[i] -= l(j, i) * b[j];
    b[i] = b[i] / l(i, i);
  }
  return b;
}

/// Symmetric eigenproblem by cyclic Jacobi: eigenvalues ascending in `w`,
/// eigenvectors as the columns of `v`.
template <class T, int N>
void sym_eigen(Mat<T, N, N> a, Vec<T, N>& w, Mat<T, N, N>& v) {
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) v(i, j) = T(i == j ? 1.0 : 0.0);
  for (int sweep = 0; sweep < 60; ++sweep) {
    T off = T(0.0), diag = T(0.0);
    for (int p = 0; p < N; ++p) {
      diag += a(p, p) * a(p, p);
      for (int q = p + 1; q < N; ++q) off += a(p, q) * a(p, q);
    }
    if (off == T(0.0) || off <= T(1.0e-36) * diag) break;
    for (int p = 0; p < N - 1; ++p)
      for (int q = p + 1; q < N; ++q) {
        const T apq = a(p, q);
        if (apq == T(0.0)) continue;
        const T theta = (a(q, q) - a(p, p)) / (T(2.0) * apq);
        const T t = (theta >= T(0.0) ? T(1.0) : T(-1.0)) /
                    (abs(theta) + sqrt(theta * theta + T(1.0)));
        const T c = T(1.0) / sqrt(t * t + T(1.0));
        const T s = t * c;
        for (int k = 0; k < N; ++k) {
          const T akp = a(k, p), akq = a(k, q);
          a(k, p) = c * akp - s * akq;
          a(k, q) = s * akp + c * akq;
        }
        for (int k = 0; k < N; ++k) {
          const T apk = a(p, k), aqk = a(q, k);
          a(p, k) = c * apk - s * aqk;
          a(q, k) = s * apk + c * aqk;
        }
        for (int k = 0; k < N; ++k) {
          const T vkp = v(k, p), vkq = v(k, q);
          v(k, p) = c * vkp - s * vkq;
          v(k, q) = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < N; ++i) w[i] = a(i, i);
  // Sort ascending (selection sort, columns of v follow).
  for (int i = 0; i < N - 1; ++i) {
    int m = i;
    for (int j = i + 1; j < N; ++j)
      if (w[j] < w[m]) m = j;
    if (m != i) {
      std::swap(w[i], w[m]);
      for (int k = 0; k < N; ++k) std::swap(v(k, i), v(k, m));
    }
  }
}

// ---------------------------------------------------------------------------
// Material (reference: include/sparlab/material/Material.hpp:148-257,
// src/material/Material.cpp:73-218).
// ---------------------------------------------------------------------------
struct Material {
  double E = 0.0, nu = 0.0;
  double sy0 = 0.0, H = 0.0, Hkin = 0.0, Q = 0.0, delta = 0.0;
  int criterion = 0;  // 0 von Mises, 1 Hill48
  double P[36] = {};  // yield matrix, tensorial Voigt, global axes
  int nback = 0;
  double Cb[kMaxBack] = {}, gb[kMaxBack] = {};
  int integration = 0;  // 0 exponential, 1 backward Euler

  double shear() const { return E / (2.0 * (1.0 + nu)); }
  double lame() const { return E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)); }
  bool enabled() const { return sy0 > 0.0; }
  bool general() const { return criterion == 1 || nback > 0; }
  bool symmetric() const {
    for (int i = 0; i < nback; ++i)
      if (gb[i] > 0.0) return false;
    return true;
  }
  int kin_terms() const { return nback + (Hkin > 0.0 ? 1 : 0); }
  double term_modulus(int i) const { return i < nback ? Cb[i] : Hkin; }
  double term_recovery(int i) const { return i < nback ? gb[i] : 0.0; }
  // Material.cpp:73-90.
  template <class T> T yield(T a) const { return T(sy0) + T(H) * a + T(Q) * -expm1(T(-delta) * a); }
  template <class T> T yield_slope(T a) const { return T(H) + T(Q) * T(delta) * exp(T(-delta) * a); }
  template <class T> T isotropic_energy(T a) const {
    T out = T(0.5) * T(H) * a * a;
    if (Q != 0.0) out += T(Q) * (a + expm1(T(-delta) * a) / T(delta));
    return out;
  }
};

/// The von Mises yield matrix (Material.cpp:92-102).
inline void von_mises_matrix(double* p) {
  for (int i = 0; i < 36; ++i) p[i] = 0.0;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) p[i * 6 + j] = -0.5;
    p[i * 6 + i] = 1.0;
    p[(3 + i) * 6 + 3 + i] = 3.0;
  }
}

/// Hill48 from r-values (RValues calibration) in the frame of `rd`, `nd`
/// (Material.cpp:117-129, 135-217). Returns false on an invalid set.
inline bool hill_from_r(double r0, double r45, double r90, double shear_l, double shear_m,
                        const double rd_in[3], const double nd_in[3], double* p_out) {
  if (!(r0 > 0 && r45 > 0 && r90 > 0)) return false;
  const double G = 1.0 / (1.0 + r0);
  const double H = r0 / (1.0 + r0);
  const double F = r0 / (r90 * (1.0 + r0));
  const double N = (r0 + r90) * (1.0 + 2.0 * r45) / (2.0 * r90 * (1.0 + r0));
  const double L = shear_l, M = shear_m;
  double nd[3], rd[3];
  double nn = std::sqrt(nd_in[0] * nd_in[0] + nd_in[1] * nd_in[1] + nd_in[2] * nd_in[2]);
  double rn = std::sqrt(rd_in[0] * rd_in[0] + rd_in[1] * rd_in[1] + rd_in[2] * rd_in[2]);
  if (!(nn > 0 && rn > 0)) return false;
  for (int i = 0; i < 3; ++i) { nd[i] = nd_in[i] / nn; rd[i] = rd_in[i] / rn; }
  const double d = rd[0] * nd[0] + rd[1] * nd[1] + rd[2] * nd[2];
  for (int i = 0; i < 3; ++i) rd[i] -= d * nd[i];
  rn = std::sqrt(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
  if (!(rn > 1.0e-6)) return false;
  for (int i = 0; i < 3; ++i) rd[i] /= rn;
  const double td[3] = {nd[1] * rd[2] - nd[2] * rd[1], nd[2] * rd[0] - nd[0] * rd[2],
                        nd[0] * rd[1] - nd[1] * rd[0]};
  double q[3][3];
  for (int i = 0; i < 3; ++i) { q[0][i] = rd[i]; q[1][i] = td[i]; q[2][i] = nd[i]; }
  double pm[6][6] = {};
  pm[0][0] = G + H; pm[1][1] = F + H; pm[2][2] = F + G;
  pm[0][1] = pm[1][0] = -H; pm[1][2] = pm[2][1] = -F; pm[0][2] = pm[2][0] = -G;
  pm[3][3] = 2.0 * N; pm[4][4] = 2.0 * L; pm[5][5] = 2.0 * M;
  // stress_rotation(q): column k is the Voigt image of q e_k q^T.
  static const int ii[6] = {0, 1, 2, 0, 1, 2};
  static const int jj[6] = {0, 1, 2, 1, 2, 0};
  double t[6][6];
  for (int k = 0; k < 6; ++k) {
    double e[3][3] = {};
    e[ii[k]][jj[k]] = 1.0;
    e[jj[k]][ii[k]] = 1.0;
    double r[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double s = 0.0;
        for (int c = 0; c < 3; ++c)
          for (int dd = 0; dd < 3; ++dd) s += q[a][c] * e[c][dd] * q[b][dd];
        r[a][b] = s;
      }
    for (int row = 0; row < 6; ++row) t[row][k] = r[ii[row]][jj[row]];
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) s += t[a][i] * pm[a][b] * t[b][j];
      p_out[i * 6 + j] = s;
    }
  return true;
}

// ---------------------------------------------------------------------------
// Plastic state and response (include/sparlab/material/Plasticity.hpp:185-214).
// ---------------------------------------------------------------------------
template <class T>
struct State {
  T ep[6];            // plastic strain, engineering shears
  T beta[6];          // whole back stress, tensorial
  T alpha[kMaxBack][6];
  T eqps;
  T thick;
  bool loading;
  State() : eqps(0.0), thick(0.0), loading(false) {
    for (int i = 0; i < 6; ++i) { ep[i] = T(0.0); beta[i] = T(0.0); }
    for (int b = 0; b < kMaxBack; ++b)
      for (int i = 0; i < 6; ++i) alpha[b][i] = T(0.0);
  }
};

template <class T>
struct Response {
  Vec<T, 6> stress;
  Mat<T, 6, 6> tangent;
  State<T> state;
  bool yielding = false;
  T energy = T(0.0);
  T strain33 = T(0.0);
  bool symmetric = true;
};

/// Failures the reference throws as SolverError / MeshError; the code is the
/// element status of the C ABI.
struct Failure {
  int code;
};
enum FailCode {
  kInverted = 1,        // det F <= 0 at a point (logarithmic kinematics)
  kReturnFail = 2,      // the return did not converge / non-finite trial
  kLocalNoConverge = 3, // 25 local iterations, or a non-finite residual
  kLocalSingular = 4,   // K_aa not invertible
  kLocalNoDescent = 5,  // no step lowers |r_alpha|
  kMeshInverted = 6,    // det J <= 0 in the reference configuration
  kNonFinite = 7,       // non-finite Green-Lagrange strain
  kDegenerate = 8,      // a principal stretch squared <= 0
};

template <class T>
T tensor_norm(const Vec<T, 6>& v) {
  return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] +
              T(2.0) * (v[3] * v[3] + v[4] * v[4] + v[5] * v[5]));
}
template <class T>
Vec<T, 6> deviatoric_stress(T g, const Vec<T, 6>& s) {
  const T mean = (s[0] + s[1] + s[2]) / T(3.0);
  Vec<T, 6> o;
  for (int i = 0; i < 3; ++i) o[i] = T(2.0) * g * (s[i] - mean);
  for (int i = 3; i < 6; ++i) o[i] = g * s[i];
  return o;
}
template <class T>
T deviatoric_norm2(const Vec<T, 6>& s) {
  const T mean = (s[0] + s[1] + s[2]) / T(3.0);
  T out = T(0.0);
  for (int i = 0; i < 3; ++i) out += (s[i] - mean) * (s[i] - mean);
  for (int i = 3; i < 6; ++i) out += T(0.5) * s[i] * s[i];
  return out;
}
template <class T>
T strain_norm2(const T* s) {
  T out = T(0.0);
  for (int i = 0; i < 3; ++i) out += s[i] * s[i];
  for (int i = 3; i < 6; ++i) out += T(0.5) * s[i] * s[i];
  return out;
}
template <class T>
Mat<T, 6, 6> elastic_tangent(T k, T g) {
  Mat<T, 6, 6> c;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) c(i, j) = k - T(2.0) * g / T(3.0);
    c(i, i) = k + T(4.0) * g / T(3.0);
    c(3 + i, 3 + i) = g;
  }
  return c;
}

/// The J2 radial return (Plasticity.cpp:66-171).
template <class T>
Response<T> return_3d(const Material& m, const Vec<T, 6>& strain, const State<T>& committed) {
  const T g = T(m.shear());
  const T k = T(m.lame()) + T(2.0) * g / T(3.0);
  const T hk = T(m.Hkin);
  Vec<T, 6> elastic;
  for (int i = 0; i < 6; ++i) elastic[i] = strain[i] - committed.ep[i];
  const T volumetric = elastic[0] + elastic[1] + elastic[2];
  const Vec<T, 6> s_trial = deviatoric_stress(g, elastic);
  Vec<T, 6> xi_trial;
  for (int i = 0; i < 6; ++i) xi_trial[i] = s_trial[i] - committed.beta[i];
  const T xi_norm = tensor_norm(xi_trial);
  const T alpha_n = committed.eqps;
  const T sq23 = T(std::sqrt(2.0 / 3.0));
  const T radius_n = sq23 * m.yield(alpha_n);
  const T f_trial = xi_norm - radius_n;

  Response<T> out;
  out.state = committed;
  out.state.loading = false;
  out.strain33 = strain[2];
  if (!m.enabled() || f_trial <= T(1.0e-12) * radius_n) {
    out.stress = s_trial;
    for (int i = 0; i < 3; ++i) out.stress[i] += k * volumetric;
    out.tangent = elastic_tangent(k, g);
    out.energy = T(0.5) * k * volumetric * volumetric + g * deviatoric_norm2(elastic) +
                 m.isotropic_energy(alpha_n) + hk / T(3.0) * strain_norm2(committed.ep);
    if (m.enabled() && committed.loading && f_trial > T(-1.0e-10) * radius_n && xi_norm > T(0.0)) {
      Vec<T, 6> n;
      for (int i = 0; i < 6; ++i) n[i] = xi_trial[i] / xi_norm;
      const T f = T(2.0) * g / (T(1.0) + (m.yield_slope(alpha_n) + hk) / (T(3.0) * g));
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) out.tangent(i, j) -= f * (n[i] * n[j]);
      out.state.loading = true;
    }
    return out;
  }
  const T stiffness = T(2.0) * g + T(2.0) / T(3.0) * hk;
  T dgamma = f_trial / (stiffness + T(2.0) / T(3.0) * m.yield_slope(alpha_n));
  if (m.Q != 0.0) {
    dgamma = T(0.0);
    bool converged = false;
    for (int it = 0; it < 60; ++it) {
      const T alpha = alpha_n + sq23 * dgamma;
      const T residual = xi_norm - stiffness * dgamma - sq23 * m.yield(alpha);
      if (abs(residual) <= T(1.0e-13) * radius_n) { converged = true; break; }
      dgamma += residual / (stiffness + T(2.0) / T(3.0) * m.yield_slope(alpha));
    }
    if (!converged) {
      const T alpha = alpha_n + sq23 * dgamma;
      const T residual = xi_norm - stiffness * dgamma - sq23 * m.yield(alpha);
      converged = abs(residual) <= T(8.0 * kEps) * xi_norm;
    }
    if (!converged) throw Failure{kReturnFail};
  }
  const T alpha = alpha_n + sq23 * dgamma;
  Vec<T, 6> n;
  for (int i = 0; i < 6; ++i) n[i] = xi_trial[i] / xi_norm;
  out.yielding = true;
  for (int i = 0; i < 6; ++i) out.stress[i] = s_trial[i] - T(2.0) * g * dgamma * n[i];
  for (int i = 0; i < 3; ++i) out.stress[i] += k * volumetric;
  State<T>& st = out.state;
  st.loading = true;
  st.eqps = alpha;
  for (int i = 0; i < 6; ++i) st.beta[i] += T(2.0) / T(3.0) * hk * dgamma * n[i];
  for (int i = 0; i < 3; ++i) st.ep[i] += dgamma * n[i];
  for (int i = 3; i < 6; ++i) st.ep[i] += T(2.0) * dgamma * n[i];
  const T theta = T(1.0) - T(2.0) * g * dgamma / xi_norm;
  const T theta_bar = T(1.0) / (T(1.0) + (m.yield_slope(alpha) + hk) / (T(3.0) * g)) - (T(1.0) - theta);
  Mat<T, 6, 6> c;
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) c(i, j) = k - T(2.0) * g * theta / T(3.0);
    c(i, i) = k + T(4.0) * g * theta / T(3.0);
    c(3 + i, 3 + i) = g * theta;
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) c(i, j) -= T(2.0) * g * theta_bar * (n[i] * n[j]);
  out.tangent = c;
  Vec<T, 6> elastic_new = elastic;
  for (int i = 0; i < 3; ++i) elastic_new[i] -= dgamma * n[i];
  for (int i = 3; i < 6; ++i) elastic_new[i] -= T(2.0) * dgamma * n[i];
  out.energy = T(0.5) * k * volumetric * volumetric + g * deviatoric_norm2(elastic_new) +
               m.isotropic_energy(alpha) + hk / T(3.0) * strain_norm2(st.ep);
  return out;
}

// --- The general return (Plasticity.cpp:178-471) ---------------------------
template <class T>
struct Decay {
  T theta = T(1.0), chi = T(0.0), dtheta = T(0.0), dchi = T(1.0);
};
template <class T>
Decay<T> decay(double gamma, T dl, int integration) {
  Decay<T> d;
  if (gamma == 0.0) { d.chi = dl; return d; }
  if (integration == 0) {
    d.theta = exp(T(-gamma) * dl);
    d.chi = -expm1(T(-gamma) * dl) / T(gamma);
    d.dtheta = T(-gamma) * d.theta;
    d.dchi = d.theta;
  } else {
    d.theta = T(1.0) / (T(1.0) + T(gamma) * dl);
    d.chi = d.theta * dl;
    d.dtheta = T(-gamma) * d.theta * d.theta;
    d.dchi = d.theta * d.theta;
  }
  return d;
}

template <class T>
struct GeneralPoint {
  T equivalent = T(0.0);
  Vec<T, 6> m, mt;
  T b = T(0.0), db = T(0.0);
  Vec<T, 6> back_rate;
  Decay<T> decays[kMaxBack];
  Vec<T, 7> residual;
};

template <class T>
struct GeneralReturn {
  const Material& mat;
  T g;
  const State<T>& committed;
  const Vec<T, 6>& s_trial;
  int count;
  GeneralReturn(const Material& m, const State<T>& c, const Vec<T, 6>& st)
      : mat(m), g(T(m.shear())), committed(c), s_trial(st), count(m.kin_terms()) {}

  bool evaluate(const Vec<T, 6>& xi, T dl, GeneralPoint<T>& e) const {
    Vec<T, 6> pxi;
    for (int i = 0; i < 6; ++i) {
      T s = T(0.0);
      for (int j = 0; j < 6; ++j) s += T(mat.P[i * 6 + j]) * xi[j];
      pxi[i] = s;
    }
    const T q = dot(xi, pxi);
    if (!(q > T(0.0)) || !isfinite(q)) return false;
    e.equivalent = sqrt(q);
    for (int i = 0; i < 6; ++i) e.m[i] = pxi[i] / e.equivalent;
    e.mt = e.m;
    for (int i = 3; i < 6; ++i) e.mt[i] = e.mt[i] * T(0.5);
    Vec<T, 6> xi_tilde = s_trial;
    e.b = T(2.0) * g * dl;
    e.db = T(2.0) * g;
    for (int i = 0; i < 6; ++i) e.back_rate[i] = T(0.0);
    for (int i = 0; i < count; ++i) {
      const Decay<T> d = decay(mat.term_recovery(i), dl, mat.integration);
      const T* an = committed.alpha[i];
      for (int c = 0; c < 6; ++c) xi_tilde[c] -= d.theta * an[c];
      e.b += T(2.0) / T(3.0) * T(mat.term_modulus(i)) * d.chi;
      e.db += T(2.0) / T(3.0) * T(mat.term_modulus(i)) * d.dchi;
      for (int c = 0; c < 6; ++c) e.back_rate[c] += d.dtheta * an[c];
      e.decays[i] = d;
    }
    for (int c = 0; c < 6; ++c) e.residual[c] = xi[c] - xi_tilde[c] + e.b * e.mt[c];
    e.residual[6] = e.equivalent - mat.yield(committed.eqps + dl);
    return true;
  }
  Mat<T, 6, 6> flow_curvature(const GeneralPoint<T>& e) const {
    Mat<T, 6, 6> c;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) c(i, j) = T(mat.P[i * 6 + j]) - e.m[i] * e.m[j];
    for (int i = 3; i < 6; ++i)
      for (int j = 0; j < 6; ++j) c(i, j) = c(i, j) * T(0.5);
    return c;
  }
  Mat<T, 7, 7> jacobian(const GeneralPoint<T>& e, T dl) const {
    Mat<T, 7, 7> j;
    const Mat<T, 6, 6> fc = flow_curvature(e);
    const T f = e.b / e.equivalent;
    for (int r = 0; r < 6; ++r)
      for (int c = 0; c < 6; ++c) j(r, c) = T(r == c ? 1.0 : 0.0) + f * fc(r, c);
    for (int r = 0; r < 6; ++r) j(r, 6) = e.back_rate[r] + e.db * e.mt[r];
    for (int c = 0; c < 6; ++c) j(6, c) = e.m[c];
    j(6, 6) = -mat.yield_slope(committed.eqps + dl);
    return j;
  }
  Mat<T, 6, 6> tangent(const GeneralPoint<T>& e, T dl, const Mat<T, 6, 6>& elastic) const {
    // rhs = [D_dev; 0], solved column by column with one LU.
    Mat<T, 7, 7> lu = jacobian(e, dl);
    int perm[7];
    lu_partial(lu, perm);
    Mat<T, 7, 6> da;
    for (int col = 0; col < 6; ++col) {
      Vec<T, 7> rhs;
      for (int i = 0; i < 3; ++i) rhs[i] = (col < 3) ? (i == col ? T(4.0) * g / T(3.0) : T(-2.0) * g / T(3.0)) : T(0.0);
      for (int i = 3; i < 6; ++i) rhs[i] = (i == col) ? g : T(0.0);
      rhs[6] = T(0.0);
      const Vec<T, 7> x = lu_partial_solve(lu, perm, rhs);
      for (int i = 0; i < 7; ++i) da(i, col) = x[i];
    }
    Mat<T, 6, 6> c = elastic;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) c(i, j) -= T(2.0) * g * (e.mt[i] * da(6, j));
    if (dl > T(0.0)) {
      const Mat<T, 6, 6> fc = flow_curvature(e);
      const T f = T(2.0) * g * dl / e.equivalent;
      for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
          T s = T(0.0);
          for (int k = 0; k < 6; ++k) s += fc(i, k) * da(k, j);
          c(i, j) -= f * s;
        }
    }
    return c;
  }
};

template <class T>
T kinematic_energy(const Material& m, const State<T>& st) {
  T out = T(0.0);
  for (int i = 0; i < m.kin_terms(); ++i) {
    Vec<T, 6> v;
    for (int c = 0; c < 6; ++c) v[c] = st.alpha[i][c];
    const T norm = tensor_norm(v);
    out += T(0.75) * norm * norm / T(m.term_modulus(i));
  }
  return out;
}

/// Plasticity.cpp:337-471.
template <class T>
Response<T> return_general_3d(const Material& m, const Vec<T, 6>& strain,
                              const State<T>& committed, bool want_tangent) {
  const T g = T(m.shear());
  const T k = T(m.lame()) + T(2.0) * g / T(3.0);
  Vec<T, 6> elastic;
  for (int i = 0; i < 6; ++i) elastic[i] = strain[i] - committed.ep[i];
  const T volumetric = elastic[0] + elastic[1] + elastic[2];
  const Vec<T, 6> s_trial = deviatoric_stress(g, elastic);
  const GeneralReturn<T> gr(m, committed, s_trial);
  Vec<T, 6> xi_trial = s_trial;
  for (int i = 0; i < gr.count; ++i)
    for (int c = 0; c < 6; ++c) xi_trial[c] -= committed.alpha[i][c];
  const T alpha_n = committed.eqps;
  const T sy_n = m.yield(alpha_n);
  T q = T(0.0);
  for (int i = 0; i < 6; ++i) {
    T s = T(0.0);
    for (int j = 0; j < 6; ++j) s += T(m.P[i * 6 + j]) * xi_trial[j];
    q += xi_trial[i] * s;
  }
  const T eq_trial = sqrt(tmax(q, T(0.0)));
  const T f_trial = eq_trial - sy_n;
  const Mat<T, 6, 6> ce = elastic_tangent(k, g);
  if (!isfinite(f_trial)) throw Failure{kReturnFail};

  Response<T> out;
  out.state = committed;
  out.state.loading = false;
  out.strain33 = strain[2];
  if (!m.enabled() || f_trial <= T(1.0e-12) * sy_n) {
    out.stress = s_trial;
    for (int i = 0; i < 3; ++i) out.stress[i] += k * volumetric;
    out.tangent = ce;
    out.energy = T(0.5) * k * volumetric * volumetric + g * deviatoric_norm2(elastic) +
                 m.isotropic_energy(alpha_n) + kinematic_energy(m, committed);
    if (m.enabled() && committed.loading && f_trial > T(-1.0e-10) * sy_n && eq_trial > T(0.0)) {
      out.state.loading = true;
      GeneralPoint<T> e;
      if (want_tangent && gr.evaluate(xi_trial, T(0.0), e)) out.tangent = gr.tangent(e, T(0.0), ce);
    }
    return out;
  }
  Vec<T, 6> xi = xi_trial;
  T dl = T(0.0);
  GeneralPoint<T> e;
  gr.evaluate(xi, dl, e);
  T scale = sy_n;
  for (int i = 0; i < 6; ++i) scale = tmax(scale, abs(s_trial[i]));
  for (int i = 0; i < 6; ++i) scale = tmax(scale, abs(xi_trial[i]));
  const T eps_scale = T(kEps) * scale;
  const T tol = tmax(T(1.0e-13) * sy_n, T(32.0) * eps_scale);
  bool converged = false;
  for (int it = 0; it < 50; ++it) {
    const T r_inf = maxabs(e.residual);
    if (r_inf <= tol) { converged = true; break; }
    Mat<T, 7, 7> lu = gr.jacobian(e, dl);
    int perm[7];
    lu_partial(lu, perm);
    Vec<T, 7> rhs;
    for (int i = 0; i < 7; ++i) rhs[i] = -e.residual[i];
    const Vec<T, 7> step = lu_partial_solve(lu, perm, rhs);
    const T r0 = norm(e.residual);
    T t = T(1.0);
    bool accepted = false;
    GeneralPoint<T> trial;
    for (int ls = 0; ls < 40; ++ls) {
      Vec<T, 6> xi_t;
      for (int i = 0; i < 6; ++i) xi_t[i] = xi[i] + t * step[i];
      const T dl_t = tmax(dl + t * step[6], T(0.0));
      if (gr.evaluate(xi_t, dl_t, trial) && norm(trial.residual) <= (T(1.0) - T(1.0e-4) * t) * r0) {
        xi = xi_t;
        dl = dl_t;
        e = trial;
        accepted = true;
        break;
      }
      t = t * T(0.5);
    }
    if (!accepted) {
      converged = r_inf <= T(4.0) * tol;
      break;
    }
  }
  if (!converged) throw Failure{kReturnFail};
  if (maxabs(e.residual) > T(4.0) * eps_scale) {
    Mat<T, 7, 7> lu = gr.jacobian(e, dl);
    int perm[7];
    lu_partial(lu, perm);
    Vec<T, 7> rhs;
    for (int i = 0; i < 7; ++i) rhs[i] = -e.residual[i];
    const Vec<T, 7> step = lu_partial_solve(lu, perm, rhs);
    Vec<T, 6> xi_p;
    for (int i = 0; i < 6; ++i) xi_p[i] = xi[i] + step[i];
    const T dl_p = tmax(dl + step[6], T(0.0));
    GeneralPoint<T> polished;
    if (gr.evaluate(xi_p, dl_p, polished) && maxabs(polished.residual) < maxabs(e.residual)) {
      xi = xi_p;
      dl = dl_p;
      e = polished;
    }
  }
  out.yielding = true;
  out.symmetric = m.symmetric();
  for (int i = 0; i < 6; ++i) out.stress[i] = s_trial[i] - T(2.0) * g * dl * e.mt[i];
  for (int i = 0; i < 3; ++i) out.stress[i] += k * volumetric;
  State<T>& st = out.state;
  st.loading = true;
  st.eqps = alpha_n + dl;
  for (int i = 0; i < 6; ++i) st.ep[i] += dl * e.m[i];
  for (int i = 0; i < 6; ++i) st.beta[i] = T(0.0);
  for (int b = 0; b < gr.count; ++b) {
    const Decay<T>& d = e.decays[b];
    const T f = T(2.0) / T(3.0) * T(m.term_modulus(b)) * d.chi;
    for (int c = 0; c < 6; ++c) st.alpha[b][c] = d.theta * committed.alpha[b][c] + f * e.mt[c];
    for (int c = 0; c < 6; ++c) st.beta[c] += st.alpha[b][c];
  }
  Vec<T, 6> elastic_new;
  for (int i = 0; i < 6; ++i) elastic_new[i] = elastic[i] - dl * e.m[i];
  out.energy = T(0.5) * k * volumetric * volumetric + g * deviatoric_norm2(elastic_new) +
               m.isotropic_energy(st.eqps) + kinematic_energy(m, st);
  out.tangent = want_tangent ? gr.tangent(e, dl, ce) : ce;
  return out;
}

/// Plasticity.cpp:513-539, three-dimensional stress state.
template <class T>
Response<T> plastic_return(const Material& m, const Vec<T, 6>& strain, const State<T>& committed,
                           bool want_tangent) {
  if (!m.general()) return return_3d(m, strain, committed);
  return return_general_3d(m, strain, committed, want_tangent);
}

// ---------------------------------------------------------------------------
// Logarithmic strain (src/material/LogarithmicStrain.cpp:1-199).
// ---------------------------------------------------------------------------
constexpr int kRow[6] = {0, 1, 2, 0, 1, 2};
constexpr int kCol[6] = {0, 1, 2, 1, 2, 0};
constexpr double kSpread = 5.0e-3;

template <class T>
struct LogStrain {
  Mat<T, 3, 3> axes;  // columns N_a
  Vec<T, 3> green;    // principal Green-Lagrange strains
  Vec<T, 6> strain;   // E_log, engineering shears
  Mat<T, 6, 6> projection;
  Mat<T, 3, 3> first;
};

template <class T>
T log_divided(T mx, T my) {
  if (mx > my) std::swap(mx, my);
  const T y = T(1.0) + T(2.0) * my;
  const T d = T(2.0) * (mx - my);
  if (d == T(0.0)) return T(1.0) / y;
  return log1p(d / y) / d;
}

template <class T>
T log_divided2(const Vec<T, 3>& mu, const Mat<T, 3, 3>& first, int a, int b, int c) {
  int i = a, j = b, k = c;
  if (mu[i] < mu[j]) std::swap(i, j);
  if (mu[j] < mu[k]) std::swap(j, k);
  if (mu[i] < mu[j]) std::swap(i, j);
  const T y = T(1.0) + T(2.0) * mu[j];
  const T spread = T(2.0) * (mu[i] - mu[k]);
  if (spread > T(kSpread) * y) return (first(i, j) - first(j, k)) / spread;
  const T u = T(2.0) * (mu[i] - mu[j]) / y;
  const T w = T(2.0) * (mu[k] - mu[j]) / y;
  T h = T(1.0), wn = T(1.0), sum = T(-0.5);
  for (int n = 1; n <= 5; ++n) {
    wn = wn * w;
    h = u * h + wn;
    sum += T(n % 2 == 1 ? 1.0 : -1.0) * h / T(double(n + 2));
  }
  return sum / (y * y);
}

template <class T>
Mat<T, 3, 3> tensor_of(const Vec<T, 6>& v, double shear) {
  Mat<T, 3, 3> t;
  t(0, 0) = v[0]; t(1, 1) = v[1]; t(2, 2) = v[2];
  t(0, 1) = t(1, 0) = T(shear) * v[3];
  t(1, 2) = t(2, 1) = T(shear) * v[4];
  t(2, 0) = t(0, 2) = T(shear) * v[5];
  return t;
}
template <class T>
Vec<T, 6> voigt_of(const Mat<T, 3, 3>& t, double shear) {
  Vec<T, 6> v;
  v[0] = t(0, 0); v[1] = t(1, 1); v[2] = t(2, 2);
  v[3] = T(shear) * t(0, 1); v[4] = T(shear) * t(1, 2); v[5] = T(shear) * t(2, 0);
  return v;
}
template <class T>
Mat<T, 6, 6> principal_rotation(const Mat<T, 3, 3>& q) {
  Mat<T, 6, 6> m;
  for (int r = 0; r < 6; ++r) {
    const int a = kRow[r], b = kCol[r];
    for (int c = 0; c < 6; ++c) {
      const int i = kRow[c], j = kCol[c];
      m(r, c) = i == j ? q(i, a) * q(i, b) : q(i, a) * q(j, b) + q(j, a) * q(i, b);
    }
  }
  return m;
}

template <class T>
LogStrain<T> logarithmic_strain(const Vec<T, 6>& green) {
  for (int i = 0; i < 6; ++i)
    if (!isfinite(green[i])) throw Failure{kNonFinite};
  LogStrain<T> out;
  sym_eigen<T, 3>(tensor_of(green, 0.5), out.green, out.axes);
  Vec<T, 3> principal;
  for (int a = 0; a < 3; ++a) {
    const T stretch2 = T(1.0) + T(2.0) * out.green[a];
    if (!(stretch2 > T(0.0)) || !isfinite(stretch2)) throw Failure{kDegenerate};
    principal[a] = T(0.5) * log1p(T(2.0) * out.green[a]);
  }
  const Mat<T, 3, 3>& q = out.axes;
  Mat<T, 3, 3> e;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      T s = T(0.0);
      for (int a = 0; a < 3; ++a) s += q(i, a) * principal[a] * q(j, a);
      e(i, j) = s;
    }
  out.strain = voigt_of(e, 2.0);
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) out.first(a, b) = out.first(b, a) = log_divided(out.green[a], out.green[b]);
  const Mat<T, 6, 6> m = principal_rotation(q);
  Vec<T, 6> sd;
  for (int k = 0; k < 6; ++k) sd[k] = T(k < 3 ? 1.0 : 2.0) * out.first(kRow[k], kCol[k]);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      T s = T(0.0);
      for (int k = 0; k < 6; ++k) s += m(k, i) * sd[k] * m(k, j);
      out.projection(i, j) = j >= 3 ? s * T(0.5) : s;
    }
  return out;
}

template <class T>
Vec<T, 6> logarithmic_stress(const LogStrain<T>& log, const Vec<T, 6>& t) {
  const Mat<T, 3, 3>& q = log.axes;
  const Mat<T, 3, 3> tt = tensor_of(t, 1.0);
  Mat<T, 3, 3> p = mul(mul(tr(q), tt), q);
  for (int i = 0; i < 9; ++i) p[i] = p[i] * log.first[i];
  return voigt_of(mul(mul(q, p), tr(q)), 1.0);
}

template <class T>
Mat<T, 6, 6> logarithmic_curvature(const LogStrain<T>& log, const Vec<T, 6>& t) {
  const Mat<T, 3, 3>& q = log.axes;
  const Mat<T, 3, 3> tp = mul(mul(tr(q), tensor_of(t, 1.0)), q);
  T second[27];
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b)
      for (int c = b; c < 3; ++c) {
        const T v = log_divided2(log.green, log.first, a, b, c);
        const int perm[6][3] = {{a, b, c}, {a, c, b}, {b, a, c}, {b, c, a}, {c, a, b}, {c, b, a}};
        for (const auto& i : perm) second[i[0] + 3 * i[1] + 9 * i[2]] = v;
      }
  auto entries = [](int k, int (&rows)[2], int (&cols)[2]) {
    rows[0] = kRow[k]; cols[0] = kCol[k];
    rows[1] = kCol[k]; cols[1] = kRow[k];
    return k < 3 ? 1 : 2;
  };
  auto half = [&](int kx, int ky) {
    int xr[2], xc[2], yr[2], yc[2];
    const int nx = entries(kx, xr, xc);
    const int ny = entries(ky, yr, yc);
    T sum = T(0.0);
    for (int s = 0; s < nx; ++s) {
      const int a = xr[s], c = xc[s];
      for (int r = 0; r < ny; ++r) {
        if (yr[r] != c) continue;
        const int b = yc[r];
        sum += tp(a, b) * second[a + 3 * b + 9 * c];
      }
    }
    return sum;
  };
  Mat<T, 6, 6> hp;
  for (int k = 0; k < 6; ++k)
    for (int l = k; l < 6; ++l) hp(k, l) = hp(l, k) = T(2.0) * (half(k, l) + half(l, k));
  Mat<T, 6, 6> m = principal_rotation(q);
  for (int r = 0; r < 6; ++r)
    for (int c = 3; c < 6; ++c) m(r, c) = m(r, c) * T(0.5);
  return mul(mul(tr(m), hp), m);
}

}  // namespace orc
