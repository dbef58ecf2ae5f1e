// ORACLE — test infrastructure only (see oracle_core.hpp). Built into
// oracle/_build/liboracle.so and called through ctypes by the tests, the
// smoke check and bench.py's CPU-baseline leg; the product never links it.
//
// The system level of the reference, restated:
//  - the element loop of detail::NonlinearSystem::evaluate with its serial
//    gather of f_int, the gross norm, the energy and the yield count
//    (src/fem/NonlinearSystem.hpp:192-268), OpenMP static over elements as
//    in the reference;
//  - the node-block sparsity pattern and the element-order scatter of the
//    element tangents (src/fem/Assembler.cpp:86-215), plus add_node_block
//    (src/fem/Forming.cpp:280-297);
//  - penalty contact with rigid tools: candidate search, evaluation with
//    Coulomb friction, the semismooth anticipation and the history commit
//    (src/fem/RigidTool.cpp:43-611).
#include "oracle_element.hpp"

#include <cstdio>
#include <map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {
thread_local long long g_flops = 0;
}

using namespace orc;

namespace {

constexpr int kNF = 39;  // per-point state: ep 6, beta 6, alpha 4x6, eqps, thick, loading

// Flat material record (the Python side fills the same layout):
// [0]E [1]nu [2]sy0 [3]H [4]Hkin [5]Q [6]delta [7]criterion [8]nback
// [9]integration [10..13]C_i [14..17]gamma_i [18]r0 [19]r45 [20]r90
// [21]L [22]M [23..25]rolling direction [26..28]sheet normal
bool make_material(const double* m, Material& mat) {
  mat.E = m[0];
  mat.nu = m[1];
  mat.sy0 = m[2];
  mat.H = m[3];
  mat.Hkin = m[4];
  mat.Q = m[5];
  mat.delta = m[6];
  mat.criterion = static_cast<int>(m[7]);
  mat.nback = static_cast<int>(m[8]);
  mat.integration = static_cast<int>(m[9]);
  if (mat.nback < 0 || mat.nback > kMaxBack || mat.kin_terms() > kMaxBack) return false;
  for (int i = 0; i < kMaxBack; ++i) {
    mat.Cb[i] = m[10 + i];
    mat.gb[i] = m[14 + i];
  }
  if (mat.criterion == 1) {
    return hill_from_r(m[18], m[19], m[20], m[21], m[22], m + 23, m + 26, mat.P);
  }
  von_mises_matrix(mat.P);
  return true;
}

template <class T>
State<T> load_state(const double* s) {
  State<T> st;
  for (int i = 0; i < 6; ++i) st.ep[i] = T(s[i]);
  for (int i = 0; i < 6; ++i) st.beta[i] = T(s[6 + i]);
  for (int b = 0; b < kMaxBack; ++b)
    for (int i = 0; i < 6; ++i) st.alpha[b][i] = T(s[12 + 6 * b + i]);
  st.eqps = T(s[36]);
  st.thick = T(s[37]);
  st.loading = s[38] != 0.0;
  return st;
}

template <class T>
void store_state(const State<T>& st, double* s) {
  for (int i = 0; i < 6; ++i) s[i] = val(st.ep[i]);
  for (int i = 0; i < 6; ++i) s[6 + i] = val(st.beta[i]);
  for (int b = 0; b < kMaxBack; ++b)
    for (int i = 0; i < 6; ++i) s[12 + 6 * b + i] = val(st.alpha[b][i]);
  s[36] = val(st.eqps);
  s[37] = val(st.thick);
  s[38] = st.loading ? 1.0 : 0.0;
}

struct ElementBatch {
  const Material* mat;
  const std::vector<QPoint>* rule;
  int kin;
  const double* X;
  const double* ue;
  const double* committed;
  const double* alpha_n;
  int want_tangent;
  double* f;
  double* K;
  double* energy;
  double* trial;
  double* alpha;
  int* yielding;
  int* iterations;
  int* status;
  signed char* yield_flags;  // nq per element, or null
};

// The element formulation of orc_elements / orc_system_evaluate: 0 the
// incompatible-mode Hex8, 1 the standard Hex8 (with g_averaged: mean
// dilatation), set by orc_set_element.
int g_standard = 0;
int g_averaged = 0;

template <class T>
void run_element(const ElementBatch& b, long long e) {
  const int nq = static_cast<int>(b.rule->size());
  IMElement<T> el(*b.mat, *b.rule, b.kin);
  StdElement<T> std_el(*b.mat, *b.rule, b.kin, g_averaged != 0);
  std::vector<State<T>> committed(static_cast<std::size_t>(nq));
  for (int q = 0; q < nq; ++q) committed[q] = load_state<T>(b.committed + (e * nq + q) * kNF);
  T ue[24], an[9];
  for (int i = 0; i < 24; ++i) ue[i] = T(b.ue[e * 24 + i]);
  for (int i = 0; i < 9; ++i) an[i] = T(b.alpha_n ? b.alpha_n[e * 9 + i] : 0.0);
  try {
    ElementOut<T> out = g_standard ? std_el.evaluate(b.X + e * 24, ue, committed, b.want_tangent != 0)
                                   : el.evaluate(b.X + e * 24, ue, committed, an, b.want_tangent != 0);
    for (int i = 0; i < 24; ++i) b.f[e * 24 + i] = val(out.force[i]);
    if (b.want_tangent && b.K)
      for (int i = 0; i < 576; ++i) b.K[e * 576 + i] = val(out.tangent[i]);
    if (b.energy) b.energy[e] = val(out.energy);
    if (b.trial)
      for (int q = 0; q < nq; ++q) store_state(out.states[q], b.trial + (e * nq + q) * kNF);
    if (b.alpha)
      for (int i = 0; i < 9; ++i) b.alpha[e * 9 + i] = val(out.alpha[i]);
    if (b.yielding) b.yielding[e] = out.yielding;
    if (b.yield_flags)
      for (int q = 0; q < nq; ++q) b.yield_flags[e * nq + q] = out.point_yield[q] ? 1 : 0;
    if (b.iterations) b.iterations[e] = out.iterations;
    b.status[e] = 0;
  } catch (const Failure& fail) {
    b.status[e] = fail.code;
  }
}

int set_threads(int threads) {
#ifdef _OPENMP
  if (threads > 0) return threads;
  return omp_get_max_threads();
#else
  (void)threads;
  return 1;
#endif
}

// ---- pattern (Assembler.cpp:86-173) ----------------------------------------
struct Pattern {
  std::vector<int> outer, inner, block_offset;
};

void build_pattern(int nn, int ne, const int* conn, Pattern& p) {
  const int npe = 8, dim = 3;
  std::vector<int> inc_ptr(static_cast<std::size_t>(nn) + 1, 0);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < npe; ++a) ++inc_ptr[conn[e * 8 + a] + 1];
  for (int n = 0; n < nn; ++n) inc_ptr[n + 1] += inc_ptr[n];
  std::vector<int> inc(static_cast<std::size_t>(inc_ptr.back()));
  {
    std::vector<int> fill(inc_ptr.begin(), inc_ptr.end() - 1);
    for (int e = 0; e < ne; ++e)
      for (int a = 0; a < npe; ++a) inc[fill[conn[e * 8 + a]]++] = e;
  }
  std::vector<int> nbr_ptr(static_cast<std::size_t>(nn) + 1, 0), nbr;
  nbr.reserve(static_cast<std::size_t>(nn) * 27);
  {
    std::vector<int> marker(static_cast<std::size_t>(nn), -1), list;
    for (int b = 0; b < nn; ++b) {
      list.clear();
      for (int k = inc_ptr[b]; k < inc_ptr[b + 1]; ++k) {
        const int* nodes = conn + static_cast<std::size_t>(inc[k]) * 8;
        for (int a = 0; a < npe; ++a)
          if (marker[nodes[a]] != b) { marker[nodes[a]] = b; list.push_back(nodes[a]); }
      }
      std::sort(list.begin(), list.end());
      nbr.insert(nbr.end(), list.begin(), list.end());
      nbr_ptr[b + 1] = static_cast<int>(nbr.size());
    }
  }
  const long long n = static_cast<long long>(nn) * dim;
  p.outer.assign(static_cast<std::size_t>(n) + 1, 0);
  for (int b = 0; b < nn; ++b) {
    const int deg = nbr_ptr[b + 1] - nbr_ptr[b];
    for (int kb = 0; kb < dim; ++kb) {
      const long long c = static_cast<long long>(b) * dim + kb;
      p.outer[c + 1] = p.outer[c] + deg * dim;
    }
  }
  p.inner.resize(static_cast<std::size_t>(p.outer.back()));
  for (int b = 0; b < nn; ++b)
    for (int kb = 0; kb < dim; ++kb) {
      int q = p.outer[static_cast<std::size_t>(b) * dim + kb];
      for (int k = nbr_ptr[b]; k < nbr_ptr[b + 1]; ++k)
        for (int ka = 0; ka < dim; ++ka) p.inner[q++] = nbr[k] * dim + ka;
    }
  p.block_offset.resize(static_cast<std::size_t>(ne) * 64);
  for (int e = 0; e < ne; ++e) {
    const int* nodes = conn + static_cast<std::size_t>(e) * 8;
    for (int b = 0; b < npe; ++b) {
      const int* begin = nbr.data() + nbr_ptr[nodes[b]];
      const int* end = nbr.data() + nbr_ptr[nodes[b] + 1];
      for (int a = 0; a < npe; ++a) {
        const int* hit = std::lower_bound(begin, end, nodes[a]);
        p.block_offset[(static_cast<std::size_t>(e) * npe + a) * npe + b] = static_cast<int>(hit - begin) * dim;
      }
    }
  }
}

}  // namespace

extern "C" {

/// The element formulation of the calls that follow: standard 0 the
/// incompatible-mode Hex8 (IncompatibleModes.cpp), 1 the standard Hex8
/// (Elastoplastic.cpp:226-340), averaged 1 its mean dilatation.
int orc_set_element(int standard, int averaged) {
  g_standard = standard;
  g_averaged = averaged;
  return 0;
}

int orc_rule_size(int in_plane, int thickness, int axis) {
  return static_cast<int>(hex8_rule(in_plane, thickness, axis).size());
}

/// The rule's points: xi, eta, zeta, weight per point.
int orc_rule(int in_plane, int thickness, int axis, double* out) {
  const auto r = hex8_rule(in_plane, thickness, axis);
  for (std::size_t i = 0; i < r.size(); ++i) {
    out[4 * i] = r[i].xi;
    out[4 * i + 1] = r[i].eta;
    out[4 * i + 2] = r[i].zeta;
    out[4 * i + 3] = r[i].weight;
  }
  return static_cast<int>(r.size());
}

/// The yield matrix of a material record (Hill48 or von Mises), row-major.
int orc_yield_matrix(const double* material, double* p) {
  Material mat;
  if (!make_material(material, mat)) return 1;
  for (int i = 0; i < 36; ++i) p[i] = mat.P[i];
  return 0;
}

/// One 3-D return (plastic_return, ThreeDimensional). state/trial: 39
/// doubles each. Returns 0, or the failure code.
int orc_return(const double* material, const double* strain, const double* committed, int want_tangent,
               double* stress, double* tangent, double* trial, double* energy, int* yielding) {
  Material mat;
  if (!make_material(material, mat)) return -1;
  Vec<double, 6> e;
  for (int i = 0; i < 6; ++i) e[i] = strain[i];
  try {
    const Response<double> r = plastic_return(mat, e, load_state<double>(committed), want_tangent != 0);
    for (int i = 0; i < 6; ++i) stress[i] = r.stress[i];
    for (int i = 0; i < 36; ++i) tangent[i] = r.tangent[i];
    store_state(r.state, trial);
    *energy = r.energy;
    *yielding = r.yielding ? 1 : 0;
    return 0;
  } catch (const Failure& f) {
    return f.code;
  }
}

/// The logarithmic strain of an engineering Green-Lagrange strain: E_log
/// (6), P (36), and T:L (36) for the stress t, S = P^T t (6).
int orc_log_strain(const double* green, const double* t, double* strain, double* projection,
                   double* curvature, double* stress) {
  Vec<double, 6> g, tt;
  for (int i = 0; i < 6; ++i) { g[i] = green[i]; tt[i] = t[i]; }
  try {
    const LogStrain<double> l = logarithmic_strain(g);
    for (int i = 0; i < 6; ++i) strain[i] = l.strain[i];
    for (int i = 0; i < 36; ++i) projection[i] = l.projection[i];
    const Mat<double, 6, 6> c = logarithmic_curvature(l, tt);
    for (int i = 0; i < 36; ++i) curvature[i] = c[i];
    const Vec<double, 6> s = logarithmic_stress(l, tt);
    for (int i = 0; i < 6; ++i) stress[i] = s[i];
    return 0;
  } catch (const Failure& f) {
    return f.code;
  }
}

/// A batch of independent elements (incompatible_elastoplastic_element per
/// element). X, ue: 24 per element (node-major); committed/trial: nq x 39
/// per element; alpha: 9. K may be null. Returns the number of failed
/// elements (per-element codes in status).
int orc_elements(const double* material, int in_plane, int thickness, int axis, int kinematics,
                 long long ne, const double* X, const double* ue, const double* committed,
                 const double* alpha_n, int want_tangent, int threads, double* f, double* K,
                 double* energy, double* trial, double* alpha, int* yielding, int* iterations,
                 int* status, signed char* yield_flags) {
  Material mat;
  if (!make_material(material, mat)) return -1;
  const std::vector<QPoint> rule = hex8_rule(in_plane, thickness, axis);
  ElementBatch b{&mat, &rule, kinematics, X, ue, committed, alpha_n, want_tangent, f, K, energy,
                 trial, alpha, yielding, iterations, status, yield_flags};
  const int nt = set_threads(threads);
  long long failed = 0;
#pragma omp parallel for schedule(static) num_threads(nt) reduction(+ : failed)
  for (long long e = 0; e < ne; ++e) {
    run_element<double>(b, e);
    if (b.status[e] != 0) ++failed;
  }
  return static_cast<int>(failed);
}

/// incompatible_elastoplastic_stress (IncompatibleModes.cpp:602-664) for a
/// batch: 28 doubles per element - Cauchy 6, second Piola-Kirchhoff 6, von
/// Mises, max eqps, max strain, min det F, Kirchhoff 6, log strain 6.
int orc_element_stress(const double* material, int in_plane, int thickness, int axis, int kinematics,
                       long long ne, const double* X, const double* ue, const double* committed,
                       const double* alpha, int threads, double* out, int* status) {
  Material mat;
  if (!make_material(material, mat)) return -1;
  const std::vector<QPoint> rule = hex8_rule(in_plane, thickness, axis);
  const int nq = static_cast<int>(rule.size());
  const int nt = set_threads(threads);
  long long failed = 0;
#pragma omp parallel for schedule(static) num_threads(nt) reduction(+ : failed)
  for (long long e = 0; e < ne; ++e) {
    IMElement<double> el(mat, rule, kinematics);
    StdElement<double> std_el(mat, rule, kinematics, g_averaged != 0);
    std::vector<State<double>> c(static_cast<std::size_t>(nq));
    for (int q = 0; q < nq; ++q) c[q] = load_state<double>(committed + (e * nq + q) * kNF);
    try {
      const ElementStress st = g_standard ? std_el.stress(X + e * 24, ue + e * 24, c)
                                          : el.stress(X + e * 24, ue + e * 24, c, alpha ? alpha + e * 9 : nullptr);
      double* o = out + e * 28;
      for (int i = 0; i < 6; ++i) {
        o[i] = st.cauchy[i];
        o[6 + i] = st.piola_kirchhoff[i];
        o[16 + i] = st.kirchhoff[i];
        o[22 + i] = st.log_strain[i];
      }
      o[12] = st.von_mises;
      o[13] = st.max_eqps;
      o[14] = st.max_strain;
      o[15] = st.min_jacobian;
      status[e] = 0;
    } catch (const Failure& f) {
      status[e] = f.code;
      ++failed;
    }
  }
  return static_cast<int>(failed);
}

/// The vector-Jacobian product lambda . d f*/d X of a batch of IM Hex8 (24
/// per element), at fixed displacements and committed history
/// (IMElement::vjp_x). Returns the number of failed elements.
int orc_vjp_x(const double* material, int in_plane, int thickness, int axis, int kinematics, long long ne,
              const double* X, const double* ue, const double* committed, const double* alpha_n,
              const double* lambda, double* out, int* status) {
  Material mat;
  if (!make_material(material, mat)) return -1;
  const std::vector<QPoint> rule = hex8_rule(in_plane, thickness, axis);
  const int nq = static_cast<int>(rule.size());
  long long failed = 0;
  for (long long e = 0; e < ne; ++e) {
    IMElement<double> el(mat, rule, kinematics);
    std::vector<State<double>> c(static_cast<std::size_t>(nq));
    for (int q = 0; q < nq; ++q) c[q] = load_state<double>(committed + (e * nq + q) * kNF);
    try {
      el.vjp_x(X + e * 24, ue + e * 24, c, alpha_n ? alpha_n + e * 9 : nullptr, lambda + e * 24, out + e * 24);
      status[e] = 0;
    } catch (const Failure& f) {
      status[e] = f.code;
      ++failed;
    }
  }
  return static_cast<int>(failed);
}

/// The algorithmic flop count of the same batch (counting scalar, one
/// thread): +, -, *, / and each sqrt/log1p/exp/expm1 count one.
long long orc_count_flops(const double* material, int in_plane, int thickness, int axis,
                          int kinematics, long long ne, const double* X, const double* ue,
                          const double* committed, const double* alpha_n, int want_tangent) {
  Material mat;
  if (!make_material(material, mat)) return -1;
  const std::vector<QPoint> rule = hex8_rule(in_plane, thickness, axis);
  const int nq = static_cast<int>(rule.size());
  std::vector<double> f(24), K(576), energy(1), trial(static_cast<std::size_t>(nq) * kNF), alpha(9);
  int y = 0, it = 0, st = 0;
  g_flops = 0;
  for (long long e = 0; e < ne; ++e) {
    // Shift the inputs so that element e sits at index 0 of the batch.
    ElementBatch b{&mat, &rule, kinematics, X + e * 24, ue + e * 24, committed + e * nq * kNF,
                   alpha_n ? alpha_n + e * 9 : nullptr, want_tangent, f.data(), K.data(),
                   energy.data(), trial.data(), alpha.data(), &y, &it, &st, nullptr};
    run_element<CD>(b, 0);
  }
  return g_flops;
}

/// Size of the node-block pattern of a Hex8 mesh.
long long orc_pattern_nnz(int nn, int ne, const int* conn) {
  Pattern p;
  build_pattern(nn, ne, conn, p);
  return static_cast<long long>(p.inner.size());
}

int orc_build_pattern(int nn, int ne, const int* conn, int* outer, int* inner, int* block_offset) {
  Pattern p;
  build_pattern(nn, ne, conn, p);
  std::copy(p.outer.begin(), p.outer.end(), outer);
  std::copy(p.inner.begin(), p.inner.end(), inner);
  if (block_offset) std::copy(p.block_offset.begin(), p.block_offset.end(), block_offset);
  return 0;
}

/// Assembler::scatter of element matrices K (576 per element, row-major)
/// into CSC values, element by element (Assembler.cpp:184-215).
int orc_scatter(int nn, int ne, const int* conn, const int* outer, const int* block_offset,
                const double* K, double* values, long long nnz) {
  (void)nn;
  std::fill(values, values + nnz, 0.0);
  for (int e = 0; e < ne; ++e) {
    const double* ke = K + static_cast<std::size_t>(e) * 576;
    const int* nodes = conn + static_cast<std::size_t>(e) * 8;
    const int* offsets = block_offset + static_cast<std::size_t>(e) * 64;
    for (int b = 0; b < 8; ++b)
      for (int kb = 0; kb < 3; ++kb) {
        const int column = 3 * b + kb;
        const int base = outer[nodes[b] * 3 + kb];
        for (int a = 0; a < 8; ++a) {
          double* target = values + base + offsets[a * 8 + b];
          for (int ka = 0; ka < 3; ++ka) target[ka] += ke[(3 * a + ka) * 24 + column];
        }
      }
  }
  return 0;
}

/// NonlinearSystem::evaluate: the element loop, then the serial gather of
/// f_int, gross, energy and yield count, and (want_tangent) the scatter.
/// u: 3 per node. Returns 0, or the code of the first failing element
/// (its index in *failed_element).
int orc_system_evaluate(const double* material, int in_plane, int thickness, int axis,
                        int kinematics, int nn, int ne, const double* coords, const int* conn,
                        const double* u, const double* committed, const double* alpha_n,
                        int want_tangent, int threads, const int* outer, const int* block_offset,
                        long long nnz, double* internal, double* gross, double* energy,
                        int* yielding_points, double* values, double* trial, double* alpha_out,
                        int* failed_element) {
  const int nq = orc_rule_size(in_plane, thickness, axis);
  std::vector<double> X(static_cast<std::size_t>(ne) * 24), ue(static_cast<std::size_t>(ne) * 24);
  for (int e = 0; e < ne; ++e)
    for (int a = 0; a < 8; ++a) {
      const int node = conn[e * 8 + a];
      for (int k = 0; k < 3; ++k) {
        X[static_cast<std::size_t>(e) * 24 + 3 * a + k] = coords[static_cast<std::size_t>(node) * 3 + k];
        ue[static_cast<std::size_t>(e) * 24 + 3 * a + k] = u[static_cast<std::size_t>(node) * 3 + k];
      }
    }
  std::vector<double> f(static_cast<std::size_t>(ne) * 24), en(static_cast<std::size_t>(ne));
  std::vector<double> K(want_tangent ? static_cast<std::size_t>(ne) * 576 : 0);
  std::vector<int> y(static_cast<std::size_t>(ne)), it(static_cast<std::size_t>(ne)), st(static_cast<std::size_t>(ne));
  (void)nq;
  orc_elements(material, in_plane, thickness, axis, kinematics, ne, X.data(), ue.data(), committed,
               alpha_n, want_tangent, threads, f.data(), want_tangent ? K.data() : nullptr, en.data(),
               trial, alpha_out, y.data(), it.data(), st.data(), nullptr);
  for (int e = 0; e < ne; ++e)
    if (st[e] != 0) {
      *failed_element = e;
      return st[e];
    }
  *failed_element = -1;
  const long long n = static_cast<long long>(nn) * 3;
  std::vector<double> gv(static_cast<std::size_t>(n), 0.0);
  std::fill(internal, internal + n, 0.0);
  double energy_sum = 0.0;
  int ysum = 0;
  for (int e = 0; e < ne; ++e) {
    for (int a = 0; a < 8; ++a)
      for (int k = 0; k < 3; ++k) {
        const long long dof = static_cast<long long>(conn[e * 8 + a]) * 3 + k;
        internal[dof] += f[static_cast<std::size_t>(e) * 24 + 3 * a + k];
        gv[dof] += std::fabs(f[static_cast<std::size_t>(e) * 24 + 3 * a + k]);
      }
    energy_sum += en[e];
    ysum += y[e];
  }
  double g2 = 0.0;
  for (long long i = 0; i < n; ++i) g2 += gv[i] * gv[i];
  *gross = std::sqrt(g2);
  *energy = energy_sum;
  *yielding_points = ysum;
  if (want_tangent) orc_scatter(nn, ne, conn, outer, block_offset, K.data(), values, nnz);
  return 0;
}

/// add_node_block (Forming.cpp:280-297) for blocks that lie in the pattern.
int orc_add_node_blocks(const int* outer, const int* inner, double* values, int nblocks,
                        const int* nodes, const double* blocks /*9 per block, row-major*/) {
  for (int i = 0; i < nblocks; ++i) {
    const int node = nodes[i];
    for (int b = 0; b < 3; ++b) {
      const int col = node * 3 + b;
      const int* begin = inner + outer[col];
      const int* end = inner + outer[col + 1];
      for (int a = 0; a < 3; ++a) {
        const int row = node * 3 + a;
        const int* it = std::lower_bound(begin, end, row);
        if (it == end || *it != row) return 1;
        values[it - inner] += blocks[9 * i + 3 * a + b];
      }
    }
  }
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Contact (src/fem/RigidTool.cpp), three-dimensional.
// ---------------------------------------------------------------------------
namespace {

struct V3 {
  double x[3] = {0, 0, 0};
  double& operator[](int i) { return x[i]; }
  double operator[](int i) const { return x[i]; }
};
V3 sub(const V3& a, const V3& b) { V3 o; for (int i = 0; i < 3; ++i) o[i] = a[i] - b[i]; return o; }
double dot3(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
double nrm(const V3& a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

struct Tool {
  int shape = 0;  // 0 sphere, 1 plane, 2 cylinder
  double radius = 0, friction = 0, tangential_ratio = 1;
  V3 normal, axis;
  std::vector<double> times;
  std::vector<V3> points;
  std::vector<int> nodes;
  std::vector<double> area, kappa;
  std::vector<int> candidates;
  mutable std::size_t hint = 0;

  std::size_t segment(double t) const {
    const std::size_t last = times.size() - 2;
    std::size_t i = std::min(hint, last);
    if (times[i] <= t && t < times[i + 1]) return i;
    if (i < last && times[i + 1] <= t && t < times[i + 2]) { hint = i + 1; return i + 1; }
    const auto it = std::upper_bound(times.begin(), times.end(), t);
    long long j = static_cast<long long>(it - times.begin()) - 1;
    if (j < 0) j = 0;
    i = std::min(static_cast<std::size_t>(j), last);
    hint = i;
    return i;
  }
  V3 position(double t) const {
    if (t <= times.front()) return points.front();
    if (t >= times.back()) return points.back();
    const std::size_t i = segment(t);
    const double w = (t - times[i]) / (times[i + 1] - times[i]);
    V3 o;
    for (int k = 0; k < 3; ++k) o[k] = (1.0 - w) * points[i][k] + w * points[i + 1][k];
    return o;
  }
  // RigidTool::gap (RigidTool.cpp:237-270); false where the node is within
  // half the radius (SolverError in the reference).
  bool gap(const V3& x, const V3& c, V3& n, double dn[9], double& d, double& g) const {
    if (shape == 1) {
      const double l = nrm(normal);
      for (int i = 0; i < 3; ++i) n[i] = normal[i] / l;
      for (int i = 0; i < 9; ++i) dn[i] = 0.0;
      d = 0.0;
      g = dot3(n, sub(x, c));
      return true;
    }
    V3 r = sub(x, c);
    double base[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (shape == 2) {
      const double l = nrm(axis);
      V3 a;
      for (int i = 0; i < 3; ++i) a[i] = axis[i] / l;
      const double ar = dot3(a, r);
      for (int i = 0; i < 3; ++i) r[i] -= ar * a[i];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) base[3 * i + j] -= a[i] * a[j];
    }
    d = nrm(r);
    if (!(d > 0.5 * radius)) return false;
    for (int i = 0; i < 3; ++i) n[i] = r[i] / d;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dn[3 * i + j] = (base[3 * i + j] - n[i] * n[j]) / d;
    g = d - radius;
    return true;
  }
};

double segment_distance(const V3& p, const V3& a, const V3& b) {
  const V3 s = sub(b, a);
  const double len2 = dot3(s, s);
  double t = 0.0;
  if (len2 > 0.0) t = std::clamp(dot3(sub(p, a), s) / len2, 0.0, 1.0);
  V3 o;
  for (int i = 0; i < 3; ++i) o[i] = p[i] - a[i] - t * s[i];
  return nrm(o);
}

struct Hist {
  V3 force, relative;
};

struct Contact {
  int nn = 0;
  const double* coords = nullptr;  // borrowed, 3 per node
  std::vector<Tool> tools;
  int friction_tangent = 0;  // 0 exact, 1 symmetric
  std::vector<std::map<int, Hist>> history, trial;
  std::vector<double> start;
  double t0 = 0.0, margin = 0.0;
  std::vector<char> active;
  V3 node(int n) const { V3 o; for (int k = 0; k < 3; ++k) o[k] = coords[static_cast<std::size_t>(n) * 3 + k]; return o; }
};

}  // namespace

extern "C" {

/// tools: per tool 12 doubles [shape, radius, friction, tangential_ratio,
/// normal xyz, axis xyz, nknots, nslaves]; knots: (t, x, y, z) per knot of
/// every tool in order; slaves: (node, area, kappa) per slave node of every
/// tool in order (ascending nodes).
void* orc_contact_create(int nn, const double* coords, int ntools, const double* tools,
                         const double* knots, const double* slaves, int friction_tangent) {
  Contact* c = new Contact();
  c->nn = nn;
  c->coords = coords;
  c->friction_tangent = friction_tangent;
  std::size_t kk = 0, ss = 0;
  for (int i = 0; i < ntools; ++i) {
    const double* t = tools + 12 * i;
    Tool tool;
    tool.shape = static_cast<int>(t[0]);
    tool.radius = t[1];
    tool.friction = t[2];
    tool.tangential_ratio = t[3];
    for (int k = 0; k < 3; ++k) { tool.normal[k] = t[4 + k]; tool.axis[k] = t[7 + k]; }
    const int nk = static_cast<int>(t[10]);
    const int ns = static_cast<int>(t[11]);
    for (int k = 0; k < nk; ++k, ++kk) {
      tool.times.push_back(knots[4 * kk]);
      V3 p;
      for (int j = 0; j < 3; ++j) p[j] = knots[4 * kk + 1 + j];
      tool.points.push_back(p);
    }
    for (int k = 0; k < ns; ++k, ++ss) {
      tool.nodes.push_back(static_cast<int>(slaves[3 * ss]));
      tool.area.push_back(slaves[3 * ss + 1]);
      tool.kappa.push_back(slaves[3 * ss + 2]);
      tool.candidates.push_back(k);
    }
    c->tools.push_back(tool);
  }
  c->history.assign(c->tools.size(), {});
  c->start.assign(static_cast<std::size_t>(nn) * 3, 0.0);
  c->t0 = c->tools.empty() ? 0.0 : c->tools.front().times.front();
  c->margin = std::numeric_limits<double>::infinity();
  c->active.assign(c->tools.size(), 1);
  return c;
}

void orc_contact_destroy(void* h) { delete static_cast<Contact*>(h); }

/// ToolContact::begin_increment (RigidTool.cpp:345-393). Returns the
/// candidate count of every tool in `counts`.
int orc_contact_begin(void* h, const double* u0, double t0, double t1, const char* active,
                      double margin, int* counts) {
  Contact& c = *static_cast<Contact*>(h);
  std::copy(u0, u0 + static_cast<std::size_t>(c.nn) * 3, c.start.begin());
  c.t0 = t0;
  c.margin = margin;
  for (std::size_t k = 0; k < c.tools.size(); ++k) c.active[k] = active[k];
  for (std::size_t k = 0; k < c.tools.size(); ++k) {
    Tool& tool = c.tools[k];
    tool.candidates.clear();
    if (!c.active[k]) { counts[k] = 0; continue; }
    const V3 c0 = tool.position(t0), c1 = tool.position(t1);
    V3 a;
    a[2] = 1.0;
    if (tool.shape == 2) { const double l = nrm(tool.axis); for (int i = 0; i < 3; ++i) a[i] = tool.axis[i] / l; }
    V3 pn;
    { const double l = nrm(tool.normal); for (int i = 0; i < 3; ++i) pn[i] = tool.normal[i] / l; }
    for (std::size_t i = 0; i < tool.nodes.size(); ++i) {
      const int node = tool.nodes[i];
      V3 x = c.node(node);
      for (int k2 = 0; k2 < 3; ++k2) x[k2] += u0[static_cast<std::size_t>(node) * 3 + k2];
      bool candidate = false;
      if (tool.shape == 0) {
        candidate = segment_distance(x, c0, c1) <= tool.radius + margin;
      } else if (tool.shape == 2) {
        double p[9];
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) p[3 * r + s] = (r == s ? 1.0 : 0.0) - a[r] * a[s];
        V3 dx = sub(x, c0), dc = sub(c1, c0), px, pc, zero;
        for (int r = 0; r < 3; ++r) {
          px[r] = p[3 * r] * dx[0] + p[3 * r + 1] * dx[1] + p[3 * r + 2] * dx[2];
          pc[r] = p[3 * r] * dc[0] + p[3 * r + 1] * dc[1] + p[3 * r + 2] * dc[2];
        }
        candidate = segment_distance(px, zero, pc) <= tool.radius + margin;
      } else {
        candidate = std::min(dot3(pn, sub(x, c0)), dot3(pn, sub(x, c1))) <= margin;
      }
      if (candidate) tool.candidates.push_back(static_cast<int>(i));
    }
    counts[k] = static_cast<int>(tool.candidates.size());
  }
  return 0;
}

/// ToolContact::evaluate (RigidTool.cpp:398-555). residual: 3 nn (full
/// length); blocks: up to max_blocks (node + 9 values each, in tool then
/// slave order); resultants: 9 per tool [centre xyz, force xyz, active,
/// slipping, max penetration]; scalars: [gross, round_off, force_norm,
/// symmetric]. Returns the block count, or -1 (a node within half a
/// radius: SolverError in the reference).
int orc_contact_evaluate(void* h, const double* u, double t, int want_tangent, double* residual,
                         int max_blocks, int* block_nodes, double* blocks, double* resultants,
                         double* scalars) {
  Contact& c = *static_cast<Contact*>(h);
  const std::size_t n = static_cast<std::size_t>(c.nn) * 3;
  std::fill(residual, residual + n, 0.0);
  std::vector<double> gross(n, 0.0), positions(n, 0.0);
  c.trial.assign(c.tools.size(), {});
  bool symmetric = true;
  int nblocks = 0;
  std::vector<int> all;
  for (std::size_t k = 0; k < c.tools.size(); ++k) {
    const Tool& tool = c.tools[k];
    double* res = resultants + 9 * k;
    for (int i = 0; i < 9; ++i) res[i] = 0.0;
    const V3 cc = tool.position(t);
    for (int i = 0; i < 3; ++i) res[i] = cc[i];
    if (!c.active[k]) continue;
    const std::vector<int>* nodes = &tool.candidates;
    double moved = 0.0;
    for (int node : tool.nodes) {
      double m2 = 0.0;
      for (int comp = 0; comp < 3; ++comp) {
        const double du = u[static_cast<std::size_t>(node) * 3 + comp] - c.start[static_cast<std::size_t>(node) * 3 + comp];
        m2 += du * du;
      }
      moved = std::max(moved, m2);
    }
    if (std::sqrt(moved) > c.margin) {
      all.resize(tool.nodes.size());
      for (std::size_t i = 0; i < tool.nodes.size(); ++i) all[i] = static_cast<int>(i);
      nodes = &all;
    }
    const double mu = tool.friction;
    const std::map<int, Hist>& committed = c.history[k];
    for (int i : *nodes) {
      const int node = tool.nodes[i];
      V3 x = c.node(node);
      for (int comp = 0; comp < 3; ++comp) x[comp] += u[static_cast<std::size_t>(node) * 3 + comp];
      V3 nv;
      double dn[9], d = 0.0, g = 0.0;
      if (!tool.gap(x, cc, nv, dn, d, g)) return -1;
      if (!(g < 0.0)) continue;
      const double ka = tool.kappa[i] * tool.area[i];
      const double pn = -ka * g;
      V3 force;
      for (int r = 0; r < 3; ++r) force[r] = pn * nv[r];
      double kn[9];
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) kn[3 * r + s] = ka * (nv[r] * nv[s]) - pn * dn[3 * r + s];
      bool slipping = false;
      const V3 rr = sub(x, cc);
      if (mu > 0.0) {
        const double kt = tool.tangential_ratio * ka;
        V3 f0, q;
        const auto it = committed.find(node);
        if (it != committed.end()) {
          f0 = it->second.force;
          q = it->second.relative;
        } else {
          V3 x0 = c.node(node);
          for (int comp = 0; comp < 3; ++comp) x0[comp] += c.start[static_cast<std::size_t>(node) * 3 + comp];
          q = sub(x0, tool.position(c.t0));
        }
        const double s0 = nrm(f0);
        const double fn = dot3(f0, nv);
        V3 ft_tilde;
        for (int r = 0; r < 3; ++r) ft_tilde[r] = f0[r] - fn * nv[r];
        const double ftn = nrm(ft_tilde);
        V3 f_hat;
        double d_hat[9] = {};
        if (s0 > 0.0 && ftn > 1.0e-12 * s0) {
          V3 e;
          for (int r = 0; r < 3; ++r) e[r] = ft_tilde[r] / ftn;
          for (int r = 0; r < 3; ++r) f_hat[r] = s0 * e[r];
          // d_tilde = -(n (f0^T dn) + (f0 . n) dn)
          double f0dn[3];
          for (int s = 0; s < 3; ++s) f0dn[s] = f0[0] * dn[s] + f0[1] * dn[3 + s] + f0[2] * dn[6 + s];
          double d_tilde[9];
          for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) d_tilde[3 * r + s] = -(nv[r] * f0dn[s] + fn * dn[3 * r + s]);
          const double sc = s0 / ftn;
          for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) {
              double acc = 0.0;
              for (int m = 0; m < 3; ++m) acc += ((r == m ? 1.0 : 0.0) - e[r] * e[m]) * d_tilde[3 * m + s];
              d_hat[3 * r + s] = sc * acc;
            }
        }
        const V3 w = sub(rr, q);
        double p[9];
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) p[3 * r + s] = (r == s ? 1.0 : 0.0) - nv[r] * nv[s];
        V3 delta;
        for (int r = 0; r < 3; ++r) delta[r] = p[3 * r] * w[0] + p[3 * r + 1] * w[1] + p[3 * r + 2] * w[2];
        const double nw = dot3(nv, w);
        double wdn[3];
        for (int s = 0; s < 3; ++s) wdn[s] = w[0] * dn[s] + w[1] * dn[3 + s] + w[2] * dn[6 + s];
        double d_delta[9], d_trial[9];
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) d_delta[3 * r + s] = p[3 * r + s] - nw * dn[3 * r + s] - nv[r] * wdn[s];
        V3 trial;
        for (int r = 0; r < 3; ++r) trial[r] = f_hat[r] - kt * delta[r];
        for (int i2 = 0; i2 < 9; ++i2) d_trial[i2] = d_hat[i2] - kt * d_delta[i2];
        const double trial_norm = nrm(trial);
        const double limit = mu * pn;
        V3 ft;
        double d_ft[9], k_sym[9];
        if (trial_norm <= limit) {
          ft = trial;
          for (int i2 = 0; i2 < 9; ++i2) { d_ft[i2] = d_trial[i2]; k_sym[i2] = kt * p[i2]; }
        } else {
          slipping = true;
          V3 e;
          for (int r = 0; r < 3; ++r) e[r] = trial[r] / trial_norm;
          for (int r = 0; r < 3; ++r) ft[r] = limit * e[r];
          const double lt = limit / trial_norm;
          for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) {
              double acc = 0.0;
              for (int m = 0; m < 3; ++m) acc += ((r == m ? 1.0 : 0.0) - e[r] * e[m]) * d_trial[3 * m + s];
              d_ft[3 * r + s] = -(mu * ka) * (e[r] * nv[s]) + lt * acc;
              k_sym[3 * r + s] = lt * kt * (p[3 * r + s] - e[r] * e[s]);
            }
        }
        for (int r = 0; r < 3; ++r) force[r] += ft[r];
        if (c.friction_tangent == 1) {
          for (int i2 = 0; i2 < 9; ++i2) kn[i2] += k_sym[i2];
        } else {
          for (int i2 = 0; i2 < 9; ++i2) kn[i2] -= d_ft[i2];
        }
        Hist hh;
        hh.force = ft;
        hh.relative = rr;
        c.trial[k].emplace(node, hh);
      }
      const double position_scale = ka * (nrm(x) + nrm(cc));
      for (int comp = 0; comp < 3; ++comp) {
        const std::size_t dof = static_cast<std::size_t>(node) * 3 + comp;
        residual[dof] -= force[comp];
        gross[dof] += std::fabs(force[comp]);
        positions[dof] += position_scale;
      }
      res[6] += 1.0;
      if (slipping) res[7] += 1.0;
      for (int r = 0; r < 3; ++r) res[3 + r] -= force[r];
      res[8] = std::max(res[8], -g);
      if (want_tangent) {
        if (c.friction_tangent == 1) {
          double ks[9];
          for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) ks[3 * r + s] = 0.5 * (kn[3 * r + s] + kn[3 * s + r]);
          std::copy(ks, ks + 9, kn);
        }
        double top = 0.0, asym = 0.0;
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) {
            top = std::max(top, std::fabs(kn[3 * r + s]));
            asym = std::max(asym, std::fabs(kn[3 * r + s] - kn[3 * s + r]));
          }
        if (asym > 1.0e-12 * top) symmetric = false;
        if (nblocks < max_blocks) {
          block_nodes[nblocks] = node;
          std::copy(kn, kn + 9, blocks + 9 * nblocks);
        }
        ++nblocks;
      }
    }
  }
  double a = 0, b = 0, f = 0;
  for (std::size_t i = 0; i < n; ++i) {
    a += gross[i] * gross[i];
    b += positions[i] * positions[i];
    f += residual[i] * residual[i];
  }
  scalars[0] = std::sqrt(a);
  scalars[1] = std::sqrt(b);
  scalars[2] = std::sqrt(f);
  scalars[3] = symmetric ? 1.0 : 0.0;
  return nblocks;
}

/// ToolContact::anticipate (RigidTool.cpp:557-603): adds to `residual` and
/// appends blocks; returns the number added.
int orc_contact_anticipate(void* h, const double* u, const double* du, double t, double* residual,
                           int max_blocks, int* block_nodes, double* blocks) {
  Contact& c = *static_cast<Contact*>(h);
  int added = 0;
  for (std::size_t k = 0; k < c.tools.size(); ++k) {
    if (!c.active[k]) continue;
    const Tool& tool = c.tools[k];
    const V3 cc = tool.position(t);
    for (int i : tool.candidates) {
      const int node = tool.nodes[i];
      V3 x = c.node(node), dx;
      for (int comp = 0; comp < 3; ++comp) {
        x[comp] += u[static_cast<std::size_t>(node) * 3 + comp];
        dx[comp] = du[static_cast<std::size_t>(node) * 3 + comp];
      }
      V3 nv;
      double dn[9], d = 0.0, g = 0.0;
      if (!tool.gap(x, cc, nv, dn, d, g)) continue;
      if (!(g > 0.0)) continue;
      double g_next = 0.0;
      V3 xn, n_next;
      for (int r = 0; r < 3; ++r) xn[r] = x[r] + dx[r];
      if (!tool.gap(xn, cc, n_next, dn, d, g_next)) g_next = -std::numeric_limits<double>::infinity();
      if (!(g_next < 0.0)) continue;
      const double ka = tool.kappa[i] * tool.area[i];
      for (int comp = 0; comp < 3; ++comp) residual[static_cast<std::size_t>(node) * 3 + comp] += ka * g * nv[comp];
      if (added < max_blocks) {
        block_nodes[added] = node;
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) blocks[9 * added + 3 * r + s] = ka * (nv[r] * nv[s]);
      }
      ++added;
    }
  }
  return added;
}

/// ToolContact::commit (RigidTool.cpp:605-611): the trial history of the
/// last evaluate becomes the committed one of every active tool.
int orc_contact_commit(void* h) {
  Contact& c = *static_cast<Contact*>(h);
  for (std::size_t k = 0; k < c.tools.size() && k < c.trial.size(); ++k) {
    if (!c.active[k]) continue;
    c.history[k] = std::move(c.trial[k]);
  }
  c.trial.clear();
  return 0;
}

/// The committed history of tool k: count, then (node, force xyz, relative
/// xyz) per entry in node order.
int orc_contact_history(void* h, int k, int max_entries, double* out) {
  Contact& c = *static_cast<Contact*>(h);
  int n = 0;
  for (const auto& [node, hh] : c.history[static_cast<std::size_t>(k)]) {
    if (n < max_entries) {
      double* o = out + 7 * n;
      o[0] = node;
      for (int r = 0; r < 3; ++r) { o[1 + r] = hh.force[r]; o[4 + r] = hh.relative[r]; }
    }
    ++n;
  }
  return n;
}

}  // extern "C"
