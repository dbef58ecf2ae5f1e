// K1: the incompatible-mode Hex8 element on the GPU.
//
// One group of G lanes (G = 8 for rules of up to 8 points, 32 for rules of
// 9 to 32 points) evaluates one element; a 32-lane warp holds 32 / G
// elements, and a block of four warps 16 (or 4) elements by default.
// Lane q owns integration point q: its kinematics, its return map and its
// share of K_aa, which a shuffle reduce-scatter sums over the group into
// shared memory. The element-level work of the local Newton iteration - the
// 9x9 factorisations, the line searches and their fallbacks - runs on lane 0
// over shared memory, every decision being read back by the whole group, so
// the group's control flow stays uniform. After convergence the lanes split
// the condensation by element node: lane a forms the rows of node a of K_ua,
// K_uu and K* = K_uu - K_ua K_aa^-1 K_au.
//
// Algorithm: incompatible_elastoplastic_element and solve_and_condense
// (src/fem/IncompatibleModes.cpp:134-600, constants
// src/fem/IncompatibleModes.hpp:98-127). The local iteration, the line
// search on the directional residual, the shifted direction, the
// Levenberg-Marquardt fallback and the condensation follow it step for
// step; the arithmetic is reorganised for the GPU (the strain operator is
// never stored: B^T D B products are formed from F, D and the gradients).
#include <cuda_runtime.h>
#include <stdint.h>

#include "sbk_element.h"
#include "sbk_material.cuh"
#include "sbk_wave.h"

namespace sbk {
namespace {

constexpr int kMaxLocal = 25;
constexpr double kFullStepReduction = 1.0 - 1.0e-4;
constexpr int kMaxLineSearch = 8;
constexpr double kLineSearchRatio = 0.5;
constexpr double kLocalShift = 1.0e-3;
constexpr double kLocalMarquardt = 1.0e-6;
constexpr double kLocalTolerance = 1.0e-8;
constexpr double kLocalRoundOff = 1.0e-13;

constexpr int kSlot = 54;  // per point: D 36 | S 6 | F 9 | w | energy | floor factor
constexpr int kSlotS = 36, kSlotF = 42, kSlotW = 51, kSlotE = 52, kSlotFl = 53;

__constant__ double kCorner[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                     {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

template <int G>
struct __align__(16) ElemShared {
  double X[24];
  double U[24];
  double jinv0[9];
  double geo[G][12];  // J^-1 (9), w det J, det0 / det
  double slot[G][kSlot];
  // K_aa (the reduced sums) during the local iteration; the coupling
  // C = K_aa^-1 K_au (9 x 24) in the condensation.
  double kc[216];
  double r[33];
  double scale[9];
  double flo[9];
  double energy;
  double alpha[9];
  double dir[9];
  double dir2[9];
  double r0[9];
  double lu[81];
  // Lane 0's scratch of the local iteration (K_aa at alpha, its symmetric
  // part, the Cholesky test, the shifted and Levenberg-Marquardt systems):
  // in shared memory, where its serial loads stay close.
  double work[243];
  double maxpivot;
  double dval[4];
  int rowp[9], colp[9], perm[9];
  int ival[4];
};

__device__ __forceinline__ void shape_grad(int a, double xi, double eta, double zeta, double dn[3]) {
  const double fx = 1.0 + xi * kCorner[a][0];
  const double fy = 1.0 + eta * kCorner[a][1];
  const double fz = 1.0 + zeta * kCorner[a][2];
  dn[0] = 0.125 * kCorner[a][0] * fy * fz;
  dn[1] = 0.125 * kCorner[a][1] * fx * fz;
  dn[2] = 0.125 * kCorner[a][2] * fx * fy;
}

__device__ __forceinline__ double det3(const double m[9]) {
  return m[0] * (m[4] * m[8] - m[7] * m[5]) - m[3] * (m[1] * m[8] - m[7] * m[2]) +
         m[6] * (m[1] * m[5] - m[4] * m[2]);
}
__device__ __forceinline__ void inv3(const double m[9], double out[9]) {
  out[0] = m[4] * m[8] - m[5] * m[7];
  out[3] = m[5] * m[6] - m[3] * m[8];
  out[6] = m[3] * m[7] - m[4] * m[6];
  const double det = m[0] * out[0] + m[1] * out[3] + m[2] * out[6];
  const double inv = 1.0 / det;
  out[1] = m[2] * m[7] - m[1] * m[8];
  out[4] = m[0] * m[8] - m[2] * m[6];
  out[7] = m[1] * m[6] - m[0] * m[7];
  out[2] = m[1] * m[5] - m[2] * m[4];
  out[5] = m[2] * m[3] - m[0] * m[5];
  out[8] = m[0] * m[4] - m[1] * m[3];
#pragma unroll
  for (int i = 0; i < 9; ++i) out[i] *= inv;
}

// Reduce-scatter of G values over the G lanes of a group: lane l returns the
// group sum of v[l]. Fixed pairing, so the result is deterministic.
template <int G>
__device__ __forceinline__ double reduce_scatter(double (&v)[G], int lane, unsigned mask) {
  double cur[G];
#pragma unroll
  for (int i = 0; i < G; ++i) cur[i] = v[i];
#pragma unroll
  for (int half = G / 2; half >= 1; half >>= 1) {
    const bool upper = (lane & half) != 0;
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const double send = upper ? cur[j] : cur[half + j];
      const double keep = upper ? cur[half + j] : cur[j];
      cur[j] = keep + __shfl_xor_sync(mask, send, half, G);
    }
  }
  return cur[0];
}

// Voigt index of the tensor pair (i, j).
__device__ __forceinline__ int voigt(int i, int j) {
  if (i == j) return i;
  const int s = i + j;  // (0,1) -> 3, (1,2) -> 4, (0,2) -> 5
  return s == 1 ? 3 : (s == 3 ? 4 : 5);
}

// Column (3 m + k) of the Green-Lagrange strain variation for an
// augmented node with gradient g (3): b[c] for Voigt c = (i, j).
__device__ __forceinline__ void bcol(const double F[9], const double g[3], int k, double b[6]) {
  b[0] = F[k * 3 + 0] * g[0];
  b[1] = F[k * 3 + 1] * g[1];
  b[2] = F[k * 3 + 2] * g[2];
  b[3] = F[k * 3 + 0] * g[1] + F[k * 3 + 1] * g[0];
  b[4] = F[k * 3 + 1] * g[2] + F[k * 3 + 2] * g[1];
  b[5] = F[k * 3 + 2] * g[0] + F[k * 3 + 0] * g[2];
}

// V(k, l, n) = sum_{j,i,m} g(j) F(k,i) F(l,m) D[v(i,j)][v(m,n)] (D, or D^T
// with `transpose`), times w, plus the geometric w S(j,n) g(j) delta_kl:
// K_ab(k, l) = sum_n V(k, l, n) g_b(n) is the block of B_a^T D B_b + G_a^T S G_b.
__device__ __forceinline__ void vtensor(const double* slot, const double g[3], bool transpose, bool geometric,
                                     double V[27]) {
  const double w = slot[kSlotW];
  const double* D = slot;
  const double* F = slot + kSlotF;
  double W[3][6];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int r = voigt(i, j);
        s += g[j] * (transpose ? D[c * 6 + r] : D[r * 6 + c]);
      }
      W[i][c] = w * s;
    }
  double Uk[3][6];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 6; ++c) Uk[k][c] = F[k * 3 + 0] * W[0][c] + F[k * 3 + 1] * W[1][c] + F[k * 3 + 2] * W[2][c];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) s += F[l * 3 + m] * Uk[k][voigt(m, n)];
        V[(k * 3 + l) * 3 + n] = s;
      }
  if (geometric) {
    const double* S = slot + kSlotS;
    double sg[3];
#pragma unroll
    for (int n = 0; n < 3; ++n)
      sg[n] = w * (g[0] * S[voigt(0, n)] + g[1] * S[voigt(1, n)] + g[2] * S[voigt(2, n)]);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int n = 0; n < 3; ++n) V[(k * 3 + k) * 3 + n] += sg[n];
  }
}

// The per-element context of a group: S is the shared-memory record of one
// element, which differs between the single element kernel and the phase
// kernels (each holds only the fields its stage reads).
template <int G, class Rec = ElemShared<G>>
struct Ctx {
  const Params* p;
  Rec* s;
  int lane;
  unsigned mask;
  int64_t e;
  int64_t npts;  // ne * nq: the state stride
  const double* state;
  double* trial;
  uint8_t* yield;
  double* hu;    // this lane's U G^T (per-lane memory)
  double* warm;  // this lane's last converged closest point (general return)
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};

// Mode gradients of point q: g~(i, m) = (det0 / det)(-2 xi_m) J0^-1(m, i).
template <int G, class Rec>
__device__ __forceinline__ void mode_grads(const Ctx<G, Rec>& c, int q, double gt[9]) {
  const double ratio = c.s->geo[q][10];
  const double nat[3] = {c.p->qp[q][0], c.p->qp[q][1], c.p->qp[q][2]};
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const double f = ratio * (-2.0 * nat[m]);
#pragma unroll
    for (int i = 0; i < 3; ++i) gt[i * 3 + m] = f * c.s->jinv0[m * 3 + i];
  }
}
// Gradient of node a at point q: g(i) = sum_c dN_a/dxi_c J^-1(c, i).
template <int G, class Rec>
__device__ __forceinline__ void node_grad(const Ctx<G, Rec>& c, int q, int a, double g[3]) {
  double dn[3];
  shape_grad(a, c.p->qp[q][0], c.p->qp[q][1], c.p->qp[q][2], dn);
  const double* ji = c.s->geo[q];
#pragma unroll
  for (int i = 0; i < 3; ++i) g[i] = dn[0] * ji[i] + dn[1] * ji[3 + i] + dn[2] * ji[6 + i];
}

// Reference geometry (set_up, IncompatibleModes.cpp:134-192). Returns 0 or
// SBK_EL_MESH_INVERTED (group-uniform).
template <int G, class Rec>
__device__ int set_up(const Ctx<G, Rec>& c) {
  Rec& s = *c.s;
  const Params& p = *c.p;
  // Centre Jacobian, every lane alike.
  double j0[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double dn[3];
    shape_grad(a, 0.0, 0.0, 0.0, dn);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) j0[i * 3 + k] += s.X[3 * a + i] * dn[k];
  }
  const double det0 = det3(j0);
  int bad = !(det0 > 0.0);
  if (c.lane == 0 && !bad) inv3(j0, s.jinv0);
  const int q = c.lane;
  if (q < p.nq && !bad) {
    double jq[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double dnq[8][3];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      shape_grad(a, p.qp[q][0], p.qp[q][1], p.qp[q][2], dnq[a]);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) jq[i * 3 + k] += s.X[3 * a + i] * dnq[a][k];
    }
    const double det = det3(jq);
    if (!(det > 0.0)) {
      bad = 1;
    } else {
      double ji[9];
      inv3(jq, ji);
#pragma unroll
      for (int i = 0; i < 9; ++i) s.geo[q][i] = ji[i];
      s.geo[q][9] = p.qp[q][3] * det;
      s.geo[q][10] = det0 / det;
      // hu = U G^T with G(i, a) = sum_c dN_a/dxi_c J^-1(c, i).
      double hu[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        double g[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) g[i] = dnq[a][0] * ji[i] + dnq[a][1] * ji[3 + i] + dnq[a][2] * ji[6 + i];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) hu[i * 3 + j] += s.U[3 * a + i] * g[j];
      }
#pragma unroll
      for (int i = 0; i < 9; ++i) c.hu[i] = hu[i];
    }
  }
  bad = __any_sync(c.mask, bad);
  c.sync();
  return bad ? SBK_EL_MESH_INVERTED : 0;
}

// The kinematics of point q at the modes `at` (kinematics_at,
// IncompatibleModes.cpp:195-225): its mode gradients gt, F, the largest
// |H| entry, the strain the return takes and, under logarithmic
// kinematics, the spectral data L of the log strain. Returns 0, or a
// point-failure code (an inverted point, a log strain out of range).
template <int G, class Rec>
__device__ __forceinline__ int point_kinematics(const Ctx<G, Rec>& c, int q, const double at[9], double gt[9],
                                                double F[9], double& hmax, double strain[6], LogKin& L) {
  const Params& p = *c.p;
  int code = 0;
  mode_grads(c, q, gt);
  double h[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double v = c.hu[i * 3 + j];
#pragma unroll
      for (int m = 0; m < 3; ++m) v += at[3 * m + i] * gt[j * 3 + m];
      h[i * 3 + j] = v;
    }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    hmax = fmax(hmax, fabs(h[i]));
    F[i] = h[i] + ((i % 4) == 0 ? 1.0 : 0.0);
  }
  if (p.kinematics == SBK_SMALL_STRAIN) {
    strain[0] = h[0];
    strain[1] = h[4];
    strain[2] = h[8];
    strain[3] = h[1] + h[3];
    strain[4] = h[5] + h[7];
    strain[5] = h[6] + h[2];
#pragma unroll
    for (int i = 0; i < 9; ++i) F[i] = (i % 4) == 0 ? 1.0 : 0.0;
  } else {
    double E[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        E[i * 3 + j] = 0.5 * (h[i * 3 + j] + h[j * 3 + i] + h[0 * 3 + i] * h[0 * 3 + j] +
                              h[1 * 3 + i] * h[1 * 3 + j] + h[2 * 3 + i] * h[2 * 3 + j]);
    double green[6] = {E[0], E[4], E[8], 2.0 * E[1], 2.0 * E[5], 2.0 * E[6]};
    if (p.kinematics == SBK_FINITE) {
#pragma unroll
      for (int i = 0; i < 6; ++i) strain[i] = green[i];
    } else {
      if (!(det3(F) > 0.0)) {
        code = SBK_EL_INVERTED_POINT;
      } else {
        code = log_strain(green, L, strain);
      }
    }
  }
  return code;
}

// After the point's response r: its yield flag, the material block M and
// stress S in the strain measure of the element (the logarithmic map, or
// as they are), and its slot for the group sums. MAPPED: r already holds
// them in the element's strain measure (the logarithmic map was applied).
template <int G, class Rec, bool MAPPED = false>
__device__ __forceinline__ void point_slot(const Ctx<G, Rec>& c, int q, const Response& r, const LogKin& L,
                                           const double F[9], double w, double hmax, double M[36], double S[6]) {
  const Params& p = *c.p;
  Rec& s = *c.s;
  c.yield[c.e * p.nq + q] = r.yielding ? 1 : 0;
#pragma unroll
  for (int i = 0; i < 36; ++i) M[i] = r.C[i];
  if (!MAPPED && p.kinematics == SBK_FINITE_LOGARITHMIC) {
    log_transform(L, r.stress, S, M);
  } else {
#pragma unroll
    for (int i = 0; i < 6; ++i) S[i] = r.stress[i];
  }
  double mmax = 0.0;
#pragma unroll
  for (int i = 0; i < 36; ++i) {
    s.slot[q][i] = M[i];
    mmax = fmax(mmax, fabs(M[i]));
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) s.slot[q][kSlotS + i] = S[i];
#pragma unroll
  for (int i = 0; i < 9; ++i) s.slot[q][kSlotF + i] = F[i];
  s.slot[q][kSlotW] = w;
  s.slot[q][kSlotE] = r.energy;
  s.slot[q][kSlotFl] = w * mmax * hmax * (1.0 + hmax);
}

// The group's side of a pass after every point has its slot (or failed):
// the first failure in the reference's order (the earliest stage, then the
// lowest point), else K_aa and the force, scale and floor sums. fail =
// (stage << 8) | q of this lane's failure (0: none), code its code.
// The nodal force f_u (24) and the energy of the pass from the points'
// slots, in point order: lane a (a < 8) node a, lane 7 the energy.
template <int G, class Rec>
__device__ __forceinline__ void force_sums(const Ctx<G, Rec>& c) {
  Rec& s = *c.s;
  const Params& p = *c.p;
  if (c.lane < 8) {
    const int a = c.lane;
    double ra[3] = {0, 0, 0}, en = 0.0;
    for (int qq = 0; qq < p.nq; ++qq) {
      const double* sl = s.slot[qq];
      const double* Fq = sl + kSlotF;
      const double* Sq = sl + kSlotS;
      const double wq = sl[kSlotW];
      double FS[9];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          FS[k * 3 + j] = Fq[k * 3 + 0] * Sq[voigt(0, j)] + Fq[k * 3 + 1] * Sq[voigt(1, j)] + Fq[k * 3 + 2] * Sq[voigt(2, j)];
      double g[3];
      node_grad(c, qq, a, g);
#pragma unroll
      for (int k = 0; k < 3; ++k) ra[k] += wq * (FS[k * 3 + 0] * g[0] + FS[k * 3 + 1] * g[1] + FS[k * 3 + 2] * g[2]);
      if (a == 7) en += wq * sl[kSlotE];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) s.r[3 * a + k] = ra[k];
    if (a == 7) s.energy = en;
  }
  c.sync();
}

// FORCES = false leaves out the nodal force and the energy (force_sums
// gives them, the same sums, for the pass that ends the iteration).
template <int G, class Rec, bool FORCES = true>
__device__ __forceinline__ int pass_sums(const Ctx<G, Rec>& c, bool active, int fail, int code, const double gt[9],
                                         const double F[9], const double M[36], const double S[6], double w) {
  Rec& s = *c.s;
  const Params& p = *c.p;
  const bool geometric = p.kinematics != SBK_SMALL_STRAIN;
  double kbuf[G];
  // The failure of the group: the first point of the earliest stage.
  int key = fail ? fail : 0x7fffffff;
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) key = min(key, __shfl_xor_sync(c.mask, key, o, G));
  if (key != 0x7fffffff) {
    const int owner = key & 0xff;
    const int out = __shfl_sync(c.mask, code, owner, G);
    c.sync();
    return out;
  }
  // K_aa: w ba^T (D ba) + geometric, streamed through the reduce-scatter in
  // chunks of G (row-major 9 x 9).
  const bool live = active;
  double Mba[6][9];
  if (live) {
#pragma unroll
    for (int col = 0; col < 9; ++col) {
      const int m = col / 3, k = col % 3;
      const double g[3] = {gt[0 * 3 + m], gt[1 * 3 + m], gt[2 * 3 + m]};
      double b[6];
      bcol(F, g, k, b);
#pragma unroll
      for (int r = 0; r < 6; ++r) {
        double v = 0.0;
#pragma unroll
        for (int d = 0; d < 6; ++d) v += M[r * 6 + d] * b[d];
        Mba[r][col] = v;
      }
    }
  }
  double geo[9];
  if (live && geometric) {
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int n = 0; n < 3; ++n) {
        double v = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) v += gt[i * 3 + m] * S[voigt(i, j)] * gt[j * 3 + n];
        geo[m * 3 + n] = w * v;
      }
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    double bi[6];
    if (live) {
      const int m = i / 3, k = i % 3;
      const double g[3] = {gt[0 * 3 + m], gt[1 * 3 + m], gt[2 * 3 + m]};
      bcol(F, g, k, bi);
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const int idx = i * 9 + j;
      double v = 0.0;
      if (live) {
#pragma unroll
        for (int r = 0; r < 6; ++r) v += bi[r] * Mba[r][j];
        v *= w;
        if (geometric && (i % 3) == (j % 3)) v += geo[(i / 3) * 3 + (j / 3)];
      }
      kbuf[idx % G] = v;
      if (idx % G == G - 1) {
        const double y = reduce_scatter<G>(kbuf, c.lane, c.mask);
        s.kc[(idx / G) * G + c.lane] = y;
      }
    }
  }
  if (81 % G != 0) {
#pragma unroll
    for (int i = 81 % G; i < G; ++i) kbuf[i] = 0.0;
    const double y = reduce_scatter<G>(kbuf, c.lane, c.mask);
    s.kc[(81 / G) * G + c.lane] = y;
  }
  c.sync();
  // The force and the scale sums over the points, in point order: lane a
  // (a < 8) node a, lanes 0-2 also mode a with its scale and floor sums,
  // lane 7 the energy.
  if (c.lane < 8) {
    const int a = c.lane;
    double ra[3] = {0, 0, 0}, rm[3] = {0, 0, 0}, sc[3] = {0, 0, 0}, fl[3] = {0, 0, 0}, en = 0.0;
    for (int qq = 0; qq < p.nq; ++qq) {
      const double* sl = s.slot[qq];
      const double* Fq = sl + kSlotF;
      const double* Sq = sl + kSlotS;
      const double wq = sl[kSlotW];
      double FS[9];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          FS[k * 3 + j] = Fq[k * 3 + 0] * Sq[voigt(0, j)] + Fq[k * 3 + 1] * Sq[voigt(1, j)] + Fq[k * 3 + 2] * Sq[voigt(2, j)];
      if (FORCES) {
        double g[3];
        node_grad(c, qq, a, g);
#pragma unroll
        for (int k = 0; k < 3; ++k) ra[k] += wq * (FS[k * 3 + 0] * g[0] + FS[k * 3 + 1] * g[1] + FS[k * 3 + 2] * g[2]);
      }
      if (a < 3) {
        double gtq[9];
        mode_grads(c, qq, gtq);
        const double gm[3] = {gtq[0 * 3 + a], gtq[1 * 3 + a], gtq[2 * 3 + a]};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          rm[k] += wq * (FS[k * 3 + 0] * gm[0] + FS[k * 3 + 1] * gm[1] + FS[k * 3 + 2] * gm[2]);
          double b[6];
          bcol(Fq, gm, k, b);
          double s1 = 0.0, s2 = 0.0;
#pragma unroll
          for (int r = 0; r < 6; ++r) {
            s1 += fabs(b[r]) * fabs(Sq[r]);
            s2 += fabs(b[r]);
          }
          sc[k] += wq * s1;
          fl[k] += sl[kSlotFl] * s2;
        }
      }
      if (FORCES && a == 7) en += wq * sl[kSlotE];
    }
    if (FORCES)
#pragma unroll
      for (int k = 0; k < 3; ++k) s.r[3 * a + k] = ra[k];
    if (a < 3) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        s.r[24 + 3 * a + k] = rm[k];
        s.scale[3 * a + k] = sc[k];
        s.flo[3 * a + k] = fl[k];
      }
    }
    if (FORCES && a == 7) s.energy = en;
  }
  c.sync();
  return 0;
}


// One pass (IncompatibleModes.cpp:337-342): the kinematics, the returns and
// the sums at `at` (9 values, identical in every lane). Returns 0 or the
// failure code of the first failing point in the reference's order.
template <int G, class Rec>
__device__ __noinline__ int pass(const Ctx<G, Rec>& c, const double at[9]) {
  const Params& p = *c.p;
  const int q = c.lane;
  const bool active = q < p.nq;
  int fail = 0;  // (stage << 8) | q, stage 1 kinematics, 2 return
  int code = 0;
  double gt[9], F[9], hmax = 0.0;
  double M[36], S[6];
  double w = 0.0;
  if (active) {
    w = c.s->geo[q][9];
    double strain[6];
    LogKin L;
    code = point_kinematics(c, q, at, gt, F, hmax, strain, L);
    if (code) fail = (1 << 8) | q;
    if (!fail) {
      PointState st{c.state + c.e * p.nq + q, c.trial + c.e * p.nq + q, c.npts};
      Response r;
      code = p.general ? general_return(p, strain, st, r, c.warm) : radial_return(p, strain, st, r);
      if (code) {
        fail = (2 << 8) | q;
      } else {
        point_slot(c, q, r, L, F, w, hmax, M, S);
      }
    }
  }
  return pass_sums(c, active, fail, code, gt, F, M, S, w);
}

// ---- element-level helpers (lane 0, shared memory) ---------------------------

// FullPivLU of a (9x9 row-major) into lu by the lanes of a group together
// (every lane calls it); true if invertible (Eigen's rank test: every |U_ii|
// above 9 eps of the largest pivot). Step k: lane l scans and eliminates
// rows k + l, k + l + G, ...; the pivot is the group's largest |entry| of
// the remaining block, ties to the first in column-major order as Eigen's
// scan takes it; rows, then columns exchanged; the column below the pivot
// multiplied by its reciprocal, then the rank-one update. rowp / colp hold
// the transpositions.
template <int G, class CT>
__device__ __forceinline__ bool fullpiv_lu9_rows_inline(const CT& c, const double* a, double* lu, int* rowp,
                                                        int* colp, double* maxpivot_out) {
  const int lane = c.lane;
  _Pragma("unroll 1") for (int i = lane; i < 81; i += G) lu[i] = a[i];
  c.sync();
  double maxpivot = 0.0;
  int nonzero = 9;
  _Pragma("unroll 1") for (int k = 0; k < 9; ++k) {
    double big = -1.0;
    int bi = k, bj = k;
    _Pragma("unroll 1") for (int j = k; j < 9; ++j)
      _Pragma("unroll 1") for (int i = k + lane; i < 9; i += G) {
        const double v = fabs(lu[i * 9 + j]);
        if (v > big) {
          big = v;
          bi = i;
          bj = j;
        }
      }
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
      const double ob = __shfl_xor_sync(c.mask, big, o, G);
      const int oi = __shfl_xor_sync(c.mask, bi, o, G);
      const int oj = __shfl_xor_sync(c.mask, bj, o, G);
      if (ob > big || (ob == big && (oj < bj || (oj == bj && oi < bi)))) {
        big = ob;
        bi = oi;
        bj = oj;
      }
    }
    if (big == 0.0) {
      nonzero = k;
      break;
    }
    if (big > maxpivot) maxpivot = big;
    if (lane == 0) {
      rowp[k] = bi;
      colp[k] = bj;
    }
    if (bi != k)
      _Pragma("unroll 1") for (int j = lane; j < 9; j += G) {
        const double t = lu[k * 9 + j];
        lu[k * 9 + j] = lu[bi * 9 + j];
        lu[bi * 9 + j] = t;
      }
    c.sync();
    if (bj != k)
      _Pragma("unroll 1") for (int i = lane; i < 9; i += G) {
        const double t = lu[i * 9 + k];
        lu[i * 9 + k] = lu[i * 9 + bj];
        lu[i * 9 + bj] = t;
      }
    c.sync();
    const double inv = 1.0 / lu[k * 9 + k];
    _Pragma("unroll 1") for (int i = k + 1 + lane; i < 9; i += G) {
      const double l = lu[i * 9 + k] * inv;
      lu[i * 9 + k] = l;
      _Pragma("unroll 1") for (int j = k + 1; j < 9; ++j) lu[i * 9 + j] -= l * lu[k * 9 + j];
    }
    c.sync();
  }
  if (lane == 0) {
    _Pragma("unroll 1") for (int i = nonzero; i < 9; ++i) rowp[i] = colp[i] = i;
    *maxpivot_out = maxpivot;
  }
  bool mine = true;
  if (nonzero == 9) {
    const double threshold = kEps * 9.0 * maxpivot;
    _Pragma("unroll 1") for (int i = lane; i < 9; i += G) mine = mine && fabs(lu[i * 9 + i]) > threshold;
  }
  const bool ok = __all_sync(c.mask, mine) && nonzero == 9;
  c.sync();
  return ok;
}

template <int G, class CT>
__device__ __noinline__ bool fullpiv_lu9_rows(const CT& c, const double* a, double* lu, int* rowp, int* colp,
                                              double* maxpivot_out) {
  return fullpiv_lu9_rows_inline<G>(c, a, lu, rowp, colp, maxpivot_out);
}

// x = A^-1 b with the FullPivLU factors (any lane; b and x may alias).
__device__ __forceinline__ void fullpiv_solve9_inline(const double* lu, const int* rowp, const int* colp,
                                                      const double* b, double* x) {
  double y[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) y[i] = b[i];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int pk = rowp[k];
#pragma unroll
    for (int i = k + 1; i < 9; ++i) {
      if (i == pk) {
        const double t = y[k];
        y[k] = y[i];
        y[i] = t;
      }
    }
  }
#pragma unroll
  for (int i = 1; i < 9; ++i)
#pragma unroll
    for (int j = 0; j < i; ++j) y[i] -= lu[i * 9 + j] * y[j];
#pragma unroll
  for (int i = 8; i >= 0; --i) {
#pragma unroll
    for (int j = i + 1; j < 9; ++j) y[i] -= lu[i * 9 + j] * y[j];
    y[i] /= lu[i * 9 + i];
  }
#pragma unroll
  for (int k = 8; k >= 0; --k) {
    const int pk = colp[k];
#pragma unroll
    for (int i = k + 1; i < 9; ++i) {
      if (i == pk) {
        const double t = y[k];
        y[k] = y[i];
        y[i] = t;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) x[i] = y[i];
}

__device__ __noinline__ void fullpiv_solve9(const double* lu, const int* rowp, const int* colp, const double* b,
                                            double* x) {
  fullpiv_solve9_inline(lu, rowp, colp, b, x);
}

// x = A^-T b with the FullPivLU factors of A (P A Q = L U, so
// A^-T = P^T L^-T U^-T Q^T): the column transpositions in order, U^T
// forward, L^T backward (unit diagonal), the row transpositions in reverse.
__device__ __noinline__ void fullpiv_solve9_t(const double* lu, const int* rowp, const int* colp, const double* b,
                                                 double* x) {
  double y[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) y[i] = b[i];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    const int pk = colp[k];
#pragma unroll
    for (int i = k + 1; i < 9; ++i) {
      if (i == pk) {
        const double t = y[k];
        y[k] = y[i];
        y[i] = t;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
#pragma unroll
    for (int j = 0; j < i; ++j) y[i] -= lu[j * 9 + i] * y[j];
    y[i] /= lu[i * 9 + i];
  }
#pragma unroll
  for (int i = 8; i >= 0; --i)
#pragma unroll
    for (int j = i + 1; j < 9; ++j) y[i] -= lu[j * 9 + i] * y[j];
#pragma unroll
  for (int k = 8; k >= 0; --k) {
    const int pk = rowp[k];
#pragma unroll
    for (int i = k + 1; i < 9; ++i) {
      if (i == pk) {
        const double t = y[k];
        y[k] = y[i];
        y[i] = t;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) x[i] = y[i];
}

// Cholesky (lower, in place); false at the first non-positive pivot.
__device__ __noinline__ bool llt9(double* a) {
  _Pragma("unroll 1") for (int k = 0; k < 9; ++k) {
    double x = a[k * 9 + k];
    _Pragma("unroll 1") for (int j = 0; j < k; ++j) x -= a[k * 9 + j] * a[k * 9 + j];
    if (x <= 0.0) return false;
    a[k * 9 + k] = sqrt(x);
    _Pragma("unroll 1") for (int i = k + 1; i < 9; ++i) {
      double v = a[i * 9 + k];
      _Pragma("unroll 1") for (int j = 0; j < k; ++j) v -= a[i * 9 + j] * a[k * 9 + j];
      a[i * 9 + k] = v / a[k * 9 + k];
    }
  }
  return true;
}
// llt9 by the lanes of a group together (every lane calls it): step k's
// diagonal by the lane of row k, then the rows below in parallel, each entry
// the same dot product in the same order - the same factor and the same
// answer.
template <int G, class CT>
__device__ __forceinline__ bool llt9_rows_inline(const CT& c, double* a) {
  const int lane = c.lane;
  _Pragma("unroll 1") for (int k = 0; k < 9; ++k) {
    int bad = 0;
    if (lane == k % G) {
      double x = a[k * 9 + k];
      _Pragma("unroll 1") for (int j = 0; j < k; ++j) x -= a[k * 9 + j] * a[k * 9 + j];
      if (x <= 0.0) {
        bad = 1;
      } else {
        a[k * 9 + k] = sqrt(x);
      }
    }
    bad = __shfl_sync(c.mask, bad, k % G, G);
    c.sync();
    if (bad) return false;
    _Pragma("unroll 1") for (int i = k + 1 + ((lane - (k + 1)) % G + G) % G; i < 9; i += G) {
      double v = a[i * 9 + k];
      _Pragma("unroll 1") for (int j = 0; j < k; ++j) v -= a[i * 9 + j] * a[k * 9 + j];
      a[i * 9 + k] = v / a[k * 9 + k];
    }
    c.sync();
  }
  return true;
}

template <int G, class CT>
__device__ __noinline__ bool llt9_rows(const CT& c, double* a) {
  return llt9_rows_inline<G>(c, a);
}

__device__ __noinline__ void llt9_solve(const double* l, const double* b, double* x) {
  double y[9];
  _Pragma("unroll 1") for (int i = 0; i < 9; ++i) {
    double v = b[i];
    _Pragma("unroll 1") for (int j = 0; j < i; ++j) v -= l[i * 9 + j] * y[j];
    y[i] = v / l[i * 9 + i];
  }
  _Pragma("unroll 1") for (int i = 8; i >= 0; --i) {
    double v = y[i];
    _Pragma("unroll 1") for (int j = i + 1; j < 9; ++j) v -= l[j * 9 + i] * y[j];
    y[i] = v / l[i * 9 + i];
  }
  _Pragma("unroll 1") for (int i = 0; i < 9; ++i) x[i] = y[i];
}

// Smallest eigenvalue and largest |eigenvalue| of a symmetric 9x9 (cyclic
// Jacobi on a copy in `a`, destroyed).
__device__ __noinline__ void sym_eig9(double* a, double* lo, double* top) {
  _Pragma("unroll 1") for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, diag = 0.0;
    _Pragma("unroll 1") for (int p = 0; p < 9; ++p) {
      diag += a[p * 9 + p] * a[p * 9 + p];
      _Pragma("unroll 1") for (int q = p + 1; q < 9; ++q) off += a[p * 9 + q] * a[p * 9 + q];
    }
    if (off == 0.0 || off <= 1.0e-36 * diag) break;
    _Pragma("unroll 1") for (int p = 0; p < 8; ++p)
      _Pragma("unroll 1") for (int q = p + 1; q < 9; ++q) {
        const double apq = a[p * 9 + q];
        if (apq == 0.0) continue;
        const double theta = (a[q * 9 + q] - a[p * 9 + p]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double cs = 1.0 / sqrt(t * t + 1.0);
        const double sn = t * cs;
        _Pragma("unroll 1") for (int k = 0; k < 9; ++k) {
          const double akp = a[k * 9 + p], akq = a[k * 9 + q];
          a[k * 9 + p] = cs * akp - sn * akq;
          a[k * 9 + q] = sn * akp + cs * akq;
        }
        _Pragma("unroll 1") for (int k = 0; k < 9; ++k) {
          const double apk = a[p * 9 + k], aqk = a[q * 9 + k];
          a[p * 9 + k] = cs * apk - sn * aqk;
          a[q * 9 + k] = sn * apk + cs * aqk;
        }
      }
  }
  double mn = a[0], mx = fabs(a[0]);
  _Pragma("unroll 1") for (int i = 1; i < 9; ++i) {
    mn = fmin(mn, a[i * 9 + i]);
    mx = fmax(mx, fabs(a[i * 9 + i]));
  }
  *lo = mn;
  *top = mx;
}

// Partial-pivoting LU solve of a 9x9 (in place), x = A^-1 b.
__device__ __noinline__ void plu9_solve(double* a, int* perm, const double* b, double* x) {
  _Pragma("unroll 1") for (int k = 0; k < 9; ++k) {
    int p = k;
    double big = fabs(a[k * 9 + k]);
    _Pragma("unroll 1") for (int i = k + 1; i < 9; ++i)
      if (fabs(a[i * 9 + k]) > big) {
        big = fabs(a[i * 9 + k]);
        p = i;
      }
    perm[k] = p;
    if (big != 0.0) {
      if (p != k)
        _Pragma("unroll 1") for (int j = 0; j < 9; ++j) {
          const double t = a[k * 9 + j];
          a[k * 9 + j] = a[p * 9 + j];
          a[p * 9 + j] = t;
        }
      const double inv = 1.0 / a[k * 9 + k];
      _Pragma("unroll 1") for (int i = k + 1; i < 9; ++i) a[i * 9 + k] *= inv;
    }
    _Pragma("unroll 1") for (int i = k + 1; i < 9; ++i)
      _Pragma("unroll 1") for (int j = k + 1; j < 9; ++j) a[i * 9 + j] -= a[i * 9 + k] * a[k * 9 + j];
  }
  double y[9];
  _Pragma("unroll 1") for (int i = 0; i < 9; ++i) y[i] = b[i];
  _Pragma("unroll 1") for (int k = 0; k < 9; ++k)
    if (perm[k] != k) {
      const double t = y[k];
      y[k] = y[perm[k]];
      y[perm[k]] = t;
    }
  _Pragma("unroll 1") for (int i = 1; i < 9; ++i)
    _Pragma("unroll 1") for (int j = 0; j < i; ++j) y[i] -= a[i * 9 + j] * y[j];
  _Pragma("unroll 1") for (int i = 8; i >= 0; --i) {
    _Pragma("unroll 1") for (int j = i + 1; j < 9; ++j) y[i] -= a[i * 9 + j] * y[j];
    y[i] /= a[i * 9 + i];
  }
  _Pragma("unroll 1") for (int i = 0; i < 9; ++i) x[i] = y[i];
}

// ---- the local iteration -------------------------------------------------------

template <int G>
struct Local {
  const Ctx<G>& c;
  ElemShared<G>& s;
  double residual;
  int iterations;
  __device__ Local(const Ctx<G>& cc) : c(cc), s(*cc.s), residual(0.0), iterations(0) {}

  __device__ double rnorm() const {
    double v = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) v += s.r[24 + i] * s.r[24 + i];
    return sqrt(v);
  }
  __device__ double rinf() const {
    double v = fabs(s.r[24]);
#pragma unroll
    for (int i = 1; i < 9; ++i) v = fmax(v, fabs(s.r[24 + i]));
    return v;
  }
  __device__ double vmax(const double* v) const {
    double m = fabs(v[0]);
#pragma unroll
    for (int i = 1; i < 9; ++i) m = fmax(m, fabs(v[i]));
    return m;
  }
  __device__ double ddot(const double* a, const double* b) const {
    double v = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) v += a[i] * b[i];
    return v;
  }
  // A pass at alpha + t d; true if every point evaluated.
  __device__ bool try_at(const double* d, double t) {
    double at[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) at[i] = s.alpha[i] + t * d[i];
    return pass<G>(c, at) == 0;
  }
  __device__ void advance(const double* d, double t) {
    c.sync();
    if (c.lane == 0)
#pragma unroll
      for (int i = 0; i < 9; ++i) s.alpha[i] += t * d[i];
    c.sync();
  }

  // search_norm (IncompatibleModes.cpp:359-383).
  __device__ __noinline__ bool search_norm(const double* d, double reach) {
    double best_step = 0.0, best = residual;
    bool last_is_best = false;
    double trial_step = reach;
    for (int search = 0; search < kMaxLineSearch; ++search, trial_step *= 0.5) {
      if (!try_at(d, trial_step)) {
        last_is_best = false;
        continue;
      }
      const double n = rnorm();
      last_is_best = n < best;
      if (last_is_best) {
        best = n;
        best_step = trial_step;
      }
      if (n <= kFullStepReduction * residual) break;
    }
    if (best_step == 0.0) return false;
    if (!last_is_best) try_at(d, best_step);
    advance(d, best_step);
    residual = best;
    return true;
  }

  // line_search (IncompatibleModes.cpp:398-456).
  __device__ __noinline__ bool line_search(const double* d) {
    const double phi0 = ddot(d, s.r0);
    double reach = 1.0;
    bool evaluated = try_at(d, 1.0);
    for (int halving = 0; !evaluated && halving < kMaxLineSearch; ++halving) {
      reach *= 0.5;
      evaluated = try_at(d, reach);
    }
    if (!evaluated) return false;
    const double full = rnorm();
    if (full <= kFullStepReduction * residual ||
        rinf() <= kLocalTolerance * vmax(s.scale) + kLocalRoundOff * vmax(s.flo)) {
      advance(d, reach);
      residual = full;
      return true;
    }
    const double phi1 = ddot(d, s.r + 24);
    if (!(phi0 < 0.0) || !(phi1 > 0.0) || !isfinite(phi1)) return search_norm(d, 0.5 * reach);
    double s0 = 0.0, f0 = phi0, s1 = reach, f1 = phi1, step = reach;
    int side = 0;
    for (int search = 0; search < kMaxLineSearch; ++search) {
      const double width = s1 - s0;
      step = fmin(fmax((s0 * f1 - s1 * f0) / (f1 - f0), s0 + 0.1 * width), s1 - 0.1 * width);
      evaluated = try_at(d, step);
      const double f = evaluated ? ddot(d, s.r + 24) : __longlong_as_double(0x7ff0000000000000LL);
      if (evaluated && fabs(f) <= kLineSearchRatio * fabs(phi0)) break;
      if (!evaluated || f > 0.0) {
        s1 = step;
        f1 = evaluated ? f : 0.5 * f1;
        if (side == 1) f0 *= 0.5;
        side = 1;
      } else {
        s0 = step;
        f0 = f;
        if (side == -1) f1 *= 0.5;
        side = -1;
      }
    }
    if (!evaluated) {
      if (s0 == 0.0) return false;
      step = s0;
      try_at(d, step);
    }
    advance(d, step);
    residual = rnorm();
    return true;
  }

  // solve_and_condense's loop (IncompatibleModes.cpp:353-546). Returns 0 or
  // a failure code; on success the last pass is at s.alpha and s.lu holds
  // the factors of its K_aa.
  __device__ __noinline__ int run() {
    // K_aa at alpha (k0), its symmetric part and scratch: lane 0's alone.
    double* work = s.work;
    {
      double at[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) at[i] = s.alpha[i];
      const int code = pass<G>(c, at);
      if (code) return code;
    }
    residual = rnorm();
    for (;;) {
      const double largest = rinf();
      const double scale = vmax(s.scale);
      const double floor_ = kLocalRoundOff * vmax(s.flo);
      const bool invertible = fullpiv_lu9_rows<G>(c, s.kc, s.lu, s.rowp, s.colp, &s.maxpivot);
      // k0 and r0 copies (the trial passes overwrite the sums).
      for (int i = c.lane; i < 81; i += G) work[i] = s.kc[i];
      for (int i = c.lane; i < 9; i += G) s.r0[i] = s.r[24 + i];
      c.sync();
      if (!invertible) return SBK_EL_LOCAL_SINGULAR;
      if (largest <= kLocalTolerance * scale + floor_ || largest == 0.0) return 0;
      if (iterations == kMaxLocal || !isfinite(largest)) return SBK_EL_LOCAL_NO_CONVERGE;
      ++iterations;
      // Newton's direction and the Cholesky test of the symmetric part.
      for (int idx = c.lane; idx < 81; idx += G) {
        const int i = idx / 9, j = idx % 9;
        const double v = 0.5 * (work[i * 9 + j] + work[j * 9 + i]);
        work[81 + idx] = v;   // sym
        work[162 + idx] = v;  // chol
      }
      c.sync();
      if (c.lane == 0) {
        double nw[9];
        fullpiv_solve9(s.lu, s.rowp, s.colp, s.r0, nw);
        for (int i = 0; i < 9; ++i) s.dir[i] = -nw[i];
      }
      const bool positive = llt9_rows<G>(c, work + 162);
      c.sync();
      if (positive) {
        if (line_search(s.dir)) continue;
      } else {
        if (try_at(s.dir, 1.0)) {
          const double full = rnorm();
          if (full <= kFullStepReduction * residual) {
            advance(s.dir, 1.0);
            residual = full;
            continue;
          }
        }
        if (c.lane == 0) {
          // The shifted direction (K_aa + mu I) d = -r_alpha.
          double* sym = work + 81;
          double* tmp = work + 162;
          for (int i = 0; i < 81; ++i) tmp[i] = sym[i];
          double lo, top;
          sym_eig9(tmp, &lo, &top);
          const double mu = kLocalShift * top - lo;
          for (int i = 0; i < 81; ++i) tmp[i] = work[i];
          for (int i = 0; i < 9; ++i) tmp[i * 9 + i] += mu;
          double x[9];
          plu9_solve(tmp, s.perm, s.r0, x);
          for (int i = 0; i < 9; ++i) s.dir2[i] = -x[i];
        }
        c.sync();
        if (line_search(s.dir2)) continue;
        if (search_norm(s.dir, 0.5)) continue;
      }
      // Levenberg-Marquardt (IncompatibleModes.cpp:522-545).
      double mu = 0.0;
      if (c.lane == 0) {
        double* normal = work + 81;
        for (int i = 0; i < 9; ++i)
          for (int j = 0; j < 9; ++j) {
            double v = 0.0;
            for (int k = 0; k < 9; ++k) v += work[k * 9 + i] * work[k * 9 + j];
            normal[i * 9 + j] = v;
          }
        double dmax = normal[0];
        for (int i = 1; i < 9; ++i) dmax = fmax(dmax, normal[i * 9 + i]);
        s.dval[0] = kLocalMarquardt * dmax;
      }
      c.sync();
      mu = s.dval[0];
      bool moved = false;
      for (int search = 0; search < kMaxLineSearch && !moved; ++search, mu *= 10.0) {
        c.sync();
        if (c.lane == 0) {
          double* normal = work + 81;
          double* a = work + 162;
          for (int i = 0; i < 81; ++i) a[i] = normal[i];
          for (int i = 0; i < 9; ++i) a[i * 9 + i] += mu;
          double grad[9];
          for (int i = 0; i < 9; ++i) {
            double v = 0.0;
            for (int j = 0; j < 9; ++j) v += work[j * 9 + i] * s.r0[j];
            grad[i] = v;
          }
          const bool ok = llt9(a);
          s.ival[2] = ok ? 1 : 0;
          if (ok) {
            double x[9];
            llt9_solve(a, grad, x);
            for (int i = 0; i < 9; ++i) s.dir2[i] = -x[i];
          }
        }
        c.sync();
        if (!s.ival[2]) continue;
        if (!try_at(s.dir2, 1.0)) continue;
        const double n = rnorm();
        if (n < residual) {
          advance(s.dir2, 1.0);
          residual = n;
          moved = true;
        }
      }
      if (!moved) return SBK_EL_LOCAL_NO_DESCENT;
    }
  }
};

// ---- the condensation ---------------------------------------------------------

// The condensation (IncompatibleModes.cpp:549-561) after the local
// iteration converged: lane a (a < 8) forms the rows of node a of K_ua (and
// K_au), the coupling C = K_aa^-1 K_au, f* = f_u - K_ua K_aa^-1 r_a and, with
// the tangent, K* = K_uu - K_ua C, symmetrised for a symmetric tangent. Reads
// the group's shared record: the last pass's slots and sums (slot, r), the
// factors of its K_aa (lu, rowp, colp) and the geometry; kc is overwritten.
// INLINE_SOLVE: the 9 x 9 solves compiled in place (their vectors stay in
// registers) rather than called.
template <int G, class Rec, bool INLINE_SOLVE = false>
__device__ __forceinline__ void condense(const Ctx<G, Rec>& c, int want_tangent, double* __restrict__ force,
                                         double* __restrict__ tangent) {
  const Params& p = *c.p;
  Rec& s = *c.s;
  const int lane = c.lane;
  const int64_t e = c.e;
  const bool sym = p.symmetric != 0;
  const bool geometric = p.kinematics != SBK_SMALL_STRAIN;
  const int nq = p.nq;
  // K_ua rows of node a (and K_au columns for a non-symmetric tangent).
  double kua[3][9], kau[3][9];
  if (lane < 8) {
    const int a = lane;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 9; ++j) kua[k][j] = kau[k][j] = 0.0;
    for (int q = 0; q < nq; ++q) {
      double g[3], gt[9], V[27];
      node_grad(c, q, a, g);
      mode_grads(c, q, gt);
      vtensor(s.slot[q], g, false, geometric, V);
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l)
            kua[k][3 * m + l] += V[(k * 3 + l) * 3 + 0] * gt[0 * 3 + m] + V[(k * 3 + l) * 3 + 1] * gt[1 * 3 + m] +
                                 V[(k * 3 + l) * 3 + 2] * gt[2 * 3 + m];
      if (!sym) {
        vtensor(s.slot[q], g, true, geometric, V);
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int l = 0; l < 3; ++l)
              kau[k][3 * m + l] += V[(k * 3 + l) * 3 + 0] * gt[0 * 3 + m] + V[(k * 3 + l) * 3 + 1] * gt[1 * 3 + m] +
                                   V[(k * 3 + l) * 3 + 2] * gt[2 * 3 + m];
      }
    }
    // The coupling C = K_aa^-1 K_au, columns of node a, into shared memory
    // (K_au(3m+l, 3a+k) = kau[k][3m+l], or kua[k][3m+l] when symmetric).
    double* C = s.kc;  // 9 x 24, column-major by DOF: C[col * 9 + i]
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double b[9];
#pragma unroll
      for (int j = 0; j < 9; ++j) b[j] = sym ? kua[k][j] : kau[k][j];
      double x[9];
      if (INLINE_SOLVE) fullpiv_solve9_inline(s.lu, s.rowp, s.colp, b, x);
      else fullpiv_solve9(s.lu, s.rowp, s.colp, b, x);
#pragma unroll
      for (int j = 0; j < 9; ++j) C[(3 * a + k) * 9 + j] = x[j];
    }
  }
  c.sync();
  if (lane < 8) {
    const int a = lane;
    // f* = f_u - K_ua K_aa^-1 r_alpha.
    double corr[9];
    if (INLINE_SOLVE) fullpiv_solve9_inline(s.lu, s.rowp, s.colp, s.r + 24, corr);
    else fullpiv_solve9(s.lu, s.rowp, s.colp, s.r + 24, corr);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double v = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) v += kua[k][j] * corr[j];
      force[e * 24 + 3 * a + k] = s.r[3 * a + k] - v;
    }
    if (want_tangent) {
      const double* C = s.kc;
#pragma unroll
      for (int chunk = 0; chunk < 2; ++chunk) {
        double acc[4][9];
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
          for (int i = 0; i < 9; ++i) acc[b][i] = 0.0;
        for (int q = 0; q < nq; ++q) {
          double g[3], V[27];
          node_grad(c, q, a, g);
          vtensor(s.slot[q], g, false, geometric, V);
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            double gb[3];
            node_grad(c, q, chunk * 4 + b, gb);
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
              for (int l = 0; l < 3; ++l)
                acc[b][k * 3 + l] += V[(k * 3 + l) * 3 + 0] * gb[0] + V[(k * 3 + l) * 3 + 1] * gb[1] +
                                     V[(k * 3 + l) * 3 + 2] * gb[2];
          }
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int bb = chunk * 4 + b;
          double* out = tangent + e * 576 + (8 * a + bb) * 9;
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int l = 0; l < 3; ++l) {
              double v = acc[b][k * 3 + l];
#pragma unroll
              for (int m = 0; m < 9; ++m) v -= kua[k][m] * C[(3 * bb + l) * 9 + m];
              out[k * 3 + l] = v;
            }
        }
      }
    }
  }
  if (want_tangent && sym) {
    // K* = (K* + K*^T) / 2: the unordered pair {(i, j), (j, i)} by the lane
    // that owns row min(i, j).
    __threadfence_block();
    c.sync();
    if (lane < 8) {
      double* Ke = tangent + e * 576;
      auto at = [&](int i, int j) -> double* { return Ke + (8 * (i / 3) + j / 3) * 9 + 3 * (i % 3) + (j % 3); };
      for (int k = 0; k < 3; ++k) {
        const int i = 3 * lane + k;
        for (int j = i + 1; j < 24; ++j) {
          double* x = at(i, j);
          double* y = at(j, i);
          const double v = 0.5 * (*x + *y);
          *x = v;
          *y = v;
        }
      }
    }
  }
}


// One element of the single kernel, start to finish: staging, set_up, the
// local iteration (Local::run), the condensation and the outputs.
template <int G>
__device__ __forceinline__ void element_body(const Params& p, int64_t ne, bool batch, int64_t e, ElemShared<G>* sh,
                                             int lane, unsigned mask, const double* __restrict__ coords,
                                             const int32_t* __restrict__ conn, const double* __restrict__ u,
                                             const double* __restrict__ state, const double* __restrict__ alpha_n,
                                             int want_tangent, double* __restrict__ force,
                                             double* __restrict__ tangent, double* __restrict__ energy,
                                             double* __restrict__ trial, double* __restrict__ alpha_out,
                                             uint8_t* __restrict__ yield, int32_t* __restrict__ iterations,
                                             int32_t* __restrict__ code, int32_t* __restrict__ first_failure) {
  double hu_lane[9];
  double warm_lane[8];
  warm_lane[7] = 0.0;  // no closest point yet
  Ctx<G> c{&p, sh, lane, mask, e, ne * p.nq, state, trial, yield, hu_lane, warm_lane};
  ElemShared<G>& s = *sh;
  // Stage the element's coordinates and displacements (lane a: node a); a
  // node index out of range fails the element before anything is read.
  int bad_node = 0;
  if (lane < 8) {
    if (batch) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        s.X[3 * lane + k] = coords[e * 24 + 3 * lane + k];
        s.U[3 * lane + k] = u[e * 24 + 3 * lane + k];
      }
    } else {
      const int64_t node = conn[e * 8 + lane];
      if (p.num_nodes > 0 && (node < 0 || node >= p.num_nodes)) {
        bad_node = 1;
      } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          s.X[3 * lane + k] = coords[node * 3 + k];
          s.U[3 * lane + k] = u[node * 3 + k];
        }
      }
    }
  }
  if (__any_sync(mask, bad_node)) {
    if (lane == 0) {
      code[e] = SBK_EL_BAD_NODE;
      if (first_failure) atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  for (int i = lane; i < 9; i += G) s.alpha[i] = alpha_n ? alpha_n[e * 9 + i] : 0.0;
  c.sync();
  int status = set_up<G>(c);
  Local<G> loc(c);
  if (!status) status = loc.run();
  if (status) {
    if (lane == 0) {
      code[e] = status;
      if (first_failure) atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  condense<G>(c, want_tangent, force, tangent);
  if (lane == 0) {
    energy[e] = s.energy;
    iterations[e] = loc.iterations;
    code[e] = 0;
  }
  for (int i = lane; i < 9; i += G) alpha_out[e * 9 + i] = s.alpha[i];
}

template <int G>
__global__ void __launch_bounds__(256) element_kernel(const __grid_constant__ Params p, int64_t ne, bool batch,
                                                      const double* __restrict__ coords,
                                                      const int32_t* __restrict__ conn, const double* __restrict__ u,
                                                      const double* __restrict__ state,
                                                      const double* __restrict__ alpha_n, int want_tangent,
                                                      double* __restrict__ force, double* __restrict__ tangent,
                                                      double* __restrict__ energy, double* __restrict__ trial,
                                                      double* __restrict__ alpha_out, uint8_t* __restrict__ yield,
                                                      int32_t* __restrict__ iterations, int32_t* __restrict__ code,
                                                      int32_t* __restrict__ first_failure,
                                                      const int32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const int64_t slot = (int64_t)blockIdx.x * epb + slot_in_block;
  ElemShared<G>* sh = reinterpret_cast<ElemShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  if (slot >= ne) return;  // whole groups leave together
  // The element of this slot: the schedule's order (elements of alike cost
  // side by side, so that the groups sharing a warp take alike paths), or
  // the mesh order. Every output is indexed by the element, so the order
  // changes no result.
  const int64_t e = order ? (int64_t)order[slot] : slot;
  element_body<G>(p, ne, batch, e, sh, lane, mask, coords, conn, u, state, alpha_n, want_tangent, force, tangent,
                  energy, trial, alpha_out, yield, iterations, code, first_failure);
}

// The single kernel over a device-counted list of elements (grid-stride):
// the phase kernels hand it the elements that leave their common road.
template <int G>
__global__ void __launch_bounds__(256) element_list_kernel(const __grid_constant__ Params p, int64_t ne, bool batch,
                                                           const double* __restrict__ coords,
                                                           const int32_t* __restrict__ conn,
                                                           const double* __restrict__ u,
                                                           const double* __restrict__ state,
                                                           const double* __restrict__ alpha_n, int want_tangent,
                                                           double* __restrict__ force, double* __restrict__ tangent,
                                                           double* __restrict__ energy, double* __restrict__ trial,
                                                           double* __restrict__ alpha_out,
                                                           uint8_t* __restrict__ yield,
                                                           int32_t* __restrict__ iterations,
                                                           int32_t* __restrict__ code,
                                                           int32_t* __restrict__ first_failure,
                                                           const int32_t* __restrict__ list,
                                                           const int32_t* __restrict__ count) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  ElemShared<G>* sh = reinterpret_cast<ElemShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  const int64_t n = *count;
  for (int64_t i = (int64_t)blockIdx.x * epb + slot_in_block; i < n; i += (int64_t)gridDim.x * epb) {
    __syncwarp(mask);
    element_body<G>(p, ne, batch, (int64_t)list[i], sh, lane, mask, coords, conn, u, state, alpha_n, want_tangent,
                    force, tangent, energy, trial, alpha_out, yield, iterations, code, first_failure);
  }
}

// ---- the local iteration as phase kernels over the whole mesh ------------------
//
// The same algorithm as element_kernel, split at its passes. Every element
// of the mesh runs its local iteration in lockstep rounds; a round is two
// launches over the elements still iterating:
//
//   wave_pass_kernel     one pass at each element's trial modes (the first
//                        round: the geometry, then the pass at alpha_n);
//   wave_control_kernel  the element-level step that follows a pass: the
//                        full-pivoting LU of K_aa and the convergence test,
//                        Newton's direction and the Cholesky test of the
//                        symmetric part, the acceptance of a full step.
//
// Most elements take only that road - every trial a full Newton step that
// the residual test accepts. An element that needs anything else (a step
// the test rejects, a trial pass that fails, an indefinite K_aa, hence the
// line searches, the shifted direction or Levenberg-Marquardt) is handed to
// element_kernel, which runs it again from the start; an element that
// converges goes to wave_condense_kernel, the condensation. Elements
// continuing to the next round are compacted into the next round's list.
// The passes, the factorisations, the tests and the condensation are the
// single kernel's own functions on the same values, so every element's
// outputs are bit-identical to element_kernel's (tested), and the rounds
// end by construction: the first pass plus at most kMaxLocal Newton steps.
//
// Why: the single kernel runs set-up, passes, 9 x 9 algebra and
// condensation back to back in one body of about 470 KB of code with 9.8 KB
// of shared memory per element - one 4-warp block per SM, its warps at
// different places in the code. Each phase kernel is a fraction of that
// code, its record a fraction of that memory, and the warps of a launch all
// run the same phase.

constexpr int kWaveRounds = kMaxLocal + 1;
constexpr int kKcStride = 88;  // K_aa as the reduce-scatter leaves it (81 used)

template <int G>
struct __align__(16) PassShared {
  double X[24];
  double U[24];
  double jinv0[9];
  double geo[G][12];
  double slot[G][kSlot];
  double kc[kKcStride];
  double r[33];
  double scale[9];
  double flo[9];
  double energy;
};

// The first pass kernel's record: the staged element and its geometry.
template <int G>
struct __align__(16) PreShared {
  double X[24];
  double U[24];
  double jinv0[9];
  double geo[G][12];
};

// Minimum resident blocks per SM (128 threads each) the compiler is told
// to fit, which bounds the registers of a thread: 2 allows 255, 3 170, 4
// 128. Measured on the 1M-element microbenchmark: these kernels lose 15-65 %
// at 3 or 4 (their spills grow), the logarithmic map 33 % at 3; the return
// kernel (sbk_return.cu) is best at 4.
#ifndef SBK_MINB_PRE
#define SBK_MINB_PRE 2
#endif
#ifndef SBK_MINB_POST
#define SBK_MINB_POST 2
#endif
#ifndef SBK_MINB_LOG
#define SBK_MINB_LOG 2
#endif
#ifndef SBK_MINB_CONDENSE
#define SBK_MINB_CONDENSE 2
#endif

// The control kernel's record: K_aa (then, once the LU has copied it, its
// symmetric part in place for the Cholesky test), the LU, the pass's sums.
// 1.9 KB per element, so that six 4-warp blocks fit an SM (the kernel's
// registers allow six).
template <int G>
struct __align__(16) ControlShared {
  double kc[81];
  double lu[81];
  double r[33];
  double scale[9];
  double flo[9];
  double alpha[9];
  double dir[9];
  double maxpivot;
  int rowp[9], colp[9];
};

template <int G>
struct __align__(16) CondenseShared {
  double jinv0[9];
  double geo[G][12];
  double slot[G][kSlot];
  double kc[216];
  double r[33];
  double lu[81];
  int rowp[9], colp[9];
  double energy;
};

__device__ __forceinline__ double modes_norm(const double* r) {
  double v = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) v += r[24 + i] * r[24 + i];
  return sqrt(v);
}
__device__ __forceinline__ double modes_inf(const double* r) {
  double v = fabs(r[24]);
#pragma unroll
  for (int i = 1; i < 9; ++i) v = fmax(v, fabs(r[24 + i]));
  return v;
}
__device__ __forceinline__ double abs_max9(const double* v) {
  double m = fabs(v[0]);
#pragma unroll
  for (int i = 1; i < 9; ++i) m = fmax(m, fabs(v[i]));
  return m;
}

// Warp-aggregated append of element e (by lane 0 of its group) to a list.
__device__ __forceinline__ void append(int32_t* list, int32_t* count, int64_t e) {
  const int pos = atomicAdd(count, 1);
  list[pos] = (int32_t)e;
}

// Pass, first kernel: per point the kinematics at the trial modes and the
// log strain; the response of every point the return takes elastically,
// here; the points that will yield listed for wave_return_kernel. The first
// round also stages the element and runs set_up.
template <int G, bool GENERAL>
__global__ void __launch_bounds__(128, SBK_MINB_PRE) wave_pre_kernel(const __grid_constant__ Params p, int64_t ne, int first,
                                                       const int32_t* __restrict__ list,
                                                       const int32_t* __restrict__ count, bool batch,
                                                       const double* __restrict__ coords,
                                                       const int32_t* __restrict__ conn,
                                                       const double* __restrict__ u, const double* __restrict__ state,
                                                       const double* __restrict__ alpha_n,
                                                       double* __restrict__ trial, uint8_t* __restrict__ yield,
                                                       int32_t* __restrict__ plastic,
                                                       int32_t* __restrict__ plastic_count,
                                                       const __grid_constant__ WaveBuffers w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  PreShared<G>* sh = reinterpret_cast<PreShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  const int64_t n = count ? (int64_t)*count : ne;
  const int nq = p.nq;
  PreShared<G>& s = *sh;
  for (int64_t i = (int64_t)blockIdx.x * epb + slot_in_block; i < n; i += (int64_t)gridDim.x * epb) {
    const int64_t e = list ? (int64_t)list[i] : i;
    double hu_lane[9];
    double* warm = w.warm + (e * 8 + lane) * 8;
    Ctx<G, PreShared<G>> c{&p, sh, lane, mask, e, ne * nq, state, trial, yield, hu_lane, warm};
    __syncwarp(mask);
    int status = 0;
    double at[9];
    if (first) {
      // The single kernel's start: staging (a node out of range fails the
      // element), alpha_n, set_up.
      int bad_node = 0;
      if (lane < 8) {
        if (batch) {
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            s.X[3 * lane + k] = coords[e * 24 + 3 * lane + k];
            s.U[3 * lane + k] = u[e * 24 + 3 * lane + k];
          }
        } else {
          const int64_t node = conn[e * 8 + lane];
          if (p.num_nodes > 0 && (node < 0 || node >= p.num_nodes)) {
            bad_node = 1;
          } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              s.X[3 * lane + k] = coords[node * 3 + k];
              s.U[3 * lane + k] = u[node * 3 + k];
            }
          }
        }
      }
      if (__any_sync(mask, bad_node)) {
        status = SBK_EL_BAD_NODE;
      } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) at[k] = alpha_n ? alpha_n[e * 9 + k] : 0.0;
        for (int k = lane; k < 9; k += G) w.alpha[e * 9 + k] = at[k];
        if (lane < 8)
#pragma unroll
          for (int k = 0; k < 8; ++k) warm[k] = 0.0;  // no closest point yet (warm[7] == 0)
        c.sync();
        status = set_up<G>(c);
        if (!status) {
          if (lane < nq) {
#pragma unroll
            for (int f = 0; f < 12; ++f) w.geo[(e * 12 + f) * G + lane] = s.geo[lane][f];
#pragma unroll
            for (int f = 0; f < 9; ++f) w.hu[(e * 9 + f) * G + lane] = hu_lane[f];
          }
          for (int k = lane; k < 9; k += G) w.jinv0[e * 9 + k] = s.jinv0[k];
        }
      }
    } else {
      // A trial at alpha + 1 dir (Local::try_at with t = 1).
#pragma unroll
      for (int k = 0; k < 9; ++k) at[k] = w.alpha[e * 9 + k] + 1.0 * w.dir[e * 9 + k];
      if (lane < nq) {
#pragma unroll
        for (int f = 0; f < 12; ++f) s.geo[lane][f] = w.geo[(e * 12 + f) * G + lane];
#pragma unroll
        for (int f = 0; f < 9; ++f) hu_lane[f] = w.hu[(e * 9 + f) * G + lane];
      }
      for (int k = lane; k < 9; k += G) s.jinv0[k] = w.jinv0[e * 9 + k];
      c.sync();
    }
    // An element that failed before its points: every point's record says
    // so (stage 0 sorts before the points' own failures).
    int fail = status ? 1 : 0, code = status;
    bool deferred = false;
    const int q = lane;
    if (!status && q < nq) {
      double gt[9], F[9], hmax = 0.0, strain[6];
      LogKin L;
      code = point_kinematics(c, q, at, gt, F, hmax, strain, L);
      if (code) fail = (1 << 8) | q;
      if (!fail) {
        PointState st{state + e * nq + q, trial + e * nq + q, ne * nq};
        Response r;
        if (GENERAL) {
          // The return's own trial test: its elastic branch outside the
          // loading window here; the rest (the whole return again) in
          // wave_return_kernel.
          GTrial T;
          general_trial(p, strain, st, T);
          if (!isfinite(T.f_trial)) {
            code = kFailReturn;
          } else if (general_is_elastic(p, T) && !general_loading_window(p, T)) {
            code = general_elastic<false>(p, T, st, r);
          } else {
            deferred = true;
#pragma unroll
            for (int k = 0; k < 6; ++k) *pw_at(w, e, kPwStrain + k, q) = strain[k];
          }
        } else {
          code = radial_return(p, strain, st, r);
        }
        if (code) fail = (2 << 8) | q;
        else if (!deferred) store_response(w, e, q, r);
      }
#pragma unroll
      for (int k = 0; k < 9; ++k) *pw_at(w, e, kPwF + k, q) = F[k];
      *pw_at(w, e, kPwHmax, q) = hmax;
#pragma unroll
      for (int k = 0; k < 9; ++k) *pw_at(w, e, kPwL + k, q) = L.q[k];
#pragma unroll
      for (int k = 0; k < 3; ++k) *pw_at(w, e, kPwL + 9 + k, q) = L.mu[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) *pw_at(w, e, kPwL + 12 + k, q) = L.first[k];
    }
    if (q < 8) {
      w.pfail[e * 8 + q] = fail;
      w.pcodes[e * 8 + q] = code;
    }
    // The group's deferred points, appended together.
    const unsigned ballot = __ballot_sync(mask, deferred);
    int base = 0;
    if (ballot) {
      const unsigned mine = ballot >> ((threadIdx.x % 32) / G * G);
      if (lane == 0) base = atomicAdd(plastic_count, __popc(mine));
      base = __shfl_sync(mask, base, 0, G);
      if (deferred) plastic[base + __popc(mine & ((1u << lane) - 1u))] = (int32_t)(e * 8 + q);
    }
  }
}

// Pass, second kernel: the general return of every listed point, in
// sbk_return.cu (launch_wave_returns).

// Pass, third kernel (logarithmic kinematics): the logarithmic map of every
// evaluated point's response (log_transform: S = P^T T, material = P^T C P
// + T : L), a thread per point, in place in the point's record. On its own
// its working set fits the registers of a thread; inside the sums kernel it
// spilled.
__global__ void __launch_bounds__(128, SBK_MINB_LOG) wave_log_kernel(int64_t ne, int nq, const int32_t* __restrict__ list,
                                                          const int32_t* __restrict__ count,
                                                          const __grid_constant__ WaveBuffers w) {
  const int64_t n = (count ? (int64_t)*count : ne) * 8;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int q = (int)(i & 7);
    if (q >= nq) continue;
    const int64_t e = list ? (int64_t)list[i >> 3] : (i >> 3);
    if (w.pfail[e * 8 + q]) continue;
    LogKin L;
#pragma unroll
    for (int k = 0; k < 9; ++k) L.q[k] = *pw_at(w, e, kPwL + k, q);
#pragma unroll
    for (int k = 0; k < 3; ++k) L.mu[k] = *pw_at(w, e, kPwL + 9 + k, q);
#pragma unroll
    for (int k = 0; k < 6; ++k) L.first[k] = *pw_at(w, e, kPwL + 12 + k, q);
    double t[6], S[6], M[36];
#pragma unroll
    for (int k = 0; k < 6; ++k) t[k] = *pw_at(w, e, kPwStress + k, q);
#pragma unroll
    for (int k = 0; k < 36; ++k) M[k] = *pw_at(w, e, kPwC + k, q);
    log_transform(L, t, S, M);
#pragma unroll
    for (int k = 0; k < 6; ++k) *pw_at(w, e, kPwStress + k, q) = S[k];
#pragma unroll
    for (int k = 0; k < 36; ++k) *pw_at(w, e, kPwC + k, q) = M[k];
  }
}

// Pass, fourth kernel: per point the yield flag and the slot; per element
// the first failure, K_aa and the sums (pass_sums) into the element's
// record.
template <int G>
__global__ void __launch_bounds__(128, SBK_MINB_POST) wave_post_kernel(const __grid_constant__ Params p, int64_t ne,
                                                        const int32_t* __restrict__ list,
                                                        const int32_t* __restrict__ count,
                                                        uint8_t* __restrict__ yield,
                                                        const __grid_constant__ WaveBuffers w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  PassShared<G>* sh = reinterpret_cast<PassShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  const int64_t n = count ? (int64_t)*count : ne;
  const int nq = p.nq;
  PassShared<G>& s = *sh;
  for (int64_t i = (int64_t)blockIdx.x * epb + slot_in_block; i < n; i += (int64_t)gridDim.x * epb) {
    const int64_t e = list ? (int64_t)list[i] : i;
    Ctx<G, PassShared<G>> c{&p, sh, lane, mask, e, ne * nq, nullptr, nullptr, yield, nullptr, nullptr};
    __syncwarp(mask);
    const int q = lane;
    const bool active = q < nq;
    int fail = 0, code = 0;
    if (q < 8) {
      fail = w.pfail[e * 8 + q];
      code = w.pcodes[e * 8 + q];
    }
    // A failure before the points (stage 0): the whole element.
    const int early = __shfl_sync(mask, fail == 1 ? code : 0, 0, G);
    if (early) {
      if (lane == 0) w.pcode[e] = early;
      continue;
    }
    if (active) {
#pragma unroll
      for (int f = 0; f < 12; ++f) s.geo[q][f] = w.geo[(e * 12 + f) * G + q];
    }
    for (int k = lane; k < 9; k += G) s.jinv0[k] = w.jinv0[e * 9 + k];
    c.sync();
    double gt[9], F[9], M[36], S[6], w_q = 0.0;
    if (active) {
      w_q = s.geo[q][9];
      mode_grads(c, q, gt);
#pragma unroll
      for (int k = 0; k < 9; ++k) F[k] = *pw_at(w, e, kPwF + k, q);
      if (!fail) {
        // The response in the element's strain measure (wave_log_kernel
        // applied the logarithmic map).
        Response r;
        LogKin L;
#pragma unroll
        for (int k = 0; k < 6; ++k) r.stress[k] = *pw_at(w, e, kPwStress + k, q);
#pragma unroll
        for (int k = 0; k < 36; ++k) r.C[k] = *pw_at(w, e, kPwC + k, q);
        r.energy = *pw_at(w, e, kPwEnergy, q);
        r.yielding = *pw_at(w, e, kPwYield, q) != 0.0;
        const double hmax = *pw_at(w, e, kPwHmax, q);
        point_slot<G, PassShared<G>, true>(c, q, r, L, F, w_q, hmax, M, S);
      }
    }
    // The sums read the point's M, S and F back from its slot in shared
    // memory, so that they need not stay in registers.
    const double* sl = s.slot[q < nq ? q : 0];
    const int status = pass_sums<G, PassShared<G>, false>(c, active, fail, code, gt, sl + kSlotF, sl, sl + kSlotS, w_q);
    if (lane == 0) w.pcode[e] = status;
    if (!status) {
      for (int k = lane; k < 81; k += G) w.kc[e * kKcStride + k] = s.kc[k];
      for (int k = lane; k < 9; k += G) {
        w.r[e * 33 + 24 + k] = s.r[24 + k];
        w.sf[e * 19 + k] = s.scale[k];
        w.sf[e * 19 + 9 + k] = s.flo[k];
      }
      if (active) {
#pragma unroll 6
        for (int f = 0; f < kSlot; ++f) w.slot[(e * kSlot + f) * G + q] = s.slot[q][f];
      }
    }
  }
}

// A failed element: its status and the lowest failing element, as the
// single kernel reports them.
__device__ __forceinline__ void wave_fail(int32_t* code, int32_t* first_failure, int64_t e, int status) {
  code[e] = status;
  if (first_failure) atomicMin(first_failure, (int32_t)e);
}

template <int G>
__global__ void __launch_bounds__(128) wave_control_kernel(const __grid_constant__ Params p, int64_t ne, int first,
                                                           const int32_t* __restrict__ list,
                                                           const int32_t* __restrict__ count,
                                                           const __grid_constant__ WaveBuffers w,
                                                           int32_t* __restrict__ next, int32_t* __restrict__ next_count,
                                                           int32_t* __restrict__ code,
                                                           int32_t* __restrict__ first_failure) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  ControlShared<G>* sh = reinterpret_cast<ControlShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  const int64_t n = count ? (int64_t)*count : ne;
  ControlShared<G>& s = *sh;
  int32_t* done_list = w.done;
  int32_t* done_count = w.counts + kWaveRounds + 1;
  int32_t* fallback_list = w.fallback;
  int32_t* fallback_count = w.counts + kWaveRounds + 2;
  for (int64_t i = (int64_t)blockIdx.x * epb + slot_in_block; i < n; i += (int64_t)gridDim.x * epb) {
    const int64_t e = list ? (int64_t)list[i] : i;
    Ctx<G, ControlShared<G>> c{&p, sh, lane, mask, e, 0, nullptr, nullptr, nullptr, nullptr, nullptr};
    __syncwarp(mask);
    const int pc = w.pcode[e];
    if (pc) {
      // A failed first pass fails the element (Local::run); a failed trial
      // is the line search's business.
      if (lane == 0) {
        if (first) wave_fail(code, first_failure, e, pc);
        else append(fallback_list, fallback_count, e);
      }
      continue;
    }
    for (int k = lane; k < 81; k += G) s.kc[k] = w.kc[e * kKcStride + k];
    for (int k = lane; k < 33; k += G) s.r[k] = w.r[e * 33 + k];
    for (int k = lane; k < 9; k += G) {
      s.scale[k] = w.sf[e * 19 + k];
      s.flo[k] = w.sf[e * 19 + 9 + k];
      s.alpha[k] = w.alpha[e * 9 + k];
      s.dir[k] = w.dir[e * 9 + k];
    }
    int iterations = first ? 0 : w.iters[e];
    double residual = first ? 0.0 : w.res[e];
    c.sync();
    if (first) {
      residual = modes_norm(s.r);
    } else {
      // line_search's full step (IncompatibleModes.cpp:398-410): accepted
      // when it reduces the residual enough or meets the tolerance.
      const double full = modes_norm(s.r);
      if (full <= kFullStepReduction * residual ||
          modes_inf(s.r) <= kLocalTolerance * abs_max9(s.scale) + kLocalRoundOff * abs_max9(s.flo)) {
        c.sync();
        if (lane == 0)
#pragma unroll
          for (int k = 0; k < 9; ++k) s.alpha[k] += 1.0 * s.dir[k];
        c.sync();
        residual = full;
      } else {
        if (lane == 0) append(fallback_list, fallback_count, e);
        continue;
      }
    }
    // The head of solve_and_condense's loop (IncompatibleModes.cpp:353-397).
    const double largest = modes_inf(s.r);
    const double scale = abs_max9(s.scale);
    const double floor_ = kLocalRoundOff * abs_max9(s.flo);
    const bool invertible = fullpiv_lu9_rows_inline<G>(c, s.kc, s.lu, s.rowp, s.colp, &s.maxpivot);
    c.sync();
    if (!invertible) {
      if (lane == 0) wave_fail(code, first_failure, e, SBK_EL_LOCAL_SINGULAR);
      continue;
    }
    if (largest <= kLocalTolerance * scale + floor_ || largest == 0.0) {
      // Converged: the factors of this K_aa for the condensation.
      for (int k = lane; k < 81; k += G) w.kc[e * kKcStride + k] = s.lu[k];
      for (int k = lane; k < 9; k += G) {
        w.piv[e * 18 + k] = s.rowp[k];
        w.piv[e * 18 + 9 + k] = s.colp[k];
        w.alpha[e * 9 + k] = s.alpha[k];
      }
      if (lane == 0) {
        w.iters[e] = iterations;
        append(done_list, done_count, e);
      }
      continue;
    }
    if (iterations == kMaxLocal || !isfinite(largest)) {
      if (lane == 0) wave_fail(code, first_failure, e, SBK_EL_LOCAL_NO_CONVERGE);
      continue;
    }
    ++iterations;
    // The symmetric part (K + K^T) / 2 in place: each lane owns the pairs
    // (a, b), a <= b, it writes, and reads nothing another lane writes.
    for (int idx = lane; idx < 45; idx += G) {
      int a = 0, rest = idx;
      while (rest >= 9 - a) {
        rest -= 9 - a;
        ++a;
      }
      const int b = a + rest;
      const double v = 0.5 * (s.kc[a * 9 + b] + s.kc[b * 9 + a]);
      s.kc[a * 9 + b] = v;
      s.kc[b * 9 + a] = v;
    }
    c.sync();
    if (lane == 0) {
      double nw[9];
      fullpiv_solve9_inline(s.lu, s.rowp, s.colp, s.r + 24, nw);
      for (int k = 0; k < 9; ++k) s.dir[k] = -nw[k];
    }
    const bool positive = llt9_rows_inline<G>(c, s.kc);
    c.sync();
    if (!positive) {
      if (lane == 0) append(fallback_list, fallback_count, e);
      continue;
    }
    for (int k = lane; k < 9; k += G) {
      w.alpha[e * 9 + k] = s.alpha[k];
      w.dir[e * 9 + k] = s.dir[k];
    }
    if (lane == 0) {
      w.iters[e] = iterations;
      w.res[e] = residual;
      append(next, next_count, e);
    }
  }
}

template <int G>
__global__ void __launch_bounds__(128, SBK_MINB_CONDENSE) wave_condense_kernel(const __grid_constant__ Params p, int64_t ne,
                                                            const __grid_constant__ WaveBuffers w, int want_tangent,
                                                            double* __restrict__ force, double* __restrict__ tangent,
                                                            double* __restrict__ energy,
                                                            double* __restrict__ alpha_out,
                                                            int32_t* __restrict__ iterations,
                                                            int32_t* __restrict__ code) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  CondenseShared<G>* sh = reinterpret_cast<CondenseShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  const int64_t n = w.counts[kWaveRounds + 1];
  const int nq = p.nq;
  CondenseShared<G>& s = *sh;
  for (int64_t i = (int64_t)blockIdx.x * epb + slot_in_block; i < n; i += (int64_t)gridDim.x * epb) {
    const int64_t e = w.done[i];
    Ctx<G, CondenseShared<G>> c{&p, sh, lane, mask, e, ne * nq, nullptr, nullptr, nullptr, nullptr, nullptr};
    __syncwarp(mask);
    if (lane < nq) {
#pragma unroll
      for (int f = 0; f < 12; ++f) s.geo[lane][f] = w.geo[(e * 12 + f) * G + lane];
#pragma unroll 6
      for (int f = 0; f < kSlot; ++f) s.slot[lane][f] = w.slot[(e * kSlot + f) * G + lane];
    }
    for (int k = lane; k < 9; k += G) {
      s.jinv0[k] = w.jinv0[e * 9 + k];
      s.rowp[k] = w.piv[e * 18 + k];
      s.colp[k] = w.piv[e * 18 + 9 + k];
    }
    for (int k = lane; k < 81; k += G) s.lu[k] = w.kc[e * kKcStride + k];
    for (int k = lane; k < 9; k += G) s.r[24 + k] = w.r[e * 33 + 24 + k];
    c.sync();
    force_sums(c);  // f_u and the energy of the last pass
    condense<G, CondenseShared<G>, true>(c, want_tangent, force, tangent);
    if (lane == 0) {
      energy[e] = s.energy;
      iterations[e] = w.iters[e];
      code[e] = 0;
    }
    for (int k = lane; k < 9; k += G) alpha_out[e * 9 + k] = w.alpha[e * 9 + k];
  }
}

// ---- the shape derivative: lambda . d f* / d X ---------------------------------
//
// For the condensed residual f*(u, X) of an IM Hex8 at fixed displacements
// and committed history, with the modes at their local equilibrium
// r_a(u, alpha, X) = 0: lambda^T d f*/dX = [lambda; mu]^T d r/dX |_alpha with
// mu = -K_aa^-T K_ua^T lambda, and r = sum_q w F S [G | G~] (nodes and
// modes). Per point the reverse chain runs r -> (w, F, S, [G | G~]);
// S -> E through the point's material tangent dS/dE; E -> F; F = I + U
// [G | G~]^T -> [G | G~]; G = dN J^-1, G~ = (det0/det)(-2 xi) J0^-1 and
// w = w_q det J -> (J, J0) -> X.

// One point's share: xb (24, node-major) and j0b (9, row-major) accumulate.
template <int G>
__device__ __noinline__ void vjp_point(const Ctx<G>& c, int q, const double* lam, const double* mu, double xb[24],
                                       double j0b[9]) {
  const ElemShared<G>& s = *c.s;
  const double* sl = s.slot[q];
  const double* Fp = sl + kSlotF;
  const double* Sv = sl + kSlotS;
  const double w = sl[kSlotW];
  const double* Ji = s.geo[q];  // J^-1, row-major
  const double ratio = s.geo[q][10];
  double S[9] = {Sv[0], Sv[3], Sv[5], Sv[3], Sv[1], Sv[4], Sv[5], Sv[4], Sv[2]};
  // Q = Lambda Ghat^T (3 x 3), FS = F S, phi = w sum Lambda . (F S Ghat).
  double Q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double dn[8][3];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    shape_grad(a, c.p->qp[q][0], c.p->qp[q][1], c.p->qp[q][2], dn[a]);
    double g[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] = dn[a][0] * Ji[i] + dn[a][1] * Ji[3 + i] + dn[a][2] * Ji[6 + i];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) Q[k * 3 + j] += lam[3 * a + k] * g[j];
  }
  double gt[9];  // G~(i, m) at gt[i * 3 + m]
  mode_grads(c, q, gt);
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) Q[k * 3 + j] += mu[3 * m + k] * gt[j * 3 + m];
  double FS[9];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) FS[k * 3 + j] = Fp[k * 3 + 0] * S[j] + Fp[k * 3 + 1] * S[3 + j] + Fp[k * 3 + 2] * S[6 + j];
  double phi = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) phi += FS[i] * Q[i];
  phi *= w;
  // Sbar = w sym(F^T Q) -> sbar (normal, 2 x shear) -> ebar = M^T sbar -> Ebar.
  double FtQ[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      FtQ[i * 3 + j] = w * (Fp[0 * 3 + i] * Q[0 * 3 + j] + Fp[1 * 3 + i] * Q[1 * 3 + j] + Fp[2 * 3 + i] * Q[2 * 3 + j]);
  const int vi[6] = {0, 1, 2, 0, 1, 2}, vj[6] = {0, 1, 2, 1, 2, 0};
  double sb[6];
#pragma unroll
  for (int cc = 0; cc < 6; ++cc) {
    const double sym = 0.5 * (FtQ[vi[cc] * 3 + vj[cc]] + FtQ[vj[cc] * 3 + vi[cc]]);
    sb[cc] = cc < 3 ? sym : 2.0 * sym;
  }
  double Eb[9];
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    double acc = 0.0;
#pragma unroll
    for (int cc = 0; cc < 6; ++cc) acc += sl[cc * 6 + d] * sb[cc];
    Eb[vi[d] * 3 + vj[d]] = acc;
    Eb[vj[d] * 3 + vi[d]] = acc;
  }
  // Fbar = w Q S + F Ebar.
  double Fb[9];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      Fb[k * 3 + j] = w * (Q[k * 3 + 0] * S[j] + Q[k * 3 + 1] * S[3 + j] + Q[k * 3 + 2] * S[6 + j]) +
                      Fp[k * 3 + 0] * Eb[j] + Fp[k * 3 + 1] * Eb[3 + j] + Fp[k * 3 + 2] * Eb[6 + j];
  // Gbar = w (F S)^T Lambda + Fbar^T U, node by node; K1 = sum_a dN_a Gbar_a^T.
  double K1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double gb[3];
#pragma unroll
    for (int j = 0; j < 3; ++j)
      gb[j] = w * (FS[0 * 3 + j] * lam[3 * a + 0] + FS[1 * 3 + j] * lam[3 * a + 1] + FS[2 * 3 + j] * lam[3 * a + 2]) +
              Fb[0 * 3 + j] * s.U[3 * a + 0] + Fb[1 * 3 + j] * s.U[3 * a + 1] + Fb[2 * 3 + j] * s.U[3 * a + 2];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
      for (int j = 0; j < 3; ++j) K1[cc * 3 + j] += dn[a][cc] * gb[j];
  }
  // Modes: Gbar~ (3 x 3), R and K2.
  double R = 0.0, K2[9];
  const double cm[3] = {-2.0 * c.p->qp[q][0], -2.0 * c.p->qp[q][1], -2.0 * c.p->qp[q][2]};
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double gbm = w * (FS[0 * 3 + i] * mu[3 * m + 0] + FS[1 * 3 + i] * mu[3 * m + 1] + FS[2 * 3 + i] * mu[3 * m + 2]) +
                         Fb[0 * 3 + i] * s.alpha[3 * m + 0] + Fb[1 * 3 + i] * s.alpha[3 * m + 1] +
                         Fb[2 * 3 + i] * s.alpha[3 * m + 2];
      R += gbm * cm[m] * s.jinv0[m * 3 + i];
      K2[m * 3 + i] = cm[m] * gbm;
    }
  // Jbar = (phi - ratio R) J^-T - J^-T K1 J^-T; J0bar += ratio R J0^-T - ratio J0^-T K2 J0^-T.
  const double* J0i = s.jinv0;
  double Jb[9];
#pragma unroll
  for (int pp = 0; pp < 3; ++pp)
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double a1 = 0.0, a2 = 0.0;
#pragma unroll
      for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          a1 += Ji[cc * 3 + pp] * K1[cc * 3 + j] * Ji[r * 3 + j];
          a2 += J0i[cc * 3 + pp] * K2[cc * 3 + j] * J0i[r * 3 + j];
        }
      Jb[pp * 3 + r] = (phi - ratio * R) * Ji[r * 3 + pp] - a1;
      j0b[pp * 3 + r] += ratio * R * J0i[r * 3 + pp] - ratio * a2;
    }
  // J = X dN: Xbar_ia += sum_c Jbar_ic dN_ac.
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      xb[3 * a + i] += Jb[i * 3 + 0] * dn[a][0] + Jb[i * 3 + 1] * dn[a][1] + Jb[i * 3 + 2] * dn[a][2];
}

template <int G>
__global__ void __launch_bounds__(256) vjp_kernel(const __grid_constant__ Params p, int64_t ne,
                                                  const double* __restrict__ coords, const int32_t* __restrict__ conn,
                                                  const double* __restrict__ u, const double* __restrict__ state,
                                                  const double* __restrict__ alpha_n,
                                                  const double* __restrict__ lambda, double* __restrict__ trial,
                                                  uint8_t* __restrict__ yield, int32_t* __restrict__ code,
                                                  int32_t* __restrict__ first_failure, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const int64_t e = (int64_t)blockIdx.x * epb + slot_in_block;
  ElemShared<G>* sh = reinterpret_cast<ElemShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  if (e >= ne) return;
  double hu_lane[9];
  double warm_lane[8];
  warm_lane[7] = 0.0;
  Ctx<G> c{&p, sh, lane, mask, e, ne * p.nq, state, trial, yield, hu_lane, warm_lane};
  ElemShared<G>& s = *sh;
  int bad_node = 0;
  double lam_a[3] = {0.0, 0.0, 0.0};
  if (lane < 8) {
    const int64_t node = conn[e * 8 + lane];
    if (p.num_nodes > 0 && (node < 0 || node >= p.num_nodes)) {
      bad_node = 1;
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        s.X[3 * lane + k] = coords[node * 3 + k];
        s.U[3 * lane + k] = u[node * 3 + k];
        lam_a[k] = lambda[node * 3 + k];
      }
    }
  }
  if (__any_sync(mask, bad_node)) {
    if (lane == 0) {
      code[e] = SBK_EL_BAD_NODE;
      atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  for (int i = lane; i < 9; i += G) s.alpha[i] = alpha_n ? alpha_n[e * 9 + i] : 0.0;
  c.sync();
  int status = set_up<G>(c);
  Local<G> loc(c);
  if (!status) status = loc.run();
  if (status) {
    if (lane == 0) {
      code[e] = status;
      atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  const bool geometric = p.kinematics != SBK_SMALL_STRAIN;
  // K_ua^T lambda, node by node (lane a), summed in node order by lane 0.
  double* part = s.work;  // 8 x 9 partial sums, then lambda (24) and mu (9)
  if (lane < 8) {
    const int a = lane;
    double kua[3][9];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 9; ++j) kua[k][j] = 0.0;
    for (int q = 0; q < p.nq; ++q) {
      double g[3], gt[9], V[27];
      node_grad(c, q, a, g);
      mode_grads(c, q, gt);
      vtensor(s.slot[q], g, false, geometric, V);
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l)
            kua[k][3 * m + l] += V[(k * 3 + l) * 3 + 0] * gt[0 * 3 + m] + V[(k * 3 + l) * 3 + 1] * gt[1 * 3 + m] +
                                 V[(k * 3 + l) * 3 + 2] * gt[2 * 3 + m];
    }
#pragma unroll
    for (int j = 0; j < 9; ++j)
      part[a * 9 + j] = kua[0][j] * lam_a[0] + kua[1][j] * lam_a[1] + kua[2][j] * lam_a[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) part[72 + 3 * a + k] = lam_a[k];
  }
  c.sync();
  if (lane == 0) {
    double b[9], y[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      double acc = 0.0;
      for (int a = 0; a < 8; ++a) acc += part[a * 9 + j];
      b[j] = acc;
    }
    fullpiv_solve9_t(s.lu, s.rowp, s.colp, b, y);
#pragma unroll
    for (int j = 0; j < 9; ++j) part[96 + j] = -y[j];
  }
  c.sync();
  // Every point's share, then the sums over the points (reduce-scatter of
  // 33 values: 24 of Xbar, 9 of J0bar), and J0 = X dN(0) folded in.
  double xb[24], j0b[9];
#pragma unroll
  for (int i = 0; i < 24; ++i) xb[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) j0b[i] = 0.0;
  if (lane < p.nq) vjp_point<G>(c, lane, part + 72, part + 96, xb, j0b);
  double* red = s.kc;  // 33 sums
#pragma unroll
  for (int chunk = 0; chunk * G < 33; ++chunk) {
    double buf[G];
#pragma unroll
    for (int i = 0; i < G; ++i) {
      const int idx = chunk * G + i;
      buf[i] = idx < 24 ? xb[idx < 24 ? idx : 0] : (idx < 33 ? j0b[idx - 24 < 9 && idx >= 24 ? idx - 24 : 0] : 0.0);
    }
    const double v = reduce_scatter<G>(buf, lane, mask);
    if (chunk * G + lane < 33) red[chunk * G + lane] = v;
  }
  c.sync();
  if (lane < 8) {
    const int a = lane;
    double dn0[3];
    shape_grad(a, 0.0, 0.0, 0.0, dn0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
      out[e * 24 + 3 * a + i] = red[3 * a + i] + red[24 + i * 3 + 0] * dn0[0] + red[24 + i * 3 + 1] * dn0[1] +
                                red[24 + i * 3 + 2] * dn0[2];
  }
  if (lane == 0) code[e] = 0;
}

// ---- the standard Hex8 -------------------------------------------------------
//
// elastoplastic_element for an element without internal modes
// (Elastoplastic.cpp:226-340, kinematics_of :104-168): per point the
// kinematics (B, B_NL or P B_NL), with mean dilatation (B-bar) the
// element's averaged dilatation in the strain and its variation, the return,
// then f = sum w b^T sigma and the tangent. Lane = point as in K1; the
// per-point material blocks go through the same slots, so the
// B_NL^T M B_NL + geometric part is K1's V-tensor form; the mean-dilatation
// terms are rank-two updates (w/3)(left s^T + s a_mc^T) of 24-vectors that
// are all B_NL^T v for a per-point 6-vector v, built node by node.

constexpr int kStdPt = 26;  // per point: pv 6 | u1 6 | u2 6 | m.C m | S(T) 6 | tr T
constexpr int kStdPv = 0, kStdU1 = 6, kStdU2 = 12, kStdMcm = 18, kStdST = 19, kStdTr = 25;

template <int G>
struct __align__(16) StdExtra {
  double pt[G][kStdPt];
  double mean_row[24];  // the volume average of the points' dilatation rows
  double red[32];       // group sums: w d (24), w, w tr(strain)
};

// [B_NL^T v] at DOF 3a + k for the node gradient g (B_NL from F; F = I: B).
__device__ __forceinline__ double bnl_t(const double F[9], const double g[3], int k, const double v[6]) {
  double b[6];
  bcol(F, g, k, b);
  return b[0] * v[0] + b[1] * v[1] + b[2] * v[2] + b[3] * v[3] + b[4] * v[4] + b[5] * v[5];
}

// The points of a standard element: kinematics, mean dilatation, returns,
// slots. Returns 0 or the failure code of the first failing point in the
// reference's order.
template <int G>
__device__ __noinline__ int std_points(const Ctx<G>& c, StdExtra<G>* x) {
  ElemShared<G>& s = *c.s;
  const Params& p = *c.p;
  const int q = c.lane;
  const bool active = q < p.nq;
  const int kin = p.kinematics;
  const bool averaged = p.averaged != 0;
  int fail = 0, code = 0;
  double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, strain[6] = {0, 0, 0, 0, 0, 0}, w = 0.0;
  LogKin L;
  if (active) {
    w = s.geo[q][9];
    const double* h = c.hu;
    if (kin == SBK_SMALL_STRAIN) {
      strain[0] = h[0];
      strain[1] = h[4];
      strain[2] = h[8];
      strain[3] = h[1] + h[3];
      strain[4] = h[5] + h[7];
      strain[5] = h[6] + h[2];
    } else {
#pragma unroll
      for (int i = 0; i < 9; ++i) F[i] = h[i] + ((i % 4) == 0 ? 1.0 : 0.0);
      double E[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          E[i * 3 + j] = 0.5 * (h[i * 3 + j] + h[j * 3 + i] + h[0 * 3 + i] * h[0 * 3 + j] +
                                h[1 * 3 + i] * h[1 * 3 + j] + h[2 * 3 + i] * h[2 * 3 + j]);
      const double green[6] = {E[0], E[4], E[8], 2.0 * E[1], 2.0 * E[5], 2.0 * E[6]};
      if (kin == SBK_FINITE) {
#pragma unroll
        for (int i = 0; i < 6; ++i) strain[i] = green[i];
      } else {
        code = det3(F) > 0.0 ? log_strain(green, L, strain) : SBK_EL_INVERTED_POINT;
        if (code) fail = (1 << 8) | q;
      }
    }
  }
  int key = fail ? fail : 0x7fffffff;
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) key = min(key, __shfl_xor_sync(c.mask, key, o, G));
  if (key != 0x7fffffff) {
    const int out = __shfl_sync(c.mask, code, key & 0xff, G);
    c.sync();
    return out;
  }
  const double m6[6] = {1.0, 1.0, 1.0, 0.0, 0.0, 0.0};
  double pv[6] = {1.0, 1.0, 1.0, 0.0, 0.0, 0.0};  // P^T m: the variation of the trace
  if (averaged) {
    if (active && kin == SBK_FINITE_LOGARITHMIC) log_stress(L, m6, pv);
    // Group sums of w d(3a + k) (d = B_NL^T pv, the point's dilatation row),
    // of w and of w tr(strain), in chunks of G through the reduce-scatter.
    const double tr = strain[0] + strain[1] + strain[2];
#pragma unroll 1
    for (int chunk = 0; chunk * G < 26; ++chunk) {
      double buf[G];
#pragma unroll
      for (int i = 0; i < G; ++i) {
        const int idx = chunk * G + i;
        double v = 0.0;
        if (active && idx < 26) {
          if (idx < 24) {
            double g[3];
            node_grad(c, q, idx / 3, g);
            v = w * bnl_t(F, g, idx % 3, pv);
          } else {
            v = idx == 24 ? w : w * tr;
          }
        }
        buf[i] = v;
      }
      const double y = reduce_scatter<G>(buf, c.lane, c.mask);
      if (chunk * G + c.lane < 32) x->red[chunk * G + c.lane] = y;
    }
    c.sync();
    const double volume = x->red[24];
    if (c.lane < 24) x->mean_row[c.lane] = x->red[c.lane] / volume;
    if (G < 24)
      for (int j = c.lane + G; j < 24; j += G) x->mean_row[j] = x->red[j] / volume;
    const double mean_trace = x->red[25] / volume;
    if (active) {
      const double shift = (mean_trace - tr) / 3.0;
      strain[0] += shift;
      strain[1] += shift;
      strain[2] += shift;
    }
    c.sync();
  }
  Response r;
  if (active) {
    PointState st{c.state + c.e * p.nq + q, c.trial + c.e * p.nq + q, c.npts};
    code = p.general ? general_return(p, strain, st, r, c.warm) : radial_return(p, strain, st, r);
    if (code) fail = (2 << 8) | q;
  }
  key = fail ? fail : 0x7fffffff;
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) key = min(key, __shfl_xor_sync(c.mask, key, o, G));
  if (key != 0x7fffffff) {
    const int out = __shfl_sync(c.mask, code, key & 0xff, G);
    c.sync();
    return out;
  }
  const double trT = active ? r.stress[0] + r.stress[1] + r.stress[2] : 0.0;
  // The element's mean Kirchhoff pressure (logarithmic + averaged): a
  // butterfly sum, the same bits in every lane.
  double mean_pressure = 0.0;
  if (averaged && kin == SBK_FINITE_LOGARITHMIC) {
    double v = active ? w * trT / 3.0 : 0.0;
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) v += __shfl_xor_sync(c.mask, v, o, G);
    mean_pressure = v / x->red[24];
  }
  if (active) {
    c.yield[c.e * p.nq + q] = r.yielding ? 1 : 0;
    double* e = x->pt[q];
    double cm[6], mc[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      cm[i] = r.C[i * 6 + 0] + r.C[i * 6 + 1] + r.C[i * 6 + 2];
      mc[i] = r.C[0 * 6 + i] + r.C[1 * 6 + i] + r.C[2 * 6 + i];
    }
    e[kStdMcm] = cm[0] + cm[1] + cm[2];
    e[kStdTr] = trT;
#pragma unroll
    for (int i = 0; i < 6; ++i) e[kStdPv + i] = pv[i];
    double S[6], M[36];
#pragma unroll
    for (int i = 0; i < 36; ++i) M[i] = r.C[i];
    if (kin == SBK_FINITE_LOGARITHMIC) {
      double t[6], u[6];
      log_stress(L, r.stress, u);
#pragma unroll
      for (int i = 0; i < 6; ++i) e[kStdST + i] = u[i];
      log_stress(L, cm, u);
#pragma unroll
      for (int i = 0; i < 6; ++i) e[kStdU1 + i] = u[i];
      log_stress(L, mc, u);
#pragma unroll
      for (int i = 0; i < 6; ++i) e[kStdU2 + i] = u[i];
#pragma unroll
      for (int i = 0; i < 6; ++i) t[i] = r.stress[i];
      if (averaged) {
        const double shift = mean_pressure - trT / 3.0;
        t[0] += shift;
        t[1] += shift;
        t[2] += shift;
      }
      log_transform(L, t, S, M);
    } else {
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        S[i] = r.stress[i];
        e[kStdST + i] = r.stress[i];
        e[kStdU1 + i] = cm[i];
        e[kStdU2 + i] = mc[i];
      }
    }
#pragma unroll
    for (int i = 0; i < 36; ++i) s.slot[q][i] = M[i];
#pragma unroll
    for (int i = 0; i < 6; ++i) s.slot[q][kSlotS + i] = S[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) s.slot[q][kSlotF + i] = F[i];
    s.slot[q][kSlotW] = w;
    s.slot[q][kSlotE] = r.energy;
  }
  c.sync();
  return 0;
}

template <int G>
__global__ void __launch_bounds__(256) standard_kernel(const __grid_constant__ Params p, int64_t ne, bool batch,
                                                       const double* __restrict__ coords,
                                                       const int32_t* __restrict__ conn, const double* __restrict__ u,
                                                       const double* __restrict__ state, int want_tangent,
                                                       double* __restrict__ force, double* __restrict__ tangent,
                                                       double* __restrict__ energy, double* __restrict__ trial,
                                                       double* __restrict__ alpha_out, uint8_t* __restrict__ yield,
                                                       int32_t* __restrict__ iterations, int32_t* __restrict__ code,
                                                       int32_t* __restrict__ first_failure,
                                                       const int32_t* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const int64_t slot = (int64_t)blockIdx.x * epb + slot_in_block;
  ElemShared<G>* sh = reinterpret_cast<ElemShared<G>*>(smem_raw) + slot_in_block;
  StdExtra<G>* xs = reinterpret_cast<StdExtra<G>*>(smem_raw + sizeof(ElemShared<G>) * epb) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  if (slot >= ne) return;
  const int64_t e = order ? (int64_t)order[slot] : slot;
  double hu_lane[9];
  double warm_lane[8];
  warm_lane[7] = 0.0;
  Ctx<G> c{&p, sh, lane, mask, e, ne * p.nq, state, trial, yield, hu_lane, warm_lane};
  ElemShared<G>& s = *sh;
  int bad_node = 0;
  if (lane < 8) {
    if (batch) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        s.X[3 * lane + k] = coords[e * 24 + 3 * lane + k];
        s.U[3 * lane + k] = u[e * 24 + 3 * lane + k];
      }
    } else {
      const int64_t node = conn[e * 8 + lane];
      if (p.num_nodes > 0 && (node < 0 || node >= p.num_nodes)) {
        bad_node = 1;
      } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          s.X[3 * lane + k] = coords[node * 3 + k];
          s.U[3 * lane + k] = u[node * 3 + k];
        }
      }
    }
  }
  if (__any_sync(mask, bad_node)) {
    if (lane == 0) {
      code[e] = SBK_EL_BAD_NODE;
      if (first_failure) atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  c.sync();
  int status = set_up<G>(c);
  if (!status) status = std_points<G>(c, xs);
  if (status) {
    if (lane == 0) {
      code[e] = status;
      if (first_failure) atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  const bool sym = p.symmetric != 0;
  const bool geometric = p.kinematics != SBK_SMALL_STRAIN;
  const bool averaged = p.averaged != 0;
  const bool finite = p.kinematics == SBK_FINITE;
  const int nq = p.nq;
  if (lane < 8) {
    const int a = lane;
    // f = sum w [B_NL^T S(T) + s (tr T) / 3], s = mean_row - d, in point order.
    double ra[3] = {0, 0, 0}, en = 0.0;
    for (int q = 0; q < nq; ++q) {
      const double* sl = s.slot[q];
      const double* ex = xs->pt[q];
      const double* Fq = sl + kSlotF;
      const double* Sq = ex + kStdST;
      const double wq = sl[kSlotW];
      double g[3];
      node_grad(c, q, a, g);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double v = bnl_t(Fq, g, k, Sq);
        if (averaged) v += (xs->mean_row[3 * a + k] - bnl_t(Fq, g, k, ex + kStdPv)) * ex[kStdTr] / 3.0;
        ra[k] += wq * v;
      }
      en += wq * sl[kSlotE];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) force[e * 24 + 3 * a + k] = ra[k];
    if (a == 0) energy[e] = en;
    if (want_tangent) {
      // The volume average of g_a . g_b (finite + averaged).
      double gbar[8];
      if (averaged && finite) {
#pragma unroll
        for (int b = 0; b < 8; ++b) gbar[b] = 0.0;
        double volume = 0.0;
        for (int q = 0; q < nq; ++q) {
          const double wq = s.slot[q][kSlotW];
          double ga[3];
          node_grad(c, q, a, ga);
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            double gb[3];
            node_grad(c, q, b, gb);
            gbar[b] += wq * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
          }
          volume += wq;
        }
#pragma unroll
        for (int b = 0; b < 8; ++b) gbar[b] /= volume;
      }
#pragma unroll 1
      for (int chunk = 0; chunk < 2; ++chunk) {
        double acc[4][9];
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
          for (int i = 0; i < 9; ++i) acc[b][i] = 0.0;
        for (int q = 0; q < nq; ++q) {
          const double* sl = s.slot[q];
          const double* ex = xs->pt[q];
          const double* Fq = sl + kSlotF;
          const double wq = sl[kSlotW];
          double g[3], V[27];
          node_grad(c, q, a, g);
          vtensor(sl, g, false, geometric, V);
          double sa[3], la[3];
          if (averaged) {
            const double third = ex[kStdMcm] / 3.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              sa[k] = xs->mean_row[3 * a + k] - bnl_t(Fq, g, k, ex + kStdPv);
              la[k] = bnl_t(Fq, g, k, ex + kStdU1) + third * sa[k];
            }
          }
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int bb = chunk * 4 + b;
            double gb[3];
            node_grad(c, q, bb, gb);
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
              for (int l = 0; l < 3; ++l)
                acc[b][k * 3 + l] += V[(k * 3 + l) * 3 + 0] * gb[0] + V[(k * 3 + l) * 3 + 1] * gb[1] +
                                     V[(k * 3 + l) * 3 + 2] * gb[2];
            if (averaged) {
              double sb[3], mb[3];
#pragma unroll
              for (int l = 0; l < 3; ++l) {
                sb[l] = xs->mean_row[3 * bb + l] - bnl_t(Fq, gb, l, ex + kStdPv);
                mb[l] = bnl_t(Fq, gb, l, ex + kStdU2);
              }
              const double w3 = wq / 3.0;
#pragma unroll
              for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int l = 0; l < 3; ++l) acc[b][k * 3 + l] += w3 * (la[k] * sb[l] + sa[k] * mb[l]);
              if (finite) {
                const double v = wq * (ex[kStdTr] / 3.0) * (gbar[bb] - (g[0] * gb[0] + g[1] * gb[1] + g[2] * gb[2]));
#pragma unroll
                for (int k = 0; k < 3; ++k) acc[b][k * 3 + k] += v;
              }
            }
          }
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          double* out = tangent + e * 576 + (8 * a + chunk * 4 + b) * 9;
#pragma unroll
          for (int i = 0; i < 9; ++i) out[i] = acc[b][i];
        }
      }
    }
  }
  if (want_tangent && sym) {
    __threadfence_block();
    c.sync();
    if (lane < 8) {
      double* Ke = tangent + e * 576;
      auto at = [&](int i, int j) -> double* { return Ke + (8 * (i / 3) + j / 3) * 9 + 3 * (i % 3) + (j % 3); };
      for (int k = 0; k < 3; ++k) {
        const int i = 3 * lane + k;
        for (int j = i + 1; j < 24; ++j) {
          double* x1 = at(i, j);
          double* y1 = at(j, i);
          const double v = 0.5 * (*x1 + *y1);
          *x1 = v;
          *y1 = v;
        }
      }
    }
  }
  if (lane == 0) {
    iterations[e] = 0;
    code[e] = 0;
  }
  for (int i = lane; i < 9; i += G) alpha_out[e * 9 + i] = 0.0;
}

// Stress recovery at the end of a step (incompatible_elastoplastic_stress,
// IncompatibleModes.cpp:602-664, called for every element by the forming
// driver, Forming.cpp:1266-1281): the kinematics at the committed modes
// without a local iteration, every point's return from its committed state
// (an elastic check that reproduces it), and per element the point averages
// of the Cauchy, second Piola-Kirchhoff and Kirchhoff stresses and the log
// strain, the von Mises stress of the average Cauchy stress, the largest
// accumulated plastic strain and strain component and the smallest det F.
// The point values go through shared memory and lane 0 sums them in point
// order, as the reference does. out: 28 per element (cauchy 6, pk2 6, von
// Mises, max eqps, max strain, min det F, kirchhoff 6, log strain 6).
template <int G>
__global__ void __launch_bounds__(128) stress_kernel(const __grid_constant__ Params p, int64_t ne,
                                                     const double* __restrict__ coords,
                                                     const int32_t* __restrict__ conn, const double* __restrict__ u,
                                                     const double* __restrict__ state,
                                                     const double* __restrict__ alpha_n, double* __restrict__ scratch,
                                                     double* __restrict__ out, int32_t* __restrict__ code,
                                                     int32_t* __restrict__ first_failure) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int epb = blockDim.x / G;
  const int slot_in_block = threadIdx.x / G;
  const int lane = threadIdx.x % G;
  const int64_t e = (int64_t)blockIdx.x * epb + slot_in_block;
  ElemShared<G>* sh = reinterpret_cast<ElemShared<G>*>(smem_raw) + slot_in_block;
  const unsigned lanes_mask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
  const unsigned mask = lanes_mask << ((threadIdx.x % 32) / G * G);
  if (e >= ne) return;
  double hu_lane[9];
  Ctx<G> c{&p, sh, lane, mask, e, ne * p.nq, state, scratch, nullptr, hu_lane, nullptr};
  ElemShared<G>& s = *sh;
  int bad_node = 0;
  if (lane < 8) {
    const int64_t node = conn[e * 8 + lane];
    if (p.num_nodes > 0 && (node < 0 || node >= p.num_nodes)) {
      bad_node = 1;
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        s.X[3 * lane + k] = coords[node * 3 + k];
        s.U[3 * lane + k] = u[node * 3 + k];
      }
    }
  }
  if (__any_sync(mask, bad_node)) {
    if (lane == 0) {
      code[e] = SBK_EL_BAD_NODE;
      atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  // The standard Hex8 has no modes: its kinematics are K1's at zero modes.
  for (int i = lane; i < 9; i += G) s.alpha[i] = (alpha_n && !p.element) ? alpha_n[e * 9 + i] : 0.0;
  c.sync();
  int status = set_up<G>(c);
  if (status) {
    if (lane == 0) {
      code[e] = status;
      atomicMin(first_failure, (int32_t)e);
    }
    return;
  }
  const int q = lane;
  int fail = 0, fcode = 0;
  double h[9], F[9], sym[9], strain[6] = {0, 0, 0, 0, 0, 0};
  LogKin L;
  if (q < p.nq) {
    double gt[9];
    mode_grads(c, q, gt);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double v = c.hu[i * 3 + j];
#pragma unroll
        for (int m = 0; m < 3; ++m) v += s.alpha[3 * m + i] * gt[j * 3 + m];
        h[i * 3 + j] = v;
      }
#pragma unroll
    for (int i = 0; i < 9; ++i) F[i] = h[i] + ((i % 4) == 0 ? 1.0 : 0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) sym[i * 3 + j] = 0.5 * (h[i * 3 + j] + h[j * 3 + i]);
    if (p.kinematics == SBK_SMALL_STRAIN) {
      strain[0] = h[0];
      strain[1] = h[4];
      strain[2] = h[8];
      strain[3] = h[1] + h[3];
      strain[4] = h[5] + h[7];
      strain[5] = h[6] + h[2];
    } else {
      double E[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          E[i * 3 + j] = 0.5 * (h[i * 3 + j] + h[j * 3 + i] + h[0 * 3 + i] * h[0 * 3 + j] +
                                h[1 * 3 + i] * h[1 * 3 + j] + h[2 * 3 + i] * h[2 * 3 + j]);
      const double green[6] = {E[0], E[4], E[8], 2.0 * E[1], 2.0 * E[5], 2.0 * E[6]};
      if (p.kinematics == SBK_FINITE) {
#pragma unroll
        for (int i = 0; i < 6; ++i) strain[i] = green[i];
      } else if (!(det3(F) > 0.0)) {
        fcode = SBK_EL_INVERTED_POINT;
      } else {
        fcode = log_strain(green, L, strain);
      }
      if (fcode) fail = (1 << 8) | q;
    }
  }
  // The standard Hex8 with mean dilatation (kinematics_of,
  // Elastoplastic.cpp:140-167): every point's trace replaced by the volume
  // average, once no point failed; the returns and the averaged measures
  // take it, the largest strain component stays the point's own.
  double own[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) own[i] = strain[i];
  if (p.averaged && !__any_sync(c.mask, fail != 0)) {
    const double w = q < p.nq ? s.geo[q][9] : 0.0;
    double wt = w * (strain[0] + strain[1] + strain[2]), vol = w;
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
      wt += __shfl_xor_sync(c.mask, wt, o, G);
      vol += __shfl_xor_sync(c.mask, vol, o, G);
    }
    const double shift = (wt / vol - (strain[0] + strain[1] + strain[2])) / 3.0;
    strain[0] += shift;
    strain[1] += shift;
    strain[2] += shift;
  }
  if (q < p.nq && !fail) {
    {
      PointState st{c.state + c.e * p.nq + q, c.trial + c.e * p.nq + q, c.npts};
      Response r;
      fcode = p.general ? general_return(p, strain, st, r) : radial_return(p, strain, st, r);
      if (fcode) {
        fail = (2 << 8) | q;
      } else {
        double* o = s.slot[q];
        double pk[6], cauchy[6], tau[6] = {0, 0, 0, 0, 0, 0}, lstr[6] = {0, 0, 0, 0, 0, 0};
        double max_strain = 0.0, jac = 1.0;
#pragma unroll
        for (int i = 0; i < 6; ++i) cauchy[i] = pk[i] = r.stress[i];
        // F T F^T of a tensorial Voigt T, as a tensorial Voigt vector.
        auto push = [&](const double t[6], double res[6]) {
          const double T3[9] = {t[0], t[3], t[5], t[3], t[1], t[4], t[5], t[4], t[2]};
          double FT[9], R[9];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
              FT[i * 3 + j] = F[i * 3 + 0] * T3[0 * 3 + j] + F[i * 3 + 1] * T3[1 * 3 + j] + F[i * 3 + 2] * T3[2 * 3 + j];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
              R[i * 3 + j] = FT[i * 3 + 0] * F[j * 3 + 0] + FT[i * 3 + 1] * F[j * 3 + 1] + FT[i * 3 + 2] * F[j * 3 + 2];
          res[0] = R[0], res[1] = R[4], res[2] = R[8], res[3] = R[1], res[4] = R[5], res[5] = R[6];
        };
        if (p.kinematics == SBK_FINITE_LOGARITHMIC) {
          log_stress(L, r.stress, pk);
          push(pk, tau);
#pragma unroll
          for (int i = 0; i < 6; ++i) lstr[i] = i < 3 ? strain[i] : 0.5 * strain[i];
          const double vol = exp(lstr[0] + lstr[1] + lstr[2]);
#pragma unroll
          for (int i = 0; i < 6; ++i) {
            cauchy[i] = tau[i] / vol;
            max_strain = fmax(max_strain, fabs(i < 3 ? own[i] : 0.5 * own[i]));
          }
          jac = det3(F);
        } else if (p.kinematics == SBK_FINITE) {
          jac = det3(F);
          double ft[6];
          push(r.stress, ft);
#pragma unroll
          for (int i = 0; i < 6; ++i) cauchy[i] = ft[i] / jac;
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const double g = sym[i * 3 + j] + 0.5 * (h[0 * 3 + i] * h[0 * 3 + j] + h[1 * 3 + i] * h[1 * 3 + j] +
                                                       h[2 * 3 + i] * h[2 * 3 + j]);
              max_strain = fmax(max_strain, fabs(g));
            }
        } else {
#pragma unroll
          for (int i = 0; i < 9; ++i) max_strain = fmax(max_strain, fabs(sym[i]));
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
          o[i] = cauchy[i];
          o[6 + i] = pk[i];
          o[12 + i] = tau[i];
          o[18 + i] = lstr[i];
        }
        o[24] = max_strain;
        o[25] = jac;
        o[26] = st.out[field_eqps(p.nterms) * st.stride];
      }
    }
  }
  int key = fail ? fail : 0x7fffffff;
#pragma unroll
  for (int o = G / 2; o >= 1; o >>= 1) key = min(key, __shfl_xor_sync(c.mask, key, o, G));
  const int owner = key & 0xff;
  const int fcode_g = __shfl_sync(c.mask, fcode, key != 0x7fffffff ? owner : 0, G);
  c.sync();
  if (lane != 0) return;
  if (key != 0x7fffffff) {
    code[e] = fcode_g;
    atomicMin(first_failure, (int32_t)e);
    return;
  }
  double acc[24];
#pragma unroll
  for (int i = 0; i < 24; ++i) acc[i] = 0.0;
  double max_eqps = 0.0, max_strain = 0.0, min_jac = __longlong_as_double(0x7ff0000000000000LL);
  for (int qq = 0; qq < p.nq; ++qq) {
    const double* o = s.slot[qq];
#pragma unroll
    for (int i = 0; i < 24; ++i) acc[i] += o[i];
    max_strain = fmax(max_strain, o[24]);
    min_jac = fmin(min_jac, o[25]);
    max_eqps = fmax(max_eqps, o[26]);
  }
  const double count = (double)p.nq;
  double* res = out + e * 28;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    res[i] = acc[i] / count;
    res[6 + i] = acc[6 + i] / count;
    res[16 + i] = acc[12 + i] / count;
    res[22 + i] = acc[18 + i] / count;
  }
  const double a0 = res[0] - res[1], a1 = res[1] - res[2], a2 = res[2] - res[0];
  res[12] = sqrt(0.5 * (a0 * a0 + a1 * a1 + a2 * a2) + 3.0 * (res[3] * res[3] + res[4] * res[4] + res[5] * res[5]));
  res[13] = max_eqps;
  res[14] = max_strain;
  res[15] = p.kinematics == SBK_SMALL_STRAIN ? 1.0 : min_jac;
  code[e] = 0;
}

template <int G>
int launch_stress_g(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                    const double* state, const double* alpha_n, double* scratch, double* out, int32_t* code,
                    int32_t* first_failure, int epb, cudaStream_t stream) {
  const size_t smem = sizeof(ElemShared<G>) * epb;
  const int64_t blocks = (ne + epb - 1) / epb;
  if (blocks == 0) return 0;
  auto kern = stress_kernel<G>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return (int)err;
  kern<<<(unsigned)blocks, epb * G, smem, stream>>>(p, ne, coords, conn, u, state, alpha_n, scratch, out, code,
                                                    first_failure);
  return (int)cudaGetLastError();
}

template <int G>
int launch_g(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
             const double* state, const double* alpha_n, int want_tangent, double* force, double* tangent,
             double* energy, double* trial, double* alpha_out, uint8_t* yield, int32_t* iterations, int32_t* code,
             int32_t* first_failure, bool batch, int epb, const int32_t* order, cudaStream_t stream) {
  const int threads = epb * G;
  const size_t smem = sizeof(ElemShared<G>) * epb;
  const int64_t blocks = (ne + epb - 1) / epb;
  if (blocks == 0) return 0;
  auto kern = element_kernel<G>;
  // The shared-memory limit is raised once per device and size, so that a
  // launch inside a stream capture (a CUDA graph of an evaluation) makes no
  // attribute call.
  static size_t raised[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || raised[dev] < smem) {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return (int)err;
    if (dev >= 0 && dev < 64) raised[dev] = smem;
  }
  kern<<<(unsigned)blocks, threads, smem, stream>>>(p, ne, batch, coords, conn, u, state, alpha_n, want_tangent,
                                                     force, tangent, energy, trial, alpha_out, yield, iterations,
                                                     code, first_failure, order);
  return (int)cudaGetLastError();
}

}  // namespace

int launch_stress(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                  const double* state, const double* alpha_n, double* scratch, double* out, int32_t* code,
                  int32_t* first_failure, cudaStream_t stream) {
  if (p.nq <= 8)
    return launch_stress_g<8>(p, ne, coords, conn, u, state, alpha_n, scratch, out, code, first_failure, 4, stream);
  return launch_stress_g<32>(p, ne, coords, conn, u, state, alpha_n, scratch, out, code, first_failure, 1, stream);
}

template <int G>
int launch_standard_g(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                      const double* state, int want_tangent, double* force, double* tangent, double* energy,
                      double* trial, double* alpha_out, uint8_t* yield, int32_t* iterations, int32_t* code,
                      int32_t* first_failure, bool batch, int epb, const int32_t* order, cudaStream_t stream) {
  const size_t per = sizeof(ElemShared<G>) + sizeof(StdExtra<G>);
  const int most = (int)((227 * 1024) / per);
  if (epb > most) epb = most;
  if (epb * G > 256) epb = 256 / G;
  const size_t smem = per * epb;
  const int64_t blocks = (ne + epb - 1) / epb;
  if (blocks == 0) return 0;
  auto kern = standard_kernel<G>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return set_error(SBK_ERR_CUDA, std::string("standard kernel attribute: ") + cudaGetErrorString(err));
  kern<<<(unsigned)blocks, epb * G, smem, stream>>>(p, ne, batch, coords, conn, u, state, want_tangent, force, tangent,
                                                    energy, trial, alpha_out, yield, iterations, code, first_failure,
                                                    order);
  err = cudaGetLastError();
  if (err != cudaSuccess) return set_error(SBK_ERR_CUDA, std::string("standard kernel launch: ") + cudaGetErrorString(err));
  return 0;
}

template <int G>
int launch_vjp_g(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                 const double* state, const double* alpha_n, const double* lambda, double* trial, uint8_t* yield,
                 int32_t* code, int32_t* first_failure, double* out, cudaStream_t stream) {
  const int epb = G == 8 ? 16 : 4;
  const size_t smem = sizeof(ElemShared<G>) * epb;
  const int64_t blocks = (ne + epb - 1) / epb;
  if (blocks == 0) return 0;
  auto kern = vjp_kernel<G>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err != cudaSuccess) return set_error(SBK_ERR_CUDA, std::string("vjp kernel attribute: ") + cudaGetErrorString(err));
  kern<<<(unsigned)blocks, epb * G, smem, stream>>>(p, ne, coords, conn, u, state, alpha_n, lambda, trial, yield, code,
                                                    first_failure, out);
  err = cudaGetLastError();
  if (err != cudaSuccess) return set_error(SBK_ERR_CUDA, std::string("vjp kernel launch: ") + cudaGetErrorString(err));
  return 0;
}

int launch_vjp(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
               const double* state, const double* alpha_n, const double* lambda, double* trial, uint8_t* yield,
               int32_t* code, int32_t* first_failure, double* out, cudaStream_t stream) {
  if (p.nq <= 8)
    return launch_vjp_g<8>(p, ne, coords, conn, u, state, alpha_n, lambda, trial, yield, code, first_failure, out,
                           stream);
  return launch_vjp_g<32>(p, ne, coords, conn, u, state, alpha_n, lambda, trial, yield, code, first_failure, out,
                          stream);
}

namespace {

// The next array of `count` T at byte offset `at` of base (256-byte
// aligned); advances `at`. With a null base only the offsets are counted.
template <class T>
T* carve(char* base, size_t& at, size_t count) {
  T* out = base ? reinterpret_cast<T*>(base + at) : nullptr;
  at += (count * sizeof(T) + 255) / 256 * 256;
  return out;
}

// The shared-memory limit of a kernel raised once per device, so that a
// launch inside a stream capture makes no attribute call.
template <class K>
int raise_smem(K kern, size_t smem, size_t* raised) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || raised[dev] < smem) {
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return (int)err;
    if (dev >= 0 && dev < 64) raised[dev] = smem;
  }
  return 0;
}

}  // namespace

namespace {

size_t carve_all(char* base, int64_t ne, WaveBuffers& w) {
  size_t at = 0;
  const size_t n = (size_t)ne;
  w.alpha = carve<double>(base, at, n * 9);
  w.dir = carve<double>(base, at, n * 9);
  w.res = carve<double>(base, at, n);
  w.iters = carve<int32_t>(base, at, n);
  w.pcode = carve<int32_t>(base, at, n);
  w.kc = carve<double>(base, at, n * kKcStride);
  w.r = carve<double>(base, at, n * 33);
  w.sf = carve<double>(base, at, n * 19);
  w.piv = carve<int32_t>(base, at, n * 18);
  w.slot = carve<double>(base, at, n * kSlot * 8);
  w.geo = carve<double>(base, at, n * 12 * 8);
  w.jinv0 = carve<double>(base, at, n * 9);
  w.hu = carve<double>(base, at, n * 9 * 8);
  w.warm = carve<double>(base, at, n * 8 * 8);
  w.pw = carve<double>(base, at, n * kPw * 8);
  w.pfail = carve<int32_t>(base, at, n * 8);
  w.pcodes = carve<int32_t>(base, at, n * 8);
  w.plastic = carve<int32_t>(base, at, n * 8);
  w.list[0] = carve<int32_t>(base, at, n);
  w.list[1] = carve<int32_t>(base, at, n);
  w.done = carve<int32_t>(base, at, n);
  w.fallback = carve<int32_t>(base, at, n);
  w.counts = carve<int32_t>(base, at, 2 * kWaveRounds + 3);
  return at;
}

}  // namespace

size_t wave_buffer_bytes(int64_t ne) {
  WaveBuffers w;
  return carve_all(nullptr, ne, w);
}

void wave_buffers_carve(void* base, int64_t ne, WaveBuffers& w) { carve_all(static_cast<char*>(base), ne, w); }

bool wave_applies(const Params& p) { return p.element == 0 && p.nq <= 8; }

int launch_elements_wave(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                         const double* state, const double* alpha_n, int want_tangent, double* force,
                         double* tangent, double* energy, double* trial, double* alpha_out, uint8_t* yield,
                         int32_t* iterations, int32_t* code, int32_t* first_failure, bool batch,
                         const int32_t* order, const WaveBuffers& w, int pass_epb, cudaStream_t stream) {
  constexpr int G = 8;
  if (!wave_applies(p)) return (int)cudaErrorInvalidValue;
  if (ne <= 0) return 0;
  constexpr int epb = 16;  // 4 warps per block
  const int threads = epb * G;
  // The first pass kernel's block: pass_epb elements (0: 16), at most 16
  // (its launch bounds assume 128 threads).
  const int pepb = pass_epb > 0 ? (pass_epb > 16 ? 16 : pass_epb) : 16;
  static size_t raised[6][64] = {};
  const size_t smem_pass = sizeof(PreShared<G>) * pepb;
  const size_t smem_post = sizeof(PassShared<G>) * epb;
  const size_t smem_ctl = sizeof(ControlShared<G>) * epb;
  const size_t smem_cond = sizeof(CondenseShared<G>) * epb;
  const size_t smem_elem = sizeof(ElemShared<G>) * epb;
  auto pre = p.general ? wave_pre_kernel<G, true> : wave_pre_kernel<G, false>;
  int rc = raise_smem(pre, smem_pass, raised[p.general ? 0 : 5]);
  if (!rc) rc = raise_smem(wave_post_kernel<G>, smem_post, raised[4]);
  if (!rc) rc = raise_smem(wave_control_kernel<G>, smem_ctl, raised[1]);
  if (!rc) rc = raise_smem(wave_condense_kernel<G>, smem_cond, raised[2]);
  if (!rc) rc = raise_smem(element_list_kernel<G>, smem_elem, raised[3]);
  if (rc) return rc;
  const int64_t need = (ne + epb - 1) / epb;
  // Grid-stride launches: enough blocks to fill every SM several times over
  // in the first rounds, few enough that the late rounds (a handful of
  // elements) cost little more than the launch.
  const int64_t cap = 148 * 16;
  const unsigned grid = (unsigned)(need < cap ? need : cap);
  const int64_t pneed = (ne + pepb - 1) / pepb;
  const unsigned pgrid = (unsigned)(pneed < cap ? pneed : cap);
  const int64_t rneed = (ne * 8 + 127) / 128;
  const unsigned rgrid = (unsigned)(rneed < 148 * 8 ? rneed : 148 * 8);
  const unsigned lgrid = rgrid;
  cudaError_t err = cudaMemsetAsync(w.counts, 0, (2 * kWaveRounds + 3) * sizeof(int32_t), stream);
  if (err != cudaSuccess) return (int)err;
  for (int r = 0; r < kWaveRounds; ++r) {
    const int32_t* list = r == 0 ? order : w.list[r & 1];
    const int32_t* count = r == 0 ? nullptr : w.counts + r;
    int32_t* plastic_count = w.counts + kWaveRounds + 3 + r;
    pre<<<pgrid, pepb * G, smem_pass, stream>>>(p, ne, r == 0, list, count, batch, coords, conn, u, state, alpha_n,
                                                trial, yield, w.plastic, plastic_count, w);
    launch_wave_returns(p, ne, w.plastic, plastic_count, state, trial, w, rgrid, stream);
    if (p.kinematics == SBK_FINITE_LOGARITHMIC)
      wave_log_kernel<<<lgrid, 128, 0, stream>>>(ne, p.nq, list, count, w);
    wave_post_kernel<G><<<grid, threads, smem_post, stream>>>(p, ne, list, count, yield, w);
    wave_control_kernel<G><<<grid, threads, smem_ctl, stream>>>(p, ne, r == 0, list, count, w, w.list[(r + 1) & 1],
                                                                w.counts + r + 1, code, first_failure);
  }
  wave_condense_kernel<G><<<grid, threads, smem_cond, stream>>>(p, ne, w, want_tangent, force, tangent, energy,
                                                                alpha_out, iterations, code);
  // The elements that left the common road, by the single kernel from the
  // start (one 4-warp block per SM holds its records).
  const unsigned fgrid = (unsigned)(need < 148 * 2 ? need : 148 * 2);
  element_list_kernel<G><<<fgrid, threads, smem_elem, stream>>>(
      p, ne, batch, coords, conn, u, state, alpha_n, want_tangent, force, tangent, energy, trial, alpha_out, yield,
      iterations, code, first_failure, w.fallback, w.counts + kWaveRounds + 2);
  return (int)cudaGetLastError();
}

size_t element_smem_bytes(int group) {
  return group == 8 ? sizeof(ElemShared<8>) : sizeof(ElemShared<32>);
}

int launch_elements(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                    const double* state, const double* alpha_n, int want_tangent, double* force, double* tangent,
                    double* energy, double* trial, double* alpha_out, uint8_t* yield, int32_t* iterations,
                    int32_t* code, int32_t* first_failure, bool batch, int elements_per_block,
                    const int32_t* order, cudaStream_t stream) {
  if (p.element == 1) {
    // The standard Hex8: the same launch shapes as K1.
    if (p.nq <= 8)
      return launch_standard_g<8>(p, ne, coords, conn, u, state, want_tangent, force, tangent, energy, trial,
                                  alpha_out, yield, iterations, code, first_failure, batch,
                                  elements_per_block > 0 ? elements_per_block : 16, order, stream);
    return launch_standard_g<32>(p, ne, coords, conn, u, state, want_tangent, force, tangent, energy, trial,
                                 alpha_out, yield, iterations, code, first_failure, batch,
                                 elements_per_block > 0 ? elements_per_block : 8, order, stream);
  }
  if (p.nq <= 8) {
    // At most what 227 KB of shared memory and 256 threads hold.
    const int most = (int)((227 * 1024) / sizeof(ElemShared<8>)) < 32 ? (int)((227 * 1024) / sizeof(ElemShared<8>)) : 32;
    // The default, 16 elements (4 warps) per block and so one block per SM:
    // the four warps of a block start together and, their elements being
    // alike under the schedule, stay close enough in the code to share its
    // instruction fetches (1.8x over one-warp blocks on the sheet
    // microbenchmark; 5 to 7 warps per block are slower).
    int epb = elements_per_block > 0 ? elements_per_block : 16;
    if (epb > most) epb = most;
    return launch_g<8>(p, ne, coords, conn, u, state, alpha_n, want_tangent, force, tangent, energy, trial,
                       alpha_out, yield, iterations, code, first_failure, batch, epb, order, stream);
  }
  // Rules of 9 to 32 points (the sheet rules 2 x 2 x 3..7, the 3 x 3 x 3
  // cube): a warp per element, lane = point. The default, 8 warps per block
  // (the most 256 threads allow), for the same shared instruction fetches:
  // 42 ms per 80,000 elements of the 2 x 2 x 5 rule, against 55 ms at 4
  // warps and 80 ms at 1.
  const int epb = elements_per_block > 0 ? (elements_per_block < 8 ? elements_per_block : 8) : 8;
  return launch_g<32>(p, ne, coords, conn, u, state, alpha_n, want_tangent, force, tangent, energy, trial,
                      alpha_out, yield, iterations, code, first_failure, batch, epb, order, stream);
}

}  // namespace sbk
