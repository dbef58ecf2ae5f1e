// Launch parameters shared by the host code and the kernels: the material
// (elastic constants, hardening, yield matrix, kinematic terms) and the
// integration rule, passed by value (kernel parameter space, broadcast to
// every thread from the constant bank).
#pragma once

#include <stdint.h>

#include "sbk.h"

namespace sbk {

// Per-point state layout (field-major on the device, see sbk.h):
//   [0, 6)   plastic strain (engineering shears)
//   [6, 12)  whole back stress (tensorial)
//   [12 + 6i, 18 + 6i)  kinematic term i of the general return
//   12 + 6n  accumulated plastic strain
//   13 + 6n  loading flag (0 / 1)
constexpr int kFieldEp = 0;
constexpr int kFieldBeta = 6;
constexpr int kFieldAlpha = 12;
inline __host__ __device__ int field_eqps(int nterms) { return 12 + 6 * nterms; }
inline __host__ __device__ int field_loading(int nterms) { return 13 + 6 * nterms; }
inline __host__ __device__ int state_fields(int nterms) { return 14 + 6 * nterms; }

struct Params {
  // Elasticity: shear modulus, bulk modulus K = lambda + 2G/3.
  double G, K;
  // sigma_y(a) = sy0 + H a + Q (1 - exp(-delta a)); Prager's H_kin.
  double sy0, H, Hkin, Q, delta;
  // Yield matrix (tensorial Voigt, global axes), row-major.
  double P[36];
  // P = S^-1 PV diag(PL) PV^T S^-1 with PV^T S^-1 PV = I, S = diag(1, 1, 1,
  // 1/2, 1/2, 1/2): the generalised eigenvectors (columns, row-major) and
  // eigenvalues of the yield matrix, for the closest-point solves.
  double PV[36];
  double PL[6];
  // Kinematic terms of the general return (Chaboche, then Prager).
  double termC[SBK_MAX_BACKSTRESSES], termG[SBK_MAX_BACKSTRESSES];
  int nterms;       // terms stored per point (0 for the radial return)
  int general;      // 1: closest-point return (Hill48 and/or backstresses)
  int enabled;      // sy0 > 0
  int integration;  // 0 exponential, 1 backward Euler
  int symmetric;    // the consistent tangent is symmetric
  int kinematics;   // sbk_kinematics
  int nq;           // integration points
  int nfields;      // doubles per point of state
  int element;      // 0 the incompatible-mode Hex8, 1 the standard Hex8
  int averaged;     // standard Hex8: mean dilatation (B-bar)
  int num_nodes;    // mesh mode: node indices are checked against it (0: batch mode, unchecked)
  // The rule: xi, eta, zeta, weight per point.
  double qp[SBK_MAX_POINTS][4];
};

}  // namespace sbk
