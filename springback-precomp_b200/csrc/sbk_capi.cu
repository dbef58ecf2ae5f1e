// The C ABI (include/sbk.h): materials and rules, the element batch, and the
// system that stands in for detail::NonlinearSystem
// (src/fem/NonlinearSystem.hpp:85-334), whose Assembler pattern
// (src/fem/Assembler.cpp:86-173) sbk_pattern.cu builds on the device. Every
// device buffer belongs to a handle; no exception crosses the ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sbk.h"
#include "sbk_element.h"
#include "sbk_params.h"
#include "sbk_pattern.h"

using sbk::Params;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& what) {
  g_error = what;
  return code;
}

#define SBK_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) return fail(SBK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(SBK_ERR_NO_EXTENSION, "no CUDA device: the element loop runs on the GPU only");
  }
  return SBK_OK;
}

bool finite_positive(double v) { return std::isfinite(v) && v > 0.0; }

// Material::set_plasticity and derive_hill (src/material/Material.cpp:135-271).
int yield_matrix(const sbk_material& m, double* P) {
  std::memset(P, 0, 36 * sizeof(double));
  if (m.criterion != SBK_HILL48) {
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) P[i * 6 + j] = -0.5;
      P[i * 6 + i] = 1.0;
      P[(3 + i) * 6 + 3 + i] = 3.0;
    }
    return SBK_OK;
  }
  if (!finite_positive(m.r0) || !finite_positive(m.r45) || !finite_positive(m.r90))
    return fail(SBK_ERR_CONFIG, "the Hill48 r-values must be finite and positive");
  const double G = 1.0 / (1.0 + m.r0);
  const double H = m.r0 / (1.0 + m.r0);
  const double F = m.r0 / (m.r90 * (1.0 + m.r0));
  const double N = (m.r0 + m.r90) * (1.0 + 2.0 * m.r45) / (2.0 * m.r90 * (1.0 + m.r0));
  const double L = m.shear_l, M = m.shear_m;
  if (!(L > 0.0 && M > 0.0 && N > 0.0) || !(F + H > 0.0) || !(F * G + G * H + H * F > 0.0))
    return fail(SBK_ERR_CONFIG, "the Hill48 coefficients do not make a convex yield surface");
  double nd[3], rd[3];
  const double nn = std::sqrt(m.sheet_normal[0] * m.sheet_normal[0] + m.sheet_normal[1] * m.sheet_normal[1] +
                              m.sheet_normal[2] * m.sheet_normal[2]);
  const double rn0 = std::sqrt(m.rolling_direction[0] * m.rolling_direction[0] +
                               m.rolling_direction[1] * m.rolling_direction[1] +
                               m.rolling_direction[2] * m.rolling_direction[2]);
  if (!(nn > 0.0) || !(rn0 > 0.0) || !std::isfinite(nn) || !std::isfinite(rn0))
    return fail(SBK_ERR_CONFIG, "the rolling direction and the sheet normal must be finite non-zero vectors");
  for (int i = 0; i < 3; ++i) {
    nd[i] = m.sheet_normal[i] / nn;
    rd[i] = m.rolling_direction[i] / rn0;
  }
  const double d = rd[0] * nd[0] + rd[1] * nd[1] + rd[2] * nd[2];
  for (int i = 0; i < 3; ++i) rd[i] -= d * nd[i];
  const double rn = std::sqrt(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
  if (!(rn > 1.0e-6)) return fail(SBK_ERR_CONFIG, "the rolling direction is parallel to the sheet normal");
  for (int i = 0; i < 3; ++i) rd[i] /= rn;
  const double td[3] = {nd[1] * rd[2] - nd[2] * rd[1], nd[2] * rd[0] - nd[0] * rd[2], nd[0] * rd[1] - nd[1] * rd[0]};
  const double* axes[3] = {rd, td, nd};
  // Material-frame matrix, then P = T^T Pm T with T the Voigt stress
  // rotation into the material axes (rows of `axes`).
  double pm[6][6] = {};
  pm[0][0] = G + H;
  pm[1][1] = F + H;
  pm[2][2] = F + G;
  pm[0][1] = pm[1][0] = -H;
  pm[1][2] = pm[2][1] = -F;
  pm[0][2] = pm[2][0] = -G;
  pm[3][3] = 2.0 * N;
  pm[4][4] = 2.0 * L;
  pm[5][5] = 2.0 * M;
  static const int ii[6] = {0, 1, 2, 0, 1, 2};
  static const int jj[6] = {0, 1, 2, 1, 2, 0};
  double t[6][6];
  for (int k = 0; k < 6; ++k) {
    // Voigt image of q e q^T, e the symmetric unit tensor of component k.
    for (int row = 0; row < 6; ++row) {
      const int a = ii[row], b = jj[row];
      const int c = ii[k], dd = jj[k];
      double v = axes[a][c] * axes[b][dd];
      if (c != dd) v += axes[a][dd] * axes[b][c];
      t[row][k] = v;
    }
  }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) s += t[a][i] * pm[a][b] * t[b][j];
      P[i * 6 + j] = s;
    }
  return SBK_OK;
}

int validate_material(const sbk_material& m) {
  if (!(m.youngs_modulus > 0.0) || !std::isfinite(m.youngs_modulus))
    return fail(SBK_ERR_CONFIG, "the material needs a positive Young's modulus");
  if (!(m.poisson_ratio > -1.0 && m.poisson_ratio < 0.5))
    return fail(SBK_ERR_CONFIG, "the material needs a Poisson ratio in (-1, 0.5)");
  const double vals[] = {m.yield_stress, m.hardening_modulus, m.kinematic_hardening_modulus, m.saturation_stress,
                         m.saturation_rate};
  for (double v : vals)
    if (!std::isfinite(v) || v < 0.0) return fail(SBK_ERR_CONFIG, "plasticity parameters must be finite and >= 0");
  if (m.saturation_stress > 0.0 && !(m.saturation_rate > 0.0))
    return fail(SBK_ERR_CONFIG, "a Voce saturation stress needs a positive saturation rate");
  if (m.num_backstresses < 0 || m.num_backstresses > SBK_MAX_BACKSTRESSES)
    return fail(SBK_ERR_CONFIG, "at most 4 backstresses are supported");
  for (int i = 0; i < m.num_backstresses; ++i)
    if (!finite_positive(m.backstress_modulus[i]) || !std::isfinite(m.backstress_recovery[i]) ||
        m.backstress_recovery[i] < 0.0)
      return fail(SBK_ERR_CONFIG, "a backstress needs a finite positive modulus and a non-negative recovery");
  const bool enabled = m.yield_stress > 0.0;
  if (!enabled && (m.hardening_modulus > 0.0 || m.kinematic_hardening_modulus > 0.0 || m.saturation_stress > 0.0 ||
                   m.num_backstresses > 0))
    return fail(SBK_ERR_CONFIG, "hardening parameters need a yield stress");
  if (!enabled && m.criterion != SBK_VON_MISES) return fail(SBK_ERR_CONFIG, "a yield criterion needs a yield stress");
  const bool general = m.criterion == SBK_HILL48 || m.num_backstresses > 0;
  const int terms = m.num_backstresses + (m.kinematic_hardening_modulus > 0.0 ? 1 : 0);
  if (general && terms > SBK_MAX_BACKSTRESSES)
    return fail(SBK_ERR_CONFIG, "backstresses plus Prager's modulus exceed 4 kinematic terms");
  if (m.kinematic_integration != SBK_EXPONENTIAL && m.kinematic_integration != SBK_BACKWARD_EULER)
    return fail(SBK_ERR_CONFIG, "unknown kinematic integration");
  return SBK_OK;
}

// Gauss-Legendre rules (src/elements/Quadrature.cpp:16-219), into fixed
// arrays (no heap): n points (x, w) of the line rule.
void line_rule(int n, double x_out[7], double w_out[7]) {
  if (n == 1) {
    x_out[0] = 0.0;
    w_out[0] = 2.0;
    return;
  }
  if (n == 2) {
    const double a = 1.0 / std::sqrt(3.0);
    x_out[0] = -a, x_out[1] = a, w_out[0] = w_out[1] = 1.0;
    return;
  }
  if (n == 3) {
    const double a = std::sqrt(3.0 / 5.0);
    x_out[0] = -a, x_out[1] = 0.0, x_out[2] = a;
    w_out[0] = w_out[2] = 5.0 / 9.0, w_out[1] = 8.0 / 9.0;
    return;
  }
  if (n == 4) {
    const double s6 = std::sqrt(6.0 / 5.0);
    const double x1 = std::sqrt((3.0 - 2.0 * s6) / 7.0), x2 = std::sqrt((3.0 + 2.0 * s6) / 7.0);
    const double s = std::sqrt(30.0);
    const double w1 = (18.0 + s) / 36.0, w2 = (18.0 - s) / 36.0;
    x_out[0] = -x2, x_out[1] = -x1, x_out[2] = x1, x_out[3] = x2;
    w_out[0] = w2, w_out[1] = w1, w_out[2] = w1, w_out[3] = w2;
    return;
  }
  const double pi = std::acos(-1.0);
  auto legendre = [n](double x, double& p0, double& p1) {
    p0 = 1.0;
    p1 = x;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
  };
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double x = std::cos(pi * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p0, p1;
      legendre(x, p0, p1);
      const double der = n * (x * p1 - p0) / (x * x - 1.0);
      const double step = p1 / der;
      x -= step;
      if (std::fabs(step) <= 1.0e-16) break;
    }
    if (2 * i + 1 == n) x = 0.0;
    double p0, p1;
    legendre(x, p0, p1);
    const double der = n * (x * p1 - p0) / (x * x - 1.0);
    const double w = 2.0 / ((1.0 - x * x) * der * der);
    x_out[i] = -x, w_out[i] = w;
    x_out[n - 1 - i] = x, w_out[n - 1 - i] = w;
  }
}

// The Hex8 stiffness rule: xi fastest, weights multiplied x * y * z
// (Hex8Kernels.hpp:125-130, Quadrature.cpp:165-219). Returns the point count
// (points with more than SBK_MAX_POINTS are counted but not stored), or a
// negative status.
int make_rule(const sbk_rule& rule, double pts[SBK_MAX_POINTS][4]) {
  int np = rule.stiffness_points, nt = rule.thickness_points, axis = rule.thickness_axis;
  if (np < 1 || np > 4) return -fail(SBK_ERR_CONFIG, "stiffness points must be 1 to 4");
  if (nt <= 0 || nt == np) {
    nt = np;
    axis = 2;
  }
  if (nt > 7) return -fail(SBK_ERR_CONFIG, "thickness points must be 1 to 7");
  if (axis < 0 || axis > 2) return -fail(SBK_ERR_CONFIG, "the thickness axis must be 0, 1 or 2");
  double px[7], pw[7], tx[7], tw[7];
  line_rule(np, px, pw);
  line_rule(nt, tx, tw);
  const int nx = axis == 0 ? nt : np, ny = axis == 1 ? nt : np, nz = axis == 2 ? nt : np;
  const double* rxx = axis == 0 ? tx : px;
  const double* rxw = axis == 0 ? tw : pw;
  const double* ryx = axis == 1 ? tx : px;
  const double* ryw = axis == 1 ? tw : pw;
  const double* rzx = axis == 2 ? tx : px;
  const double* rzw = axis == 2 ? tw : pw;
  int q = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i, ++q) {
        if (q >= SBK_MAX_POINTS) continue;
        pts[q][0] = rxx[i];
        pts[q][1] = ryx[j];
        pts[q][2] = rzx[k];
        pts[q][3] = rxw[i] * ryw[j] * rzw[k];
      }
  return q;
}

// The generalised eigenvectors of the yield matrix, P v = l S^-1 v with
// V^T S^-1 V = I (S = diag(1, 1, 1, 1/2, 1/2, 1/2)), through the ordinary
// eigenproblem of Q = S^1/2 P S^1/2 = U diag(l) U^T by cyclic Jacobi
// (V = S^1/2 U). The closest-point solves of the general return use them
// (B^-1 = V (I + f diag(l))^-1 V^T).
void yield_eigenbasis(const double* P, double* V, double* L) {
  const double h = std::sqrt(0.5);
  double s[6] = {1.0, 1.0, 1.0, h, h, h};
  double a[6][6], u[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      a[i][j] = s[i] * P[i * 6 + j] * s[j];
      u[i][j] = i == j ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < 6; ++i) {
      diag += a[i][i] * a[i][i];
      for (int j = i + 1; j < 6; ++j) off += a[i][j] * a[i][j];
    }
    if (off == 0.0 || off <= 1e-40 * diag) break;
    for (int pp = 0; pp < 5; ++pp)
      for (int q = pp + 1; q < 6; ++q) {
        const double apq = a[pp][q];
        if (apq == 0.0) continue;
        const double theta = (a[q][q] - a[pp][pp]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < 6; ++k) {
          const double akp = a[k][pp], akq = a[k][q];
          a[k][pp] = c * akp - sn * akq;
          a[k][q] = sn * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {
          const double apk = a[pp][k], aqk = a[q][k];
          a[pp][k] = c * apk - sn * aqk;
          a[q][k] = sn * apk + c * aqk;
        }
        for (int k = 0; k < 6; ++k) {
          const double ukp = u[k][pp], ukq = u[k][q];
          u[k][pp] = c * ukp - sn * ukq;
          u[k][q] = sn * ukp + c * ukq;
        }
      }
  }
  for (int k = 0; k < 6; ++k) {
    L[k] = std::max(a[k][k], 0.0);  // P is positive semi-definite; clip round-off below zero
    for (int i = 0; i < 6; ++i) V[i * 6 + k] = s[i] * u[i][k];
  }
}

int make_params(const sbk_material* mat, const sbk_rule* rule, int kinematics, Params& p) {
  if (!mat || !rule) return fail(SBK_ERR_ARGUMENT, "null material or rule");
  int rc = validate_material(*mat);
  if (rc) return rc;
  if (kinematics < SBK_SMALL_STRAIN || kinematics > SBK_FINITE_LOGARITHMIC)
    return fail(SBK_ERR_ARGUMENT, "unknown kinematics");
  double pts[SBK_MAX_POINTS][4];
  const int nq = make_rule(*rule, pts);
  if (nq < 0) return -nq;
  if (nq > SBK_MAX_POINTS) return fail(SBK_ERR_UNSUPPORTED, "rules of more than 32 points are not supported");
  std::memset(&p, 0, sizeof(Params));
  const double E = mat->youngs_modulus, nu = mat->poisson_ratio;
  p.G = E / (2.0 * (1.0 + nu));
  const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  p.K = lam + 2.0 * p.G / 3.0;
  p.sy0 = mat->yield_stress;
  p.H = mat->hardening_modulus;
  p.Hkin = mat->kinematic_hardening_modulus;
  p.Q = mat->saturation_stress;
  p.delta = mat->saturation_rate;
  rc = yield_matrix(*mat, p.P);
  if (rc) return rc;
  yield_eigenbasis(p.P, p.PV, p.PL);
  p.general = (mat->criterion == SBK_HILL48 || mat->num_backstresses > 0) ? 1 : 0;
  p.enabled = p.sy0 > 0.0 ? 1 : 0;
  p.integration = mat->kinematic_integration;
  p.symmetric = 1;
  for (int i = 0; i < mat->num_backstresses; ++i)
    if (mat->backstress_recovery[i] > 0.0) p.symmetric = 0;
  p.nterms = 0;
  if (p.general) {
    for (int i = 0; i < mat->num_backstresses; ++i) {
      p.termC[p.nterms] = mat->backstress_modulus[i];
      p.termG[p.nterms] = mat->backstress_recovery[i];
      ++p.nterms;
    }
    if (p.Hkin > 0.0) {
      p.termC[p.nterms] = p.Hkin;
      p.termG[p.nterms] = 0.0;
      ++p.nterms;
    }
  }
  p.kinematics = kinematics;
  p.nq = nq;
  p.nfields = sbk::state_fields(p.nterms);
  for (int q = 0; q < nq; ++q)
    for (int k = 0; k < 4; ++k) p.qp[q][k] = pts[q][k];
  return SBK_OK;
}

template <class T>
int dalloc(T** ptr, size_t count) {
  *ptr = nullptr;
  if (count == 0) return SBK_OK;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(ptr), count * sizeof(T));
  if (e != cudaSuccess) return fail(SBK_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return SBK_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
struct sbk_system {
  Params p;
  int64_t nn = 0, ne = 0, nnz = 0, num_blocks = 0;
  cudaStream_t stream = nullptr;
  bool plastic = false;
  bool frozen = false;            // committed plastic state frozen: no return
  int material_symmetric = 1;     // Params::symmetric of the material
  // mesh
  double* coords = nullptr;
  int32_t* conn = nullptr;
  // history and trial
  double* committed = nullptr;
  double* trial = nullptr;
  double* alpha_c = nullptr;
  double* alpha_t = nullptr;
  // element outputs
  double* force = nullptr;
  double* tangent = nullptr;
  double* energy_e = nullptr;
  uint8_t* yield = nullptr;
  int32_t* iters = nullptr;
  int32_t* code = nullptr;
  int32_t* first_fail = nullptr;
  // assembly
  int32_t* outer = nullptr;
  int32_t* inner = nullptr;
  double* values = nullptr;       // where the assembly writes the tangent values
  double* own_values = nullptr;   // the system's own buffer (values unless the caller set one)
  double* internal = nullptr;
  double* scratch = nullptr;
  double* scalars = nullptr;
  int32_t* missing = nullptr;
  int32_t* block_col = nullptr;
  int64_t* block_value = nullptr;
  int32_t* block_ptr = nullptr;
  int32_t* block_src = nullptr;
  int32_t* node_ptr = nullptr;
  int32_t* node_src = nullptr;
  double* product = nullptr;  // |K| |u| per DOF (stiffness_gross)
  int32_t* order = nullptr;    // the element schedule of the next launch
  int32_t* sched = nullptr;    // its bucket counters
  bool order_valid = false;
  bool schedule = true;
  bool stable = false;  // commit copies instead of swapping (captured graphs stay valid)
  int elements_per_block = 0;
  bool has_trial = false;
  bool has_values = false;  // values hold the tangent of the last evaluate
  bool timing = false;
  int local_mode = SBK_LOCAL_PHASES;
  void* wave_mem = nullptr;  // the phase kernels' records (one allocation)
  sbk::WaveBuffers wave{};
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double last_ms[3] = {0.0, 0.0, 0.0};

  sbk::GatherMaps maps() const {
    sbk::GatherMaps m;
    m.num_nodes = nn;
    m.num_elements = ne;
    m.nnz = nnz;
    m.num_blocks = num_blocks;
    m.block_col = block_col;
    m.block_value = block_value;
    m.block_ptr = block_ptr;
    m.block_src = block_src;
    m.outer = outer;
    m.node_ptr = node_ptr;
    m.node_src = node_src;
    return m;
  }
};

namespace {

void free_system(sbk_system* s) {
  void* ptrs[] = {s->coords, s->conn, s->committed, s->trial, s->alpha_c, s->alpha_t, s->force,
                  s->tangent, s->energy_e, s->yield, s->iters, s->code, s->first_fail, s->outer,
                  s->inner, s->own_values, s->internal, s->scratch, s->scalars, s->missing, s->block_col,
                  s->block_value, s->block_ptr, s->block_src, s->node_ptr, s->node_src, s->product,
                  s->order, s->sched, s->wave_mem};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : s->ev)
    if (e) cudaEventDestroy(e);
  delete s;
}

std::atomic<int> g_local_mode{SBK_LOCAL_PHASES};

// The phase kernels' records of a system whose element takes them
// (allocated once, outside any stream capture).
int ensure_wave(sbk_system* s) {
  if (s->wave_mem || !sbk::wave_applies(s->p)) return SBK_OK;
  const size_t bytes = sbk::wave_buffer_bytes(s->ne);
  cudaError_t e = cudaMalloc(&s->wave_mem, bytes);
  if (e != cudaSuccess) {
    s->wave_mem = nullptr;
    return fail(SBK_ERR_CUDA, std::string("cudaMalloc (local-iteration records): ") + cudaGetErrorString(e));
  }
  sbk::wave_buffers_carve(s->wave_mem, s->ne, s->wave);
  return SBK_OK;
}

// Whether K1 of the system runs as the phase kernels.
bool uses_phases(const sbk_system* sys) {
  return sys->local_mode == SBK_LOCAL_PHASES && sys->wave_mem && sbk::wave_applies(sys->p);
}

// Whether the element schedule runs after an evaluation: for the single
// kernel only. The phase kernels take the elements in mesh order (on the
// 1M-element microbenchmark the schedule's order was 0.5 % slower there:
// every phase is a short body of code that all warps share anyway).
bool schedules(const sbk_system* sys) { return sys->schedule && !uses_phases(sys); }

// K1 of a system: the phase kernels where they apply, else the single kernel.
int system_elements(sbk_system* sys, const double* u_dev, int want_tangent, cudaStream_t st) {
  const int32_t* order = sys->schedule && sys->order_valid ? sys->order : nullptr;
  if (uses_phases(sys))
    return sbk::launch_elements_wave(sys->p, sys->ne, sys->coords, sys->conn, u_dev, sys->committed, sys->alpha_c,
                                     want_tangent, sys->force, sys->tangent, sys->energy_e, sys->trial, sys->alpha_t,
                                     sys->yield, sys->iters, sys->code, sys->first_fail, false, nullptr, sys->wave,
                                     sys->elements_per_block, st);
  return sbk::launch_elements(sys->p, sys->ne, sys->coords, sys->conn, u_dev, sys->committed, sys->alpha_c,
                              want_tangent, sys->force, sys->tangent, sys->energy_e, sys->trial, sys->alpha_t,
                              sys->yield, sys->iters, sys->code, sys->first_fail, false, sys->elements_per_block, order,
                              st);
}

template <class T>
int upload(T** dst, const std::vector<T>& src, cudaStream_t s) {
  int rc = dalloc(dst, src.size());
  if (rc) return rc;
  if (!src.empty()) SBK_CUDA(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return SBK_OK;
}

}  // namespace

namespace sbk {
int set_error(int code, const std::string& what) { return fail(code, what); }
int make_launch_params(const sbk_material* material, const sbk_rule* rule, int kinematics, Params& p) {
  return make_params(material, rule, kinematics, p);
}
}  // namespace sbk

extern "C" {

const char* sbk_last_error(void) { return g_error.c_str(); }

int sbk_rule_size(const sbk_rule* rule) {
  if (!rule) return 0;
  double pts[SBK_MAX_POINTS][4];
  const int n = make_rule(*rule, pts);
  return n < 0 ? 0 : n;
}

int sbk_state_fields(const sbk_material* material) {
  if (!material) return 0;
  const bool general = material->criterion == SBK_HILL48 || material->num_backstresses > 0;
  int terms = 0;
  if (general) terms = material->num_backstresses + (material->kinematic_hardening_modulus > 0.0 ? 1 : 0);
  return sbk::state_fields(terms);
}

int sbk_yield_matrix(const sbk_material* material, double* p_out) {
  if (!material || !p_out) return fail(SBK_ERR_ARGUMENT, "null argument");
  int rc = validate_material(*material);
  if (rc) return rc;
  return yield_matrix(*material, p_out);
}

int sbk_element_batch(const sbk_material* material, const sbk_rule* rule, int kinematics, int64_t ne,
                      const double* x_dev, const double* u_dev, const double* state_dev, const double* alpha_dev,
                      double* force_dev, double* tangent_dev, double* energy_dev, double* trial_dev,
                      double* alpha_out_dev, uint8_t* yield_dev, int32_t* iterations_dev, int32_t* code_dev,
                      void* stream) {
  int rc = check_device();
  if (rc) return rc;
  Params p;
  rc = make_params(material, rule, kinematics, p);
  if (rc) return rc;
  if (ne < 0) return fail(SBK_ERR_ARGUMENT, "negative element count");
  if (ne == 0) return SBK_OK;
  if (!x_dev || !u_dev || !state_dev || !force_dev || !energy_dev || !trial_dev || !alpha_out_dev || !yield_dev ||
      !iterations_dev || !code_dev)
    return fail(SBK_ERR_ARGUMENT, "null device buffer");
  if (ne * p.nq > 0x7fffffffLL) return fail(SBK_ERR_UNSUPPORTED, "too many points for one batch");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g_local_mode.load() == SBK_LOCAL_PHASES && sbk::wave_applies(p)) {
    // The phase kernels' records, stream-ordered on the caller's stream.
    void* mem = nullptr;
    SBK_CUDA(cudaMallocAsync(&mem, sbk::wave_buffer_bytes(ne), s));
    sbk::WaveBuffers w;
    sbk::wave_buffers_carve(mem, ne, w);
    rc = sbk::launch_elements_wave(p, ne, x_dev, nullptr, u_dev, state_dev, alpha_dev, tangent_dev != nullptr,
                                   force_dev, tangent_dev, energy_dev, trial_dev, alpha_out_dev, yield_dev,
                                   iterations_dev, code_dev, nullptr, true, nullptr, w, 0, s);
    cudaError_t e = cudaFreeAsync(mem, s);
    if (rc) return fail(SBK_ERR_CUDA, std::string("element kernels: ") + cudaGetErrorString((cudaError_t)rc));
    if (e != cudaSuccess) return fail(SBK_ERR_CUDA, std::string("cudaFreeAsync: ") + cudaGetErrorString(e));
    return SBK_OK;
  }
  rc = sbk::launch_elements(p, ne, x_dev, nullptr, u_dev, state_dev, alpha_dev, tangent_dev != nullptr, force_dev,
                            tangent_dev, energy_dev, trial_dev, alpha_out_dev, yield_dev, iterations_dev, code_dev,
                            nullptr, true, 0, nullptr, s);
  if (rc) return fail(SBK_ERR_CUDA, std::string("element kernel launch: ") + cudaGetErrorString((cudaError_t)rc));
  return SBK_OK;
}

int sbk_system_create(const sbk_mesh* mesh, const sbk_material* material, const sbk_rule* rule, int kinematics,
                      sbk_system** out) {
  if (!out) return fail(SBK_ERR_ARGUMENT, "null output handle");
  *out = nullptr;
  int rc = check_device();
  if (rc) return rc;
  if (!mesh || !mesh->coords || !mesh->connectivity || mesh->num_nodes <= 0 || mesh->num_elements <= 0)
    return fail(SBK_ERR_ARGUMENT, "an empty or null mesh");
  Params p;
  rc = make_params(material, rule, kinematics, p);
  if (rc) return rc;
  sbk_system* s = new sbk_system();
  p.num_nodes = mesh->num_nodes;
  s->p = p;
  s->nn = mesh->num_nodes;
  s->ne = mesh->num_elements;
  s->plastic = p.enabled != 0;
  s->material_symmetric = p.symmetric;
  if (s->ne * p.nq > 0x7fffffffLL) {
    free_system(s);
    return fail(SBK_ERR_UNSUPPORTED, "too many points");
  }
  const int64_t npts = s->ne * p.nq;
  const size_t state_size = static_cast<size_t>(npts) * p.nfields;
  std::vector<double> coords(mesh->coords, mesh->coords + 3 * s->nn);
  std::vector<int32_t> conn(mesh->connectivity, mesh->connectivity + 8 * s->ne);
#define TRY(x)          \
  do {                  \
    rc = (x);           \
    if (rc) {           \
      free_system(s);   \
      return rc;        \
    }                   \
  } while (0)
  TRY(upload(&s->coords, coords, nullptr));
  TRY(upload(&s->conn, conn, nullptr));
  {
    // The reference's pattern and the assembly's gather maps, built on the
    // device from the connectivity (sbk_pattern.cu).
    sbk::DevicePattern dp;
    TRY(sbk::build_device_pattern(s->nn, s->ne, s->conn, dp, nullptr));
    s->outer = dp.outer;
    s->inner = dp.inner;
    s->block_col = dp.block_col;
    s->block_value = dp.block_value;
    s->block_ptr = dp.block_ptr;
    s->block_src = dp.block_src;
    s->node_ptr = dp.node_ptr;
    s->node_src = dp.node_src;
    s->nnz = dp.nnz;
    s->num_blocks = dp.num_blocks;
  }
  TRY(dalloc(&s->committed, state_size));
  TRY(dalloc(&s->trial, state_size));
  TRY(dalloc(&s->alpha_c, static_cast<size_t>(s->ne) * 9));
  TRY(dalloc(&s->alpha_t, static_cast<size_t>(s->ne) * 9));
  TRY(dalloc(&s->force, static_cast<size_t>(s->ne) * 24));
  TRY(dalloc(&s->tangent, static_cast<size_t>(s->ne) * 576));
  TRY(dalloc(&s->energy_e, static_cast<size_t>(s->ne)));
  TRY(dalloc(&s->yield, static_cast<size_t>(npts)));
  TRY(dalloc(&s->iters, static_cast<size_t>(s->ne)));
  TRY(dalloc(&s->code, static_cast<size_t>(s->ne)));
  TRY(dalloc(&s->first_fail, 1));
  TRY(dalloc(&s->own_values, static_cast<size_t>(s->nnz)));
  s->values = s->own_values;
  TRY(dalloc(&s->internal, static_cast<size_t>(s->nn) * 3));
  TRY(dalloc(&s->product, static_cast<size_t>(s->nn) * 3));
  TRY(dalloc(&s->order, static_cast<size_t>(s->ne)));
  TRY(dalloc(&s->sched, sbk::schedule_scratch_ints(s->ne)));
  TRY(dalloc(&s->scratch, sbk::assemble_scratch_doubles()));
  TRY(dalloc(&s->scalars, 4));
  TRY(dalloc(&s->missing, 1));
  s->local_mode = g_local_mode.load();
  TRY(ensure_wave(s));
#undef TRY
  // Virgin points and zero modes (initialise_history).
  cudaMemset(s->committed, 0, state_size * sizeof(double));
  cudaMemset(s->alpha_c, 0, static_cast<size_t>(s->ne) * 9 * sizeof(double));
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    free_system(s);
    return fail(SBK_ERR_CUDA, std::string("system upload: ") + cudaGetErrorString(e));
  }
  *out = s;
  return SBK_OK;
}

int sbk_system_destroy(sbk_system* sys) {
  if (!sys) return SBK_OK;
  cudaStreamSynchronize(sys->stream);
  free_system(sys);
  return SBK_OK;
}

int sbk_system_set_stream(sbk_system* sys, void* stream) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  sys->stream = static_cast<cudaStream_t>(stream);
  return SBK_OK;
}

int sbk_system_set_schedule(sbk_system* sys, int by_cost) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  sys->schedule = by_cost != 0;
  if (!sys->schedule) sys->order_valid = false;
  return SBK_OK;
}

int sbk_system_set_element(sbk_system* sys, int element, int mean_dilatation) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  if (element != SBK_ELEMENT_INCOMPATIBLE_MODES && element != SBK_ELEMENT_STANDARD)
    return fail(SBK_ERR_ARGUMENT, "unknown element formulation");
  if (mean_dilatation < SBK_MEAN_DILATATION_AUTO || mean_dilatation > SBK_MEAN_DILATATION_NONE)
    return fail(SBK_ERR_ARGUMENT, "unknown mean_dilatation");
  // NonlinearSystem's constructor (NonlinearSystem.hpp:283-309): the
  // incompatible-mode Hex8 refuses "all"; the standard Hex8 averages with
  // "all" or "auto" when its rule has more than one point.
  if (element == SBK_ELEMENT_INCOMPATIBLE_MODES && mean_dilatation == SBK_MEAN_DILATATION_ALL)
    return fail(SBK_ERR_CONFIG,
                "\"mean_dilatation\": \"all\" is not combined with the incompatible-mode Hex8: averaging the "
                "dilatation of its modes leaves a zero-energy mode; use \"auto\" or \"none\"");
  sys->p.element = element == SBK_ELEMENT_STANDARD ? 1 : 0;
  sys->p.averaged = (element == SBK_ELEMENT_STANDARD && mean_dilatation != SBK_MEAN_DILATATION_NONE && sys->p.nq > 1)
                        ? 1
                        : 0;
  sys->order_valid = false;
  if (!sbk::wave_applies(sys->p) && sys->wave_mem) {
    cudaFree(sys->wave_mem);
    sys->wave_mem = nullptr;
  }
  return sys->local_mode == SBK_LOCAL_PHASES ? ensure_wave(sys) : SBK_OK;
}

int sbk_system_set_frozen(sbk_system* sys, int frozen) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  sys->frozen = frozen != 0;
  sys->p.enabled = (sys->plastic && !sys->frozen) ? 1 : 0;
  sys->p.symmetric = sys->frozen ? 1 : sys->material_symmetric;
  sys->order_valid = false;
  return SBK_OK;
}

int sbk_system_set_coordinates(sbk_system* sys, const double* coords_dev) {
  if (!sys || !coords_dev) return fail(SBK_ERR_ARGUMENT, "null argument");
  SBK_CUDA(cudaMemcpyAsync(sys->coords, coords_dev, static_cast<size_t>(sys->nn) * 3 * sizeof(double),
                           cudaMemcpyDeviceToDevice, sys->stream));
  return SBK_OK;
}

int sbk_system_element(const sbk_system* sys, int* element, int* averaged) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  if (element) *element = sys->p.element ? SBK_ELEMENT_STANDARD : SBK_ELEMENT_INCOMPATIBLE_MODES;
  if (averaged) *averaged = sys->p.averaged;
  return SBK_OK;
}

int sbk_set_local_iteration(int mode) {
  if (mode != SBK_LOCAL_PHASES && mode != SBK_LOCAL_SINGLE_KERNEL) return fail(SBK_ERR_ARGUMENT, "unknown mode");
  g_local_mode.store(mode);
  return SBK_OK;
}

int sbk_system_set_local_iteration(sbk_system* sys, int mode) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  if (mode != SBK_LOCAL_PHASES && mode != SBK_LOCAL_SINGLE_KERNEL) return fail(SBK_ERR_ARGUMENT, "unknown mode");
  sys->local_mode = mode;
  return mode == SBK_LOCAL_PHASES ? ensure_wave(sys) : SBK_OK;
}

int sbk_system_set_values_buffer(sbk_system* sys, double* values_dev) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  sys->values = values_dev ? values_dev : sys->own_values;
  sys->has_values = false;
  return SBK_OK;
}

int sbk_system_set_elements_per_block(sbk_system* sys, int epb) {
  if (!sys || epb < 0 || epb > 32) return fail(SBK_ERR_ARGUMENT, "bad elements per block");
  sys->elements_per_block = epb;
  return SBK_OK;
}

int sbk_system_pattern(const sbk_system* sys, sbk_pattern* out) {
  if (!sys || !out) return fail(SBK_ERR_ARGUMENT, "null argument");
  out->num_dofs = sys->nn * 3;
  out->nnz = sys->nnz;
  out->outer_dev = sys->outer;
  out->inner_dev = sys->inner;
  return SBK_OK;
}

int sbk_system_evaluate(sbk_system* sys, const double* u_dev, double lambda, int want_tangent,
                        sbk_evaluation* out) {
  (void)lambda;  // the forming system carries no dead load: f_ext = 0 (NonlinearSystem.hpp:87-92)
  if (!sys || !u_dev || !out) return fail(SBK_ERR_ARGUMENT, "null argument");
  cudaStream_t st = sys->stream;
  std::memset(out, 0, sizeof(*out));
  out->failed_element = -1;
  SBK_CUDA(cudaMemsetAsync(sys->first_fail, 0x7f, sizeof(int32_t), st));
  if (sys->timing) SBK_CUDA(cudaEventRecord(sys->ev[0], st));
  int rc = system_elements(sys, u_dev, want_tangent, st);
  if (rc) return fail(SBK_ERR_CUDA, std::string("element kernel: ") + cudaGetErrorString((cudaError_t)rc));
  if (sys->timing) SBK_CUDA(cudaEventRecord(sys->ev[1], st));
  // The assembly runs unconditionally; a failed element is reported after
  // it, with the scalars, in a single synchronisation (its sums are then
  // discarded, as the reference discards them when it throws).
  rc = sbk::launch_assemble_forces(sys->maps(), sys->force, sys->energy_e, sys->yield, sys->p.nq, sys->internal,
                                   sys->scratch, sys->scalars, st);
  if (rc) return fail(SBK_ERR_CUDA, std::string("assembly: ") + cudaGetErrorString((cudaError_t)rc));
  if (sys->timing) SBK_CUDA(cudaEventRecord(sys->ev[2], st));
  if (want_tangent) {
    rc = sbk::launch_assemble_values(sys->maps(), sys->tangent, sys->values, st);
    if (rc) return fail(SBK_ERR_CUDA, std::string("assembly: ") + cudaGetErrorString((cudaError_t)rc));
  }
  if (sys->timing) SBK_CUDA(cudaEventRecord(sys->ev[3], st));
  if (schedules(sys)) {
    rc = sbk::launch_schedule(sys->ne, sys->p.nq, sys->iters, sys->yield, sys->sched, sys->order, st);
    if (rc) return fail(SBK_ERR_CUDA, std::string("schedule: ") + cudaGetErrorString((cudaError_t)rc));
    sys->order_valid = true;
  }
  double sc[3];
  int32_t first = 0;
  SBK_CUDA(cudaMemcpyAsync(sc, sys->scalars, sizeof(sc), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaMemcpyAsync(&first, sys->first_fail, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaStreamSynchronize(st));
  if (sys->timing) {
    float ms = 0.0f;
    for (int i = 0; i < 3; ++i) {
      SBK_CUDA(cudaEventElapsedTime(&ms, sys->ev[i], sys->ev[i + 1]));
      sys->last_ms[i] = ms;
    }
  }
  if (first != 0x7f7f7f7f) {
    int32_t code = 0;
    SBK_CUDA(cudaMemcpy(&code, sys->code + first, sizeof(int32_t), cudaMemcpyDeviceToHost));
    out->failed_element = first;
    out->failure_code = code;
    sys->has_trial = false;
    sys->has_values = false;
    char buf[160];
    std::snprintf(buf, sizeof(buf), "Hex8 element %d: SolverError (code %d)", first, code);
    return fail(SBK_ERR_SOLVER, buf);
  }
  out->internal_dev = sys->internal;
  out->residual_dev = sys->internal;
  out->values_dev = want_tangent ? sys->values : nullptr;
  out->energy = sc[0];
  out->gross = std::sqrt(sc[1]);
  out->yielding_points = static_cast<int32_t>(sc[2]);
  sys->has_trial = true;
  sys->has_values = want_tangent != 0;
  return SBK_OK;
}

int sbk_system_set_timing(sbk_system* sys, int enable) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  if (enable && !sys->ev[0])
    for (cudaEvent_t& e : sys->ev) SBK_CUDA(cudaEventCreate(&e));
  sys->timing = enable != 0;
  return SBK_OK;
}

int sbk_system_last_timings(const sbk_system* sys, double* ms3) {
  if (!sys || !ms3) return fail(SBK_ERR_ARGUMENT, "null argument");
  for (int i = 0; i < 3; ++i) ms3[i] = sys->last_ms[i];
  return SBK_OK;
}

int sbk_system_commit(sbk_system* sys) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  // With stable buffers the trial state may come from a replayed graph,
  // which the host does not see: the caller checked its summary.
  if (!sys->has_trial && !sys->stable) return fail(SBK_ERR_ARGUMENT, "no successful evaluation to commit");
  if (sys->stable) {
    const size_t ns = static_cast<size_t>(sys->ne) * sys->p.nq * sys->p.nfields;
    SBK_CUDA(cudaMemcpyAsync(sys->committed, sys->trial, ns * sizeof(double), cudaMemcpyDeviceToDevice, sys->stream));
    SBK_CUDA(cudaMemcpyAsync(sys->alpha_c, sys->alpha_t, static_cast<size_t>(sys->ne) * 9 * sizeof(double),
                             cudaMemcpyDeviceToDevice, sys->stream));
  } else {
    std::swap(sys->committed, sys->trial);
    std::swap(sys->alpha_c, sys->alpha_t);
  }
  sys->has_trial = false;
  return SBK_OK;
}

int sbk_system_set_stable_buffers(sbk_system* sys, int stable) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  sys->stable = stable != 0;
  return SBK_OK;
}

int sbk_system_enqueue(sbk_system* sys, const double* u_dev, int want_tangent, double* summary_dev) {
  if (!sys || !u_dev || !summary_dev) return fail(SBK_ERR_ARGUMENT, "null argument");
  cudaStream_t st = sys->stream;
  SBK_CUDA(cudaMemsetAsync(sys->first_fail, 0x7f, sizeof(int32_t), st));
  int rc = system_elements(sys, u_dev, want_tangent, st);
  if (rc) return fail(SBK_ERR_CUDA, std::string("element kernel: ") + cudaGetErrorString((cudaError_t)rc));
  rc = sbk::launch_assemble_forces(sys->maps(), sys->force, sys->energy_e, sys->yield, sys->p.nq, sys->internal,
                                   sys->scratch, sys->scalars, st);
  if (!rc && want_tangent) rc = sbk::launch_assemble_values(sys->maps(), sys->tangent, sys->values, st);
  if (!rc && schedules(sys) && sys->order_valid)
    rc = sbk::launch_schedule(sys->ne, sys->p.nq, sys->iters, sys->yield, sys->sched, sys->order, st);
  if (!rc) rc = sbk::launch_summary(sys->scalars, sys->first_fail, sys->code, summary_dev, st);
  if (rc) return fail(SBK_ERR_CUDA, std::string("enqueue: ") + cudaGetErrorString((cudaError_t)rc));
  // The caller reads the summary after its own synchronisation; a commit
  // then takes this evaluation's trial state.
  sys->has_trial = true;
  sys->has_values = want_tangent != 0;
  return SBK_OK;
}

int sbk_system_get_committed(const sbk_system* sys, double* state, double* alpha) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  const size_t ns = static_cast<size_t>(sys->ne) * sys->p.nq * sys->p.nfields;
  if (state) SBK_CUDA(cudaMemcpy(state, sys->committed, ns * sizeof(double), cudaMemcpyDeviceToHost));
  if (alpha) SBK_CUDA(cudaMemcpy(alpha, sys->alpha_c, static_cast<size_t>(sys->ne) * 9 * sizeof(double),
                                 cudaMemcpyDeviceToHost));
  return SBK_OK;
}

int sbk_system_set_committed(sbk_system* sys, const double* state, const double* alpha) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  const size_t ns = static_cast<size_t>(sys->ne) * sys->p.nq * sys->p.nfields;
  if (state) {
    for (size_t i = 0; i < ns; ++i)
      if (!std::isfinite(state[i])) return fail(SBK_ERR_CONFIG, "the saved plastic history is not finite");
    SBK_CUDA(cudaMemcpy(sys->committed, state, ns * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (alpha) {
    for (size_t i = 0; i < static_cast<size_t>(sys->ne) * 9; ++i)
      if (!std::isfinite(alpha[i])) return fail(SBK_ERR_CONFIG, "the saved internal-mode parameters are not finite");
    SBK_CUDA(cudaMemcpy(sys->alpha_c, alpha, static_cast<size_t>(sys->ne) * 9 * sizeof(double),
                        cudaMemcpyHostToDevice));
  }
  return SBK_OK;
}

int sbk_system_get_trial(const sbk_system* sys, double* state, double* alpha, uint8_t* yield) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  const size_t npts = static_cast<size_t>(sys->ne) * sys->p.nq;
  if (state) SBK_CUDA(cudaMemcpy(state, sys->trial, npts * sys->p.nfields * sizeof(double), cudaMemcpyDeviceToHost));
  if (alpha) SBK_CUDA(cudaMemcpy(alpha, sys->alpha_t, static_cast<size_t>(sys->ne) * 9 * sizeof(double),
                                 cudaMemcpyDeviceToHost));
  if (yield) SBK_CUDA(cudaMemcpy(yield, sys->yield, npts, cudaMemcpyDeviceToHost));
  return SBK_OK;
}

int sbk_system_buffers(const sbk_system* sys, const double** committed_state_dev, const double** committed_alpha_dev,
                       const double** trial_state_dev, const double** trial_alpha_dev) {
  if (!sys) return fail(SBK_ERR_ARGUMENT, "null system");
  if (committed_state_dev) *committed_state_dev = sys->committed;
  if (committed_alpha_dev) *committed_alpha_dev = sys->alpha_c;
  if (trial_state_dev) *trial_state_dev = sys->trial;
  if (trial_alpha_dev) *trial_alpha_dev = sys->alpha_t;
  return SBK_OK;
}

int sbk_system_symmetric(const sbk_system* sys) { return sys && sys->p.symmetric ? 1 : 0; }
int sbk_system_plastic(const sbk_system* sys) { return sys && sys->plastic ? 1 : 0; }

int sbk_system_add_node_blocks(sbk_system* sys, int32_t n, const int32_t* nodes_dev, const double* blocks_dev) {
  if (!sys || (n > 0 && (!nodes_dev || !blocks_dev))) return fail(SBK_ERR_ARGUMENT, "null argument");
  if (n <= 0) return SBK_OK;
  cudaStream_t st = sys->stream;
  SBK_CUDA(cudaMemsetAsync(sys->missing, 0, sizeof(int32_t), st));
  int rc = sbk::launch_add_node_blocks(sys->nn, sys->outer, sys->inner, sys->values, n, nodes_dev, blocks_dev,
                                       sys->missing, st);
  if (rc) return fail(SBK_ERR_CUDA, "add_node_blocks launch");
  int32_t missing = 0;
  SBK_CUDA(cudaMemcpyAsync(&missing, sys->missing, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaStreamSynchronize(st));
  if (missing) return fail(SBK_ERR_ARGUMENT, "a node block names a node out of range or lies outside the pattern");
  return SBK_OK;
}

int sbk_system_stress(sbk_system* sys, const double* u_dev, double* out_dev) {
  if (!sys || !u_dev || !out_dev) return fail(SBK_ERR_ARGUMENT, "null argument");
  cudaStream_t st = sys->stream;
  SBK_CUDA(cudaMemsetAsync(sys->first_fail, 0x7f, sizeof(int32_t), st));
  // The returns reproduce the committed states into the trial buffer, which
  // the last evaluate's trial state no longer occupies after a commit.
  sys->has_trial = false;
  int rc = sbk::launch_stress(sys->p, sys->ne, sys->coords, sys->conn, u_dev, sys->committed, sys->alpha_c, sys->trial,
                              out_dev, sys->code, sys->first_fail, st);
  if (rc) return fail(SBK_ERR_CUDA, std::string("stress kernel: ") + cudaGetErrorString((cudaError_t)rc));
  int32_t first = 0;
  SBK_CUDA(cudaMemcpyAsync(&first, sys->first_fail, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaStreamSynchronize(st));
  if (first != 0x7f7f7f7f) {
    int32_t code = 0;
    SBK_CUDA(cudaMemcpy(&code, sys->code + first, sizeof(int32_t), cudaMemcpyDeviceToHost));
    char buf[160];
    std::snprintf(buf, sizeof(buf), "Hex8 element %d: SolverError in stress recovery (code %d)", first, code);
    return fail(SBK_ERR_SOLVER, buf);
  }
  return SBK_OK;
}

int sbk_system_vjp_x(sbk_system* sys, const double* u_dev, const double* lambda_dev, int frozen, double* gx_dev) {
  if (!sys || !u_dev || !lambda_dev || !gx_dev) return fail(SBK_ERR_ARGUMENT, "null argument");
  if (sys->p.element != 0 || sys->p.kinematics == SBK_SMALL_STRAIN)
    return fail(SBK_ERR_UNSUPPORTED, "the shape derivative is built for the incompatible-mode Hex8 under finite or "
                                     "logarithmic kinematics");
  cudaStream_t st = sys->stream;
  Params p = sys->p;
  if (frozen) p.enabled = 0;  // the committed plastic state, no return
  SBK_CUDA(cudaMemsetAsync(sys->first_fail, 0x7f, sizeof(int32_t), st));
  sys->has_trial = false;  // the trial buffers are overwritten
  int rc = sbk::launch_vjp(p, sys->ne, sys->coords, sys->conn, u_dev, sys->committed, sys->alpha_c, lambda_dev,
                           sys->trial, sys->yield, sys->code, sys->first_fail, sys->force, st);
  if (rc) return rc;
  int32_t first = 0;
  SBK_CUDA(cudaMemcpyAsync(&first, sys->first_fail, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaStreamSynchronize(st));
  if (first != 0x7f7f7f7f) {
    int32_t code = 0;
    SBK_CUDA(cudaMemcpy(&code, sys->code + first, sizeof(int32_t), cudaMemcpyDeviceToHost));
    return fail(SBK_ERR_SOLVER, "element " + std::to_string(first) + " failed in the shape derivative (code " +
                                    std::to_string(code) + ")");
  }
  rc = sbk::launch_assemble_forces(sys->maps(), sys->force, sys->energy_e, sys->yield, sys->p.nq, gx_dev, sys->scratch,
                                   sys->scalars, st);
  if (rc) return fail(SBK_ERR_CUDA, "shape derivative gather");
  return SBK_OK;
}

int sbk_system_stiffness_gross(sbk_system* sys, const double* u_dev, int32_t num_free, const int32_t* free_dev,
                               double* out) {
  if (!sys || !u_dev || !out || num_free < 0 || (num_free > 0 && !free_dev))
    return fail(SBK_ERR_ARGUMENT, "null argument");
  if (!sys->has_values) return fail(SBK_ERR_ARGUMENT, "stiffness_gross needs an evaluate with the tangent first");
  cudaStream_t st = sys->stream;
  SBK_CUDA(cudaMemsetAsync(sys->missing, 0, sizeof(int32_t), st));
  int rc = sbk::launch_stiffness_gross(sys->nn, sys->outer, sys->inner, sys->values, u_dev, num_free, free_dev,
                                       sys->product, sys->scratch, sys->scalars, sys->missing, st);
  if (rc) return fail(SBK_ERR_CUDA, "stiffness_gross launch");
  double sum = 0.0;
  int32_t bad = 0;
  SBK_CUDA(cudaMemcpyAsync(&sum, sys->scalars, sizeof(double), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaMemcpyAsync(&bad, sys->missing, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SBK_CUDA(cudaStreamSynchronize(st));
  if (bad) return fail(SBK_ERR_ARGUMENT, "a free DOF lies outside the model");
  *out = std::sqrt(sum);
  return SBK_OK;
}

}  // extern "C"
