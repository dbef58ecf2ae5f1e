// The free-free tangent of one Dirichlet partition on the device:
// PartitionedFactor (src/fem/Forming.cpp:59-241) - the block's pattern built
// once per partition, its values gathered from the full tangent every
// iteration, and a sparse factorisation fed on the device.
//
// Layout. The full tangent is the reference's CSC node-block pattern
// (structurally symmetric). The block K_ff keeps the entries whose row and
// column are free, in the full pattern's order (ff_src: the full index of
// each block entry, the inverse of the reference's positions_ map), so that
// assemble is one gather. The factorisation takes B = K_ff(p, p) in CSR
// with p a METIS nested-dissection order; fac_src maps every entry of B
// straight to its full index (transposition and permutation composed on
// the host at build time), so that factorize also reads the full tangent
// once, with no intermediate copy of the block.
//
// A symmetric block takes a sparse Cholesky. A non-symmetric one (Chaboche
// backstresses with recovery, the exact friction tangent), or one whose
// Cholesky fails, takes a dense LU with partial pivoting while it has at most
// kDenseMax rows (n^2 doubles: 3.2 GB at the bound); a larger one takes
// restarted GMRES preconditioned by the Cholesky of its symmetric part, and
// a sparse QR when that stalls or the symmetric part is not positive
// definite. The factorisations (cuSOLVER's device sparse Cholesky, dense LU
// and sparse QR) are library code; the gathers, the permutations, the
// densification, the Krylov iteration and the backward-error check are this
// file's.
#define DISABLE_CUSOLVER_DEPRECATED
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <cusolverSp.h>
#include <cusolverSp_LOWLEVEL_PREVIEW.h>
#include <cusparse.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "sbk.h"

namespace sbk {
int set_error(int code, const std::string& what);
}

namespace {

int pfail(int code, const std::string& what) { return sbk::set_error(code, what); }

#define PCUDA(call)                                                                                 \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) return pfail(SBK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define PSOLVER(call)                                                                                 \
  do {                                                                                                \
    cusolverStatus_t s_ = (call);                                                                     \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                                                \
      return pfail(SBK_ERR_CUDA, std::string(#call) + ": cuSOLVER status " + std::to_string((int)s_)); \
  } while (0)

// A correction is accepted when max|B x - b| <= kBackward max(|B| |x| + |b|).
constexpr double kBackward = 1.0e-10;
// The QR calls the block singular below this fraction of its largest entry
// (the reference's LDL^T takes pivots above 1e-13 of the largest).
constexpr double kSingular = 1.0e-13;

constexpr int kThreads = 256;
// GMRES: Krylov space of up to kRestart vectors, at most kRestarts cycles;
// a cycle ends when the estimated residual falls below kInner of |b|, the
// iteration when the backward error falls below kConverged.
constexpr int kRestart = 30;
constexpr int kRestarts = 8;
constexpr double kInner = 1.0e-13;
constexpr double kConverged = 1.0e-14;
// Blocks of at most this many rows take the dense LU (the default limit).
constexpr int32_t kDenseMax = 20000;

// counts[]: solves by method, fallbacks, singular blocks, Krylov steps, solves.
enum { kCholesky, kGmres, kLu, kQr, kCholeskyFellBack, kGmresFellBack, kSingularCount, kKrylovSteps, kSolves,
       kNumCounts };

unsigned grid_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b > 148 * 32) b = 148 * 32;  // grid-stride beyond 32 blocks per SM
  return (unsigned)(b > 0 ? b : 1);
}

__global__ void gather_kernel(const double* __restrict__ src, const int32_t* __restrict__ idx, int64_t n,
                              double* __restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = src[idx[j]];
}

// full[idx[i]] = v[i] (add false) or full[idx[i]] += scale v[i], the
// product rounded before the sum as the reference's x86-64 build (no FMA)
// rounds it; the indices are distinct, so no two threads write one entry.
__global__ void scatter_kernel(const double* __restrict__ v, const int32_t* __restrict__ idx, int64_t n,
                               double scale, bool add, double* __restrict__ full) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (add)
      full[idx[i]] = __dadd_rn(full[idx[i]], __dmul_rn(scale, v[i]));
    else
      full[idx[i]] = v[i];
  }
}

// The symmetric part (B + B^T) / 2; mirror[j] is the position of B's entry
// mirrored from j, so both halves of a pair get the same value.
__global__ void symmetric_part_kernel(const double* __restrict__ val, const int32_t* __restrict__ mirror,
                                      int64_t n, double* __restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = 0.5 * (val[j] + val[mirror[j]]);
}

// y = B x (residual false) or y = b - B x (residual true), row by row.
__global__ void spmv_kernel(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                            const double* __restrict__ val, const double* __restrict__ x,
                            const double* __restrict__ b, bool residual, int32_t n, double* __restrict__ y) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) s += val[k] * x[col[k]];
    y[i] = residual ? b[i] - s : s;
  }
}

// out[c] = V[:, c] . w for c < ncols, one block per column, summed by a
// fixed tree: the same inputs give the same bits.
__global__ void dots_kernel(const double* __restrict__ V, int64_t ld, const double* __restrict__ w, int32_t n,
                            double* __restrict__ out) {
  __shared__ double part[kThreads];
  const double* v = V + (int64_t)blockIdx.x * ld;
  double s = 0.0;
  for (int32_t i = threadIdx.x; i < n; i += blockDim.x) s += v[i] * w[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = part[0];
}

// w -= V[:, 0:ncols] h (sub true) or w = V[:, 0:ncols] h (sub false).
__global__ void combine_kernel(const double* __restrict__ V, int64_t ld, const double* __restrict__ h, int ncols,
                               bool sub, int32_t n, double* __restrict__ w) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < ncols; ++c) s += h[c] * V[(int64_t)c * ld + i];
    w[i] = sub ? w[i] - s : s;
  }
}

// y = x / d (d on the host).
__global__ void divide_kernel(const double* __restrict__ x, double d, int32_t n, double* __restrict__ y) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] / d;
}

__global__ void add_kernel(const double* __restrict__ z, int32_t n, double* __restrict__ x) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += z[i];
}

// The block B (CSR) into a zeroed dense column-major n x n matrix.
__global__ void densify_kernel(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                               const double* __restrict__ val, int32_t n, double* __restrict__ A) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) A[(int64_t)col[k] * n + i] = val[k];
}

// Smallest |U(i, i)| of a dense LU (bits of a non-negative double; the
// buffer starts at +infinity's bits).
__global__ void min_pivot_kernel(const double* __restrict__ A, int32_t n, unsigned long long* out) {
  double m = INFINITY;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    m = fmin(m, fabs(A[(int64_t)i * n + i]));
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMin(out, (unsigned long long)__double_as_longlong(m));
}

// Largest |entry| of the block (non-negative doubles order as their bits).
__global__ void max_abs_kernel(const double* __restrict__ a, int64_t n, unsigned long long* out) {
  double m = 0.0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(a[j]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// The backward error of a correction: per row r_i = (B x - b)_i and
// s_i = (|B| |x|)_i + |b_i|; out[0] = max |r_i|, out[1] = max s_i, out[2]
// counts rows whose sums are not finite. A max does not depend on the
// order the rows finish in.
__global__ void backward_error_kernel(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                      const double* __restrict__ val, const double* __restrict__ x,
                                      const double* __restrict__ b, int32_t n, unsigned long long* out) {
  double rmax = 0.0, smax = 0.0;
  int bad = 0;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double r = -b[i], s = fabs(b[i]);
    for (int32_t k = rowptr[i]; k < rowptr[i + 1]; ++k) {
      const double t = val[k] * x[col[k]];
      r += t;
      s += fabs(t);
    }
    if (!isfinite(r) || !isfinite(s)) {
      bad = 1;
    } else {
      rmax = fmax(rmax, fabs(r));
      smax = fmax(smax, s);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (rmax > 0.0) atomicMax(&out[0], (unsigned long long)__double_as_longlong(rmax));
    if (smax > 0.0) atomicMax(&out[1], (unsigned long long)__double_as_longlong(smax));
    if (bad) atomicAdd(&out[2], 1ull);
  }
}

template <class T>
int alloc(T** p, int64_t n) {
  *p = nullptr;
  if (n <= 0) return SBK_OK;
  PCUDA(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (size_t)n));
  return SBK_OK;
}

template <class T>
int upload(T** p, const std::vector<T>& h) {
  if (int rc = alloc(p, (int64_t)h.size())) return rc;
  if (!h.empty()) PCUDA(cudaMemcpy(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return SBK_OK;
}

}  // namespace

struct sbk_partition {
  int64_t n = 0, nnz = 0, nnz_ff = 0;
  int32_t nf = 0;
  cudaStream_t stream = nullptr;
  // the block (CSC, free numbering) and its sources in the full values
  int32_t* free_dofs = nullptr;
  int32_t* ff_outer = nullptr;
  int32_t* ff_inner = nullptr;
  int32_t* ff_src = nullptr;
  // the factorisation's matrix B = K_ff(p, p), CSR
  int32_t* perm = nullptr;  // B's row i is the block's row perm[i]
  int32_t* fac_rowptr = nullptr;
  int32_t* fac_col = nullptr;
  int32_t* fac_src = nullptr;
  int32_t* fac_mirror = nullptr;  // position in B of the entry mirrored from each entry
  double* fac_val = nullptr;
  double* sym_val = nullptr;      // (B + B^T) / 2, the GMRES preconditioner's matrix
  double* krylov = nullptr;       // GMRES basis, kRestart + 1 vectors of nf
  double* work_a = nullptr;       // nf each
  double* work_b = nullptr;
  double* coeffs = nullptr;       // 2 (kRestart + 1) + 1 projections and a norm
  double* rhs = nullptr;  // permuted right-hand side
  double* sol = nullptr;  // permuted solution
  unsigned long long* check = nullptr;  // backward error: max|r|, max s, non-finite rows, max|B|
  // cuSOLVER
  cusolverSpHandle_t handle = nullptr;
  cusparseMatDescr_t descr = nullptr;
  csrcholInfo_t chol = nullptr;
  void* chol_work = nullptr;
  bool analysed = false;
  int kind = 0;           // the factorisation in use: 0 none, SBK_FACTOR_*
  double scale = 0.0;     // max |B| of the factorised values
  int64_t counts[kNumCounts] = {};
  // dense LU
  cusolverDnHandle_t dense = nullptr;
  int32_t dense_max = kDenseMax;
  double* lu = nullptr;  // n x n, column-major
  int* ipiv = nullptr;
  int* lu_info = nullptr;
  double* lu_work = nullptr;

  ~sbk_partition() {
    for (void* p : {(void*)free_dofs, (void*)ff_outer, (void*)ff_inner, (void*)ff_src, (void*)perm,
                    (void*)fac_rowptr, (void*)fac_col, (void*)fac_src, (void*)fac_mirror, (void*)fac_val,
                    (void*)sym_val, (void*)krylov, (void*)work_a, (void*)work_b, (void*)coeffs, (void*)rhs,
                    (void*)sol, (void*)check, chol_work})
      if (p) cudaFree(p);
    for (void* p : {(void*)lu, (void*)ipiv, (void*)lu_info, (void*)lu_work})
      if (p) cudaFree(p);
    if (dense) cusolverDnDestroy(dense);
    if (chol) cusolverSpDestroyCsrcholInfo(chol);
    if (descr) cusparseDestroyMatDescr(descr);
    if (handle) cusolverSpDestroy(handle);
  }
};

namespace {

// reset + build (Forming.cpp:73-84, 213-241) on the host, once per
// partition, then the factorisation's order and its composed gather map.
int build_partition(sbk_partition* P, const std::vector<int32_t>& outer, const std::vector<int32_t>& inner,
                    const int32_t* free_host) {
  const int64_t n = P->n;
  const int32_t nf = P->nf;
  std::vector<int32_t> map((size_t)n, -1);
  std::vector<int32_t> free(free_host, free_host + nf);
  for (int32_t i = 0; i < nf; ++i) map[(size_t)free[i]] = i;
  // The block: for every free column in ascending order, its free rows in
  // the full column's order (sorted, since the free DOFs ascend).
  std::vector<int32_t> ff_outer((size_t)nf + 1, 0), ff_inner, ff_src;
  ff_inner.reserve(inner.size());
  ff_src.reserve(inner.size());
  for (int64_t col = 0; col < n; ++col) {
    const int32_t c = map[(size_t)col];
    if (c < 0) continue;
    for (int32_t k = outer[(size_t)col]; k < outer[(size_t)col + 1]; ++k) {
      const int32_t r = map[(size_t)inner[(size_t)k]];
      if (r < 0) continue;
      ff_inner.push_back(r);
      ff_src.push_back(k);
    }
    ff_outer[(size_t)c + 1] = (int32_t)ff_inner.size();
  }
  const int64_t m = (int64_t)ff_inner.size();
  P->nnz_ff = m;
  // Transposition: tr[t] is the position of the block entry mirrored from
  // t; the full pattern is structurally symmetric, so it exists.
  std::vector<int32_t> tr((size_t)m);
  for (int32_t c = 0; c < nf; ++c) {
    for (int32_t t = ff_outer[(size_t)c]; t < ff_outer[(size_t)c + 1]; ++t) {
      const int32_t r = ff_inner[(size_t)t];
      const auto lo = ff_inner.begin() + ff_outer[(size_t)r], hi = ff_inner.begin() + ff_outer[(size_t)r + 1];
      const auto it = std::lower_bound(lo, hi, c);
      if (it == hi || *it != c) return pfail(SBK_ERR_ARGUMENT, "the tangent's pattern is not structurally symmetric");
      tr[(size_t)t] = (int32_t)(it - ff_inner.begin());
    }
  }
  // Fill-reducing order: the block's pattern read as CSR is its own (it is
  // symmetric).
  std::vector<int32_t> p((size_t)nf), pinv((size_t)nf);
  PSOLVER(cusolverSpXcsrmetisndHost(P->handle, nf, (int)m, P->descr, ff_outer.data(), ff_inner.data(), nullptr,
                                    p.data()));
  {
    std::vector<char> seen((size_t)nf, 0);
    for (int32_t i = 0; i < nf; ++i) {
      if (p[(size_t)i] < 0 || p[(size_t)i] >= nf || seen[(size_t)p[(size_t)i]])
        return pfail(SBK_ERR_CUDA, "the fill-reducing order is not a permutation");
      seen[(size_t)p[(size_t)i]] = 1;
      pinv[(size_t)p[(size_t)i]] = i;
    }
  }
  // B = K_ff(p, p) in CSR. Row i of B is the block's row r = p[i]; its
  // entries (r, q) sit, in the CSC block, in column q at row r: the mirror
  // tr[t] of entry t = (q, r) of column r.
  std::vector<int32_t> rowptr((size_t)nf + 1, 0), col((size_t)m), src((size_t)m);
  std::vector<std::pair<int32_t, int32_t>> row;
  int64_t w = 0;
  for (int32_t i = 0; i < nf; ++i) {
    const int32_t r = p[(size_t)i];
    row.clear();
    for (int32_t t = ff_outer[(size_t)r]; t < ff_outer[(size_t)r + 1]; ++t)
      row.emplace_back(pinv[(size_t)ff_inner[(size_t)t]], ff_src[(size_t)tr[(size_t)t]]);
    std::sort(row.begin(), row.end());
    for (const auto& e : row) {
      col[(size_t)w] = e.first;
      src[(size_t)w] = e.second;
      ++w;
    }
    rowptr[(size_t)i + 1] = (int32_t)w;
  }
  std::vector<int32_t> mirror((size_t)m);
  for (int32_t i = 0; i < nf; ++i) {
    for (int32_t k = rowptr[(size_t)i]; k < rowptr[(size_t)i + 1]; ++k) {
      const int32_t j = col[(size_t)k];
      const auto lo = col.begin() + rowptr[(size_t)j], hi = col.begin() + rowptr[(size_t)j + 1];
      const auto it = std::lower_bound(lo, hi, i);
      mirror[(size_t)k] = (int32_t)(it - col.begin());  // exists: the block's pattern is symmetric
    }
  }
  if (int rc = upload(&P->free_dofs, free)) return rc;
  if (int rc = upload(&P->ff_outer, ff_outer)) return rc;
  if (int rc = upload(&P->ff_inner, ff_inner)) return rc;
  if (int rc = upload(&P->ff_src, ff_src)) return rc;
  if (int rc = upload(&P->perm, p)) return rc;
  if (int rc = upload(&P->fac_rowptr, rowptr)) return rc;
  if (int rc = upload(&P->fac_col, col)) return rc;
  if (int rc = upload(&P->fac_src, src)) return rc;
  if (int rc = upload(&P->fac_mirror, mirror)) return rc;
  if (int rc = alloc(&P->fac_val, m)) return rc;
  if (int rc = alloc(&P->rhs, nf)) return rc;
  if (int rc = alloc(&P->sol, nf)) return rc;
  if (int rc = alloc(&P->check, 4)) return rc;
  return SBK_OK;
}

// The backward error of sol for B sol = rhs: max|B sol - rhs| / max(|B| |sol|
// + |rhs|), or infinity when a row's sums are not finite.
int backward_error(sbk_partition* P, double* omega) {
  PCUDA(cudaMemsetAsync(P->check, 0, 3 * sizeof(unsigned long long), P->stream));
  backward_error_kernel<<<grid_for(P->nf), kThreads, 0, P->stream>>>(P->fac_rowptr, P->fac_col, P->fac_val, P->sol,
                                                                     P->rhs, P->nf, P->check);
  PCUDA(cudaGetLastError());
  unsigned long long h[3];
  PCUDA(cudaMemcpyAsync(h, P->check, sizeof(h), cudaMemcpyDeviceToHost, P->stream));
  PCUDA(cudaStreamSynchronize(P->stream));
  double r, s;
  std::memcpy(&r, &h[0], sizeof(double));
  std::memcpy(&s, &h[1], sizeof(double));
  *omega = h[2] != 0 ? INFINITY : (s > 0.0 ? r / s : (r > 0.0 ? INFINITY : 0.0));
  return SBK_OK;
}

int solve_qr(sbk_partition* P) {
  int singular = -1;
  PSOLVER(cusolverSpDcsrlsvqr(P->handle, P->nf, (int)P->nnz_ff, P->descr, P->fac_val, P->fac_rowptr, P->fac_col,
                              P->rhs, kSingular * P->scale, 0, P->sol, &singular));
  if (singular >= 0) {
    ++P->counts[kSingularCount];
    return pfail(SBK_ERR_SOLVER, "the tangent is singular - a rigid-body motion or a mechanism the step's "
                                 "constraints and tools leave free (QR pivot " + std::to_string(singular) + ")");
  }
  return SBK_OK;
}

int chol_apply(sbk_partition* P, const double* b, double* x) {
  PSOLVER(cusolverSpDcsrcholSolve(P->handle, P->nf, b, x, P->chol, P->chol_work));
  return SBK_OK;
}

// Restarted GMRES on B sol = rhs, right-preconditioned by the Cholesky M of
// the symmetric part (sym_val): the Krylov space of B M^-1, orthogonalised by
// classical Gram-Schmidt applied twice, the least-squares problem reduced
// by Givens rotations on the host. *converged: the backward error reached
// kConverged (or kBackward once the cycles ran out).
int gmres(sbk_partition* P, bool* converged) {
  const int32_t n = P->nf;
  const int64_t ld = n;
  const unsigned g = grid_for(n);
  cudaStream_t st = P->stream;
  *converged = false;
  if (!P->krylov) {
    if (int rc = alloc(&P->krylov, (int64_t)(kRestart + 1) * ld)) return rc;
    if (int rc = alloc(&P->work_a, n)) return rc;
    if (int rc = alloc(&P->work_b, n)) return rc;
    if (int rc = alloc(&P->coeffs, 2 * (kRestart + 1) + 1)) return rc;
  }
  double* V = P->krylov;
  double* w = P->work_a;
  double* z = P->work_b;
  PCUDA(cudaMemsetAsync(P->sol, 0, sizeof(double) * (size_t)n, st));
  dots_kernel<<<1, kThreads, 0, st>>>(P->rhs, ld, P->rhs, n, P->coeffs);
  double bb = 0.0;
  PCUDA(cudaMemcpyAsync(&bb, P->coeffs, sizeof(double), cudaMemcpyDeviceToHost, st));
  PCUDA(cudaStreamSynchronize(st));
  if (bb == 0.0) {
    *converged = true;
    return SBK_OK;
  }
  const double bnorm = std::sqrt(bb);
  std::vector<double> H((size_t)(kRestart + 1) * kRestart), cs(kRestart), sn(kRestart), gv(kRestart + 1),
      y(kRestart), hh(2 * (kRestart + 1) + 1);
  double omega = INFINITY;
  for (int cycle = 0; cycle < kRestarts; ++cycle) {
    // v0 = (rhs - B sol) / beta
    spmv_kernel<<<g, kThreads, 0, st>>>(P->fac_rowptr, P->fac_col, P->fac_val, P->sol, P->rhs, true, n, w);
    dots_kernel<<<1, kThreads, 0, st>>>(w, ld, w, n, P->coeffs);
    double rr = 0.0;
    PCUDA(cudaMemcpyAsync(&rr, P->coeffs, sizeof(double), cudaMemcpyDeviceToHost, st));
    PCUDA(cudaStreamSynchronize(st));
    const double beta = std::sqrt(rr);
    if (!std::isfinite(beta)) break;
    if (beta == 0.0) {
      omega = 0.0;
      break;
    }
    divide_kernel<<<g, kThreads, 0, st>>>(w, beta, n, V);
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int k = 0;
    for (int j = 0; j < kRestart; ++j) {
      ++P->counts[kKrylovSteps];
      double* vj = V + (int64_t)j * ld;
      if (int rc = chol_apply(P, vj, z)) return rc;
      spmv_kernel<<<g, kThreads, 0, st>>>(P->fac_rowptr, P->fac_col, P->fac_val, z, nullptr, false, n, w);
      const int c = j + 1;
      dots_kernel<<<c, kThreads, 0, st>>>(V, ld, w, n, P->coeffs);
      combine_kernel<<<g, kThreads, 0, st>>>(V, ld, P->coeffs, c, true, n, w);
      dots_kernel<<<c, kThreads, 0, st>>>(V, ld, w, n, P->coeffs + c);
      combine_kernel<<<g, kThreads, 0, st>>>(V, ld, P->coeffs + c, c, true, n, w);
      dots_kernel<<<1, kThreads, 0, st>>>(w, ld, w, n, P->coeffs + 2 * c);
      PCUDA(cudaGetLastError());
      PCUDA(cudaMemcpyAsync(hh.data(), P->coeffs, sizeof(double) * (size_t)(2 * c + 1), cudaMemcpyDeviceToHost, st));
      PCUDA(cudaStreamSynchronize(st));
      double* col = &H[(size_t)j * (kRestart + 1)];
      for (int i = 0; i < c; ++i) col[i] = hh[(size_t)i] + hh[(size_t)(c + i)];
      const double hn = std::sqrt(hh[(size_t)(2 * c)]);
      col[c] = hn;
      if (!std::isfinite(hn)) break;
      if (hn > 0.0 && j + 1 <= kRestart) divide_kernel<<<g, kThreads, 0, st>>>(w, hn, n, V + (int64_t)c * ld);
      for (int i = 0; i < j; ++i) {  // earlier rotations
        const double a = col[i], b = col[i + 1];
        col[i] = cs[(size_t)i] * a + sn[(size_t)i] * b;
        col[i + 1] = -sn[(size_t)i] * a + cs[(size_t)i] * b;
      }
      const double r = std::hypot(col[j], col[j + 1]);
      cs[(size_t)j] = r > 0.0 ? col[j] / r : 1.0;
      sn[(size_t)j] = r > 0.0 ? col[j + 1] / r : 0.0;
      col[j] = r;
      col[j + 1] = 0.0;
      gv[(size_t)j + 1] = -sn[(size_t)j] * gv[(size_t)j];
      gv[(size_t)j] = cs[(size_t)j] * gv[(size_t)j];
      k = j + 1;
      if (std::fabs(gv[(size_t)j + 1]) <= kInner * bnorm || hn == 0.0) break;
    }
    if (k == 0) break;
    for (int i = k - 1; i >= 0; --i) {  // H y = g, upper triangular
      double t = gv[(size_t)i];
      for (int l = i + 1; l < k; ++l) t -= H[(size_t)l * (kRestart + 1) + i] * y[(size_t)l];
      y[(size_t)i] = t / H[(size_t)i * (kRestart + 1) + i];
    }
    PCUDA(cudaMemcpyAsync(P->coeffs, y.data(), sizeof(double) * (size_t)k, cudaMemcpyHostToDevice, st));
    combine_kernel<<<g, kThreads, 0, st>>>(V, ld, P->coeffs, k, false, n, w);
    if (int rc = chol_apply(P, w, z)) return rc;
    add_kernel<<<g, kThreads, 0, st>>>(z, n, P->sol);
    PCUDA(cudaGetLastError());
    const double before = omega;
    if (int rc = backward_error(P, &omega)) return rc;
    if (omega <= kConverged) break;
    if (cycle > 0 && !(omega < 0.5 * before)) break;  // stagnating
  }
  *converged = omega <= kBackward;
  return SBK_OK;
}

// The dense LU of B (partial pivoting, cuSOLVER): *singular when a pivot is
// zero or below kSingular of the block's largest entry.
int dense_factor(sbk_partition* P, bool* singular) {
  const int32_t n = P->nf;
  cudaStream_t st = P->stream;
  *singular = false;
  if (!P->dense) {
    if (cusolverDnCreate(&P->dense) != CUSOLVER_STATUS_SUCCESS) return pfail(SBK_ERR_CUDA, "cusolverDnCreate failed");
    if (int rc = alloc(&P->lu, (int64_t)n * n)) return rc;
    if (int rc = alloc(&P->ipiv, n)) return rc;
    if (int rc = alloc(&P->lu_info, 1)) return rc;
    int lwork = 0;
    PSOLVER(cusolverDnDgetrf_bufferSize(P->dense, n, n, P->lu, n, &lwork));
    if (int rc = alloc(&P->lu_work, lwork > 0 ? lwork : 1)) return rc;
  }
  PSOLVER(cusolverDnSetStream(P->dense, st));
  PCUDA(cudaMemsetAsync(P->lu, 0, sizeof(double) * (size_t)n * (size_t)n, st));
  densify_kernel<<<grid_for(n), kThreads, 0, st>>>(P->fac_rowptr, P->fac_col, P->fac_val, n, P->lu);
  PCUDA(cudaGetLastError());
  PSOLVER(cusolverDnDgetrf(P->dense, n, n, P->lu, n, P->lu_work, P->ipiv, P->lu_info));
  const double inf = INFINITY;
  PCUDA(cudaMemcpyAsync(P->check + 3, &inf, sizeof(double), cudaMemcpyHostToDevice, st));
  min_pivot_kernel<<<grid_for(n), kThreads, 0, st>>>(P->lu, n, P->check + 3);
  PCUDA(cudaGetLastError());
  int info = 0;
  unsigned long long low = 0;
  PCUDA(cudaMemcpyAsync(&info, P->lu_info, sizeof(int), cudaMemcpyDeviceToHost, st));
  PCUDA(cudaMemcpyAsync(&low, P->check + 3, sizeof(low), cudaMemcpyDeviceToHost, st));
  PCUDA(cudaStreamSynchronize(st));
  double pivot;
  std::memcpy(&pivot, &low, sizeof(double));
  *singular = info != 0 || !(pivot > kSingular * P->scale);
  return SBK_OK;
}

int dense_solve(sbk_partition* P, bool transpose = false) {
  PCUDA(cudaMemcpyAsync(P->sol, P->rhs, sizeof(double) * (size_t)P->nf, cudaMemcpyDeviceToDevice, P->stream));
  PSOLVER(cusolverDnDgetrs(P->dense, transpose ? CUBLAS_OP_T : CUBLAS_OP_N, P->nf, 1, P->lu, P->nf, P->ipiv, P->sol,
                           P->nf, P->lu_info));
  return SBK_OK;
}

}  // namespace

extern "C" {

int sbk_partition_create(int64_t num_dofs, const int32_t* outer_dev, const int32_t* inner_dev, int64_t nnz,
                         int32_t num_free, const int32_t* free_host, sbk_partition** out) {
  if (!out || !outer_dev || !inner_dev || !free_host || num_dofs <= 0 || nnz <= 0 || num_free <= 0 ||
      num_free > num_dofs || nnz > INT32_MAX)
    return pfail(SBK_ERR_ARGUMENT, "sbk_partition_create: bad arguments");
  *out = nullptr;
  for (int32_t i = 0; i < num_free; ++i) {
    if (free_host[i] < 0 || free_host[i] >= num_dofs || (i > 0 && free_host[i] <= free_host[i - 1]))
      return pfail(SBK_ERR_ARGUMENT, "the free DOFs must be strictly ascending and within the model");
  }
  std::vector<int32_t> outer((size_t)num_dofs + 1), inner((size_t)nnz);
  PCUDA(cudaMemcpy(outer.data(), outer_dev, sizeof(int32_t) * outer.size(), cudaMemcpyDeviceToHost));
  PCUDA(cudaMemcpy(inner.data(), inner_dev, sizeof(int32_t) * inner.size(), cudaMemcpyDeviceToHost));
  if (outer[0] != 0 || outer[(size_t)num_dofs] != nnz)
    return pfail(SBK_ERR_ARGUMENT, "sbk_partition_create: the pattern's offsets do not span nnz");
  for (int64_t c = 0; c < num_dofs; ++c) {
    if (outer[(size_t)c + 1] < outer[(size_t)c])
      return pfail(SBK_ERR_ARGUMENT, "sbk_partition_create: the pattern's offsets decrease");
    for (int32_t k = outer[(size_t)c]; k < outer[(size_t)c + 1]; ++k)
      if (inner[(size_t)k] < 0 || inner[(size_t)k] >= num_dofs || (k > outer[(size_t)c] && inner[(size_t)k] <= inner[(size_t)k - 1]))
        return pfail(SBK_ERR_ARGUMENT, "sbk_partition_create: a column's rows are out of range or not ascending");
  }
  sbk_partition* P = new sbk_partition;
  P->n = num_dofs;
  P->nnz = nnz;
  P->nf = num_free;
  int rc = SBK_OK;
  if (cusolverSpCreate(&P->handle) != CUSOLVER_STATUS_SUCCESS) {
    rc = pfail(SBK_ERR_CUDA, "cusolverSpCreate failed");
  } else if (cusparseCreateMatDescr(&P->descr) != CUSPARSE_STATUS_SUCCESS) {
    rc = pfail(SBK_ERR_CUDA, "cusparseCreateMatDescr failed");
  } else {
    cusparseSetMatType(P->descr, CUSPARSE_MATRIX_TYPE_GENERAL);
    cusparseSetMatIndexBase(P->descr, CUSPARSE_INDEX_BASE_ZERO);
    rc = build_partition(P, outer, inner, free_host);
  }
  if (rc != SBK_OK) {
    delete P;
    return rc;
  }
  *out = P;
  return SBK_OK;
}

int sbk_partition_destroy(sbk_partition* part) {
  delete part;
  return SBK_OK;
}

int sbk_partition_set_stream(sbk_partition* part, void* stream) {
  if (!part) return pfail(SBK_ERR_ARGUMENT, "null partition");
  part->stream = static_cast<cudaStream_t>(stream);
  PSOLVER(cusolverSpSetStream(part->handle, part->stream));
  return SBK_OK;
}

int sbk_partition_set_dense_limit(sbk_partition* part, int32_t max_rows) {
  if (!part || max_rows < 0) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_set_dense_limit: bad arguments");
  part->dense_max = max_rows;
  return SBK_OK;
}

int sbk_partition_info(const sbk_partition* part, int32_t* num_free, int64_t* nnz_ff) {
  if (!part) return pfail(SBK_ERR_ARGUMENT, "null partition");
  if (num_free) *num_free = part->nf;
  if (nnz_ff) *nnz_ff = part->nnz_ff;
  return SBK_OK;
}

int sbk_partition_pattern(const sbk_partition* part, int32_t* outer_dev, int32_t* inner_dev) {
  if (!part) return pfail(SBK_ERR_ARGUMENT, "null partition");
  if (outer_dev)
    PCUDA(cudaMemcpyAsync(outer_dev, part->ff_outer, sizeof(int32_t) * ((size_t)part->nf + 1),
                          cudaMemcpyDeviceToDevice, part->stream));
  if (inner_dev)
    PCUDA(cudaMemcpyAsync(inner_dev, part->ff_inner, sizeof(int32_t) * (size_t)part->nnz_ff, cudaMemcpyDeviceToDevice,
                          part->stream));
  return SBK_OK;
}

int sbk_partition_assemble(sbk_partition* part, const double* values_dev, double* kff_dev) {
  if (!part || !values_dev || !kff_dev) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_assemble: null argument");
  gather_kernel<<<grid_for(part->nnz_ff), kThreads, 0, part->stream>>>(values_dev, part->ff_src, part->nnz_ff,
                                                                       kff_dev);
  PCUDA(cudaGetLastError());
  return SBK_OK;
}

int sbk_partition_restrict(sbk_partition* part, const double* full_dev, double* out_dev) {
  if (!part || !full_dev || !out_dev) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_restrict: null argument");
  gather_kernel<<<grid_for(part->nf), kThreads, 0, part->stream>>>(full_dev, part->free_dofs, part->nf, out_dev);
  PCUDA(cudaGetLastError());
  return SBK_OK;
}

int sbk_partition_add_to(sbk_partition* part, double* full_dev, const double* v_dev, double alpha) {
  if (!part || !full_dev || !v_dev) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_add_to: null argument");
  scatter_kernel<<<grid_for(part->nf), kThreads, 0, part->stream>>>(v_dev, part->free_dofs, part->nf, alpha, true,
                                                                    full_dev);
  PCUDA(cudaGetLastError());
  return SBK_OK;
}

int sbk_partition_factorize(sbk_partition* part, const double* values_dev, int symmetric, int* kind) {
  if (!part || !values_dev) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_factorize: null argument");
  sbk_partition* P = part;
  P->kind = 0;
  gather_kernel<<<grid_for(P->nnz_ff), kThreads, 0, P->stream>>>(values_dev, P->fac_src, P->nnz_ff, P->fac_val);
  PCUDA(cudaGetLastError());
  PCUDA(cudaMemsetAsync(P->check + 3, 0, sizeof(unsigned long long), P->stream));
  max_abs_kernel<<<grid_for(P->nnz_ff), kThreads, 0, P->stream>>>(P->fac_val, P->nnz_ff, P->check + 3);
  PCUDA(cudaGetLastError());
  unsigned long long top = 0;
  PCUDA(cudaMemcpyAsync(&top, P->check + 3, sizeof(top), cudaMemcpyDeviceToHost, P->stream));
  PCUDA(cudaStreamSynchronize(P->stream));
  std::memcpy(&P->scale, &top, sizeof(double));
  const bool small = P->nf <= P->dense_max;
  if (symmetric || !small) {
    // The Cholesky factorises the block itself, or for a large
    // non-symmetric block its symmetric part, GMRES's preconditioner.
    const double* chol_val = P->fac_val;
    if (!symmetric) {
      if (!P->sym_val) {
        if (int rc = alloc(&P->sym_val, P->nnz_ff)) return rc;
      }
      symmetric_part_kernel<<<grid_for(P->nnz_ff), kThreads, 0, P->stream>>>(P->fac_val, P->fac_mirror,
                                                                             P->nnz_ff, P->sym_val);
      PCUDA(cudaGetLastError());
      chol_val = P->sym_val;
    }
    if (!P->analysed) {
      PSOLVER(cusolverSpCreateCsrcholInfo(&P->chol));
      PSOLVER(cusolverSpXcsrcholAnalysis(P->handle, P->nf, (int)P->nnz_ff, P->descr, P->fac_rowptr, P->fac_col,
                                         P->chol));
      size_t internal = 0, work = 0;
      PSOLVER(cusolverSpDcsrcholBufferInfo(P->handle, P->nf, (int)P->nnz_ff, P->descr, chol_val, P->fac_rowptr,
                                           P->fac_col, P->chol, &internal, &work));
      PCUDA(cudaMalloc(&P->chol_work, work > 0 ? work : 1));
      P->analysed = true;
    }
    PSOLVER(cusolverSpDcsrcholFactor(P->handle, P->nf, (int)P->nnz_ff, P->descr, chol_val, P->fac_rowptr,
                                     P->fac_col, P->chol, P->chol_work));
    int position = -1;
    PSOLVER(cusolverSpDcsrcholZeroPivot(P->handle, P->chol, 0.0, &position));
    if (position < 0) {
      P->kind = symmetric ? SBK_FACTOR_CHOLESKY : SBK_FACTOR_GMRES;
      ++P->counts[symmetric ? kCholesky : kGmres];
    } else {
      ++P->counts[symmetric ? kCholeskyFellBack : kGmresFellBack];
    }
  }
  if (P->kind == 0) {
    if (small) {
      bool singular = false;
      if (int rc = dense_factor(P, &singular)) return rc;
      P->kind = SBK_FACTOR_LU;
      ++P->counts[kLu];
      if (singular) {
        P->kind = 0;
        ++P->counts[kSingularCount];
        return pfail(SBK_ERR_SOLVER, "the tangent is singular - a rigid-body motion or a mechanism the step's "
                                     "constraints and tools leave free (a vanishing LU pivot)");
      }
    } else {
      P->kind = SBK_FACTOR_QR;  // factorised with each solve
      ++P->counts[kQr];
    }
  }
  if (kind) *kind = P->kind;
  return SBK_OK;
}

// Leaves a Cholesky or a GMRES whose correction was not accepted for the
// dense LU (small blocks) or the QR.
static int fall_back(sbk_partition* P, int from_count, int fell_back_count) {
  --P->counts[from_count];
  ++P->counts[fell_back_count];
  if (P->nf <= P->dense_max) {
    bool singular = false;
    if (int rc = dense_factor(P, &singular)) return rc;
    ++P->counts[kLu];
    P->kind = SBK_FACTOR_LU;
    if (singular) {
      P->kind = 0;
      ++P->counts[kSingularCount];
      return pfail(SBK_ERR_SOLVER, "the tangent is singular - a rigid-body motion or a mechanism the step's "
                                   "constraints and tools leave free (a vanishing LU pivot)");
    }
  } else {
    ++P->counts[kQr];
    P->kind = SBK_FACTOR_QR;
  }
  return SBK_OK;
}

int sbk_partition_solve(sbk_partition* part, const double* b_dev, double* x_dev) {
  if (!part || !b_dev || !x_dev) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_solve: null argument");
  sbk_partition* P = part;
  if (P->kind == 0) return pfail(SBK_ERR_ARGUMENT, "the free-free block was solved before it was factorised");
  ++P->counts[kSolves];
  gather_kernel<<<grid_for(P->nf), kThreads, 0, P->stream>>>(b_dev, P->perm, P->nf, P->rhs);
  PCUDA(cudaGetLastError());
  if (P->kind == SBK_FACTOR_CHOLESKY) {
    if (int rc = chol_apply(P, P->rhs, P->sol)) return rc;
    double omega = INFINITY;
    if (int rc = backward_error(P, &omega)) return rc;
    if (!(omega <= kBackward)) {  // not positive definite after all
      if (int rc = fall_back(P, kCholesky, kCholeskyFellBack)) return rc;
    }
  } else if (P->kind == SBK_FACTOR_GMRES) {
    bool converged = false;
    if (int rc = gmres(P, &converged)) return rc;
    if (!converged) {  // the skew part is too large for the preconditioner
      if (int rc = fall_back(P, kGmres, kGmresFellBack)) return rc;
    }
  }
  if (P->kind == SBK_FACTOR_LU) {
    if (int rc = dense_solve(P)) return rc;
  } else if (P->kind == SBK_FACTOR_QR) {
    if (int rc = solve_qr(P)) return rc;
  }
  scatter_kernel<<<grid_for(P->nf), kThreads, 0, P->stream>>>(P->sol, P->perm, P->nf, 0.0, false, x_dev);
  PCUDA(cudaGetLastError());
  return SBK_OK;
}

int sbk_partition_solve_transpose(sbk_partition* part, const double* b_dev, double* x_dev) {
  if (!part || !b_dev || !x_dev) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_solve_transpose: null argument");
  sbk_partition* P = part;
  if (P->kind == 0) return pfail(SBK_ERR_ARGUMENT, "the free-free block was solved before it was factorised");
  if (P->kind == SBK_FACTOR_CHOLESKY) return sbk_partition_solve(part, b_dev, x_dev);  // symmetric
  if (P->kind != SBK_FACTOR_LU)
    return pfail(SBK_ERR_UNSUPPORTED, "the transposed solve takes a Cholesky or a dense LU factorisation");
  // K^T x = b with B = K(p, p): B^T (x(p)) = b(p), the permutations as solve's.
  ++P->counts[kSolves];
  gather_kernel<<<grid_for(P->nf), kThreads, 0, P->stream>>>(b_dev, P->perm, P->nf, P->rhs);
  PCUDA(cudaGetLastError());
  if (int rc = dense_solve(P, true)) return rc;
  scatter_kernel<<<grid_for(P->nf), kThreads, 0, P->stream>>>(P->sol, P->perm, P->nf, 0.0, false, x_dev);
  PCUDA(cudaGetLastError());
  return SBK_OK;
}

int sbk_partition_counts(const sbk_partition* part, int64_t counts[9]) {
  if (!part || !counts) return pfail(SBK_ERR_ARGUMENT, "sbk_partition_counts: null argument");
  for (int i = 0; i < kNumCounts; ++i) counts[i] = part->counts[i];
  return SBK_OK;
}

}  // extern "C"
