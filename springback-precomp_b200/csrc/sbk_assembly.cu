// K2: assembly of the element forces and tangents into the node-block
// pattern, by gather.
//
// The reference scatters every element's 24 x 24 tangent into the CSC value
// array in element order (src/fem/Assembler.cpp:184-215) and gathers f_int,
// the gross sums, the energy and the yield count serially
// (src/fem/NonlinearSystem.hpp:240-266). Here every value entry (and every
// DOF of f_int) is owned by one thread, which sums its contributions in
// ascending element order from 0.0 - the reference's own order, so the
// assembled values equal its bit for bit given the same element matrices,
// with no atomics and the same result on every run. Scalar norms and sums
// use a fixed two-stage tree.
#include <cuda_runtime.h>

#include "sbk_element.h"

namespace sbk {
namespace {

constexpr int kReduceBlocks = 296;  // 2 x 148 SMs; fixed for a fixed tree
constexpr int kReduceThreads = 256;

// One thread per node block (A, B): 9 values from the element blocks that
// couple A and B, in ascending element order.
__global__ void __launch_bounds__(256) assemble_values_kernel(int64_t num_blocks, const int32_t* __restrict__ block_col,
                                                              const int64_t* __restrict__ block_value,
                                                              const int32_t* __restrict__ block_ptr,
                                                              const int32_t* __restrict__ block_src,
                                                              const int32_t* __restrict__ outer,
                                                              const double* __restrict__ tangent,
                                                              double* __restrict__ values) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < num_blocks;
       b += (int64_t)gridDim.x * blockDim.x) {
    double acc[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) acc[i] = 0.0;
    const int32_t end = block_ptr[b + 1];
    for (int32_t k = block_ptr[b]; k < end; ++k) {
      const double* src = tangent + (int64_t)block_src[k] * 9;
#pragma unroll
      for (int i = 0; i < 9; ++i) acc[i] += src[i];
    }
    const int32_t B = block_col[b];
    const int64_t stride = (int64_t)outer[3 * B + 1] - outer[3 * B];
    const int64_t base = block_value[b];
    // acc[3 ka + kb] is entry (3A + ka, 3B + kb): column 3B + kb, row offset ka.
#pragma unroll
    for (int kb = 0; kb < 3; ++kb)
#pragma unroll
      for (int ka = 0; ka < 3; ++ka) values[base + kb * stride + ka] = acc[3 * ka + kb];
  }
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double out = sh[0];
  __syncthreads();
  return out;
}

// f_int and |f| per DOF by node (ascending element order), and per-block
// partials of gross^2, the energy and the yield count.
__global__ void __launch_bounds__(kReduceThreads) assemble_forces_kernel(
    int64_t nn, int64_t ne, int nq, const int32_t* __restrict__ node_ptr, const int32_t* __restrict__ node_src,
    const double* __restrict__ force, const double* __restrict__ energy_e, const uint8_t* __restrict__ yield,
    double* __restrict__ internal, double* __restrict__ partial) {
  __shared__ double sh[kReduceThreads];
  double g2 = 0.0, en = 0.0, yc = 0.0;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < nn; n += (int64_t)gridDim.x * blockDim.x) {
    double f[3] = {0, 0, 0}, g[3] = {0, 0, 0};
    const int32_t end = node_ptr[n + 1];
    for (int32_t k = node_ptr[n]; k < end; ++k) {
      const int32_t src = node_src[k];  // e * 8 + a
      const double* fe = force + (int64_t)(src >> 3) * 24 + 3 * (src & 7);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        f[c] += fe[c];
        g[c] += fabs(fe[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      internal[3 * n + c] = f[c];
      g2 += g[c] * g[c];
    }
  }
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    en += energy_e[e];
    int y = 0;
    for (int q = 0; q < nq; ++q) y += yield[e * nq + q];
    yc += (double)y;
  }
  g2 = block_sum(g2, sh);
  en = block_sum(en, sh);
  yc = block_sum(yc, sh);
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x + 0] = en;
    partial[3 * blockIdx.x + 1] = g2;
    partial[3 * blockIdx.x + 2] = yc;
  }
}

__global__ void __launch_bounds__(kReduceThreads) finish_kernel(int nblocks, const double* __restrict__ partial,
                                                                double* __restrict__ scalars) {
  __shared__ double sh[kReduceThreads];
  double v[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x)
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] += partial[3 * i + c];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double s = block_sum(v[c], sh);
    if (threadIdx.x == 0) scalars[c] = s;
  }
}

__global__ void add_node_blocks_kernel(int64_t nn, const int32_t* __restrict__ outer, const int32_t* __restrict__ inner,
                                       double* __restrict__ values, int32_t n, const int32_t* __restrict__ nodes,
                                       const double* __restrict__ blocks, int32_t* missing) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t node = nodes[i];
  if (node < 0 || node >= nn) {  // out of range: nothing is read or written
    atomicExch(missing, 1);
    return;
  }
  for (int b = 0; b < 3; ++b) {
    const int32_t col = 3 * node + b;
    int32_t lo = outer[col], hi = outer[col + 1];
    for (int a = 0; a < 3; ++a) {
      const int32_t row = 3 * node + a;
      // lower_bound over the sorted rows of the column.
      int32_t l = lo, h = hi;
      while (l < h) {
        const int32_t mid = l + (h - l) / 2;
        if (inner[mid] < row) l = mid + 1; else h = mid;
      }
      if (l < hi && inner[l] == row) {
        values[l] += blocks[9 * i + 3 * a + b];
      } else {
        atomicExch(missing, 1);
      }
    }
  }
}

// stiffness_gross (src/fem/NonlinearSystem.hpp:55-67), first half: |K| |u|
// per row. The reference walks the CSC columns in ascending order and adds
// |K(r, c)| |u(c)| to every row r of the column; here one thread owns a row
// node A and visits its columns in the same ascending order (its neighbours
// B, then the three columns of B), so every row sum is the reference's, bit
// for bit. Column 3B's rows are sorted, so the entry (3A, 3B) is found by a
// binary search over them; columns whose displacement is zero are skipped,
// as there.
__global__ void __launch_bounds__(256) stiffness_rows_kernel(int64_t nn, const int32_t* __restrict__ outer,
                                                             const int32_t* __restrict__ inner,
                                                             const double* __restrict__ values,
                                                             const double* __restrict__ u,
                                                             double* __restrict__ product) {
  for (int64_t A = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; A < nn; A += (int64_t)gridDim.x * blockDim.x) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int32_t lo = outer[3 * A], count = (outer[3 * A + 1] - lo) / 3;
    for (int32_t k = 0; k < count; ++k) {
      const int32_t B = inner[lo + 3 * k] / 3;
      const int32_t c0 = outer[3 * B], c1 = outer[3 * B + 1];
      int32_t l = c0, h = c1;
      while (l < h) {
        const int32_t mid = l + (h - l) / 2;
        if (inner[mid] < 3 * A) l = mid + 1; else h = mid;
      }
      const int64_t stride = (int64_t)c1 - c0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double uc = fabs(u[3 * B + j]);
        if (uc == 0.0) continue;
#pragma unroll
        for (int i = 0; i < 3; ++i) acc[i] += fabs(values[l + j * stride + i]) * uc;
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) product[3 * A + i] = acc[i];
  }
}

// Second half: the sum of squares over the listed free DOFs, per block.
__global__ void __launch_bounds__(kReduceThreads) free_squares_kernel(int32_t n, const int32_t* __restrict__ free_dofs,
                                                                      int64_t ndofs,
                                                                      const double* __restrict__ product,
                                                                      double* __restrict__ partial, int32_t* bad) {
  __shared__ double sh[kReduceThreads];
  double s = 0.0;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int32_t d = free_dofs[i];
    if (d < 0 || d >= ndofs) {  // out of range: skipped and reported
      atomicExch(bad, 1);
      continue;
    }
    const double v = product[d];
    s += v * v;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x + 0] = s;
    partial[3 * blockIdx.x + 1] = 0.0;
    partial[3 * blockIdx.x + 2] = 0.0;
  }
}

// The summary of an evaluation for a caller that does not synchronise:
// energy, gross, yielding points, the lowest failing element (-1: none) and
// its code.
__global__ void summary_kernel(const double* __restrict__ scalars, const int32_t* __restrict__ first_failure,
                               const int32_t* __restrict__ code, double* __restrict__ summary) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  summary[0] = scalars[0];
  summary[1] = sqrt(scalars[1]);
  summary[2] = scalars[2];
  const int32_t first = *first_failure;
  const bool failed = first != 0x7f7f7f7f;
  summary[3] = failed ? (double)first : -1.0;
  summary[4] = failed ? (double)code[first] : 0.0;
}

}  // namespace

int launch_summary(const double* scalars, const int32_t* first_failure, const int32_t* code, double* summary,
                   cudaStream_t stream) {
  summary_kernel<<<1, 32, 0, stream>>>(scalars, first_failure, code, summary);
  return (int)cudaGetLastError();
}

int launch_stiffness_gross(int64_t nn, const int32_t* outer, const int32_t* inner, const double* values,
                           const double* u, int32_t num_free, const int32_t* free_dofs, double* product,
                           double* scratch, double* scalars, int32_t* bad, cudaStream_t stream) {
  int64_t blocks = (nn + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks > 0)
    stiffness_rows_kernel<<<(unsigned)blocks, 256, 0, stream>>>(nn, outer, inner, values, u, product);
  free_squares_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(num_free, free_dofs, 3 * nn, product, scratch,
                                                                     bad);
  finish_kernel<<<1, kReduceThreads, 0, stream>>>(kReduceBlocks, scratch, scalars);
  return (int)cudaGetLastError();
}

int launch_assemble_values(const GatherMaps& m, const double* tangent, double* values, cudaStream_t stream) {
  if (m.num_blocks == 0) return 0;
  const int threads = 256;
  int64_t blocks = (m.num_blocks + threads - 1) / threads;
  if (blocks > 148 * 64) blocks = 148 * 64;
  assemble_values_kernel<<<(unsigned)blocks, threads, 0, stream>>>(m.num_blocks, m.block_col, m.block_value,
                                                                     m.block_ptr, m.block_src, m.outer, tangent,
                                                                     values);
  return (int)cudaGetLastError();
}

int launch_assemble_forces(const GatherMaps& m, const double* force, const double* energy_e, const uint8_t* yield,
                           int nq, double* internal, double* scratch, double* scalars, cudaStream_t stream) {
  assemble_forces_kernel<<<kReduceBlocks, kReduceThreads, 0, stream>>>(
      m.num_nodes, m.num_elements, nq, m.node_ptr, m.node_src, force, energy_e, yield, internal, scratch);
  finish_kernel<<<1, kReduceThreads, 0, stream>>>(kReduceBlocks, scratch, scalars);
  return (int)cudaGetLastError();
}

int launch_add_node_blocks(int64_t nn, const int32_t* outer, const int32_t* inner, double* values, int32_t n,
                           const int32_t* nodes, const double* blocks, int32_t* missing, cudaStream_t stream) {
  if (n <= 0) return 0;
  add_node_blocks_kernel<<<(n + 127) / 128, 128, 0, stream>>>(nn, outer, inner, values, n, nodes, blocks, missing);
  return (int)cudaGetLastError();
}

size_t assemble_scratch_doubles() { return 3 * kReduceBlocks; }

}  // namespace sbk
