// The node-block sparsity pattern of a Hex8 mesh and the assembly's gather
// maps, built on the device from the device connectivity.
//
// What it must produce is the reference's pattern (Assembler::build_pattern,
// src/fem/Assembler.cpp:86-173): one 3 x 3 block per pair of nodes that share
// an element, stored column-major (CSC) by DOF, column 3B + kb listing the
// rows 3A + ka of its column node B's neighbours A in ascending order. The
// construction here is a sort, not a neighbourhood walk:
//
//   1. every element emits its 64 (column node, row node) pairs as one 64-bit
//      key col * nn + row, with the source e * 64 + a * 8 + b as its value;
//   2. a stable radix sort by key puts each node block's contributions side
//      by side, in ascending element order (the order in which the
//      reference's scatter adds them), and the blocks themselves in CSC
//      order (by column node, then row node);
//   3. the first position of every run of equal keys is a block: a scan of
//      the run heads numbers the blocks, and their positions are the gather
//      map's block pointers;
//   4. per column node, the number of its blocks (its degree) and, by a scan,
//      the first block of its column give every CSC offset directly: column
//      3B + kb starts at 9 first[B] + 3 kb deg[B], and block j of column B
//      holds rows 3A .. 3A + 2 at 3 j within each of its three columns.
//
// The node incidences (node -> e * 8 + a, ascending) of the force gather
// come from a second stable sort of the connectivity by node. Everything runs
// on one stream; the host reads back only the connectivity check and the
// block count. CUB's radix sort and scans do the sorting and scanning.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <string>

#include "sbk.h"
#include "sbk_element.h"
#include "sbk_pattern.h"

namespace sbk {
namespace {

constexpr int kThreads = 256;

unsigned grid_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  if (b > (int64_t)148 * 64) b = (int64_t)148 * 64;  // grid-stride beyond 64 blocks per SM
  return (unsigned)(b > 0 ? b : 1);
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b) != 0) ++b;
  return b > 0 ? b : 1;
}

__global__ void check_nodes_kernel(int64_t count, const int32_t* __restrict__ conn, int64_t nn, int32_t* bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t n = conn[i];
    if (n < 0 || n >= nn) atomicOr(bad, 1);
  }
}

__global__ void iota_kernel(int64_t count, int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)i;
}

__global__ void count_kernel(int64_t count, const int32_t* __restrict__ idx, int32_t* __restrict__ counts) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&counts[idx[i]], 1);
}

// Pair k = e * 64 + a * 8 + b of element e: key (node b) * nn + node a.
__global__ void pair_keys_kernel(int64_t ne, int64_t nn, const int32_t* __restrict__ conn, uint64_t* __restrict__ keys,
                                 int32_t* __restrict__ src) {
  const int64_t count = ne * 64;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = k >> 6;
    const int a = (int)((k >> 3) & 7), b = (int)(k & 7);
    keys[k] = (uint64_t)conn[e * 8 + b] * (uint64_t)nn + (uint64_t)conn[e * 8 + a];
    src[k] = (int32_t)k;
  }
}

__global__ void run_heads_kernel(int64_t count, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// At every run head i (block number id[i] - 1): the block's first
// contribution and its key; the column node's degree counted.
__global__ void blocks_kernel(int64_t count, int64_t nn, const uint64_t* __restrict__ keys,
                              const int32_t* __restrict__ head, const int32_t* __restrict__ id,
                              int32_t* __restrict__ block_ptr, uint64_t* __restrict__ block_key,
                              int32_t* __restrict__ degree) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    const int32_t blk = id[i] - 1;
    block_ptr[blk] = (int32_t)i;
    block_key[blk] = keys[i];
    atomicAdd(&degree[keys[i] / (uint64_t)nn], 1);
  }
}

// outer[3B + kb] = 9 first[B] + 3 kb deg[B]; outer[3 nn] = 9 nb.
__global__ void outer_kernel(int64_t nn, const int32_t* __restrict__ first, int32_t* __restrict__ outer) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= 3 * nn; c += (int64_t)gridDim.x * blockDim.x) {
    if (c == 3 * nn) {
      outer[c] = 9 * first[nn];
      continue;
    }
    const int64_t B = c / 3;
    const int kb = (int)(c % 3);
    outer[c] = 9 * first[B] + 3 * kb * (first[B + 1] - first[B]);
  }
}

// Block blk (column node B, row node A, j-th of its column): its column
// node, its first value (3A, 3B) and the nine row indices of its three
// columns.
__global__ void inner_kernel(int64_t nb, int64_t nn, const uint64_t* __restrict__ block_key,
                             const int32_t* __restrict__ first, int32_t* __restrict__ inner,
                             int32_t* __restrict__ block_col, int64_t* __restrict__ block_value) {
  for (int64_t blk = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; blk < nb; blk += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = block_key[blk];
    const int64_t B = (int64_t)(key / (uint64_t)nn);
    const int32_t A = (int32_t)(key % (uint64_t)nn);
    const int64_t f = first[B];
    const int64_t deg = first[B + 1] - f;
    const int64_t j = blk - f;
    block_col[blk] = (int32_t)B;
    block_value[blk] = 9 * f + 3 * j;
#pragma unroll
    for (int kb = 0; kb < 3; ++kb)
#pragma unroll
      for (int ka = 0; ka < 3; ++ka) inner[9 * f + 3 * kb * deg + 3 * j + ka] = 3 * A + ka;
  }
}

template <class T>
int dmalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
  if (e != cudaSuccess) return set_error(SBK_ERR_CUDA, std::string("cudaMalloc (pattern): ") + cudaGetErrorString(e));
  return SBK_OK;
}

struct Temp {
  void* ptrs[24] = {};
  int n = 0;
  template <class T>
  int get(T** p, size_t count) {
    if (n == 24) return set_error(SBK_ERR_CUDA, "pattern build: too many temporaries");
    int rc = dmalloc(p, count);
    if (!rc) ptrs[n++] = *p;
    return rc;
  }
  ~Temp() {
    for (int i = 0; i < n; ++i) cudaFree(ptrs[i]);
  }
};

#define PAT_CUDA(call)                                                                            \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return set_error(SBK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define PAT_TRY(x)      \
  do {                  \
    int rc_ = (x);      \
    if (rc_) return rc_; \
  } while (0)

// Exclusive sum of n + 1 counts (the last one zero) into out (n + 1).
int exclusive_sum(const int32_t* counts, int32_t* out, int64_t n, Temp& tmp, cudaStream_t s) {
  size_t bytes = 0;
  PAT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, counts, out, (int)(n + 1), s));
  void* t = nullptr;
  PAT_TRY(tmp.get(reinterpret_cast<char**>(&t), bytes));
  PAT_CUDA(cub::DeviceScan::ExclusiveSum(t, bytes, counts, out, (int)(n + 1), s));
  return SBK_OK;
}

}  // namespace

void free_pattern(DevicePattern& p) {
  void* ptrs[] = {p.outer, p.inner, p.block_col, p.block_value, p.block_ptr, p.block_src, p.node_ptr, p.node_src};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  p = DevicePattern{};
}

int build_device_pattern(int64_t nn, int64_t ne, const int32_t* conn, DevicePattern& out, cudaStream_t s) {
  out = DevicePattern{};
  if (nn <= 0 || ne <= 0) return set_error(SBK_ERR_ARGUMENT, "an empty mesh");
  if (ne * 64 > 0x7fffffffLL) return set_error(SBK_ERR_UNSUPPORTED, "too many element blocks for int32 maps");
  if (3 * nn + 1 > 0x7fffffffLL) return set_error(SBK_ERR_UNSUPPORTED, "too many nodes for int32 indices");
  Temp tmp;
  // 0. Every node index inside the mesh.
  int32_t* bad = nullptr;
  PAT_TRY(tmp.get(&bad, 1));
  PAT_CUDA(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  check_nodes_kernel<<<grid_for(ne * 8), kThreads, 0, s>>>(ne * 8, conn, nn, bad);
  PAT_CUDA(cudaGetLastError());
  int32_t bad_h = 0;
  PAT_CUDA(cudaMemcpyAsync(&bad_h, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PAT_CUDA(cudaStreamSynchronize(s));
  if (bad_h) return set_error(SBK_ERR_MESH, "connectivity names a node out of range");

  DevicePattern p;
  int rc = SBK_OK;
  auto fail_free = [&](int code) {
    free_pattern(p);
    return code;
  };
#define PAT_OWN(x)              \
  do {                          \
    rc = (x);                   \
    if (rc) return fail_free(rc); \
  } while (0)
#define PAT_OWN_CUDA(call)                                                                             \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return fail_free(set_error(SBK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)));   \
  } while (0)

  // 1. Node incidences: the connectivity sorted by node, stably.
  const int64_t ni = ne * 8;
  int32_t *inc_key = nullptr, *inc_idx = nullptr, *sorted_key = nullptr, *counts = nullptr;
  PAT_OWN(tmp.get(&inc_idx, ni));
  PAT_OWN(tmp.get(&sorted_key, ni));
  PAT_OWN(tmp.get(&counts, nn + 1));
  PAT_OWN(dmalloc(&p.node_src, ni));
  PAT_OWN(dmalloc(&p.node_ptr, nn + 1));
  inc_key = const_cast<int32_t*>(conn);
  iota_kernel<<<grid_for(ni), kThreads, 0, s>>>(ni, inc_idx);
  const int node_bits = bits_for((uint64_t)nn);
  {
    size_t bytes = 0;
    PAT_OWN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, inc_key, sorted_key, inc_idx, p.node_src, (int)ni, 0,
                                                 node_bits, s));
    void* t = nullptr;
    PAT_OWN(tmp.get(reinterpret_cast<char**>(&t), bytes));
    PAT_OWN_CUDA(cub::DeviceRadixSort::SortPairs(t, bytes, inc_key, sorted_key, inc_idx, p.node_src, (int)ni, 0,
                                                 node_bits, s));
  }
  PAT_OWN_CUDA(cudaMemsetAsync(counts, 0, (nn + 1) * sizeof(int32_t), s));
  count_kernel<<<grid_for(ni), kThreads, 0, s>>>(ni, conn, counts);
  PAT_OWN(exclusive_sum(counts, p.node_ptr, nn, tmp, s));

  // 2. The 64 node pairs of every element, sorted by (column, row) node.
  const int64_t np = ne * 64;
  uint64_t *keys = nullptr, *keys_alt = nullptr;
  int32_t* src_alt = nullptr;
  PAT_OWN(tmp.get(&keys, np));
  PAT_OWN(tmp.get(&keys_alt, np));
  PAT_OWN(tmp.get(&src_alt, np));
  PAT_OWN(dmalloc(&p.block_src, np));
  pair_keys_kernel<<<grid_for(np), kThreads, 0, s>>>(ne, nn, conn, keys, src_alt);
  PAT_OWN_CUDA(cudaGetLastError());
  const int key_bits = bits_for((uint64_t)nn * (uint64_t)nn - 1);
  {
    size_t bytes = 0;
    PAT_OWN_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, keys_alt, src_alt, p.block_src, (int)np, 0,
                                                 key_bits, s));
    void* t = nullptr;
    PAT_OWN(tmp.get(reinterpret_cast<char**>(&t), bytes));
    PAT_OWN_CUDA(cub::DeviceRadixSort::SortPairs(t, bytes, keys, keys_alt, src_alt, p.block_src, (int)np, 0, key_bits,
                                                 s));
  }
  const uint64_t* sorted = keys_alt;

  // 3. Run heads numbered: the blocks.
  // The unsorted keys are no longer needed: their 2 np int32 hold the run
  // heads and their numbers.
  int32_t* head = reinterpret_cast<int32_t*>(keys);
  int32_t* id = head + np;
  run_heads_kernel<<<grid_for(np), kThreads, 0, s>>>(np, sorted, head);
  {
    size_t bytes = 0;
    PAT_OWN_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, head, id, (int)np, s));
    void* t = nullptr;
    PAT_OWN(tmp.get(reinterpret_cast<char**>(&t), bytes));
    PAT_OWN_CUDA(cub::DeviceScan::InclusiveSum(t, bytes, head, id, (int)np, s));
  }
  int32_t nb32 = 0;
  PAT_OWN_CUDA(cudaMemcpyAsync(&nb32, id + np - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  PAT_OWN_CUDA(cudaStreamSynchronize(s));
  const int64_t nb = nb32;
  if (9 * nb > 0x7fffffffLL)
    return fail_free(set_error(SBK_ERR_UNSUPPORTED, "the pattern exceeds 2^31 entries (int32 indices)"));
  uint64_t* block_key = nullptr;
  int32_t* degree = counts;  // nn + 1 counts again
  PAT_OWN(tmp.get(&block_key, nb));
  PAT_OWN(dmalloc(&p.block_ptr, nb + 1));
  PAT_OWN_CUDA(cudaMemsetAsync(degree, 0, (nn + 1) * sizeof(int32_t), s));
  blocks_kernel<<<grid_for(np), kThreads, 0, s>>>(np, nn, sorted, head, id, p.block_ptr, block_key, degree);
  const int32_t total = (int32_t)np;
  PAT_OWN_CUDA(cudaMemcpyAsync(p.block_ptr + nb, &total, sizeof(int32_t), cudaMemcpyHostToDevice, s));

  // 4. Column starts, then the CSC arrays and the block maps.
  int32_t* first = nullptr;
  PAT_OWN(tmp.get(&first, nn + 1));
  PAT_OWN(exclusive_sum(degree, first, nn, tmp, s));
  PAT_OWN(dmalloc(&p.outer, 3 * nn + 1));
  PAT_OWN(dmalloc(&p.inner, 9 * nb));
  PAT_OWN(dmalloc(&p.block_col, nb));
  PAT_OWN(dmalloc(&p.block_value, nb));
  outer_kernel<<<grid_for(3 * nn + 1), kThreads, 0, s>>>(nn, first, p.outer);
  inner_kernel<<<grid_for(nb), kThreads, 0, s>>>(nb, nn, block_key, first, p.inner, p.block_col, p.block_value);
  PAT_OWN_CUDA(cudaGetLastError());
  // The temporaries are freed when `tmp` goes: finish the work first.
  PAT_OWN_CUDA(cudaStreamSynchronize(s));
  p.nnz = 9 * nb;
  p.num_blocks = nb;
  out = p;
  return SBK_OK;
#undef PAT_OWN
#undef PAT_OWN_CUDA
}

}  // namespace sbk
