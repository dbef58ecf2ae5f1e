// The element schedule: which element each slot of the next element launch
// evaluates.
//
// The element kernel runs four elements per warp (one 8-lane group each).
// Elements that take different paths - more local iterations, a line
// search, more plastic points - serialise inside the warp and fetch more
// distinct code, and the kernel is bound by that code fetch. Elements keep
// much of their behaviour from one Newton iteration to the next, so after
// each evaluation the elements are bucketed by what their last evaluation
// cost (local iterations, yielding points) and the next launch walks them
// bucket by bucket. The bucketing is a stable counting sort: within a
// bucket the elements keep their mesh order, so that a warp's elements stay
// neighbours where their costs agree (their nodes are then shared in cache),
// and the order is the same on every run. No result depends on the order:
// every output of the element kernel is indexed by the element, and the
// assembly sums in element order.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include "sbk_element.h"

namespace sbk {
namespace {

constexpr int kIterationBuckets = 32;             // local iterations 0..31 (the limit is 25)
constexpr int kYieldBuckets = SBK_MAX_POINTS + 1;  // yielding points 0..32
constexpr int kBuckets = kIterationBuckets * kYieldBuckets;
constexpr int kChunk = 1024;                       // elements per block, in mesh order

__device__ __forceinline__ int bucket_of(int64_t e, int nq, const int32_t* iterations, const uint8_t* yield) {
  int it = iterations[e];
  it = it < 0 ? 0 : (it >= kIterationBuckets ? kIterationBuckets - 1 : it);
  int y = 0;
  for (int q = 0; q < nq; ++q) y += yield[e * nq + q] != 0;
  return it * kYieldBuckets + y;
}

// Pass 1: the bucket counts of every chunk, bucket-major (count[k * nb + b]).
__global__ void __launch_bounds__(256) schedule_count_kernel(int64_t ne, int nq, int64_t nb,
                                                             const int32_t* __restrict__ iterations,
                                                             const uint8_t* __restrict__ yield,
                                                             int32_t* __restrict__ count, int16_t* __restrict__ keys) {
  __shared__ int32_t h[kBuckets];
  for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int64_t b = blockIdx.x;
  const int64_t lo = b * kChunk, hi = lo + kChunk < ne ? lo + kChunk : ne;
  for (int64_t e = lo + threadIdx.x; e < hi; e += blockDim.x) {
    const int k = bucket_of(e, nq, iterations, yield);
    keys[e] = (int16_t)k;
    atomicAdd(&h[k], 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) count[(int64_t)i * nb + b] = h[i];
}

// Pass 2: exclusive prefix sum of the counts in bucket-major order into the
// starts, by CUB's device-wide scan (its temporary storage after the keys).

// Pass 3: each chunk places its elements in mesh order at its buckets'
// offsets (one thread walks the chunk, so the order within a bucket is the
// mesh order).
__global__ void schedule_place_kernel(int64_t ne, int64_t nb, const int16_t* __restrict__ keys,
                                      const int32_t* __restrict__ start, int32_t* __restrict__ order) {
  if (threadIdx.x != 0) return;
  const int64_t b = blockIdx.x;
  const int64_t lo = b * kChunk, hi = lo + kChunk < ne ? lo + kChunk : ne;
  int32_t used[kBuckets];
  for (int i = 0; i < kBuckets; ++i) used[i] = 0;
  for (int64_t e = lo; e < hi; ++e) {
    const int k = keys[e];
    order[start[(int64_t)k * nb + b] + used[k]++] = (int32_t)e;
  }
}

}  // namespace

namespace {
// The counts (kBuckets per chunk), their scan (the starts), the int16 keys,
// then the scan's temporary storage at a 256-byte boundary: offsets in ints.
int64_t counts_of(int64_t ne) {
  const int64_t nb = (ne + kChunk - 1) / kChunk;
  return (int64_t)kBuckets * (nb > 0 ? nb : 1);
}
int64_t temp_offset(int64_t ne) {
  const int64_t ints = 2 * counts_of(ne) + (ne + 1) / 2;
  return (ints + 63) / 64 * 64;
}
size_t scan_temp_bytes(int64_t n) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int32_t*)nullptr, (int32_t*)nullptr, (int)n);
  return bytes;
}
}  // namespace

size_t schedule_scratch_ints(int64_t ne) {
  return (size_t)temp_offset(ne) + (scan_temp_bytes(counts_of(ne)) + 3) / 4;
}

int launch_schedule(int64_t ne, int nq, const int32_t* iterations, const uint8_t* yield, int32_t* scratch,
                    int32_t* order, cudaStream_t stream) {
  if (ne <= 0) return 0;
  const int64_t nb = (ne + kChunk - 1) / kChunk;
  const int64_t n = (int64_t)kBuckets * nb;
  int32_t* starts = scratch + n;
  int16_t* keys = reinterpret_cast<int16_t*>(scratch + 2 * n);
  schedule_count_kernel<<<(unsigned)nb, 256, 0, stream>>>(ne, nq, nb, iterations, yield, scratch, keys);
  size_t bytes = scan_temp_bytes(n);
  cudaError_t err = cub::DeviceScan::ExclusiveSum(scratch + temp_offset(ne), bytes, scratch, starts, (int)n, stream);
  if (err != cudaSuccess) return (int)err;
  schedule_place_kernel<<<(unsigned)nb, 32, 0, stream>>>(ne, nb, keys, starts, order);
  return (int)cudaGetLastError();
}

}  // namespace sbk
