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
// bucket by bucket. No result depends on the order: every output of the
// element kernel is indexed by the element, and the assembly sums in
// element order. Within a bucket the order is that of the atomic
// reservations, which may vary from run to run; the results do not.
#include <cuda_runtime.h>

#include "sbk_element.h"

namespace sbk {
namespace {

constexpr int kIterationBuckets = 32;             // local iterations 0..31 (the limit is 25)
constexpr int kYieldBuckets = SBK_MAX_POINTS + 1;  // yielding points 0..32
constexpr int kBuckets = kIterationBuckets * kYieldBuckets;

__device__ __forceinline__ int bucket_of(int64_t e, int nq, const int32_t* iterations, const uint8_t* yield) {
  int it = iterations[e];
  it = it < 0 ? 0 : (it >= kIterationBuckets ? kIterationBuckets - 1 : it);
  int y = 0;
  for (int q = 0; q < nq; ++q) y += yield[e * nq + q] != 0;
  return it * kYieldBuckets + y;
}

__global__ void __launch_bounds__(256) schedule_count_kernel(int64_t ne, int nq, const int32_t* __restrict__ iterations,
                                                             const uint8_t* __restrict__ yield,
                                                             int32_t* __restrict__ count) {
  __shared__ int32_t h[kBuckets];
  for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) h[i] = 0;
  __syncthreads();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&h[bucket_of(e, nq, iterations, yield)], 1);
  __syncthreads();
  for (int i = threadIdx.x; i < kBuckets; i += blockDim.x)
    if (h[i]) atomicAdd(&count[i], h[i]);
}

// Exclusive prefix sum of the bucket counts into the bucket cursors.
__global__ void schedule_scan_kernel(const int32_t* __restrict__ count, int32_t* __restrict__ cursor) {
  if (threadIdx.x != 0) return;
  int32_t run = 0;
  for (int i = 0; i < kBuckets; ++i) {
    cursor[i] = run;
    run += count[i];
  }
}

__global__ void __launch_bounds__(256) schedule_place_kernel(int64_t ne, int nq, const int32_t* __restrict__ iterations,
                                                             const uint8_t* __restrict__ yield,
                                                             int32_t* __restrict__ cursor, int32_t* __restrict__ order) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ne; e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t pos = atomicAdd(&cursor[bucket_of(e, nq, iterations, yield)], 1);
    order[pos] = (int32_t)e;
  }
}

}  // namespace

size_t schedule_scratch_ints() { return 2 * kBuckets; }

int launch_schedule(int64_t ne, int nq, const int32_t* iterations, const uint8_t* yield, int32_t* scratch,
                    int32_t* order, cudaStream_t stream) {
  if (ne <= 0) return 0;
  int32_t* count = scratch;
  int32_t* cursor = scratch + kBuckets;
  cudaError_t err = cudaMemsetAsync(count, 0, kBuckets * sizeof(int32_t), stream);
  if (err != cudaSuccess) return (int)err;
  int64_t blocks = (ne + 255) / 256;
  if (blocks > 148 * 4) blocks = 148 * 4;
  schedule_count_kernel<<<(unsigned)blocks, 256, 0, stream>>>(ne, nq, iterations, yield, count);
  schedule_scan_kernel<<<1, 32, 0, stream>>>(count, cursor);
  schedule_place_kernel<<<(unsigned)blocks, 256, 0, stream>>>(ne, nq, iterations, yield, cursor, order);
  return (int)cudaGetLastError();
}

}  // namespace sbk
