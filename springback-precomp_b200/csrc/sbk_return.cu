// The return kernel of the local iteration's phase kernels: the general
// (Hill48 / Chaboche) closest-point return of every point the first pass
// kernel listed as yielding, a thread per point, so that the 32 lanes of a
// warp all run the Newton iteration of a return.
//
// In its own translation unit so that the return's helpers - the residual
// evaluation, the consistent tangent, the backstress decay - are compiled
// inline here (SBK_RETURN_HELPER), while the other kernels keep them as
// calls: inline, their arguments stay in registers instead of a stack frame
// (measured on the 1M-element microbenchmark: 29.4 -> 22.1 ms per
// evaluation for this kernel; elsewhere the larger code cost more than it
// saved).
#define SBK_RETURN_HELPER __forceinline__

#include <cuda_runtime.h>

#include "sbk_element.h"
#include "sbk_material.cuh"
#include "sbk_wave.h"

// Minimum resident 128-thread blocks per SM, which bounds a thread's
// registers: at 4 (128 registers) the kernel's latency is hidden by 16
// warps per SM; 3 and 2 measured 4 % and 12 % slower.
#ifndef SBK_MINB_RETURN
#define SBK_MINB_RETURN 4
#endif

namespace sbk {
namespace {

__global__ void __launch_bounds__(128, SBK_MINB_RETURN) wave_return_kernel(const __grid_constant__ Params p, int64_t ne,
                                                          const int32_t* __restrict__ plastic,
                                                          const int32_t* __restrict__ plastic_count,
                                                          const double* __restrict__ state,
                                                          double* __restrict__ trial,
                                                          const __grid_constant__ WaveBuffers w) {
  const int64_t n = *plastic_count;
  const int nq = p.nq;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pt = plastic[i];
    const int64_t e = pt >> 3;
    const int q = (int)(pt & 7);
    double strain[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) strain[k] = *pw_at(w, e, kPwStrain + k, q);
    PointState st{state + e * nq + q, trial + e * nq + q, ne * nq};
    Response r;
    const int code = general_return(p, strain, st, r, w.warm + pt * 8);
    if (code) {
      w.pfail[pt] = (2 << 8) | q;
      w.pcodes[pt] = code;
    } else {
      store_response(w, e, q, r);
    }
  }
}

}  // namespace

void launch_wave_returns(const Params& p, int64_t ne, const int32_t* plastic, const int32_t* plastic_count,
                         const double* state, double* trial, const WaveBuffers& w, unsigned grid,
                         cudaStream_t stream) {
  wave_return_kernel<<<grid, 128, 0, stream>>>(p, ne, plastic, plastic_count, state, trial, w);
}

}  // namespace sbk
