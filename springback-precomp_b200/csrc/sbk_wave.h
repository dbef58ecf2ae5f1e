// The point records the phase kernels of the local iteration hand each other
// (sbk_element.cu, sbk_return.cu): field f of point q of element e at
// (e * kPw + f) * 8 + q, so that the eight points of an element read a field
// as one 64-byte run.
#pragma once

#include "sbk_element.h"
#include "sbk_material.cuh"

namespace sbk {

constexpr int kPwF = 0;        // F 9
constexpr int kPwHmax = 9;     // the largest |H| entry
constexpr int kPwL = 10;       // LogKin: axes 9, mu 3, first 6
constexpr int kPwStrain = 28;  // the strain the return takes, 6
constexpr int kPwStress = 34;  // the response: stress 6
constexpr int kPwC = 40;       // C 36
constexpr int kPwEnergy = 76;
constexpr int kPwYield = 77;
constexpr int kPw = 78;

__device__ __forceinline__ double* pw_at(const WaveBuffers& w, int64_t e, int f, int q) {
  return w.pw + (e * kPw + f) * 8 + q;
}

__device__ __forceinline__ void store_response(const WaveBuffers& w, int64_t e, int q, const Response& r) {
#pragma unroll
  for (int i = 0; i < 6; ++i) *pw_at(w, e, kPwStress + i, q) = r.stress[i];
#pragma unroll
  for (int i = 0; i < 36; ++i) *pw_at(w, e, kPwC + i, q) = r.C[i];
  *pw_at(w, e, kPwEnergy, q) = r.energy;
  *pw_at(w, e, kPwYield, q) = r.yielding ? 1.0 : 0.0;
}

// The return kernel (sbk_return.cu): the general return of `plastic_count`
// listed points (e * 8 + q), their responses into the point records.
void launch_wave_returns(const Params& p, int64_t ne, const int32_t* plastic, const int32_t* plastic_count,
                         const double* state, double* trial, const WaveBuffers& w, unsigned grid,
                         cudaStream_t stream);

}  // namespace sbk
