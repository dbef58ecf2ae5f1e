// sbk_evaluate_noalloc: the element loop of a small mesh for callers that
// cannot allocate device memory - a solver that runs on a fixed device
// arena handed to it by its host application, or code that must not call
// cudaMalloc while it works (a hard real-time loop, a stream being
// captured). The caller passes every input and output; the element
// tangents and forces between the element kernel and the assembly live in
// one file-scope device array of fixed size, which every GPU that loads this
// library holds until the process exits.
//
// Limits: SBK_NOALLOC_MAX_ELEMENTS elements and SBK_NOALLOC_MAX_NODES nodes
// per call; larger meshes are refused (use sbk_system_create).
//
// The array's address is looked up once per device (cudaGetSymbolAddress
// with that device current) by the first call made on it, which should
// therefore come before any stream capture. Calls share the array: two calls
// that overlap on the GPU (on different streams) race; calls on one stream
// are ordered. Each call clears what it accumulates before using it, and
// reads an element's slots only when the element kernel of the same call
// reported it evaluated (code 0).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "sbk.h"
#include "sbk_element.h"
#include "sbk_params.h"

namespace {

constexpr int kMaxElements = SBK_NOALLOC_MAX_ELEMENTS;
constexpr int kMaxNodes = SBK_NOALLOC_MAX_NODES;
constexpr int kMaxDevices = 64;

struct Scratch {
  double tangent[kMaxElements * 576];
  double force[kMaxElements * 24];
  double energy[kMaxElements];
  double gross[3 * kMaxNodes];
  int32_t iterations[kMaxElements];
  int32_t code[kMaxElements];
  int32_t first_failure;
};

static __device__ __align__(256) Scratch g_scratch;

std::mutex g_mutex;
Scratch* g_address[kMaxDevices] = {};

// The device address of the scratch on the current device.
int scratch_address(Scratch** out) {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return sbk::set_error(SBK_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
  if (dev < 0 || dev >= kMaxDevices) return sbk::set_error(SBK_ERR_UNSUPPORTED, "device index beyond 64");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_address[dev]) {
    void* p = nullptr;
    err = cudaGetSymbolAddress(&p, g_scratch);
    if (err != cudaSuccess || !p)
      return sbk::set_error(SBK_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
    g_address[dev] = static_cast<Scratch*>(p);
  }
  *out = g_address[dev];
  return SBK_OK;
}

// Position of (row, col) in the CSC pattern, or -1 if the pattern lacks it.
__device__ __forceinline__ int32_t csc_position(const int32_t* __restrict__ outer, const int32_t* __restrict__ inner,
                                                int32_t row, int32_t col) {
  int32_t lo = outer[col], hi = outer[col + 1];
  const int32_t end = hi;
  while (lo < hi) {
    const int32_t mid = lo + (hi - lo) / 2;
    if (inner[mid] < row) lo = mid + 1; else hi = mid;
  }
  return (lo < end && inner[lo] == row) ? lo : -1;
}

// One block: the element tangents and forces added into the CSC values,
// f_int and the gross sums element by element in element order (the
// reference's Assembler::scatter order, src/fem/Assembler.cpp:184-215), then
// the energy (in element order), the yield count and the gross norm. The
// element kernel writes code[e] for every element (0: evaluated); a failed
// element wrote none of its force, tangent, energy or yield flags, so its
// slots hold an earlier call's values, and it is left out of every sum. An
// element naming one node twice sends two of its blocks to one CSC entry:
// such an element is added by one thread, entry after entry in row-major
// block order, so no addition is lost.
__global__ void __launch_bounds__(576) scatter_small_kernel(
    int32_t nn, int32_t ne, int nq, const int32_t* __restrict__ conn, const int32_t* __restrict__ outer,
    const int32_t* __restrict__ inner, int64_t nnz, const Scratch* __restrict__ s, double* __restrict__ gross,
    double* __restrict__ internal, double* __restrict__ values, const uint8_t* __restrict__ yield,
    double* __restrict__ summary) {
  __shared__ double red[576];
  const int t = threadIdx.x;
  for (int64_t i = t; i < nnz && values; i += blockDim.x) values[i] = 0.0;
  for (int i = t; i < 3 * nn; i += blockDim.x) {
    internal[i] = 0.0;
    gross[i] = 0.0;
  }
  __syncthreads();
  const int r = t / 24, c = t % 24;
  const int a = r / 3, ka = r % 3, b = c / 3, kb = c % 3;
  __shared__ int mismatch;
  if (t == 0) mismatch = 0;
  __syncthreads();
  for (int e = 0; e < ne; ++e) {
    const int32_t* nodes = conn + 8 * (int64_t)e;
    // A failed element (a node out of range among the reasons) is left out;
    // a block the caller's pattern lacks is reported. Both tests give the
    // same answer in every thread.
    if (s->code[e] != 0) continue;
    bool repeated = false;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = i + 1; j < 8; ++j) repeated = repeated || nodes[i] == nodes[j];
    if (!repeated) {
      if (values) {
        const int32_t pos = csc_position(outer, inner, 3 * nodes[a] + ka, 3 * nodes[b] + kb);
        if (pos >= 0)
          values[pos] += s->tangent[(int64_t)e * 576 + (8 * a + b) * 9 + 3 * ka + kb];
        else
          mismatch = 1;
      }
      if (t < 24) {
        const int32_t dof = 3 * nodes[t / 3] + t % 3;
        const double f = s->force[(int64_t)e * 24 + t];
        internal[dof] += f;
        gross[dof] += fabs(f);
      }
    } else if (t == 0) {
      for (int i = 0; i < 576 && values; ++i) {
        const int ra = i / 24, cb = i % 24;
        const int aa = ra / 3, kka = ra % 3, bb = cb / 3, kkb = cb % 3;
        const int32_t pos = csc_position(outer, inner, 3 * nodes[aa] + kka, 3 * nodes[bb] + kkb);
        if (pos >= 0)
          values[pos] += s->tangent[(int64_t)e * 576 + (8 * aa + bb) * 9 + 3 * kka + kkb];
        else
          mismatch = 1;
      }
      for (int i = 0; i < 24; ++i) {
        const int32_t dof = 3 * nodes[i / 3] + i % 3;
        const double f = s->force[(int64_t)e * 24 + i];
        internal[dof] += f;
        gross[dof] += fabs(f);
      }
    }
    __syncthreads();
  }
  double g2 = 0.0;
  for (int i = t; i < 3 * nn; i += blockDim.x) g2 += gross[i] * gross[i];
  red[t] = g2;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (t < w && t + w < 576) red[t] += red[t + w];
    __syncthreads();
  }
  if (t == 0) {
    double en = 0.0;
    int64_t y = 0;
    for (int e = 0; e < ne; ++e) {
      if (s->code[e] != 0) continue;
      en += s->energy[e];
      for (int q = 0; q < nq; ++q) y += yield[(int64_t)e * nq + q];
    }
    const int32_t first = s->first_failure;
    summary[0] = en;
    summary[1] = sqrt(red[0]);
    summary[2] = (double)y;
    summary[3] = first == 0x7f7f7f7f ? -1.0 : (double)first;
    summary[4] = first == 0x7f7f7f7f ? 0.0 : (double)s->code[first];
    if (mismatch && first == 0x7f7f7f7f) {  // the pattern does not cover the mesh
      summary[3] = -2.0;
      summary[4] = (double)SBK_EL_BAD_NODE;
    }
  }
}

}  // namespace

extern "C" int sbk_evaluate_noalloc(const sbk_material* material, const sbk_rule* rule, int kinematics,
                                    int32_t num_nodes, int32_t num_elements, const double* coords_dev,
                                    const int32_t* connectivity_dev, const double* u_dev, const double* state_dev,
                                    const double* alpha_dev, const int32_t* outer_dev, const int32_t* inner_dev,
                                    int64_t nnz, double* internal_dev, double* values_dev, double* trial_dev,
                                    double* alpha_out_dev, uint8_t* yield_dev, double* summary_dev,
                                    void* stream) {
  if (num_elements < 1 || num_nodes < 1) return sbk::set_error(SBK_ERR_ARGUMENT, "an empty mesh");
  if (num_elements > kMaxElements || num_nodes > kMaxNodes)
    return sbk::set_error(SBK_ERR_UNSUPPORTED, "sbk_evaluate_noalloc takes at most " + std::to_string(kMaxElements) +
                                                   " elements and " + std::to_string(kMaxNodes) +
                                                   " nodes; use sbk_system_create for larger meshes");
  if (!coords_dev || !connectivity_dev || !u_dev || !state_dev || !internal_dev || !trial_dev || !alpha_out_dev ||
      !yield_dev || !summary_dev || (values_dev && (!outer_dev || !inner_dev)))
    return sbk::set_error(SBK_ERR_ARGUMENT, "null device buffer");
  sbk::Params p;
  int rc = sbk::make_launch_params(material, rule, kinematics, p);
  if (rc) return rc;
  p.num_nodes = num_nodes;  // the element kernel checks the caller's connectivity against it
  Scratch* s = nullptr;
  rc = scratch_address(&s);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t err = cudaMemsetAsync(&s->first_failure, 0x7f, sizeof(int32_t), st);
  if (err != cudaSuccess) return sbk::set_error(SBK_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(err));
  rc = sbk::launch_elements(p, num_elements, coords_dev, connectivity_dev, u_dev, state_dev, alpha_dev,
                            values_dev != nullptr, s->force, s->tangent, s->energy, trial_dev, alpha_out_dev,
                            yield_dev, s->iterations, s->code, &s->first_failure, false, 0, nullptr, st);
  if (rc) return sbk::set_error(SBK_ERR_CUDA, std::string("element kernel: ") + cudaGetErrorString((cudaError_t)rc));
  scatter_small_kernel<<<1, 576, 0, st>>>(num_nodes, num_elements, p.nq, connectivity_dev, outer_dev, inner_dev, nnz,
                                          s, s->gross, internal_dev, values_dev, yield_dev, summary_dev);
  err = cudaGetLastError();
  if (err != cudaSuccess) return sbk::set_error(SBK_ERR_CUDA, std::string("scatter: ") + cudaGetErrorString(err));
  return SBK_OK;
}
