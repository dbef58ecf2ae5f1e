// The node-block CSC pattern of a Hex8 mesh and the assembly's gather maps,
// built on the device (sbk_pattern.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sbk {

// Device arrays (cudaMalloc'd; free_pattern releases them).
struct DevicePattern {
  int32_t* outer = nullptr;        // 3 nn + 1 CSC column pointers
  int32_t* inner = nullptr;        // nnz row indices
  int32_t* block_col = nullptr;    // num_blocks: the column node of each block, CSC order
  int64_t* block_value = nullptr;  // num_blocks: value index of (3A, 3B)
  int32_t* block_ptr = nullptr;    // num_blocks + 1: contributions of each block
  int32_t* block_src = nullptr;    // 64 ne: e * 64 + a * 8 + b, ascending per block
  int32_t* node_ptr = nullptr;     // nn + 1
  int32_t* node_src = nullptr;     // 8 ne: e * 8 + a, ascending per node
  int64_t nnz = 0;
  int64_t num_blocks = 0;
};

// Builds the pattern of ne elements over nn nodes from the device
// connectivity `conn` (8 per element) on stream `s` and waits for it. A node
// out of range is SBK_ERR_MESH; a pattern beyond int32 indices
// SBK_ERR_UNSUPPORTED.
int build_device_pattern(int64_t nn, int64_t ne, const int32_t* conn, DevicePattern& out, cudaStream_t s);
void free_pattern(DevicePattern& p);

}  // namespace sbk
