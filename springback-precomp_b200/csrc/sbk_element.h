// Kernel launchers of the element loop (K1), the assembly (K2) and the
// contact (K3), called by the C ABI in sbk_capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "sbk_params.h"

namespace sbk {

// Records the message sbk_last_error returns; returns `code`.
int set_error(int code, const std::string& what);
// The launch parameters of a material, rule and kinematics (validated; no
// allocation).
int make_launch_params(const sbk_material* material, const sbk_rule* rule, int kinematics, Params& p);

// K1: ne elements (slot i evaluates element order[i]; order NULL: i). Mesh mode (batch = false): coords 3 per node, conn 8 per
// element, u 3 per node. Batch mode: coords and u hold 24 per element.
int launch_elements(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                    const double* state, const double* alpha_n, int want_tangent, double* force, double* tangent,
                    double* energy, double* trial, double* alpha_out, uint8_t* yield, int32_t* iterations,
                    int32_t* code, int32_t* first_failure, bool batch, int elements_per_block,
                    const int32_t* order, cudaStream_t stream);
size_t element_smem_bytes(int group);

// The local iteration of the incompatible-mode Hex8 (rules of up to 8
// points) as phase kernels over the whole mesh (sbk_element.cu): per-element
// records between the kernels. Field-major within an element where the
// lanes of a group read alike fields (field f of point q at (e * F + f) * 8
// + q).
struct WaveBuffers {
  double* alpha;    // ne x 9: the modes of the current iterate
  double* dir;      // ne x 9: Newton's direction of the pending trial
  double* res;      // ne: the residual norm of the current iterate
  int32_t* iters;   // ne: local Newton steps
  int32_t* pcode;   // ne: status of the last pass
  double* kc;       // ne x 88: K_aa of the last pass, then its LU factors
  double* r;        // ne x 33: f_u 24, r_a 9 of the last pass
  double* sf;       // ne x 19: scale 9, floor 9, energy
  int32_t* piv;     // ne x 18: the LU's row and column transpositions
  double* slot;     // ne x 54 x 8: the points' material blocks
  double* geo;      // ne x 12 x 8: J^-1, w det J, det0 / det per point
  double* jinv0;    // ne x 9
  double* hu;       // ne x 9 x 8: U G^T per point
  double* warm;     // ne x 8 x 8: the points' last closest points (8 per point, together)
  double* pw;       // ne x 78 x 8: the points' records between the pass kernels
  int32_t* pfail;   // ne x 8: (stage << 8) | point of a point's failure (1: the element's, before its points)
  int32_t* pcodes;  // ne x 8: its code
  int32_t* plastic; // ne x 8: points (e * 8 + q) listed for the return kernel
  int32_t* list[2]; // ne each: the elements of a round
  int32_t* done;    // ne: converged elements
  int32_t* fallback;  // ne: elements handed to the single kernel
  int32_t* counts;  // 2 rounds + 3: each round's count, done, fallback, each round's listed points
};
// Bytes of one allocation that wave_buffers_carve splits for ne elements.
size_t wave_buffer_bytes(int64_t ne);
void wave_buffers_carve(void* base, int64_t ne, WaveBuffers& w);
// Whether the phase kernels take this material, rule and element.
bool wave_applies(const Params& p);
// K1 by the phase kernels (mesh or batch mode, as launch_elements); no
// host synchronisation, so it can be captured in a CUDA graph.
int launch_elements_wave(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                         const double* state, const double* alpha_n, int want_tangent, double* force,
                         double* tangent, double* energy, double* trial, double* alpha_out, uint8_t* yield,
                         int32_t* iterations, int32_t* code, int32_t* first_failure, bool batch,
                         const int32_t* order, const WaveBuffers& w, int pass_elements_per_block,
                         cudaStream_t stream);
// The shape derivative: per element lambda . d f*/d X (24, node-major) into
// out, at u with the committed points (state) and modes (alpha_n) as the
// history and lambda a global DOF vector; the local iteration runs again to
// the modes' equilibrium (its trial state and yield flags into trial and
// yield). Mesh mode only.
int launch_vjp(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
               const double* state, const double* alpha_n, const double* lambda, double* trial, uint8_t* yield,
               int32_t* code, int32_t* first_failure, double* out, cudaStream_t stream);
// Stress recovery of ne mesh elements at u from the committed points and
// modes: 28 doubles per element into out (see stress_kernel); the returns
// write their (reproduced) states into scratch (the state layout).
int launch_stress(const Params& p, int64_t ne, const double* coords, const int32_t* conn, const double* u,
                  const double* state, const double* alpha_n, double* scratch, double* out, int32_t* code,
                  int32_t* first_failure, cudaStream_t stream);

// The gather maps of the assembly (built once on the host).
struct GatherMaps {
  int64_t num_nodes, num_elements, nnz, num_blocks;
  // Node blocks of the pattern in CSC order (column node B, its sorted
  // neighbours A): the block's first value index in column 3B (the rows of
  // the same block in columns 3B+1, 3B+2 follow at +col_stride[B]).
  const int32_t* block_col;     // num_blocks: column node B
  const int64_t* block_value;   // num_blocks: index of value (3A, 3B)
  const int32_t* block_ptr;     // num_blocks + 1: contributions of each block
  const int32_t* block_src;     // e * 64 + a * 8 + b, ascending e per block
  const int32_t* outer;         // CSC column pointers (3 nn + 1)
  // Node incidences (node -> e * 8 + a, ascending e) for f_int and gross.
  const int32_t* node_ptr;      // nn + 1
  const int32_t* node_src;      // 8 ne
};

// K2: values (nnz) from the element tangents, in element order per entry.
int launch_assemble_values(const GatherMaps& m, const double* tangent, double* values, cudaStream_t stream);
// K2: f_int and the per-DOF gross sums from the element forces; the partial
// sums of energy, gross^2 and the yield count into `scalars`
// (double[3]: energy, gross^2, yielding).
int launch_assemble_forces(const GatherMaps& m, const double* force, const double* energy_e,
                           const uint8_t* yield, int nq, double* internal, double* scratch, double* scalars,
                           cudaStream_t stream);
size_t assemble_scratch_doubles();
// Energy, gross, yielding points, lowest failing element (-1) and its code
// into summary (5 doubles, device), from the reductions' scalars.
int launch_summary(const double* scalars, const int32_t* first_failure, const int32_t* code, double* summary,
                   cudaStream_t stream);
// stiffness_gross: |K| |u| per row into `product` (3 nn), then the sum of
// squares of its listed free DOFs into scalars[0] (scratch as for the forces).
int launch_stiffness_gross(int64_t nn, const int32_t* outer, const int32_t* inner, const double* values,
                           const double* u, int32_t num_free, const int32_t* free_dofs, double* product,
                           double* scratch, double* scalars, int32_t* bad, cudaStream_t stream);
// The schedule of the next element launch: the elements bucketed by the
// cost of their last evaluation (local iterations, yielding points), so
// that elements of alike cost share a warp. scratch: schedule_scratch_ints().
int launch_schedule(int64_t ne, int nq, const int32_t* iterations, const uint8_t* yield, int32_t* scratch,
                    int32_t* order, cudaStream_t stream);
size_t schedule_scratch_ints(int64_t ne);
// add_node_block for n blocks, in list order.
int launch_add_node_blocks(int64_t nn, const int32_t* outer, const int32_t* inner, double* values, int32_t n,
                          const int32_t* nodes, const double* blocks, int32_t* missing, cudaStream_t stream);

}  // namespace sbk
