// K3: penalty contact of rigid tools with the slave nodes of the mesh
// (ToolContact, src/fem/RigidTool.cpp:43-611): the candidate search of an
// increment, the evaluation with Coulomb friction and its exact
// node-diagonal tangent, the semismooth anticipation and the friction
// history.
//
// One thread per slave node and tool. The candidate search of an increment
// (the slave nodes within R + margin of the tool's swept segment,
// RigidTool.cpp:345-393, a linear scan there) runs for a spherical tool on
// a uniform-grid hash of the slave nodes: they are binned by their position
// at the start of the increment into cells of edge R + margin, and only the
// cells the segment's box, grown by R + margin, overlaps are tested - with
// the reference's distance test, so the candidates are the same set. Other
// shapes (a plane's half space, a cylinder's infinite axis) and unbounded
// margins take the flat scan of every slave. Results are compacted in slave
// order - the reference's order - so the block list and every per-node sum
// match it; the gap and the candidate distances use explicitly rounded
// products and sums (no fused multiply-add), as a plain IEEE CPU build
// computes them, so the active set agrees bit for bit. The tool's reference
// point c(t) is interpolated on the host, as the reference does.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sbk.h"
#include "sbk_element.h"

namespace {

constexpr double kVanishing = 1.0e-12;

struct DTool {
  int shape;
  double radius, friction, ratio;
  double n[3];  // plane normal, unit
  double a[3];  // cylinder axis, unit
};

__device__ __forceinline__ double rn_dot3(const double* a, const double* b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}
__device__ __forceinline__ double rn_norm3(const double* a) { return sqrt(rn_dot3(a, a)); }

// RigidTool::gap (RigidTool.cpp:237-270); false within half the radius.
__device__ bool gap_of(const DTool& t, const double x[3], const double c[3], double n[3], double dn[9], double& g) {
  if (t.shape == 1) {
    double r[3] = {__dsub_rn(x[0], c[0]), __dsub_rn(x[1], c[1]), __dsub_rn(x[2], c[2])};
    for (int i = 0; i < 3; ++i) n[i] = t.n[i];
    for (int i = 0; i < 9; ++i) dn[i] = 0.0;
    g = rn_dot3(t.n, r);
    return true;
  }
  double r[3] = {__dsub_rn(x[0], c[0]), __dsub_rn(x[1], c[1]), __dsub_rn(x[2], c[2])};
  double base[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (t.shape == 2) {
    const double ar = rn_dot3(t.a, r);
    for (int i = 0; i < 3; ++i) r[i] = __dsub_rn(r[i], __dmul_rn(ar, t.a[i]));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) base[3 * i + j] -= t.a[i] * t.a[j];
  }
  const double d = rn_norm3(r);
  if (!(d > 0.5 * t.radius)) return false;
  for (int i = 0; i < 3; ++i) n[i] = r[i] / d;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) dn[3 * i + j] = (base[3 * i + j] - n[i] * n[j]) / d;
  g = __dsub_rn(d, t.radius);
  return true;
}

__device__ double segment_distance(const double p[3], const double a[3], const double b[3]) {
  const double s[3] = {__dsub_rn(b[0], a[0]), __dsub_rn(b[1], a[1]), __dsub_rn(b[2], a[2])};
  const double len2 = rn_dot3(s, s);
  double t = 0.0;
  if (len2 > 0.0) {
    const double pa[3] = {__dsub_rn(p[0], a[0]), __dsub_rn(p[1], a[1]), __dsub_rn(p[2], a[2])};
    t = fmin(fmax(__ddiv_rn(rn_dot3(pa, s), len2), 0.0), 1.0);
  }
  double o[3];
  for (int i = 0; i < 3; ++i) o[i] = __dsub_rn(__dsub_rn(p[i], a[i]), __dmul_rn(t, s[i]));
  return rn_norm3(o);
}

__device__ __forceinline__ void position(const double* coords, const double* u, int node, double x[3]) {
  for (int k = 0; k < 3; ++k) x[k] = __dadd_rn(coords[3 * (int64_t)node + k], u[3 * (int64_t)node + k]);
}

// The reference's candidate test of one node at x (RigidTool.cpp:345-393).
__device__ bool candidate_test(const DTool& t, const double x[3], const double c0[3], const double c1[3],
                               double margin) {
  if (t.shape == 0) return segment_distance(x, c0, c1) <= __dadd_rn(t.radius, margin);
  if (t.shape == 2) {
    double px[3], pc[3];
    const double dx[3] = {__dsub_rn(x[0], c0[0]), __dsub_rn(x[1], c0[1]), __dsub_rn(x[2], c0[2])};
    const double dc[3] = {__dsub_rn(c1[0], c0[0]), __dsub_rn(c1[1], c0[1]), __dsub_rn(c1[2], c0[2])};
    for (int r = 0; r < 3; ++r) {
      double pr[3];
      for (int s = 0; s < 3; ++s) pr[s] = __dsub_rn(r == s ? 1.0 : 0.0, __dmul_rn(t.a[r], t.a[s]));
      px[r] = rn_dot3(pr, dx);
      pc[r] = rn_dot3(pr, dc);
    }
    const double zero[3] = {0, 0, 0};
    return segment_distance(px, zero, pc) <= __dadd_rn(t.radius, margin);
  }
  const double d0[3] = {__dsub_rn(x[0], c0[0]), __dsub_rn(x[1], c0[1]), __dsub_rn(x[2], c0[2])};
  const double d1[3] = {__dsub_rn(x[0], c1[0]), __dsub_rn(x[1], c1[1]), __dsub_rn(x[2], c1[2])};
  return fmin(rn_dot3(t.n, d0), rn_dot3(t.n, d1)) <= margin;
}

// The flat scan: every slave node tested.
__global__ void candidates_kernel(DTool t, int n, const int32_t* __restrict__ nodes, const double* __restrict__ coords,
                                  const double* __restrict__ u0, double c0x, double c0y, double c0z, double c1x,
                                  double c1y, double c1z, double margin, uint8_t* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x[3];
  position(coords, u0, nodes[i], x);
  const double c0[3] = {c0x, c0y, c0z}, c1[3] = {c1x, c1y, c1z};
  flag[i] = candidate_test(t, x, c0, c1, margin) ? 1 : 0;
}

// ---- the uniform-grid hash of the slave nodes ----------------------------------
// Cell (ix, iy, iz) = floor(x / h) of a position; its bucket a hash of the
// three integers into a power-of-two table (colliding cells share a bucket;
// the exact test sorts their nodes out).
__device__ __host__ __forceinline__ uint32_t cell_bucket(long long ix, long long iy, long long iz, uint32_t mask) {
  const unsigned long long hx = (unsigned long long)ix * 73856093ull;
  const unsigned long long hy = (unsigned long long)iy * 19349663ull;
  const unsigned long long hz = (unsigned long long)iz * 83492791ull;
  return (uint32_t)((hx ^ hy ^ hz) & mask);
}

// The cell index of a coordinate; positions far outside any query (or not a
// number) share one sentinel cell.
__device__ __forceinline__ long long cell_of(double v, double inv_h) {
  const double f = floor(v * inv_h);
  return (f > 4.0e15 || f < -4.0e15 || f != f) ? (long long)4e15 : (long long)f;
}

__global__ void bin_kernel(int n, const int32_t* __restrict__ nodes, const double* __restrict__ coords,
                           const double* __restrict__ u0, double inv_h, uint32_t mask, int32_t* __restrict__ key,
                           int32_t* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x[3];
  position(coords, u0, nodes[i], x);
  const uint32_t b = cell_bucket(cell_of(x[0], inv_h), cell_of(x[1], inv_h), cell_of(x[2], inv_h), mask);
  key[i] = (int32_t)b;
  atomicAdd(&count[b], 1);
}

__global__ void bin_place_kernel(int n, const int32_t* __restrict__ key, const int32_t* __restrict__ start,
                                 int32_t* __restrict__ fill, int32_t* __restrict__ binned) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t b = key[i];
  binned[start[b] + atomicAdd(&fill[b], 1)] = i;
}

// One block per cell of the query box (first cell ix0, iy0, iz0, extents
// nx, ny): the nodes of its bucket through the exact test.
__global__ void grid_query_kernel(DTool t, long long ix0, long long iy0, long long iz0, int nx, int ny,
                                  uint32_t mask, const int32_t* __restrict__ start,
                                  const int32_t* __restrict__ binned, const int32_t* __restrict__ nodes,
                                  const double* __restrict__ coords, const double* __restrict__ u0, double c0x,
                                  double c0y, double c0z, double c1x, double c1y, double c1z, double margin,
                                  uint8_t* __restrict__ flag) {
  const int cell = blockIdx.x;
  const long long ix = ix0 + cell % nx, iy = iy0 + (cell / nx) % ny, iz = iz0 + cell / (nx * ny);
  const uint32_t b = cell_bucket(ix, iy, iz, mask);
  const double c0[3] = {c0x, c0y, c0z}, c1[3] = {c1x, c1y, c1z};
  const int32_t end = start[b + 1];
  for (int j = start[b] + threadIdx.x; j < end; j += blockDim.x) {
    const int i = binned[j];
    double x[3];
    position(coords, u0, nodes[i], x);
    if (candidate_test(t, x, c0, c1, margin)) flag[i] = 1;
  }
}

// ---- ordered compaction over many blocks ---------------------------------------
// out[k] = i for the k-th i with flag[i], *count their number: per-block
// counts, their offsets (one block), the placement by ballots - the list in
// slave order, the reference's order.
constexpr int kCompactBlock = 256;
// A query box of more cells than this takes the flat scan.
constexpr long long kMaxQueryCells = 1 << 16;

__global__ void flag_count_kernel(int n, const uint8_t* __restrict__ flag, int32_t* __restrict__ block_count) {
  __shared__ int32_t warp_count[kCompactBlock / 32];
  const int i = blockIdx.x * kCompactBlock + threadIdx.x;
  const unsigned ballot = __ballot_sync(0xffffffffu, i < n && flag[i]);
  if ((threadIdx.x & 31) == 0) warp_count[threadIdx.x >> 5] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t s = 0;
    for (int w = 0; w < kCompactBlock / 32; ++w) s += warp_count[w];
    block_count[blockIdx.x] = s;
  }
}

// Exclusive offsets of nb block counts, in place; the total into *count.
__global__ void block_offsets_kernel(int nb, int32_t* __restrict__ block_count, int32_t* __restrict__ count) {
  __shared__ int32_t warp_sums[32];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int f = i < nb ? block_count[i] : 0;
    int v = f;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
      int w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    if (i < nb) block_count[i] = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + v - f;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = carry;
}

__global__ void flag_place_kernel(int n, const uint8_t* __restrict__ flag, const int32_t* __restrict__ block_offset,
                                  int32_t* __restrict__ out) {
  __shared__ int32_t warp_base[kCompactBlock / 32];
  const int i = blockIdx.x * kCompactBlock + threadIdx.x;
  const bool f = i < n && flag[i];
  const unsigned ballot = __ballot_sync(0xffffffffu, f);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_base[warp] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    int32_t s = block_offset[blockIdx.x];
    for (int w = 0; w < kCompactBlock / 32; ++w) {
      const int32_t c = warp_base[w];
      warp_base[w] = s;
      s += c;
    }
  }
  __syncthreads();
  if (f) out[warp_base[warp] + __popc(ballot & ((1u << lane) - 1u))] = i;
}

void ordered_compact(int n, const uint8_t* flag, int32_t* out, int32_t* count, int32_t* block_scratch,
                     cudaStream_t st) {
  const int nb = (n + kCompactBlock - 1) / kCompactBlock;
  if (nb == 0) {
    cudaMemsetAsync(count, 0, sizeof(int32_t), st);
    return;
  }
  flag_count_kernel<<<nb, kCompactBlock, 0, st>>>(n, flag, block_scratch);
  block_offsets_kernel<<<1, 1024, 0, st>>>(nb, block_scratch, count);
  flag_place_kernel<<<nb, kCompactBlock, 0, st>>>(n, flag, block_scratch, out);
}

__global__ void moved_kernel(int n, const int32_t* __restrict__ nodes, const double* __restrict__ u,
                             const double* __restrict__ start, unsigned long long* __restrict__ moved) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t node = nodes[i];
  double m2 = 0.0;
  for (int c = 0; c < 3; ++c) {
    const double du = u[3 * node + c] - start[3 * node + c];
    m2 += du * du;
  }
  atomicMax(moved, (unsigned long long)__double_as_longlong(m2));  // m2 >= 0: bit order is value order
}

struct EvalOut {
  uint8_t* act;      // per slot
  uint8_t* slip;
  int32_t* node;
  double* force;     // 3 per slot
  double* k;         // 9 per slot
  double* pen;       // per slot
  double* pscale;    // per slot
};

// ToolContact::evaluate for one tool (RigidTool.cpp:398-555).
__global__ void evaluate_kernel(DTool t, int nslaves, const int32_t* __restrict__ nodes,
                                const double* __restrict__ area, const double* __restrict__ kappa,
                                const int32_t* __restrict__ cand, const int32_t* __restrict__ ncand,
                                const unsigned long long* __restrict__ moved, double margin,
                                const double* __restrict__ coords, const double* __restrict__ u,
                                const double* __restrict__ start, double cx, double cy, double cz, double c0x,
                                double c0y, double c0z, int symmetric_tangent, const uint8_t* __restrict__ h_flag,
                                const double* __restrict__ h_force, const double* __restrict__ h_rel,
                                uint8_t* __restrict__ t_flag, double* __restrict__ t_force,
                                double* __restrict__ t_rel, EvalOut out, int32_t* __restrict__ failed) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= nslaves) return;
  out.act[slot] = 0;
  const bool all = sqrt(__longlong_as_double((long long)*moved)) > margin;
  int i = slot;
  if (!all) {
    if (slot >= *ncand) return;
    i = cand[slot];
  }
  const int node = nodes[i];
  double x[3];
  position(coords, u, node, x);
  const double c[3] = {cx, cy, cz};
  double nrm[3], dn[9], g = 0.0;
  if (!gap_of(t, x, c, nrm, dn, g)) {
    atomicExch(failed, 1);
    return;
  }
  if (!(g < 0.0)) return;
  const double ka = kappa[i] * area[i];
  const double pn = -ka * g;
  double force[3], kn[9];
  for (int r = 0; r < 3; ++r) force[r] = pn * nrm[r];
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) kn[3 * r + s] = ka * (nrm[r] * nrm[s]) - pn * dn[3 * r + s];
  bool slipping = false;
  const double rr[3] = {x[0] - c[0], x[1] - c[1], x[2] - c[2]};
  if (t.friction > 0.0) {
    const double mu = t.friction;
    const double kt = t.ratio * ka;
    double f0[3] = {0, 0, 0}, q[3];
    if (h_flag[i]) {
      for (int r = 0; r < 3; ++r) {
        f0[r] = h_force[3 * i + r];
        q[r] = h_rel[3 * i + r];
      }
    } else {
      for (int r = 0; r < 3; ++r) q[r] = (coords[3 * (int64_t)node + r] + start[3 * (int64_t)node + r]) - (r == 0 ? c0x : (r == 1 ? c0y : c0z));
    }
    const double s0 = sqrt(f0[0] * f0[0] + f0[1] * f0[1] + f0[2] * f0[2]);
    const double fn = f0[0] * nrm[0] + f0[1] * nrm[1] + f0[2] * nrm[2];
    double ftl[3];
    for (int r = 0; r < 3; ++r) ftl[r] = f0[r] - fn * nrm[r];
    const double ftn = sqrt(ftl[0] * ftl[0] + ftl[1] * ftl[1] + ftl[2] * ftl[2]);
    double f_hat[3] = {0, 0, 0}, d_hat[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (s0 > 0.0 && ftn > kVanishing * s0) {
      double e[3];
      for (int r = 0; r < 3; ++r) {
        e[r] = ftl[r] / ftn;
        f_hat[r] = s0 * e[r];
      }
      double f0dn[3], d_tilde[9];
      for (int s = 0; s < 3; ++s) f0dn[s] = f0[0] * dn[s] + f0[1] * dn[3 + s] + f0[2] * dn[6 + s];
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) d_tilde[3 * r + s] = -(nrm[r] * f0dn[s] + fn * dn[3 * r + s]);
      const double sc = s0 / ftn;
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) {
          double acc = 0.0;
          for (int m = 0; m < 3; ++m) acc += ((r == m ? 1.0 : 0.0) - e[r] * e[m]) * d_tilde[3 * m + s];
          d_hat[3 * r + s] = sc * acc;
        }
    }
    const double w[3] = {rr[0] - q[0], rr[1] - q[1], rr[2] - q[2]};
    double p[9], delta[3], d_delta[9], d_trial[9], trial[3];
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) p[3 * r + s] = (r == s ? 1.0 : 0.0) - nrm[r] * nrm[s];
    for (int r = 0; r < 3; ++r) delta[r] = p[3 * r] * w[0] + p[3 * r + 1] * w[1] + p[3 * r + 2] * w[2];
    const double nw = nrm[0] * w[0] + nrm[1] * w[1] + nrm[2] * w[2];
    double wdn[3];
    for (int s = 0; s < 3; ++s) wdn[s] = w[0] * dn[s] + w[1] * dn[3 + s] + w[2] * dn[6 + s];
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) d_delta[3 * r + s] = p[3 * r + s] - nw * dn[3 * r + s] - nrm[r] * wdn[s];
    for (int r = 0; r < 3; ++r) trial[r] = f_hat[r] - kt * delta[r];
    for (int m = 0; m < 9; ++m) d_trial[m] = d_hat[m] - kt * d_delta[m];
    const double tn = sqrt(trial[0] * trial[0] + trial[1] * trial[1] + trial[2] * trial[2]);
    const double limit = mu * pn;
    double ft[3], d_ft[9], k_sym[9];
    if (tn <= limit) {
      for (int r = 0; r < 3; ++r) ft[r] = trial[r];
      for (int m = 0; m < 9; ++m) {
        d_ft[m] = d_trial[m];
        k_sym[m] = kt * p[m];
      }
    } else {
      slipping = true;
      double e[3];
      for (int r = 0; r < 3; ++r) {
        e[r] = trial[r] / tn;
        ft[r] = limit * e[r];
      }
      const double lt = limit / tn;
      for (int r = 0; r < 3; ++r)
        for (int s = 0; s < 3; ++s) {
          double acc = 0.0;
          for (int m = 0; m < 3; ++m) acc += ((r == m ? 1.0 : 0.0) - e[r] * e[m]) * d_trial[3 * m + s];
          d_ft[3 * r + s] = -(mu * ka) * (e[r] * nrm[s]) + lt * acc;
          k_sym[3 * r + s] = lt * kt * (p[3 * r + s] - e[r] * e[s]);
        }
    }
    for (int r = 0; r < 3; ++r) force[r] += ft[r];
    for (int m = 0; m < 9; ++m) kn[m] = symmetric_tangent ? kn[m] + k_sym[m] : kn[m] - d_ft[m];
    t_flag[i] = 1;
    for (int r = 0; r < 3; ++r) {
      t_force[3 * i + r] = ft[r];
      t_rel[3 * i + r] = rr[r];
    }
  }
  if (symmetric_tangent) {
    double ks[9];
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) ks[3 * r + s] = 0.5 * (kn[3 * r + s] + kn[3 * s + r]);
    for (int m = 0; m < 9; ++m) kn[m] = ks[m];
  }
  const double xn = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  const double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  out.act[slot] = 1;
  out.slip[slot] = slipping ? 1 : 0;
  out.node[slot] = node;
  for (int r = 0; r < 3; ++r) out.force[3 * slot + r] = force[r];
  for (int m = 0; m < 9; ++m) out.k[9 * slot + m] = kn[m];
  out.pen[slot] = -g;
  out.pscale[slot] = ka * (xn + cn);
}

// Active slots of one tool into the residual, the gross and round-off
// vectors and the block list (at block offset `base`, slot order).
__global__ void scatter_kernel(int nslots, const int32_t* __restrict__ list, const int32_t* __restrict__ nlist,
                               EvalOut ev, double* __restrict__ residual, double* __restrict__ gross,
                               double* __restrict__ positions, int32_t* __restrict__ block_nodes,
                               double* __restrict__ blocks, int base, int want_tangent, int32_t* __restrict__ asym) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *nlist) return;
  const int slot = list[k];
  const int64_t node = ev.node[slot];
  for (int c = 0; c < 3; ++c) {
    const double f = ev.force[3 * slot + c];
    residual[3 * node + c] -= f;
    gross[3 * node + c] += fabs(f);
    positions[3 * node + c] += ev.pscale[slot];
  }
  if (want_tangent) {
    block_nodes[base + k] = (int32_t)node;
    double top = 0.0, d = 0.0;
    for (int r = 0; r < 3; ++r)
      for (int s = 0; s < 3; ++s) {
        const double v = ev.k[9 * slot + 3 * r + s];
        blocks[9 * (base + k) + 3 * r + s] = v;
        top = fmax(top, fabs(v));
        d = fmax(d, fabs(v - ev.k[9 * slot + 3 * s + r]));
      }
    if (d > 1.0e-12 * top) atomicExch(asym, 1);
  }
}

// Per tool resultants: force sum, active and slipping counts, max
// penetration (one block, fixed order).
__global__ void resultant_kernel(const int32_t* __restrict__ list, const int32_t* __restrict__ nlist, EvalOut ev,
                                 double* __restrict__ out) {
  __shared__ double sh[256][5];
  double f[3] = {0, 0, 0}, slips = 0.0, pen = 0.0;
  const int n = *nlist;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const int slot = list[k];
    for (int c = 0; c < 3; ++c) f[c] -= ev.force[3 * slot + c];
    slips += ev.slip[slot];
    pen = fmax(pen, ev.pen[slot]);
  }
  sh[threadIdx.x][0] = f[0];
  sh[threadIdx.x][1] = f[1];
  sh[threadIdx.x][2] = f[2];
  sh[threadIdx.x][3] = slips;
  sh[threadIdx.x][4] = pen;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      for (int c = 0; c < 4; ++c) sh[threadIdx.x][c] += sh[threadIdx.x + s][c];
      sh[threadIdx.x][4] = fmax(sh[threadIdx.x][4], sh[threadIdx.x + s][4]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sh[0][0];
    out[1] = sh[0][1];
    out[2] = sh[0][2];
    out[3] = (double)n;
    out[4] = sh[0][3];
    out[5] = sh[0][4];
  }
}

// The Euclidean norms of three n-vectors in two fixed-shape stages (the
// same sums in the same order every call): kNormBlocks blocks of partial
// sums of squares, then one block over the partials.
constexpr int kNormBlocks = 296;

__global__ void norms_partial_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                     const double* __restrict__ c, double* __restrict__ partial) {
  __shared__ double sh[256][3];
  double s[3] = {0, 0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    s[0] += a[i] * a[i];
    s[1] += b[i] * b[i];
    s[2] += c[i] * c[i];
  }
  for (int k = 0; k < 3; ++k) sh[threadIdx.x][k] = s[k];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 3; ++k) sh[threadIdx.x][k] += sh[threadIdx.x + st][k];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partial[3 * blockIdx.x + k] = sh[0][k];
}

__global__ void norms_kernel(int nb, const double* __restrict__ partial, double* __restrict__ out) {
  __shared__ double sh[256][3];
  double s[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    for (int k = 0; k < 3; ++k) s[k] += partial[3 * i + k];
  for (int k = 0; k < 3; ++k) sh[threadIdx.x][k] = s[k];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int k = 0; k < 3; ++k) sh[threadIdx.x][k] += sh[threadIdx.x + st][k];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) out[k] = sqrt(sh[0][k]);
}

// ToolContact::anticipate for one tool (RigidTool.cpp:557-603).
__global__ void anticipate_kernel(DTool t, const int32_t* __restrict__ nodes, const double* __restrict__ area,
                                  const double* __restrict__ kappa, const int32_t* __restrict__ cand,
                                  const int32_t* __restrict__ ncand, const double* __restrict__ coords,
                                  const double* __restrict__ u, const double* __restrict__ du, double cx, double cy,
                                  double cz, uint8_t* __restrict__ flag, double* __restrict__ kn_out,
                                  int32_t* __restrict__ node_out, double* __restrict__ add_out) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= *ncand) return;
  flag[slot] = 0;
  const int i = cand[slot];
  const int node = nodes[i];
  double x[3], xn[3];
  position(coords, u, node, x);
  for (int r = 0; r < 3; ++r) xn[r] = __dadd_rn(x[r], du[3 * (int64_t)node + r]);
  const double c[3] = {cx, cy, cz};
  double nrm[3], dn[9], g = 0.0, nn2[3], g_next = 0.0;
  if (!gap_of(t, x, c, nrm, dn, g)) return;
  if (!(g > 0.0)) return;
  if (!gap_of(t, xn, c, nn2, dn, g_next)) g_next = -__longlong_as_double(0x7ff0000000000000LL);
  if (!(g_next < 0.0)) return;
  const double ka = kappa[i] * area[i];
  flag[slot] = 1;
  node_out[slot] = node;
  for (int r = 0; r < 3; ++r) add_out[3 * slot + r] = ka * g * nrm[r];
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) kn_out[9 * slot + 3 * r + s] = ka * (nrm[r] * nrm[s]);
}

__global__ void anticipate_scatter_kernel(const int32_t* __restrict__ list, const int32_t* __restrict__ nlist,
                                          const int32_t* __restrict__ node_in, const double* __restrict__ add_in,
                                          const double* __restrict__ kn_in, double* __restrict__ residual,
                                          int32_t* __restrict__ block_nodes, double* __restrict__ blocks, int base) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *nlist) return;
  const int slot = list[k];
  const int64_t node = node_in[slot];
  for (int c = 0; c < 3; ++c) residual[3 * node + c] += add_in[3 * slot + c];
  block_nodes[base + k] = (int32_t)node;
  for (int m = 0; m < 9; ++m) blocks[9 * (base + k) + m] = kn_in[9 * slot + m];
}

// ---------------------------------------------------------------------------
int cfail(int code, const std::string& what) { return sbk::set_error(code, what); }
#define SBK_C(call)                                                                                   \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) return cfail(SBK_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct HostTool {
  DTool d;
  std::vector<double> times, points;
  mutable size_t hint = 0;
  int nslaves = 0;
  int32_t* nodes = nullptr;
  double* area = nullptr;
  double* kappa = nullptr;
  uint8_t* cflag = nullptr;    // candidate flags (scratch)
  int32_t* cand = nullptr;     // candidate positions
  int32_t* ncand = nullptr;    // device count
  uint8_t* h_flag = nullptr;   // committed history
  double* h_force = nullptr;
  double* h_rel = nullptr;
  uint8_t* t_flag = nullptr;   // trial history of the last evaluate
  double* t_force = nullptr;
  double* t_rel = nullptr;
  unsigned long long* moved = nullptr;
  // per-slot evaluation scratch
  uint8_t* act = nullptr;
  uint8_t* slip = nullptr;
  int32_t* enode = nullptr;
  double* eforce = nullptr;
  double* ek = nullptr;
  double* epen = nullptr;
  double* epscale = nullptr;
  int32_t* alist = nullptr;
  int32_t* nalist = nullptr;
  int32_t* cblocks = nullptr;   // ordered compaction: per-block counts
  // The uniform-grid hash of the slave nodes (rebuilt each increment).
  uint32_t gmask = 0;           // table size - 1 (a power of two)
  int32_t* gkey = nullptr;      // per slave: its bucket
  int32_t* gcount = nullptr;    // per bucket (+1): count, then fill
  int32_t* gstart = nullptr;    // per bucket (+1): first position in gbinned
  int32_t* gbinned = nullptr;   // slaves by bucket
  void* gscan = nullptr;        // the bucket scan's scratch
  size_t gscan_bytes = 0;

  // ToolTrajectory::position (RigidTool.cpp:83-105), evaluated on the host.
  void position(double t, double out[3]) const {
    const size_t nk = times.size();
    if (t <= times.front()) {
      for (int k = 0; k < 3; ++k) out[k] = points[k];
      return;
    }
    if (t >= times.back()) {
      for (int k = 0; k < 3; ++k) out[k] = points[3 * (nk - 1) + k];
      return;
    }
    const size_t last = nk - 2;
    size_t i = std::min(hint, last);
    if (!(times[i] <= t && t < times[i + 1])) {
      if (i < last && times[i + 1] <= t && t < times[i + 2]) {
        i = i + 1;
      } else {
        const auto it = std::upper_bound(times.begin(), times.end(), t);
        long long j = static_cast<long long>(it - times.begin()) - 1;
        if (j < 0) j = 0;
        i = std::min(static_cast<size_t>(j), last);
      }
      hint = i;
    }
    const double w = (t - times[i]) / (times[i + 1] - times[i]);
    for (int k = 0; k < 3; ++k) out[k] = (1.0 - w) * points[3 * i + k] + w * points[3 * (i + 1) + k];
  }
  EvalOut ev() const { return EvalOut{act, slip, enode, eforce, ek, epen, epscale}; }
};

}  // namespace

struct sbk_contact {
  int64_t nn = 0;
  double* coords = nullptr;
  std::vector<HostTool> tools;
  int friction_tangent = 0;
  double* start = nullptr;
  double t0 = 0.0, margin = 0.0;
  std::vector<uint8_t> active;
  cudaStream_t stream = nullptr;
  double* residual = nullptr;
  double* gross = nullptr;
  double* positions = nullptr;
  int32_t* block_nodes = nullptr;
  double* blocks = nullptr;
  int capacity = 0;  // blocks
  int num_blocks = 0;
  int32_t* flags = nullptr;  // [0] failed, [1] asym
  double* norms = nullptr;
  double* norm_partial = nullptr;  // 3 per block of the norms' first stage
  double* res_dev = nullptr;  // 6 per tool
  std::vector<double> resultants;
  int search = SBK_SEARCH_GRID;
};

namespace {
template <class T>
int calloc_dev(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  SBK_C(cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)));
  SBK_C(cudaMemset(*p, 0, n * sizeof(T)));
  return SBK_OK;
}
void free_contact(sbk_contact* c) {
  for (HostTool& t : c->tools) {
    void* ptrs[] = {t.nodes, t.area, t.kappa, t.cflag, t.cand, t.ncand, t.h_flag, t.h_force, t.h_rel, t.t_flag,
                    t.t_force, t.t_rel, t.moved, t.act, t.slip, t.enode, t.eforce, t.ek, t.epen, t.epscale,
                    t.alist, t.nalist, t.cblocks, t.gkey, t.gcount, t.gstart, t.gbinned, t.gscan};
    for (void* p : ptrs)
      if (p) cudaFree(p);
  }
  void* ptrs[] = {c->coords, c->start, c->residual, c->gross, c->positions, c->block_nodes, c->blocks, c->flags,
                  c->norms, c->norm_partial, c->res_dev};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete c;
}
double norm3h(const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
}  // namespace

extern "C" {

int sbk_contact_create(const sbk_mesh* mesh, int32_t num_tools, const sbk_tool* tools, int friction_tangent,
                       sbk_contact** out) {
  if (!out || !mesh || !mesh->coords || mesh->num_nodes <= 0 || num_tools < 0 || (num_tools > 0 && !tools))
    return cfail(SBK_ERR_ARGUMENT, "null or empty argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return cfail(SBK_ERR_NO_EXTENSION, "no CUDA device: contact runs on the GPU only");
  }
  sbk_contact* c = new sbk_contact();
  c->nn = mesh->num_nodes;
  c->friction_tangent = friction_tangent ? 1 : 0;
  int rc;
#define TRYC(x)        \
  do {                 \
    rc = (x);          \
    if (rc) {          \
      free_contact(c); \
      return rc;       \
    }                  \
  } while (0)
  TRYC(calloc_dev(&c->coords, 3 * c->nn));
  if (cudaMemcpy(c->coords, mesh->coords, 3 * c->nn * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    free_contact(c);
    return cfail(SBK_ERR_CUDA, "coordinate upload");
  }
  TRYC(calloc_dev(&c->start, 3 * c->nn));
  TRYC(calloc_dev(&c->residual, 3 * c->nn));
  TRYC(calloc_dev(&c->gross, 3 * c->nn));
  TRYC(calloc_dev(&c->positions, 3 * c->nn));
  TRYC(calloc_dev(&c->flags, 4));
  TRYC(calloc_dev(&c->norms, 4));
  TRYC(calloc_dev(&c->norm_partial, 3 * kNormBlocks));
  int total = 0;
  for (int k = 0; k < num_tools; ++k) {
    const sbk_tool& s = tools[k];
    if (s.shape < 0 || s.shape > 2 || s.num_knots < 2 || s.num_slaves < 0 || !s.times || !s.points ||
        (s.num_slaves > 0 && (!s.nodes || !s.area || !s.kappa))) {
      free_contact(c);
      return cfail(SBK_ERR_ARGUMENT, "an invalid tool");
    }
    for (int32_t i = 0; i < s.num_slaves; ++i) {
      // Every slave node inside the mesh and in ascending order, its area and
      // penalty finite and non-negative: the kernels index by them.
      if (s.nodes[i] < 0 || s.nodes[i] >= mesh->num_nodes || (i > 0 && s.nodes[i] <= s.nodes[i - 1]) ||
          !std::isfinite(s.area[i]) || !(s.area[i] >= 0.0) || !std::isfinite(s.kappa[i]) || !(s.kappa[i] >= 0.0)) {
        free_contact(c);
        return cfail(SBK_ERR_ARGUMENT, "a tool's slave nodes must lie in the mesh, ascending, with finite "
                                       "non-negative areas and penalties");
      }
    }
    if (s.shape != 1 && !(s.radius > 0.0)) {
      free_contact(c);
      return cfail(SBK_ERR_CONFIG, "a sphere or cylinder needs a positive radius");
    }
    if (!(s.friction >= 0.0) || !(s.tangential_ratio > 0.0)) {
      free_contact(c);
      return cfail(SBK_ERR_CONFIG, "friction must be >= 0 and the tangential ratio > 0");
    }
    HostTool t;
    t.d.shape = s.shape;
    t.d.radius = s.radius;
    t.d.friction = s.friction;
    t.d.ratio = s.tangential_ratio;
    const double ln = norm3h(s.normal), la = norm3h(s.axis);
    for (int i = 0; i < 3; ++i) {
      t.d.n[i] = ln > 0.0 ? s.normal[i] / ln : 0.0;
      t.d.a[i] = la > 0.0 ? s.axis[i] / la : 0.0;
    }
    if ((s.shape == 1 && !(ln > 0.0)) || (s.shape == 2 && !(la > 0.0))) {
      free_contact(c);
      return cfail(SBK_ERR_CONFIG, "a plane needs a normal and a cylinder an axis");
    }
    t.times.assign(s.times, s.times + s.num_knots);
    t.points.assign(s.points, s.points + 3 * s.num_knots);
    for (int i = 1; i < s.num_knots; ++i)
      if (!(t.times[i] > t.times[i - 1])) {
        free_contact(c);
        return cfail(SBK_ERR_CONFIG, "trajectory times must increase strictly");
      }
    t.nslaves = s.num_slaves;
    c->tools.push_back(t);
    HostTool& h = c->tools.back();
    const size_t n = static_cast<size_t>(std::max(1, s.num_slaves));
    TRYC(calloc_dev(&h.nodes, n));
    TRYC(calloc_dev(&h.area, n));
    TRYC(calloc_dev(&h.kappa, n));
    if (s.num_slaves > 0) {
      cudaMemcpy(h.nodes, s.nodes, s.num_slaves * sizeof(int32_t), cudaMemcpyHostToDevice);
      cudaMemcpy(h.area, s.area, s.num_slaves * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(h.kappa, s.kappa, s.num_slaves * sizeof(double), cudaMemcpyHostToDevice);
    }
    TRYC(calloc_dev(&h.cflag, n));
    TRYC(calloc_dev(&h.cand, n));
    TRYC(calloc_dev(&h.ncand, 1));
    TRYC(calloc_dev(&h.h_flag, n));
    TRYC(calloc_dev(&h.h_force, 3 * n));
    TRYC(calloc_dev(&h.h_rel, 3 * n));
    TRYC(calloc_dev(&h.t_flag, n));
    TRYC(calloc_dev(&h.t_force, 3 * n));
    TRYC(calloc_dev(&h.t_rel, 3 * n));
    TRYC(calloc_dev(&h.moved, 1));
    TRYC(calloc_dev(&h.act, n));
    TRYC(calloc_dev(&h.slip, n));
    TRYC(calloc_dev(&h.enode, n));
    TRYC(calloc_dev(&h.eforce, 3 * n));
    TRYC(calloc_dev(&h.ek, 9 * n));
    TRYC(calloc_dev(&h.epen, n));
    TRYC(calloc_dev(&h.epscale, n));
    TRYC(calloc_dev(&h.alist, n));
    TRYC(calloc_dev(&h.nalist, 1));
    TRYC(calloc_dev(&h.cblocks, (n + kCompactBlock - 1) / kCompactBlock + 1));
    {
      size_t table = 1024;
      while (table < 2 * n) table <<= 1;
      h.gmask = static_cast<uint32_t>(table - 1);
      TRYC(calloc_dev(&h.gkey, n));
      TRYC(calloc_dev(&h.gcount, table + 1));
      TRYC(calloc_dev(&h.gstart, table + 1));
      TRYC(calloc_dev(&h.gbinned, n));
      if (cub::DeviceScan::ExclusiveSum(nullptr, h.gscan_bytes, h.gcount, h.gstart, static_cast<int>(table + 1)) !=
          cudaSuccess) {
        free_contact(c);
        return cfail(SBK_ERR_CUDA, "grid scan size");
      }
      TRYC(calloc_dev(reinterpret_cast<char**>(&h.gscan), h.gscan_bytes));
    }
    // Every slave a candidate until an increment is prepared.
    std::vector<int32_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = static_cast<int32_t>(i);
    int32_t cnt = s.num_slaves;
    cudaMemcpy(h.cand, idx.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice);
    cudaMemcpy(h.ncand, &cnt, sizeof(int32_t), cudaMemcpyHostToDevice);
    total += 2 * s.num_slaves;
  }
  c->capacity = std::max(1, total);
  TRYC(calloc_dev(&c->block_nodes, c->capacity));
  TRYC(calloc_dev(&c->blocks, 9 * static_cast<size_t>(c->capacity)));
  TRYC(calloc_dev(&c->res_dev, 6 * std::max<size_t>(1, c->tools.size())));
#undef TRYC
  c->t0 = c->tools.empty() ? 0.0 : c->tools.front().times.front();
  c->margin = __builtin_inf();
  c->active.assign(c->tools.size(), 1);
  c->resultants.assign(9 * c->tools.size(), 0.0);
  *out = c;
  return SBK_OK;
}

int sbk_contact_destroy(sbk_contact* c) {
  if (c) {
    cudaStreamSynchronize(c->stream);
    free_contact(c);
  }
  return SBK_OK;
}

int sbk_contact_set_stream(sbk_contact* c, void* stream) {
  if (!c) return cfail(SBK_ERR_ARGUMENT, "null contact");
  c->stream = static_cast<cudaStream_t>(stream);
  return SBK_OK;
}

int sbk_contact_begin(sbk_contact* c, const double* u0_dev, double t0, double t1, const uint8_t* active,
                      double margin) {
  if (!c || !u0_dev || (!c->tools.empty() && !active)) return cfail(SBK_ERR_ARGUMENT, "null argument");
  cudaStream_t st = c->stream;
  SBK_C(cudaMemcpyAsync(c->start, u0_dev, 3 * c->nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
  c->t0 = t0;
  c->margin = margin;
  for (size_t k = 0; k < c->tools.size(); ++k) {
    HostTool& t = c->tools[k];
    c->active[k] = active[k] ? 1 : 0;
    if (!c->active[k] || t.nslaves == 0) {
      SBK_C(cudaMemsetAsync(t.ncand, 0, sizeof(int32_t), st));
      continue;
    }
    double c0[3], c1[3];
    t.position(t0, c0);
    t.position(t1, c1);
    // The grid for a sphere with a bounded reach: cells of edge R + margin,
    // the query the cells of the segment's box grown by the reach (and by a
    // hair more, for the rounding of the distance test).
    const double reach = t.d.radius + margin;
    bool grid = c->search == SBK_SEARCH_GRID && t.d.shape == 0 && std::isfinite(reach) && reach > 0.0;
    long long lo[3] = {0, 0, 0}, ext[3] = {1, 1, 1};
    const double inv_h = grid ? 1.0 / reach : 0.0;
    if (grid) {
      double scale = reach;
      for (int k = 0; k < 3; ++k) scale = std::max(scale, std::max(std::fabs(c0[k]), std::fabs(c1[k])));
      const double hair = 1.0e-9 * scale;
      long long cells = 1;
      for (int k = 0; k < 3; ++k) {
        const double a = std::floor((std::min(c0[k], c1[k]) - reach - hair) * inv_h);
        const double b = std::floor((std::max(c0[k], c1[k]) + reach + hair) * inv_h);
        if (!std::isfinite(a) || !std::isfinite(b) || std::fabs(a) > 1.0e15 || std::fabs(b) > 1.0e15) {
          grid = false;
          break;
        }
        lo[k] = static_cast<long long>(a);
        ext[k] = static_cast<long long>(b) - lo[k] + 1;
        cells *= ext[k];
        if (cells > kMaxQueryCells) {
          grid = false;
          break;
        }
      }
    }
    const int blocks = (t.nslaves + 127) / 128;
    if (grid) {
      const size_t table = static_cast<size_t>(t.gmask) + 1;
      SBK_C(cudaMemsetAsync(t.gcount, 0, (table + 1) * sizeof(int32_t), st));
      bin_kernel<<<blocks, 128, 0, st>>>(t.nslaves, t.nodes, c->coords, u0_dev, inv_h, t.gmask, t.gkey, t.gcount);
      size_t bytes = t.gscan_bytes;
      SBK_C(cub::DeviceScan::ExclusiveSum(t.gscan, bytes, t.gcount, t.gstart, static_cast<int>(table + 1), st));
      SBK_C(cudaMemsetAsync(t.gcount, 0, table * sizeof(int32_t), st));
      bin_place_kernel<<<blocks, 128, 0, st>>>(t.nslaves, t.gkey, t.gstart, t.gcount, t.gbinned);
      SBK_C(cudaMemsetAsync(t.cflag, 0, t.nslaves, st));
      const int cells = static_cast<int>(ext[0] * ext[1] * ext[2]);
      grid_query_kernel<<<cells, 128, 0, st>>>(t.d, lo[0], lo[1], lo[2], static_cast<int>(ext[0]),
                                               static_cast<int>(ext[1]), t.gmask, t.gstart, t.gbinned, t.nodes,
                                               c->coords, u0_dev, c0[0], c0[1], c0[2], c1[0], c1[1], c1[2], margin,
                                               t.cflag);
    } else {
      candidates_kernel<<<blocks, 128, 0, st>>>(t.d, t.nslaves, t.nodes, c->coords, u0_dev, c0[0], c0[1], c0[2],
                                                c1[0], c1[1], c1[2], margin, t.cflag);
    }
    ordered_compact(t.nslaves, t.cflag, t.cand, t.ncand, t.cblocks, st);
  }
  SBK_C(cudaGetLastError());
  return SBK_OK;
}

int sbk_contact_set_search(sbk_contact* c, int mode) {
  if (!c) return cfail(SBK_ERR_ARGUMENT, "null contact");
  if (mode != SBK_SEARCH_GRID && mode != SBK_SEARCH_SCAN) return cfail(SBK_ERR_ARGUMENT, "unknown search mode");
  c->search = mode;
  return SBK_OK;
}

int sbk_contact_candidates(const sbk_contact* c, int32_t k, int32_t* count) {
  if (!c || !count || k < 0 || k >= static_cast<int32_t>(c->tools.size())) return cfail(SBK_ERR_ARGUMENT, "bad tool");
  const HostTool& h = c->tools[k];
  SBK_C(cudaMemcpyAsync(count, h.ncand, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  SBK_C(cudaStreamSynchronize(c->stream));
  return SBK_OK;
}

int sbk_contact_evaluate(sbk_contact* c, const double* u_dev, double t, int want_tangent, sbk_contact_result* out) {
  if (!c || !u_dev || !out) return cfail(SBK_ERR_ARGUMENT, "null argument");
  cudaStream_t st = c->stream;
  std::memset(out, 0, sizeof(*out));
  const size_t nd = 3 * static_cast<size_t>(c->nn);
  SBK_C(cudaMemsetAsync(c->residual, 0, nd * sizeof(double), st));
  SBK_C(cudaMemsetAsync(c->gross, 0, nd * sizeof(double), st));
  SBK_C(cudaMemsetAsync(c->positions, 0, nd * sizeof(double), st));
  SBK_C(cudaMemsetAsync(c->flags, 0, 4 * sizeof(int32_t), st));
  SBK_C(cudaMemsetAsync(c->res_dev, 0, 6 * std::max<size_t>(1, c->tools.size()) * sizeof(double), st));
  std::vector<int32_t> counts(c->tools.size(), 0);
  int base = 0;
  for (size_t k = 0; k < c->tools.size(); ++k) {
    HostTool& h = c->tools[k];
    double cc[3];
    h.position(t, cc);
    for (int i = 0; i < 3; ++i) c->resultants[9 * k + i] = cc[i];
    if (h.nslaves > 0) SBK_C(cudaMemsetAsync(h.t_flag, 0, h.nslaves, st));
    if (!c->active[k] || h.nslaves == 0) continue;
    double c0[3];
    h.position(c->t0, c0);
    SBK_C(cudaMemsetAsync(h.moved, 0, sizeof(unsigned long long), st));
    const int blocks = (h.nslaves + 127) / 128;
    moved_kernel<<<blocks, 128, 0, st>>>(h.nslaves, h.nodes, u_dev, c->start, h.moved);
    evaluate_kernel<<<blocks, 128, 0, st>>>(h.d, h.nslaves, h.nodes, h.area, h.kappa, h.cand, h.ncand, h.moved,
                                            c->margin, c->coords, u_dev, c->start, cc[0], cc[1], cc[2], c0[0],
                                            c0[1], c0[2], c->friction_tangent, h.h_flag, h.h_force, h.h_rel,
                                            h.t_flag, h.t_force, h.t_rel, h.ev(), c->flags);
    ordered_compact(h.nslaves, h.act, h.alist, h.nalist, h.cblocks, st);
    // The block offset of this tool needs the count of the previous ones.
    SBK_C(cudaMemcpyAsync(&counts[k], h.nalist, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SBK_C(cudaStreamSynchronize(st));
    scatter_kernel<<<(h.nslaves + 127) / 128, 128, 0, st>>>(h.nslaves, h.alist, h.nalist, h.ev(), c->residual,
                                                            c->gross, c->positions, c->block_nodes, c->blocks, base,
                                                            want_tangent, c->flags + 1);
    resultant_kernel<<<1, 256, 0, st>>>(h.alist, h.nalist, h.ev(), c->res_dev + 6 * k);
    if (want_tangent) base += counts[k];
  }
  norms_partial_kernel<<<kNormBlocks, 256, 0, st>>>(static_cast<int64_t>(nd), c->gross, c->positions, c->residual,
                                                   c->norm_partial);
  norms_kernel<<<1, 256, 0, st>>>(kNormBlocks, c->norm_partial, c->norms);
  SBK_C(cudaGetLastError());
  double norms[3];
  int32_t flags[2];
  std::vector<double> res(6 * std::max<size_t>(1, c->tools.size()));
  SBK_C(cudaMemcpyAsync(norms, c->norms, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  SBK_C(cudaMemcpyAsync(flags, c->flags, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SBK_C(cudaMemcpyAsync(res.data(), c->res_dev, res.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  SBK_C(cudaStreamSynchronize(st));
  for (size_t k = 0; k < c->tools.size(); ++k) {
    for (int i = 0; i < 3; ++i) c->resultants[9 * k + 3 + i] = res[6 * k + i];
    c->resultants[9 * k + 6] = res[6 * k + 3];
    c->resultants[9 * k + 7] = res[6 * k + 4];
    c->resultants[9 * k + 8] = res[6 * k + 5];
  }
  c->num_blocks = base;
  out->residual_dev = c->residual;
  out->block_nodes_dev = c->block_nodes;
  out->blocks_dev = c->blocks;
  out->num_blocks = base;
  out->symmetric = flags[1] ? 0 : 1;
  out->gross = norms[0];
  out->round_off = norms[1];
  out->force_norm = norms[2];
  out->failed = flags[0];
  if (flags[0]) return cfail(SBK_ERR_SOLVER, "a node lies within half the radius of a tool: the tool is through the surface");
  return SBK_OK;
}

int sbk_contact_resultants(const sbk_contact* c, double* out) {
  if (!c || !out) return cfail(SBK_ERR_ARGUMENT, "null argument");
  std::copy(c->resultants.begin(), c->resultants.end(), out);
  return SBK_OK;
}

int sbk_contact_anticipate(sbk_contact* c, const double* u_dev, const double* du_dev, double t, double* residual_dev,
                           int32_t* added, sbk_contact_result* out) {
  if (!c || !u_dev || !du_dev || !residual_dev || !added) return cfail(SBK_ERR_ARGUMENT, "null argument");
  cudaStream_t st = c->stream;
  int base = c->num_blocks;
  int total = 0;
  for (size_t k = 0; k < c->tools.size(); ++k) {
    HostTool& h = c->tools[k];
    if (!c->active[k] || h.nslaves == 0) continue;
    double cc[3];
    h.position(t, cc);
    const int blocks = (h.nslaves + 127) / 128;
    anticipate_kernel<<<blocks, 128, 0, st>>>(h.d, h.nodes, h.area, h.kappa, h.cand, h.ncand, c->coords, u_dev,
                                              du_dev, cc[0], cc[1], cc[2], h.act, h.ek, h.enode, h.eforce);
    // Slots past the candidate count are never written: clear their flags.
    int32_t nc = 0;
    SBK_C(cudaMemcpyAsync(&nc, h.ncand, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SBK_C(cudaStreamSynchronize(st));
    if (nc < h.nslaves) SBK_C(cudaMemsetAsync(h.act + nc, 0, h.nslaves - nc, st));
    ordered_compact(h.nslaves, h.act, h.alist, h.nalist, h.cblocks, st);
    int32_t n = 0;
    SBK_C(cudaMemcpyAsync(&n, h.nalist, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SBK_C(cudaStreamSynchronize(st));
    if (base + n > c->capacity) return cfail(SBK_ERR_ARGUMENT, "contact block capacity exceeded");
    anticipate_scatter_kernel<<<(h.nslaves + 127) / 128, 128, 0, st>>>(h.alist, h.nalist, h.enode, h.eforce, h.ek,
                                                                       residual_dev, c->block_nodes, c->blocks,
                                                                       base);
    base += n;
    total += n;
  }
  SBK_C(cudaGetLastError());
  SBK_C(cudaStreamSynchronize(st));
  c->num_blocks = base;
  *added = total;
  if (out) {
    out->block_nodes_dev = c->block_nodes;
    out->blocks_dev = c->blocks;
    out->num_blocks = base;
  }
  return SBK_OK;
}

int sbk_contact_commit(sbk_contact* c) {
  if (!c) return cfail(SBK_ERR_ARGUMENT, "null contact");
  cudaStream_t st = c->stream;
  for (size_t k = 0; k < c->tools.size(); ++k) {
    HostTool& h = c->tools[k];
    if (!c->active[k] || h.nslaves == 0) continue;
    SBK_C(cudaMemcpyAsync(h.h_flag, h.t_flag, h.nslaves, cudaMemcpyDeviceToDevice, st));
    SBK_C(cudaMemcpyAsync(h.h_force, h.t_force, 3 * h.nslaves * sizeof(double), cudaMemcpyDeviceToDevice, st));
    SBK_C(cudaMemcpyAsync(h.h_rel, h.t_rel, 3 * h.nslaves * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  return SBK_OK;
}

int sbk_contact_history(const sbk_contact* c, int32_t k, int32_t max_entries, double* out, int32_t* count) {
  if (!c || !count || k < 0 || k >= static_cast<int32_t>(c->tools.size())) return cfail(SBK_ERR_ARGUMENT, "bad tool");
  const HostTool& h = c->tools[k];
  std::vector<uint8_t> f(std::max(1, h.nslaves));
  std::vector<double> force(3 * std::max(1, h.nslaves)), rel(3 * std::max(1, h.nslaves));
  std::vector<int32_t> nodes(std::max(1, h.nslaves));
  SBK_C(cudaStreamSynchronize(c->stream));
  if (h.nslaves > 0) {
    SBK_C(cudaMemcpy(f.data(), h.h_flag, h.nslaves, cudaMemcpyDeviceToHost));
    SBK_C(cudaMemcpy(force.data(), h.h_force, 3 * h.nslaves * sizeof(double), cudaMemcpyDeviceToHost));
    SBK_C(cudaMemcpy(rel.data(), h.h_rel, 3 * h.nslaves * sizeof(double), cudaMemcpyDeviceToHost));
    SBK_C(cudaMemcpy(nodes.data(), h.nodes, h.nslaves * sizeof(int32_t), cudaMemcpyDeviceToHost));
  }
  int32_t n = 0;
  for (int i = 0; i < h.nslaves; ++i) {
    if (!f[i]) continue;
    if (out && n < max_entries) {
      double* o = out + 7 * n;
      o[0] = nodes[i];
      for (int r = 0; r < 3; ++r) {
        o[1 + r] = force[3 * i + r];
        o[4 + r] = rel[3 * i + r];
      }
    }
    ++n;
  }
  *count = n;
  return SBK_OK;
}

}  // extern "C"
