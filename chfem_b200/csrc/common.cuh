// common.cuh -- shared definitions of the chfem_b200 solver library (sm_100a).
//
// Geometry conventions follow chfem exactly so that vectors crossing the cudapcg C ABI
// keep the reference's layout:
//   * node / voxel index i = row + col*nrows + layer*nrows*ncols, row (= -y) fastest
//     (chfem/src/femhmg/cudapcg/kernels/utils.h:82);
//   * local node k of a voxel element sits at (row,col,layer) offset
//     (drow,dcol,dlay)(k) from local node 0, with local node 0 = (0,0,0), 1 = (0,+1,0),
//     2 = (-1,+1,0), 3 = (-1,0,0) and 4..7 the same one layer further
//     (chfem/src/femhmg/cudapcg/kernels/matrix_free.cu:147-160);
//   * the per-node material key packs the material of the element in which the node is
//     local node e into bits [2e, 2e+2) (chfem/src/femhmg/physical_phenomena/femhmg_3D.c:19-75).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace chfem {

// ---- element geometry, usable in constant expressions after unrolling ----------------
__host__ __device__ constexpr int drow(int k) { return -((k & 3) >> 1); }
__host__ __device__ constexpr int dcol(int k) { return ((k & 3) == 1 || (k & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int dlay(int k) { return k >> 2; }
// Nodes a and b of one element share an edge when they differ along exactly one axis;
// the Q1 conductivity matrix is zero exactly there.
__host__ __device__ constexpr bool shares_edge(int a, int b) {
  return ((drow(a) != drow(b)) + (dcol(a) != dcol(b)) + (dlay(a) != dlay(b))) == 1;
}

__host__ __device__ inline int wrap(int v, int n) { v %= n; return v < 0 ? v + n : v; }

// L2 prefetch of [p, p + bytes) rounded out to 16-byte boundaries (sm_90+ bulk prefetch); the
// rounded range stays inside the 16-byte granules of the buffer it starts in
__device__ __forceinline__ void asm_prefetch_l2(const void* p, size_t bytes) {
  const size_t a0 = (size_t)p & ~(size_t)15, a1 = ((size_t)p + bytes + 15) & ~(size_t)15;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a0), "r"((unsigned)(a1 - a0)) : "memory");
}

// ---- solver scalars living on the device (one record per right-hand side) -----------
struct DevScalars {
  double delta;      // current r^T M^-1 r (PCG) or (M^-1 r)^T A (M^-1 r) (PMINRES)
  double delta0;     // zero-guess value, the stopping reference
  double delta_old;
  double alpha;
  double beta;
  double res0;       // stopping reference for the INF / PMINRES norms
  double metric;     // last stopping metric
  double red[6];     // scratch results of the last reductions
  int iteration;
  int done;          // 1 once the stopping test passed or max iterations were reached
  int found;         // 1 when the stopping test passed
  int status;        // 0 ok, else an error code
};

// ---- block-wide FP64 reduction helpers ---------------------------------------------
template <int NT>
__device__ inline double block_sum(double v, double* sred) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x / 32 + (threadIdx.y * blockDim.x) / 32, lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
  (void)warp;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  if (lane == 0) sred[tid >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (tid < 32) {
    t = (tid < NT / 32) ? sred[tid] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;  // valid in thread 0
}
template <int NT>
__device__ inline double block_max(double v, double* sred) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tid = threadIdx.x + threadIdx.y * blockDim.x, lane = tid & 31;
  if (lane == 0) sred[tid >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (tid < 32) {
    t = (tid < NT / 32) ? sred[tid] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
  }
  __syncthreads();
  return t;
}

// Grid-level reduction control.  Every block writes its partials to part[k*nblocks+b];
// the last block to arrive (ticket counter) reduces them in block order, so results are
// deterministic run to run, and then runs the caller's finisher.  No thread ever waits
// on another block.
struct RedCtl {
  double* part;        // [NRED][nblocks]
  unsigned int* ticket;
  int nblocks;
};

template <int NT, int NRED>
__device__ inline bool grid_reduce(const double (&v)[NRED], const bool (&is_max)[NRED], RedCtl rc, int bid, double (&out)[NRED], double* sred) {
  double b[NRED];
#pragma unroll
  for (int k = 0; k < NRED; k++) b[k] = is_max[k] ? block_max<NT>(v[k], sred) : block_sum<NT>(v[k], sred);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  __shared__ unsigned int s_last;
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NRED; k++) rc.part[k * rc.nblocks + bid] = b[k];
    __threadfence();
    unsigned int t = atomicAdd(rc.ticket, 1u);
    s_last = (t == (unsigned int)rc.nblocks - 1u);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NRED; k++) {
    double acc = 0.0;
    // fixed order: thread tid sums blocks tid, tid+NT, ... then a fixed-shape tree
    for (int j = tid; j < rc.nblocks; j += NT) {
      double p = __ldcg(rc.part + k * rc.nblocks + j);
      acc = is_max[k] ? fmax(acc, p) : acc + p;
    }
    out[k] = is_max[k] ? block_max<NT>(acc, sred) : block_sum<NT>(acc, sred);
  }
  if (tid == 0) *rc.ticket = 0u;
  return true;  // out[] valid in thread 0 of the last block
}

}  // namespace chfem
