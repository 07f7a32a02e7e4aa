// pore_maps.cu -- the Stokes DOF-number maps built on the device from the voxel image.
//
// The reference numbers the unknowns on the host (chfem/src/femhmg/physical_phenomena/
// femhmg_fluid_3D.c:370-491): node i gets an 8-bit fluid key (bit e set when the voxel in which
// i is local node e is pore, i.e. material 0); nodes with key 255 (all 8 voxels pore) are
// numbered first, in node order, then the interface nodes (0 < key < 255), in node order; DOF
// d's node is node_of_dof[d]; interface DOF d keeps its key in border_keys[d - nV].  Here the
// same numbering is a stable two-class compaction: per chunk of PM_CHUNK nodes the CTA counts
// both classes, one CTA scans the chunk counts, and each chunk then numbers its nodes from its
// offsets with a CTA-wide scan -- every node keeps its rank in node order within its class, so
// the maps are equal to the host's bit for bit.
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"
#include "pore_maps.h"

namespace chfem {

constexpr int PM_NT = 1024;               // threads per CTA
constexpr int PM_PER = 4;                 // consecutive nodes per thread
constexpr int PM_CHUNK = PM_NT * PM_PER;  // nodes per chunk

// fluid key of every node from the colours (x fastest in the file, refinement^3 model voxels
// per image voxel; the node's voxel e sits at (row - drow(e) - 1, col - dcol(e), layer - dlay(e)))
__global__ void k_fluid_keys(const uint8_t* colors, PoreColorMap cm, uint8_t* fk, int R, int C, int L, int ref, int* bad) {
  const long N = (long)R * C * L;
  const int frows = R / ref, fcols = C / ref;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    unsigned k = 0;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int vr = wrap(r - drow(e) - 1, R), vc = wrap(c - dcol(e), C), vl = wrap(l - dlay(e), L);
      const long f = (long)(vl / ref) * frows * fcols + (long)(vr / ref) * fcols + vc / ref;
      const int m = cm.mat[colors[f]];
      if (m < 0) { *bad = 1; continue; }
      k |= (unsigned)(m == 0) << e;
    }
    fk[i] = (uint8_t)k;
  }
}

// CTA-wide exclusive scan of two counters (warp shuffles, then the warps' totals)
__device__ inline void pm_scan2(unsigned& a, unsigned& b, unsigned& ta, unsigned& tb, unsigned* sa, unsigned* sb) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned ia = a, ib = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned xa = __shfl_up_sync(0xffffffffu, ia, o), xb = __shfl_up_sync(0xffffffffu, ib, o);
    if (lane >= o) { ia += xa; ib += xb; }
  }
  if (lane == 31) { sa[warp] = ia; sb[warp] = ib; }
  __syncthreads();
  if (warp == 0) {
    unsigned wa = sa[lane], wb = sb[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned xa = __shfl_up_sync(0xffffffffu, wa, o), xb = __shfl_up_sync(0xffffffffu, wb, o);
      if (lane >= o) { wa += xa; wb += xb; }
    }
    sa[lane] = wa; sb[lane] = wb;  // inclusive over warps
  }
  __syncthreads();
  const unsigned wa0 = warp ? sa[warp - 1] : 0u, wb0 = warp ? sb[warp - 1] : 0u;
  ta = sa[PM_NT / 32 - 1]; tb = sb[PM_NT / 32 - 1];
  a = wa0 + ia - a;  // exclusive
  b = wb0 + ib - b;
  __syncthreads();
}

// per chunk: pore nodes (key 255) and interface nodes (0 < key < 255)
__global__ void __launch_bounds__(PM_NT) k_pore_count(const uint8_t* fk, long N, unsigned* cnt) {
  __shared__ unsigned sa[32], sb[32];
  const long base = (long)blockIdx.x * PM_CHUNK + (long)threadIdx.x * PM_PER;
  unsigned a = 0, b = 0;
#pragma unroll
  for (int j = 0; j < PM_PER; j++) {
    const long i = base + j;
    if (i < N) { const unsigned k = fk[i]; a += (k == 255u); b += (k != 0u && k != 255u); }
  }
  unsigned ta, tb;
  pm_scan2(a, b, ta, tb, sa, sb);
  if (threadIdx.x == 0) { cnt[2 * blockIdx.x] = ta; cnt[2 * blockIdx.x + 1] = tb; }
}

// exclusive scan of the chunk counts in place (one CTA); totals[0..1] = pore, interface nodes
__global__ void __launch_bounds__(PM_NT) k_pore_scan(unsigned* cnt, long nchunks, unsigned long long* totals) {
  __shared__ unsigned sa[32], sb[32];
  unsigned long long ca = 0, cb = 0;
  for (long s = 0; s < nchunks; s += PM_NT) {
    const long c = s + threadIdx.x;
    unsigned a = c < nchunks ? cnt[2 * c] : 0u, b = c < nchunks ? cnt[2 * c + 1] : 0u;
    unsigned ta, tb;
    pm_scan2(a, b, ta, tb, sa, sb);
    if (c < nchunks) { cnt[2 * c] = (unsigned)(ca + a); cnt[2 * c + 1] = (unsigned)(cb + b); }
    ca += ta;
    cb += tb;
  }
  if (threadIdx.x == 0) { totals[0] = ca; totals[1] = cb; }
}

// the numbering: pore node -> its rank among pore nodes; interface node -> nV + its rank among
// interface nodes; solid nodes -> 0 (the host's initial value)
__global__ void __launch_bounds__(PM_NT) k_pore_number(const uint8_t* fk, long N, const unsigned* off, unsigned nV,
                                                       uint32_t* dof_of_node, uint32_t* node_of_dof, uint8_t* border_keys) {
  __shared__ unsigned sa[32], sb[32];
  const long base = (long)blockIdx.x * PM_CHUNK + (long)threadIdx.x * PM_PER;
  uint8_t k[PM_PER];
  unsigned a = 0, b = 0;
#pragma unroll
  for (int j = 0; j < PM_PER; j++) {
    const long i = base + j;
    k[j] = i < N ? fk[i] : (uint8_t)0;
    a += (k[j] == 255u);
    b += (k[j] != 0u && k[j] != 255u);
  }
  unsigned ta, tb;
  pm_scan2(a, b, ta, tb, sa, sb);
  unsigned pa = off[2 * blockIdx.x] + a, pb = nV + off[2 * blockIdx.x + 1] + b;
#pragma unroll
  for (int j = 0; j < PM_PER; j++) {
    const long i = base + j;
    if (i >= N) break;
    uint32_t d = 0;
    if (k[j] == 255u) d = pa++;
    else if (k[j] != 0u) { d = pb++; border_keys[d - nV] = k[j]; }
    dof_of_node[i] = d;
    if (k[j]) node_of_dof[d] = (uint32_t)i;
  }
}

bool pore_maps_count(const uint8_t* d_colors, const PoreColorMap& cm, int R, int C, int L, int ref, uint8_t* d_fk,
                     unsigned* d_cnt, unsigned long long* d_tot, int* d_bad, unsigned long long* nV, unsigned long long* nB,
                     cudaStream_t st, const char** err) {
  const long N = (long)R * C * L;
  const long nchunks = (N + PM_CHUNK - 1) / PM_CHUNK;
  int bad = 0;
  unsigned long long tot[2] = {0, 0};
  cudaError_t e = cudaMemsetAsync(d_bad, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    const long g = std::min<long>((N + 255) / 256, 8L * 148);
    k_fluid_keys<<<(int)std::max(1L, g), 256, 0, st>>>(d_colors, cm, d_fk, R, C, L, ref, d_bad);
    k_pore_count<<<(int)nchunks, PM_NT, 0, st>>>(d_fk, N, d_cnt);
    k_pore_scan<<<1, PM_NT, 0, st>>>(d_cnt, nchunks, d_tot);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) { *err = cudaGetErrorString(e); return false; }
  if (bad) { *err = "the image holds a colour without a material"; return false; }
  *nV = tot[0];
  *nB = tot[1];
  return true;
}

bool pore_maps_number(const uint8_t* d_fk, int R, int C, int L, const unsigned* d_cnt, unsigned nV, uint32_t* d_dof_of_node,
                      uint32_t* d_node_of_dof, uint8_t* d_border, cudaStream_t st, const char** err) {
  const long N = (long)R * C * L;
  const long nchunks = (N + PM_CHUNK - 1) / PM_CHUNK;
  k_pore_number<<<(int)nchunks, PM_NT, 0, st>>>(d_fk, N, d_cnt, nV, d_dof_of_node, d_node_of_dof, d_border);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { *err = cudaGetErrorString(e); return false; }
  return true;
}

long pore_maps_chunks(long N) { return (N + PM_CHUNK - 1) / PM_CHUNK; }

}  // namespace chfem
