// loadcase.cuh -- homogenization load cases on the device: the right-hand side of a periodic
// load case and the volume term of the effective tensor, so that a native homogenization run
// never moves full-length vectors between host and device.
//
// Thermal / elastic (chfem/src/femhmg/physical_phenomena/femhmg_thermal_3D.c:122-236,
// femhmg_elastic_3D.c:130-511): the macroscopic jump along `axis` enters through the voxels on
// the +axis boundary of the cell (last column for x, first row for y, first layer for z), as
// b_n -= jump * sum over the 4 +axis face nodes f of K(node n, f; component comp).  Evaluated
// node by node: the node key gives the material of each of the node's 8 voxels, so every node
// gathers its own contributions (no atomics).
// Effective tensor (femhmg_thermal_3D.c:355-500, femhmg_elastic_3D.c:1075-1343): the volume
// term sum over voxels of CB_e x_e, rearranged per node as sum_k CB[mat_k](rows, k) x_n.
// Stokes (femhmg_fluid_3D.c:112-182, :184-285): unit body force along the flow direction on the
// velocity DOFs of pore nodes (all 8 voxels fluid), and the mean velocity as a weighted sum.
#pragma once
#include "common.cuh"
#include "stencil_te.cuh"

namespace chfem {

// local nodes on the +x, +y, +z faces of a voxel
__host__ __device__ constexpr int face_node(int axis, int f) {
  return axis == 0 ? (f == 0 ? 1 : f == 1 ? 2 : f == 2 ? 5 : 6) : axis == 1 ? (f + 2 + (f >= 2 ? 2 : 0)) : f;
}

template <int ND, typename T>
__global__ void k_rhs_load_case(const uint16_t* keys, const double* Kd, int R, int C, int L, int axis, int comp, double jump,
                                double* b, T* r) {
  constexpr int ED = 8 * ND;
  const long N = (long)R * C * L;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x) {
    const int rr = (int)(n % R), cc = (int)((n / R) % C), ll = (int)(n / ((long)R * C));
    const unsigned key = keys[n];
    double v[ND];
#pragma unroll
    for (int ci = 0; ci < ND; ci++) v[ci] = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      // the voxel in which this node is local node k
      const int er = wrap(rr - drow(k) - 1, R), ec = wrap(cc - dcol(k), C), el = wrap(ll - dlay(k), L);
      const bool boundary = axis == 0 ? ec == C - 1 : (axis == 1 ? er == 0 : el == 0);
      if (!boundary) continue;
      const double* K = Kd + (size_t)((key >> (2 * k)) & 3u) * ED * ED;
#pragma unroll
      for (int ci = 0; ci < ND; ci++) {
        double s = 0.0;
        for (int f = 0; f < 4; f++) s += K[(k * ND + ci) * ED + face_node(axis, f) * ND + comp];
        v[ci] -= s * jump;
      }
    }
#pragma unroll
    for (int ci = 0; ci < ND; ci++) {
      b[n * ND + ci] = v[ci];
      r[n * ND + ci] = T(v[ci]);
    }
  }
}

// out[s] = sum_n sum_k sum_ci CB[mat_k(n)][s][k ND + ci] x[n ND + ci], s < NS (3 thermal, 6 elastic);
// CB: [4][NS][8 ND] in device memory (material slots past nmat unused).
template <int ND, int NS>
__global__ void __launch_bounds__(PW_NT) k_cb_moments(const uint16_t* keys, const double* CB, const double* x, long N, RedCtl rc,
                                                      double* out) {
  constexpr int EC = 8 * ND;
  __shared__ double sCB[4 * NS * EC];
  __shared__ double sred[PW_NT / 32];
  for (int i = threadIdx.x; i < 4 * NS * EC; i += PW_NT) sCB[i] = CB[i];
  __syncthreads();
  double acc[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) acc[s] = 0.0;
  for (long n = blockIdx.x * (long)PW_NT + threadIdx.x; n < N; n += (long)gridDim.x * PW_NT) {
    const unsigned key = keys[n];
    double xv[ND];
#pragma unroll
    for (int ci = 0; ci < ND; ci++) xv[ci] = x[n * ND + ci];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const double* cb = sCB + ((key >> (2 * k)) & 3u) * NS * EC + k * ND;
#pragma unroll
      for (int s = 0; s < NS; s++)
#pragma unroll
        for (int ci = 0; ci < ND; ci++) acc[s] = fma(cb[s * EC + ci], xv[ci], acc[s]);
    }
  }
  bool ismax[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) ismax[s] = false;
  double res[NS];
  if (grid_reduce<PW_NT, NS>(acc, ismax, rc, blockIdx.x, res, sred) && threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; s++) out[s] = res[s];
  }
}

// Stokes: b = w on the velocity component `dir` of every pore node, 0 elsewhere.
template <typename T>
__global__ void k_fl_rhs(long nV, long n, int dir, double w, double* b, T* r) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double v = (i < 3 * nV && (int)(i % 3) == dir) ? w : 0.0;
    b[i] = v;
    r[i] = T(v);
  }
}

// Stokes: out[j] = w_j * sum over pore nodes of the velocity component j.
static __global__ void __launch_bounds__(PW_NT) k_fl_moments(const double* x, long nV, double w0, double w1, double w2, RedCtl rc, double* out) {
  __shared__ double sred[PW_NT / 32];
  double acc[3] = {0.0, 0.0, 0.0};
  for (long t = blockIdx.x * (long)PW_NT + threadIdx.x; t < nV; t += (long)gridDim.x * PW_NT) {
    acc[0] += x[3 * t];
    acc[1] += x[3 * t + 1];
    acc[2] += x[3 * t + 2];
  }
  const bool ismax[3] = {false, false, false};
  double res[3];
  if (grid_reduce<PW_NT, 3>(acc, ismax, rc, blockIdx.x, res, sred) && threadIdx.x == 0) {
    out[0] = w0 * res[0]; out[1] = w1 * res[1]; out[2] = w2 * res[2];
  }
}

}  // namespace chfem
