// stencil_el.cuh -- the elastic (3 DOF/node) voxel operator with vector shared-memory
// layouts.  Same arithmetic as te_node<3,T> (chfem/src/femhmg/cudapcg/kernels/matrix_free.cu:
// 410-459: per node, 8 voxels x one 3x24 row block of the voxel's 24x24 stiffness), but
// laid out so every shared-memory access is a 128-bit load:
//   * each 3x3 block K[3e+ci][3b+cj] of a material is stored as three 4-wide rows
//     (the 4th lane zero), so one (voxel e, local node b) pair costs three vector loads;
//   * field values are stored 4-wide per node (x, y, z, 0), one vector load per neighbour.
// The measured bound of the scalar layout was the shared-memory load pipe (one 32-bit load
// per FMA); this layout cuts the load instructions per node from ~770 to ~220.
#pragma once
#include "common.cuh"
#include "stencil_te.cuh"

namespace chfem {

template <typename T> struct V4;
template <> struct V4<float> {
  float4 v;
  __device__ __forceinline__ float x() const { return v.x; }
  __device__ __forceinline__ float y() const { return v.y; }
  __device__ __forceinline__ float z() const { return v.z; }
  __device__ __forceinline__ void set(float a, float b, float c) { v = make_float4(a, b, c, 0.f); }
};
template <> struct V4<double> {
  double2 a, b;
  __device__ __forceinline__ double x() const { return a.x; }
  __device__ __forceinline__ double y() const { return a.y; }
  __device__ __forceinline__ double z() const { return b.x; }
  __device__ __forceinline__ void set(double p, double q, double r) { a = make_double2(p, q); b = make_double2(r, 0.0); }
};

constexpr int EL_BLK = 64 * 3;        // vector rows per material: 8 x 8 blocks x 3 rows
constexpr int EL_KST = EL_BLK + 1;    // padded material stride (spreads materials over banks)

template <typename T>
inline size_t el_smem_bytes() {
  return (size_t)4 * EL_KST * sizeof(V4<T>) + (size_t)3 * TE_PP * sizeof(V4<T>) + 32;
}

template <typename T>
__device__ __forceinline__ void el_node(const V4<T>* __restrict__ sK, unsigned key, const V4<T>* pm, const V4<T>* p0,
                                        const V4<T>* pp, int ctr, T& o0, T& o1, T& o2) {
  o0 = T(0); o1 = T(0); o2 = T(0);
#pragma unroll
  for (int e = 0; e < 8; e++) {
    const V4<T>* K = sK + ((key >> (2 * e)) & 3u) * EL_KST + e * 24;
#pragma unroll
    for (int b = 0; b < 8; b++) {
      const int dr = drow(b) - drow(e), dc = dcol(b) - dcol(e), dl = dlay(b) - dlay(e);
      const V4<T>* P = dl < 0 ? pm : (dl == 0 ? p0 : pp);
      const V4<T> v = P[ctr + dr + dc * TE_PR];
      const V4<T> k0 = K[3 * b], k1 = K[3 * b + 1], k2 = K[3 * b + 2];
      o0 = fma(k0.x(), v.x(), fma(k0.y(), v.y(), fma(k0.z(), v.z(), o0)));
      o1 = fma(k1.x(), v.x(), fma(k1.y(), v.y(), fma(k1.z(), v.z(), o1)));
      o2 = fma(k2.x(), v.x(), fma(k2.y(), v.y(), fma(k2.z(), v.z(), o2)));
    }
  }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(TE_NT) k_el_apply(TeArgs<3, T> a) {
  constexpr int ED = 24;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[TE_NT / 32];
  __shared__ T sD[4 * 24];
  if (a.skip_if_done && a.sc->done) return;
  V4<T>* sK = reinterpret_cast<V4<T>*>(smem_raw);
  V4<T>* sP = sK + 4 * EL_KST;
  const int tid = threadIdx.x + TE_TR * threadIdx.y;
  // blocks: row index e (local node of the row), column index b, rows ci
  for (int i = tid; i < 4 * EL_BLK; i += TE_NT) {
    const int m = i / EL_BLK, rem = i % EL_BLK, e = rem / 24, b = (rem % 24) / 3, ci = rem % 3;
    V4<T> row;
    if (m < a.nmat) {
      const T* Kr = a.Kd + (size_t)m * ED * ED + (size_t)(3 * e + ci) * ED + 3 * b;
      row.set(Kr[0], Kr[1], Kr[2]);
    } else {
      row.set(T(0), T(0), T(0));
    }
    sK[m * EL_KST + rem] = row;
  }
  if (MODE == TE_MR) {
    for (int i = tid; i < 4 * 24; i += TE_NT) {
      const int m = i / 24, k = i % 24;
      sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)k * ED + k] : T(1);
    }
  }
  __syncthreads();
  const T beta = (MODE == TE_PCG) ? T(a.sc->beta) : T(0);
  const T alpha = (MODE == TE_MR) ? T(a.sc->alpha) : T(0);
  const bool pre = a.cfg.precond != 0;
  const int R = a.R, C = a.C, L = a.L;
  const int r0 = blockIdx.x * TE_TR, c0 = blockIdx.y * TE_TC, l0 = blockIdx.z * a.lchunk;
  const int l1 = min(l0 + a.lchunk, L);
  const size_t RC = (size_t)R * C;

  auto slot_of = [&](int l) { return ((l % 3) + 3) % 3; };
  auto load_plane = [&](int l) {
    const int lw = wrap(l, L);
    V4<T>* dst = sP + slot_of(l) * TE_PP;
    for (int p = tid; p < TE_PP; p += TE_NT) {
      const int hr = p % TE_PR, hc = p / TE_PR;
      const int gr = wrap(r0 + hr - 1, R), gc = wrap(c0 + hc - 1, C);
      const size_t node = (size_t)gr + (size_t)gc * R + (size_t)lw * RC;
      T v[3];
#pragma unroll
      for (int c = 0; c < 3; c++) v[c] = a.in0[node * 3 + c];
      if (MODE == TE_PCG) {
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = fma(beta, a.in1[node * 3 + c], v[c]);
      }
      if (MODE == TE_MR) {
        T inv[3] = {T(1), T(1), T(1)};
        if (pre) te_invdiag<3, T>(sD, a.keys[node], inv);
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = fma(-alpha, a.in1[node * 3 + c], v[c]) * inv[c];
      }
      dst[p].set(v[0], v[1], v[2]);
    }
  };

  load_plane(l0 - 1);
  load_plane(l0);
  double acc = 0.0, acc_rz = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  const int r = r0 + threadIdx.x, c = c0 + threadIdx.y;
  const bool active = (r < R) && (c < C);
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * TE_PR;
  for (int l = l0; l < l1; l++) {
    load_plane(l + 1);
    __syncthreads();
    if (active) {
      const size_t node = (size_t)r + (size_t)c * R + (size_t)l * RC;
      const unsigned key = a.keys[node];
      const V4<T>* pm = sP + slot_of(l - 1) * TE_PP;
      const V4<T>* p0 = sP + slot_of(l) * TE_PP;
      const V4<T>* pp = sP + slot_of(l + 1) * TE_PP;
      T out[3];
      el_node<T>(sK, key, pm, p0, pp, ctr, out[0], out[1], out[2]);
      const V4<T> vc = p0[ctr];
      const T vv[3] = {vc.x(), vc.y(), vc.z()};
#pragma unroll
      for (int cc = 0; cc < 3; cc++) {
        const size_t j = node * 3 + cc;
        a.y[j] = out[cc];
        if (MODE == TE_PCG) a.vout[j] = vv[cc];
        if (MODE == TE_MR) {
          const T rn = fma(-alpha, a.in1[j], a.in0[j]);
          a.vout[j] = rn;
          const T dv = a.d[j];
          const double xv = fma((double)alpha, (double)dv, a.x[j]);
          a.x[j] = xv;
          acc_rz += (double)rn * (double)vv[cc];
          mr = fmax(mr, fabs((double)rn));
          md = fmax(md, fabs((double)dv));
          mx = fmax(mx, fabs(xv));
        }
        acc += (double)vv[cc] * (double)out[cc];
      }
    }
    __syncthreads();
  }
  if (a.finish == FIN_NONE) return;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (MODE == TE_MR) {
    const double vals[5] = {acc, acc_rz, mr, md, mx};
    const bool ismax[5] = {false, false, true, true, true};
    double out[5];
    if (grid_reduce<TE_NT, 5>(vals, ismax, a.rc, bid, out, sred) && tid == 0) {
      for (int k = 0; k < 5; k++) a.sc->red[k] = out[k];
      mr_finish(a.finish, out, a.sc, a.cfg);
    }
  } else {
    const double vals[1] = {acc};
    const bool ismax[1] = {false};
    double out[1];
    if (grid_reduce<TE_NT, 1>(vals, ismax, a.rc, bid, out, sred) && tid == 0) {
      a.sc->red[0] = out[0];
      if (a.finish == FIN_ALPHA) a.sc->alpha = a.sc->delta / out[0];
    }
  }
}

}  // namespace chfem
