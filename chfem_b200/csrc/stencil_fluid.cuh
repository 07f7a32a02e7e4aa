// stencil_fluid.cuh -- matrix-free Stokes operator (4 DOF per pore node: 3 velocities and
// a pressure; interface nodes carry a pressure only), on the DOF-number pore map of the
// reference (chfem/src/femhmg/physical_phenomena/femhmg_fluid_3D.c:370-424): pore nodes
// (all 8 voxels fluid) are numbered first in ascending node order, then interface nodes.
// Vector layout: [3*nVel interleaved velocities | nVel+nBorder pressures]
// (matrix_free.cu:5012-5047).  Rows follow matrix_free.cu:674-732 (pore) and :926-977
// (interface): the 32x32 stabilised Q1-Q1 element matrix [K G; G^T Stab] enters as
// [K G; G^T -Stab], velocity columns of non-pore neighbours are dropped (no slip).
//
// B200 design: one thread per unknown row set (pore node or interface node); the 27
// neighbours are gathered once each through the node->DOF map and every (voxel, local node)
// pair that lands on a neighbour is accumulated while its values are in registers.  The
// element matrix is uniform across the warp, so it lives in __constant__ memory and every
// coefficient is a broadcast operand.
#pragma once
#include "common.cuh"
#include "stencil_te.cuh"
#include "pointwise.cuh"

namespace chfem {

constexpr int FL_NT = 256;

template <typename T>
struct FlArgs {
  const T* v;          // PLAIN: field | PCG: s | MR: r
  const T* vd;         // PCG: d_old | MR: q
  T* vout;             // PCG: formed direction | MR: updated residual r'
  T* y;
  double* x;           // MR: x += alpha d (FP64 in every precision mode)
  const T* d;          // MR
  const uint32_t* dof_of_node;   // periodic2DOF_map
  const uint32_t* node_of_dof;   // DOF2periodic_map
  const uint8_t* bkeys;          // fluid keys of interface nodes
  int R, C, L;
  long nV, nB;
  DevScalars* sc;
  RedCtl rc;
  int finish;          // TeFinish codes
  int skip_if_done;
  MrCfg cfg;
};

__constant__ double c_flK64[1024];
__constant__ float c_flK32[1024];

template <typename T> __device__ __forceinline__ T flK(int i);
template <> __device__ __forceinline__ double flK<double>(int i) { return c_flK64[i]; }
template <> __device__ __forceinline__ float flK<float>(int i) { return c_flK32[i]; }

// Jacobi inverse diagonal of a row set: pore rows have fixed values (all 8 voxels fluid);
// interface rows depend on their fluid key.  Tabulated on the host (256 keys).
struct FlDiag {
  double pore[4];
  double border[256];
};
__constant__ FlDiag c_fldiag;

// Value of the operator's input at DOF `dof` (component comp: 0..DIM-1 velocity, DIM pressure),
// formed per MODE.  `off` is the vector offset of that entry.
template <typename T, int MODE>
__device__ __forceinline__ T fl_in(const FlArgs<T>& a, size_t off, T beta, T alpha, T inv) {
  T v = a.v[off];
  if (MODE == TE_PCG) v = fma(beta, a.vd[off], v);
  if (MODE == TE_MR) v = fma(-alpha, a.vd[off], v) * inv;
  return v;
}

// DIM = 3: voxels, 8 elements, 27 neighbours, element matrix 32 x 32 (3 velocities + pressure
// per node); DIM = 2: pixels (one layer), 4 elements, 9 neighbours, 12 x 12 (2 velocities +
// pressure; matrix_free.cu:484-518 pore rows, :628-660 interface rows).  Vector layout
// [DIM nVel interleaved velocities | nVel + nBorder pressures].
template <typename T, int MODE, int DIM = 3>
__global__ void __launch_bounds__(FL_NT) k_fl_apply(FlArgs<T> a) {
  constexpr int NE = 1 << DIM, ED = (DIM + 1) * NE, PC = DIM * NE, NO = DIM == 3 ? 27 : 9;
  constexpr unsigned FULL = (1u << NE) - 1u;
  __shared__ double sred[FL_NT / 32];
  __shared__ T sbd[256];  // interface-node inverse diagonals by fluid key (per-thread keys: shared, not constant, memory)
  if (a.skip_if_done && a.sc->done) return;
  for (int i = threadIdx.x; i < 256; i += FL_NT) sbd[i] = T(c_fldiag.border[i]);
  __syncthreads();
  const long nV = a.nV, nT = a.nV + a.nB;
  const int R = a.R, C = a.C, L = a.L;
  const T beta = (MODE == TE_PCG) ? T(a.sc->beta) : T(0);
  const T alpha = (MODE == TE_MR && mr_steps(a.finish)) ? T(a.sc->alpha) : T(0);
  const bool pre = a.cfg.precond != 0;
  T ivv[DIM];
#pragma unroll
  for (int k = 0; k < DIM; k++) ivv[k] = pre ? T(c_fldiag.pore[k]) : T(1);
  const T ivp = pre ? T(c_fldiag.pore[DIM]) : T(1);
  double acc = 0.0, acc_rz = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  for (long t = blockIdx.x * (long)FL_NT + threadIdx.x; t < nT; t += (long)gridDim.x * FL_NT) {
    const uint32_t node = a.node_of_dof[t];
    const int r = (int)(node % (uint32_t)R), c = (int)((node / (uint32_t)R) % (uint32_t)C), l = (int)(node / ((uint32_t)R * (uint32_t)C));
    const bool pore = t < nV;
    const unsigned fk = pore ? FULL : a.bkeys[t - nV];
    const int rr[3] = {wrap(r - 1, R), r, wrap(r + 1, R)};
    const int cc[3] = {wrap(c - 1, C), c, wrap(c + 1, C)};
    const int ll[3] = {wrap(l - 1, L), l, wrap(l + 1, L)};
    T ov[DIM], op = 0;
#pragma unroll
    for (int k = 0; k < DIM; k++) ov[k] = 0;
#pragma unroll
    for (int o = 0; o < NO; o++) {
      const int orr = o % 3 - 1, occ = (o / 3) % 3 - 1, oll = DIM == 3 ? o / 9 - 1 : 0;
      // elements of this node that also contain the neighbour
      unsigned emask = 0;
#pragma unroll
      for (int e = 0; e < NE; e++)
#pragma unroll
        for (int b = 0; b < NE; b++)
          if (drow(b) - drow(e) == orr && dcol(b) - dcol(e) == occ && dlay(b) - dlay(e) == oll) emask |= 1u << e;
      if (!(fk & emask)) continue;
      const uint32_t nb = (uint32_t)rr[orr + 1] + (uint32_t)cc[occ + 1] * (uint32_t)R + (uint32_t)ll[oll + 1] * (uint32_t)R * (uint32_t)C;
      const uint32_t dof = a.dof_of_node[nb];
      T vv[DIM];
#pragma unroll
      for (int k = 0; k < DIM; k++) vv[k] = 0;
      const bool vel = dof < (uint32_t)nV;
      if (vel) {
#pragma unroll
        for (int k = 0; k < DIM; k++) vv[k] = fl_in<T, MODE>(a, DIM * (size_t)dof + k, beta, alpha, ivv[k]);
      }
      T ip = ivp;
      if (MODE == TE_MR && pre && !vel) ip = sbd[a.bkeys[dof - (uint32_t)nV]];
      const T vp = fl_in<T, MODE>(a, DIM * (size_t)nV + dof, beta, alpha, ip);
#pragma unroll
      for (int e = 0; e < NE; e++) {
#pragma unroll
        for (int b = 0; b < NE; b++) {
          if (!(drow(b) - drow(e) == orr && dcol(b) - dcol(e) == occ && dlay(b) - dlay(e) == oll)) continue;
          if (!((fk >> e) & 1u)) continue;
          if (pore) {
#pragma unroll
            for (int ci = 0; ci < DIM; ci++) {
              T sum = flK<T>((DIM * e + ci) * ED + DIM * b) * vv[0];
#pragma unroll
              for (int cj = 1; cj < DIM; cj++) sum += flK<T>((DIM * e + ci) * ED + DIM * b + cj) * vv[cj];
              ov[ci] += sum + flK<T>((DIM * e + ci) * ED + PC + b) * vp;
            }
          }
          T sp = flK<T>((PC + e) * ED + DIM * b) * vv[0];
#pragma unroll
          for (int cj = 1; cj < DIM; cj++) sp += flK<T>((PC + e) * ED + DIM * b + cj) * vv[cj];
          op += sp - flK<T>((PC + e) * ED + PC + b) * vp;
        }
      }
    }
    // own rows: formed input (dot), ping-pong outputs, MR updates
    const int cnt = pore ? DIM + 1 : 1;
    T outv[DIM + 1];
    size_t offs[DIM + 1];
#pragma unroll
    for (int k = 0; k < DIM; k++) { outv[k] = ov[k]; offs[k] = DIM * (size_t)t + k; }
    outv[DIM] = op;
    offs[DIM] = DIM * (size_t)nV + t;
    if (!pore) { outv[0] = op; offs[0] = DIM * (size_t)nV + t; }
    for (int k = 0; k < cnt; k++) {
      const size_t j = offs[k];
      T iv = T(1);
      if (MODE == TE_MR && pre) iv = pore ? (k == DIM ? ivp : ivv[k < DIM ? k : 0]) : sbd[fk];
      const T v = fl_in<T, MODE>(a, j, beta, alpha, iv);
      a.y[j] = outv[k];
      if (MODE == TE_PCG) a.vout[j] = v;
      if (MODE == TE_MR) {
        const T rn = fma(-alpha, a.vd[j], a.v[j]);
        a.vout[j] = rn;
        const T dv = a.d[j];
        const double xv = fma((double)alpha, (double)dv, a.x[j]);
        a.x[j] = xv;
        acc_rz += (double)rn * (double)v;
        mr = fmax(mr, fabs((double)rn));
        if ((long)j < a.cfg.nhmg) { md = fmax(md, fabs((double)dv)); mx = fmax(mx, fabs((double)xv)); }
      }
      acc += (double)v * (double)outv[k];
    }
  }
  if (a.finish == 0) return;
  if (MODE == TE_MR) {
    const double vals[5] = {acc, acc_rz, mr, md, mx};
    const bool ismax[5] = {false, false, true, true, true};
    double out[5];
    if (grid_reduce<FL_NT, 5>(vals, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
      for (int k = 0; k < 5; k++) a.sc->red[k] = out[k];
      mr_finish(a.finish, out, a.sc, a.cfg);
    }
  } else {
    const double vals[1] = {acc};
    const bool ismax[1] = {false};
    double out[1];
    if (grid_reduce<FL_NT, 1>(vals, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
      a.sc->red[0] = out[0];
      if (a.finish == FIN_ALPHA) a.sc->alpha = a.sc->delta / out[0];
    }
  }
}

template <typename T>
struct FlPw {
  double* x; T* d; T* r; const T* q; T* s; const T* dold;
  const uint8_t* bkeys;
  long nV, nB;
  DevScalars* sc;
  RedCtl rc;
  SolveCfg cfg;
};

template <typename T, int MODE, int DIM = 3>
__global__ void __launch_bounds__(PW_NT) k_fl_point(FlPw<T> a) {
  __shared__ double sred[PW_NT / 32];
  __shared__ double sbd[256];  // interface-node inverse diagonals by fluid key
  if (MODE != PW_INIT && MODE != PW_CHECK && a.sc->done) return;
  for (int i = threadIdx.x; i < 256; i += PW_NT) sbd[i] = c_fldiag.border[i];
  __syncthreads();
  const long nV = a.nV, nT = a.nV + a.nB;
  const double alpha64 = (MODE == PW_PCG) ? a.sc->alpha : 0.0;
  const T alpha = T(alpha64);
  const T beta = (MODE == PW_DIR) ? T(a.sc->beta) : T(0);
  double sum = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  for (long t = blockIdx.x * (long)PW_NT + threadIdx.x; t < nT; t += (long)gridDim.x * PW_NT) {
    const bool pore = t < nV;
    long idx[4];
    double inv[4];
    int cnt;
    if (pore) {
      for (int k = 0; k < DIM; k++) idx[k] = DIM * t + k;
      idx[DIM] = DIM * nV + t;
      cnt = DIM + 1;
      for (int k = 0; k <= DIM; k++) inv[k] = c_fldiag.pore[k];
    } else {
      idx[0] = DIM * nV + t; cnt = 1;
      inv[0] = sbd[a.bkeys[t - nV]];
    }
    for (int k = 0; k < cnt; k++) {
      const long j = idx[k];
      if (MODE == PW_DIR) { a.d[j] = fma(beta, a.dold[j], a.s[j]); continue; }
      const T iv = a.cfg.precond ? T(inv[k]) : T(1);
      T rv = a.r[j];
      if (MODE == PW_X0) { rv -= a.q[j]; a.r[j] = rv; }
      if (MODE == PW_PCG) {
        const T dv = a.d[j];
        const double xv = fma(alpha64, (double)dv, a.x[j]);
        a.x[j] = xv;
        rv = fma(-alpha, a.q[j], rv);
        a.r[j] = rv;
        if (j < a.cfg.nhmg) { md = fmax(md, fabs((double)dv)); mx = fmax(mx, fabs((double)xv)); }
      }
      const T sv = rv * iv;
      a.s[j] = sv;
      sum += (double)rv * (double)sv;
      mr = fmax(mr, fabs((double)rv));
    }
  }
  if (MODE == PW_DIR) return;
  const double vals[4] = {sum, mr, md, mx};
  const bool ismax[4] = {false, true, true, true};
  double out[4];
  if (grid_reduce<PW_NT, 4>(vals, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
    for (int k = 0; k < 4; k++) a.sc->red[k] = out[k];
    pcg_finish(MODE, out, a.sc, a.cfg);
  }
}

}  // namespace chfem
