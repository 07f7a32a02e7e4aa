// stencil_fluid_block.cuh -- block (P)MINRES passes of the Stokes operator: the flow
// directions of one pore model (3 right-hand sides) advance together.
//
// The reference solves the three flow directions one after the other
// (chfem/src/femhmg/femhmg.c:1017-1119), each operator pass gathering the 27 neighbours of a
// row set through the node->DOF map again.  Here one thread gathers each neighbour once for
// all NR right-hand sides and applies every element-matrix coefficient (a broadcast
// __constant__ operand) to the NR fields.  Every right-hand side keeps its own scalars and
// stopping test (one DevScalars record each) and follows the single-solve recurrence of
// pminres.cu:100-204; a right-hand side that has stopped takes alpha = 0, so its x and r stay
// put while the others continue.
#pragma once
#include <utility>
#include "stencil_fluid.cuh"
#include "stencil_block.cuh"
#include "minres.cuh"

namespace chfem {

template <typename T>
struct FlBlkArgs {
  const T* r;      // [NR][n] current residual
  const T* q;      // [NR][n] q = A d (recursive)
  T* rout;         // [NR][n] r' = r - alpha q
  T* s;            // [NR][n] s = A M^-1 r'
  double* x;       // [NR][n]
  const T* d;      // [NR][n]
  const uint32_t* dof_of_node;
  const uint32_t* node_of_dof;
  const uint8_t* bkeys;
  int R, C, L;
  long nV, nB, n;  // n: unknowns per right-hand side
  DevScalars* sc;  // [NR]
  RedCtl rc;
  MrCfg cfg;
};

// voxels e of a node that also hold its neighbour O (O = (drow+1) + 3 (dcol+1) + 9 (dlay+1))
__host__ __device__ constexpr unsigned fl_emask(int O) {
  unsigned m = 0;
  for (int e = 0; e < 8; e++)
    for (int b = 0; b < 8; b++)
      if (pair_nbr(e, b) == O) m |= 1u << e;
  return m;
}

// One neighbour O of a row set: gather its values for all right-hand sides once, then every
// (voxel e, local node b) pair of this node that lands on it.
template <typename T, int NR, int O>
__device__ __forceinline__ void fl_blk_nbr(const FlBlkArgs<T>& a, unsigned fk, bool pore, const int (&rr)[3], const int (&cc)[3],
                                           const int (&ll)[3], const T* salpha, bool pre, T ivv0, T ivv1, T ivv2, T ivp,
                                           T (&ov0)[NR], T (&ov1)[NR], T (&ov2)[NR], T (&op)[NR]) {
  constexpr int orr = O % 3 - 1, occ = (O / 3) % 3 - 1, oll = O / 9 - 1;
  constexpr unsigned emask = fl_emask(O);
  if (!(fk & emask)) return;
  const int R = a.R, C = a.C;
  const long nV = a.nV, n = a.n;
  const uint32_t nb = (uint32_t)rr[orr + 1] + (uint32_t)cc[occ + 1] * (uint32_t)R + (uint32_t)ll[oll + 1] * (uint32_t)R * (uint32_t)C;
  const uint32_t dof = a.dof_of_node[nb];
  const bool vel = dof < (uint32_t)nV;
  T ip = ivp;
  if (pre && !vel) ip = T(c_fldiag.border[a.bkeys[dof - (uint32_t)nV]]);
  T vx[NR], vy[NR], vz[NR], vp[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) {
    const T* rk = a.r + k * n;
    const T* qk = a.q + k * n;
    vx[k] = vy[k] = vz[k] = T(0);
    if (vel) {
      const size_t o = 3 * (size_t)dof;
      vx[k] = fma(-salpha[k], qk[o], rk[o]) * ivv0;
      vy[k] = fma(-salpha[k], qk[o + 1], rk[o + 1]) * ivv1;
      vz[k] = fma(-salpha[k], qk[o + 2], rk[o + 2]) * ivv2;
    }
    const size_t op_ = 3 * (size_t)nV + dof;
    vp[k] = fma(-salpha[k], qk[op_], rk[op_]) * ip;
  }
#pragma unroll
  for (int e = 0; e < 8; e++) {
#pragma unroll
    for (int b = 0; b < 8; b++) {
      if (pair_nbr(e, b) != O) continue;
      if (!((fk >> e) & 1u)) continue;
      if (pore) {
#pragma unroll
        for (int row = 0; row < 3; row++) {
          const T k0 = flK<T>((3 * e + row) * 32 + 3 * b), k1 = flK<T>((3 * e + row) * 32 + 3 * b + 1);
          const T k2 = flK<T>((3 * e + row) * 32 + 3 * b + 2), k3 = flK<T>((3 * e + row) * 32 + 24 + b);
#pragma unroll
          for (int k = 0; k < NR; k++) {
            const T add = k0 * vx[k] + k1 * vy[k] + k2 * vz[k] + k3 * vp[k];
            if (row == 0) ov0[k] += add;
            else if (row == 1) ov1[k] += add;
            else ov2[k] += add;
          }
        }
      }
      const T g0 = flK<T>((24 + e) * 32 + 3 * b), g1 = flK<T>((24 + e) * 32 + 3 * b + 1);
      const T g2 = flK<T>((24 + e) * 32 + 3 * b + 2), st = flK<T>((24 + e) * 32 + 24 + b);
#pragma unroll
      for (int k = 0; k < NR; k++) op[k] += g0 * vx[k] + g1 * vy[k] + g2 * vz[k] - st * vp[k];
    }
  }
}
template <typename T, int NR, int... Os>
__device__ __forceinline__ void fl_blk_all_nbrs(std::integer_sequence<int, Os...>, const FlBlkArgs<T>& a, unsigned fk, bool pore,
                                                const int (&rr)[3], const int (&cc)[3], const int (&ll)[3], const T* salpha, bool pre,
                                                T ivv0, T ivv1, T ivv2, T ivp, T (&ov0)[NR], T (&ov1)[NR], T (&ov2)[NR], T (&op)[NR]) {
  (fl_blk_nbr<T, NR, Os>(a, fk, pore, rr, cc, ll, salpha, pre, ivv0, ivv1, ivv2, ivp, ov0, ov1, ov2, op), ...);
}

// MAXN: the stopping test needs the max-norms (infinity / error norm); the L2 test needs only
// the two sums (z'.A z', r'.z') per right-hand side.  Two CTAs per SM at least: the pass is a
// gather whose latency wants the warps.
template <typename T, int NR, bool MAXN>
__global__ void __launch_bounds__(FL_NT, 2) k_fl_blk_apply(FlBlkArgs<T> a) {
  __shared__ double sred[FL_NT / 32];
  __shared__ T salpha[NR];
  __shared__ int sdone[NR];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < NR; k++) all_done = all_done && a.sc[k].done;
  if (all_done) return;
  if (threadIdx.x < NR) {
    sdone[threadIdx.x] = a.sc[threadIdx.x].done;
    salpha[threadIdx.x] = sdone[threadIdx.x] ? T(0) : T(a.sc[threadIdx.x].alpha);
  }
  __syncthreads();
  const long nV = a.nV, nT = a.nV + a.nB, n = a.n;
  const int R = a.R, C = a.C, L = a.L;
  const bool pre = a.cfg.precond != 0;
  const T ivv0 = pre ? T(c_fldiag.pore[0]) : T(1), ivv1 = pre ? T(c_fldiag.pore[1]) : T(1), ivv2 = pre ? T(c_fldiag.pore[2]) : T(1);
  const T ivp = pre ? T(c_fldiag.pore[3]) : T(1);
  constexpr int NV = MAXN ? 5 : 2;
  double vals[NV * NR];
#pragma unroll
  for (int k = 0; k < NV * NR; k++) vals[k] = 0.0;
  // z' = M^-1 (r - alpha q) at vector offset off of right-hand side k
  auto zin = [&](int k, size_t off, T inv) { return fma(-salpha[k], a.q[k * n + off], a.r[k * n + off]) * inv; };
  for (long t = blockIdx.x * (long)FL_NT + threadIdx.x; t < nT; t += (long)gridDim.x * FL_NT) {
    const uint32_t node = a.node_of_dof[t];
    const int r = (int)(node % (uint32_t)R), c = (int)((node / (uint32_t)R) % (uint32_t)C), l = (int)(node / ((uint32_t)R * (uint32_t)C));
    const bool pore = t < nV;
    const unsigned fk = pore ? 255u : a.bkeys[t - nV];
    const int rr[3] = {wrap(r - 1, R), r, wrap(r + 1, R)};
    const int cc[3] = {wrap(c - 1, C), c, wrap(c + 1, C)};
    const int ll[3] = {wrap(l - 1, L), l, wrap(l + 1, L)};
    T ov0[NR], ov1[NR], ov2[NR], op[NR];
#pragma unroll
    for (int k = 0; k < NR; k++) ov0[k] = ov1[k] = ov2[k] = op[k] = T(0);
    fl_blk_all_nbrs<T, NR>(std::make_integer_sequence<int, 27>{}, a, fk, pore, rr, cc, ll, salpha, pre, ivv0, ivv1, ivv2, ivp, ov0, ov1, ov2, op);
    // own rows: r' = r - alpha q, s = A z', x += alpha d, dots and norms
    const int cnt = pore ? 4 : 1;
    const size_t offs[4] = {pore ? 3 * (size_t)t : 3 * (size_t)nV + t, 3 * (size_t)t + 1, 3 * (size_t)t + 2, 3 * (size_t)nV + t};
    const T ivs[4] = {pore ? ivv0 : T(1), ivv1, ivv2, ivp};
    const T ivb = (pre && !pore) ? T(c_fldiag.border[fk]) : T(1);
#pragma unroll
    for (int k = 0; k < NR; k++) {
      const T outv[4] = {pore ? ov0[k] : op[k], ov1[k], ov2[k], op[k]};
#pragma unroll
      for (int m = 0; m < 4; m++) {
        if (m >= cnt) break;
        const size_t j = offs[m];
        const T iv = pore ? ivs[m] : ivb;
        const T z = zin(k, j, iv);
        const size_t jk = (size_t)k * n + j;
        a.s[jk] = outv[m];
        const T rn = fma(-salpha[k], a.q[jk], a.r[jk]);
        a.rout[jk] = rn;
        const T dv = a.d[jk];
        const double xv = fma((double)salpha[k], (double)dv, a.x[jk]);
        if (!sdone[k]) a.x[jk] = xv;
        vals[NV * k] += (double)z * (double)outv[m];
        vals[NV * k + 1] += (double)rn * (double)z;
        if constexpr (MAXN) {
          vals[NV * k + 2] = fmax(vals[NV * k + 2], fabs((double)rn));
          if ((long)j < a.cfg.nhmg) { vals[NV * k + 3] = fmax(vals[NV * k + 3], fabs((double)dv)); vals[NV * k + 4] = fmax(vals[NV * k + 4], fabs(xv)); }
        }
      }
    }
  }
  bool ismax[NV * NR];
  double out[NV * NR];
#pragma unroll
  for (int k = 0; k < NV * NR; k++) ismax[k] = (k % NV) >= 2;
  if (grid_reduce<FL_NT, NV * NR>(vals, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NR; k++) {
      if (sdone[k]) continue;
      double s5[5] = {out[NV * k], out[NV * k + 1], 0.0, 0.0, 0.0};
      if constexpr (MAXN) { s5[2] = out[NV * k + 2]; s5[3] = out[NV * k + 3]; s5[4] = out[NV * k + 4]; }
      for (int m = 0; m < 5; m++) a.sc[k].red[m] = s5[m];
      mr_finish(FIN_MR_STEP, s5, a.sc + k, a.cfg);
    }
  }
}

// Direction pass for all right-hand sides: d = M^-1 r + beta d, q = s + beta q, and
// alpha = delta / (q . M^-1 q) per right-hand side (pminres.cu:100-128).
template <typename T>
struct FlBlkDir {
  T* d; T* q; const T* r; const T* s;
  const uint8_t* bkeys; long nV, nB, n;
  DevScalars* sc; RedCtl rc; int precond;
};

template <typename T, int NR>
__global__ void __launch_bounds__(PW_NT) k_fl_blk_dir(FlBlkDir<T> a) {
  __shared__ double sred[PW_NT / 32];
  __shared__ T sbeta[NR];
  __shared__ int sdone[NR];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < NR; k++) all_done = all_done && a.sc[k].done;
  if (all_done) return;
  if (threadIdx.x < NR) { sdone[threadIdx.x] = a.sc[threadIdx.x].done; sbeta[threadIdx.x] = T(a.sc[threadIdx.x].beta); }
  __syncthreads();
  const long nV = a.nV, nT = a.nV + a.nB, n = a.n;
  double sum[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) sum[k] = 0.0;
  for (long t = blockIdx.x * (long)PW_NT + threadIdx.x; t < nT; t += (long)gridDim.x * PW_NT) {
    const bool pore = t < nV;
    const int cnt = pore ? 4 : 1;
    for (int m = 0; m < cnt; m++) {
      const long j = pore ? (m < 3 ? 3 * t + m : 3 * nV + t) : 3 * nV + t;
      T inv = T(1);
      if (a.precond) inv = pore ? T(c_fldiag.pore[m]) : T(c_fldiag.border[a.bkeys[t - nV]]);
#pragma unroll
      for (int k = 0; k < NR; k++) {
        if (sdone[k]) continue;
        const long jk = (long)k * n + j;
        const T z = a.r[jk] * inv;
        a.d[jk] = fma(sbeta[k], a.d[jk], z);
        const T qn = fma(sbeta[k], a.q[jk], a.s[jk]);
        a.q[jk] = qn;
        sum[k] += (double)qn * (double)(qn * inv);
      }
    }
  }
  bool ismax[NR];
  double out[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) ismax[k] = false;
  if (grid_reduce<PW_NT, NR>(sum, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NR; k++) {
      if (sdone[k]) continue;
      a.sc[k].red[5] = out[k];
      a.sc[k].alpha = a.sc[k].delta / out[k];
    }
  }
}

}  // namespace chfem
