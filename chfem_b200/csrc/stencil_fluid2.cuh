// stencil_fluid2.cuh -- the 2-vector Stokes solvers (CG2 / PCG2 / MINRES2 / PMINRES2) with
// on-the-fly reduction of the solution (chfem/src/femhmg/cudapcg/solvers/cg2.cu, pcg2.cu,
// minres2.cu, pminres2.cu, xreduce.cu:4-27).
//
// Only r and d are stored.  The solution is never formed: each step adds alpha d to the
// per-component sums of its velocity part (the effective-permeability column), optionally
// through an accumulator of the velocity part (FULL) or of the loaded component (ONLYDIR).
// Without a q = A d vector the operator is applied twice per step (for d.Ad -- or
// Ad.M^-1 Ad -- and for the residual update), and once more on z = M^-1 r for PMINRES2's
// delta.  The B200 passes fold every BLAS-1 step and reduction into those applies:
//   F2_DAD  d.(A d)                                 -> alpha = delta / .       (PCG2 / CG2)
//   F2_AMA  (A d).M^-1 (A d)                        -> alpha = delta / .       ((P)MINRES2)
//   F2_UPD  r -= alpha A d in place; r.M^-1 r, max|r|, max|d|, the reductions of the
//           solution (sums of alpha d or of the accumulator), max|x|; stopping test
//   F2_ZAZ  z.(A z) with z = M^-1 r formed on the fly -> delta           ((P)MINRES2)
//   F2_X0   r -= A x0 (x0 held in d); the x0 sums; the accumulator seeded from x0
// plus one pointwise pass d = M^-1 r + beta d (in place).  A pass never writes a vector that
// another thread of the same pass reads as a neighbour value, so r and d are updated in place.
//
// Rows follow the Stokes operator of stencil_fluid.cuh (one thread per pore or interface
// node; the 27 neighbours -- 9 on a 2D image -- gathered once through the node -> DOF map).
// DIM = 2: pixel images, 2 velocities + pressure per pore node; the reference's 2-vector
// solvers are generic over its 2D and 3D Stokes operators (nvarspernode = 2 or 3).
#pragma once
#include "common.cuh"
#include "stencil_fluid.cuh"

namespace chfem {

enum Fl2Mode : int { F2_DAD = 0, F2_AMA = 1, F2_UPD = 2, F2_ZAZ = 3, F2_X0 = 4 };
enum Fl2Fin : int { F2F_NONE = 0, F2F_ALPHA = 1, F2F_STEP = 2, F2F_ZAZ_INIT = 3, F2F_ZAZ_X0 = 4, F2F_ZAZ_STEP = 5, F2F_X0 = 6 };
enum XRMode : int { XR_NONE = 0, XR_ONLYDIR = 1, XR_FULL = 2 };

struct Fl2Cfg {
  double tol;
  int maxit;
  int norm;      // ResNorm
  int precond;
  int minres;    // 1: (P)MINRES2 recurrence, 0: (P)CG2
  int xmode;     // XRMode
  int shift;     // ONLYDIR: the accumulated velocity component
};

struct Fl2Args {
  const double* in;  // operator input: d (DAD, AMA, UPD, X0) or r (ZAZ, formed z = M^-1 r)
  double* r;         // UPD / X0: the residual, updated in place
  const double* d;   // UPD / X0: the direction (= in)
  double* xa;        // accumulator: ONLYDIR nV values, FULL 3 nV values, NONE none
  double* hist;      // [3][maxit + 1] per-step reductions of the solution (unscaled)
  const uint32_t* dof_of_node;
  const uint32_t* node_of_dof;
  const uint8_t* bkeys;
  int R, C, L;
  long nV, nB;
  DevScalars* sc;
  RedCtl rc;
  int finish;
  Fl2Cfg cfg;
};

// Jacobi inverse of the row at vector offset j (velocity rows DIM id + c, pressure rows
// DIM nV + id)
template <int DIM>
__device__ __forceinline__ double fl2_inv(long j, long nV, const uint8_t* bkeys) {
  if (j < DIM * nV) return c_fldiag.pore[j % DIM];
  const long id = j - DIM * nV;
  return id < nV ? c_fldiag.pore[DIM] : c_fldiag.border[bkeys[id - nV]];
}

// 2D rows (pixels: 4 elements, 9 neighbours, 12 x 12 element matrix, 2 velocities + pressure
// per node; matrix_free.cu:484-518, :628-660), in the order of the 3D statement below
template <bool FORM_Z>
__device__ __forceinline__ void fl2_rows_2d(const Fl2Args& a, long t, bool pre, double (&out)[4], unsigned& fk_out) {
  constexpr int NE = 4, ED = 12, PC = 8;
  const long nV = a.nV;
  const int R = a.R, C = a.C;
  const uint32_t node = a.node_of_dof[t];
  const int r = (int)(node % (uint32_t)R), c = (int)((node / (uint32_t)R) % (uint32_t)C);
  const bool pore = t < nV;
  const unsigned fk = pore ? 15u : a.bkeys[t - nV];
  fk_out = fk;
  const int rr[3] = {wrap(r - 1, R), r, wrap(r + 1, R)};
  const int cc[3] = {wrap(c - 1, C), c, wrap(c + 1, C)};
  double ov0 = 0, ov1 = 0, op = 0;
  const double ivv0 = (FORM_Z && pre) ? c_fldiag.pore[0] : 1.0, ivv1 = (FORM_Z && pre) ? c_fldiag.pore[1] : 1.0;
  const double ivp = (FORM_Z && pre) ? c_fldiag.pore[2] : 1.0;
#pragma unroll
  for (int o = 0; o < 9; o++) {
    const int orr = o % 3 - 1, occ = o / 3 - 1;
    unsigned emask = 0;
#pragma unroll
    for (int e = 0; e < NE; e++)
#pragma unroll
      for (int b = 0; b < NE; b++)
        if (drow(b) - drow(e) == orr && dcol(b) - dcol(e) == occ) emask |= 1u << e;
    if (!(fk & emask)) continue;
    const uint32_t nb = (uint32_t)rr[orr + 1] + (uint32_t)cc[occ + 1] * (uint32_t)R;
    const uint32_t dof = a.dof_of_node[nb];
    double vx = 0, vy = 0;
    const bool vel = dof < (uint32_t)nV;
    if (vel) {
      vx = a.in[2 * (size_t)dof] * ivv0;
      vy = a.in[2 * (size_t)dof + 1] * ivv1;
    }
    double ip = ivp;
    if (FORM_Z && pre && !vel) ip = c_fldiag.border[a.bkeys[dof - (uint32_t)nV]];
    const double vp = a.in[2 * (size_t)nV + dof] * ip;
#pragma unroll
    for (int e = 0; e < NE; e++) {
#pragma unroll
      for (int b = 0; b < NE; b++) {
        if (!(drow(b) - drow(e) == orr && dcol(b) - dcol(e) == occ)) continue;
        if (!((fk >> e) & 1u)) continue;
        if (pore) {
          ov0 += c_flK64[(2 * e + 0) * ED + 2 * b] * vx + c_flK64[(2 * e + 0) * ED + 2 * b + 1] * vy + c_flK64[(2 * e + 0) * ED + PC + b] * vp;
          ov1 += c_flK64[(2 * e + 1) * ED + 2 * b] * vx + c_flK64[(2 * e + 1) * ED + 2 * b + 1] * vy + c_flK64[(2 * e + 1) * ED + PC + b] * vp;
        }
        op += c_flK64[(PC + e) * ED + 2 * b] * vx + c_flK64[(PC + e) * ED + 2 * b + 1] * vy - c_flK64[(PC + e) * ED + PC + b] * vp;
      }
    }
  }
  out[0] = pore ? ov0 : op;
  out[1] = ov1;
  out[2] = op;
  out[3] = op;
}

// Operator rows of row set t (pore node: 3 velocities + pressure; interface node: pressure)
// applied to the vector `in`, formed as in * M^-1 when FORM_Z.  The dropped velocity columns
// of non-pore neighbours and the voxel mask of interface rows follow k_fl_apply.  out holds
// the DIM velocity rows then the pressure row (out[0] the pressure row of an interface node).
template <bool FORM_Z, int DIM = 3>
__device__ __forceinline__ void fl2_rows(const Fl2Args& a, long t, bool pre, double (&out)[4], unsigned& fk_out) {
  if constexpr (DIM == 2) {
    fl2_rows_2d<FORM_Z>(a, t, pre, out, fk_out);
    return;
  }
  const long nV = a.nV;
  const int R = a.R, C = a.C, L = a.L;
  const uint32_t node = a.node_of_dof[t];
  const int r = (int)(node % (uint32_t)R), c = (int)((node / (uint32_t)R) % (uint32_t)C), l = (int)(node / ((uint32_t)R * (uint32_t)C));
  const bool pore = t < nV;
  const unsigned fk = pore ? 255u : a.bkeys[t - nV];
  fk_out = fk;
  const int rr[3] = {wrap(r - 1, R), r, wrap(r + 1, R)};
  const int cc[3] = {wrap(c - 1, C), c, wrap(c + 1, C)};
  const int ll[3] = {wrap(l - 1, L), l, wrap(l + 1, L)};
  double ov0 = 0, ov1 = 0, ov2 = 0, op = 0;
  const double ivv0 = (FORM_Z && pre) ? c_fldiag.pore[0] : 1.0, ivv1 = (FORM_Z && pre) ? c_fldiag.pore[1] : 1.0;
  const double ivv2 = (FORM_Z && pre) ? c_fldiag.pore[2] : 1.0, ivp = (FORM_Z && pre) ? c_fldiag.pore[3] : 1.0;
#pragma unroll
  for (int o = 0; o < 27; o++) {
    const int orr = o % 3 - 1, occ = (o / 3) % 3 - 1, oll = o / 9 - 1;
    unsigned emask = 0;
#pragma unroll
    for (int e = 0; e < 8; e++)
#pragma unroll
      for (int b = 0; b < 8; b++)
        if (drow(b) - drow(e) == orr && dcol(b) - dcol(e) == occ && dlay(b) - dlay(e) == oll) emask |= 1u << e;
    if (!(fk & emask)) continue;
    const uint32_t nb = (uint32_t)rr[orr + 1] + (uint32_t)cc[occ + 1] * (uint32_t)R + (uint32_t)ll[oll + 1] * (uint32_t)R * (uint32_t)C;
    const uint32_t dof = a.dof_of_node[nb];
    double vx = 0, vy = 0, vz = 0;
    const bool vel = dof < (uint32_t)nV;
    if (vel) {
      vx = a.in[3 * (size_t)dof] * ivv0;
      vy = a.in[3 * (size_t)dof + 1] * ivv1;
      vz = a.in[3 * (size_t)dof + 2] * ivv2;
    }
    double ip = ivp;
    if (FORM_Z && pre && !vel) ip = c_fldiag.border[a.bkeys[dof - (uint32_t)nV]];
    const double vp = a.in[3 * (size_t)nV + dof] * ip;
#pragma unroll
    for (int e = 0; e < 8; e++) {
#pragma unroll
      for (int b = 0; b < 8; b++) {
        if (!(drow(b) - drow(e) == orr && dcol(b) - dcol(e) == occ && dlay(b) - dlay(e) == oll)) continue;
        if (!((fk >> e) & 1u)) continue;
        if (pore) {
          ov0 += c_flK64[(3 * e + 0) * 32 + 3 * b] * vx + c_flK64[(3 * e + 0) * 32 + 3 * b + 1] * vy + c_flK64[(3 * e + 0) * 32 + 3 * b + 2] * vz + c_flK64[(3 * e + 0) * 32 + 24 + b] * vp;
          ov1 += c_flK64[(3 * e + 1) * 32 + 3 * b] * vx + c_flK64[(3 * e + 1) * 32 + 3 * b + 1] * vy + c_flK64[(3 * e + 1) * 32 + 3 * b + 2] * vz + c_flK64[(3 * e + 1) * 32 + 24 + b] * vp;
          ov2 += c_flK64[(3 * e + 2) * 32 + 3 * b] * vx + c_flK64[(3 * e + 2) * 32 + 3 * b + 1] * vy + c_flK64[(3 * e + 2) * 32 + 3 * b + 2] * vz + c_flK64[(3 * e + 2) * 32 + 24 + b] * vp;
        }
        op += c_flK64[(24 + e) * 32 + 3 * b] * vx + c_flK64[(24 + e) * 32 + 3 * b + 1] * vy + c_flK64[(24 + e) * 32 + 3 * b + 2] * vz - c_flK64[(24 + e) * 32 + 24 + b] * vp;
      }
    }
  }
  out[0] = pore ? ov0 : op;
  out[1] = ov1;
  out[2] = ov2;
  out[3] = op;
}

// Step finisher of the 2-vector recurrences, run by thread 0 of the last CTA of F2_UPD.
// s: [0] r.M^-1 r, [1] max|r|, [2] max|d| (velocity rows), [3] max|x| (accumulator),
// [4..6] the velocity-component sums (of d for NONE, of the accumulator otherwise).
__device__ inline void fl2_step_finish(const double* s, const Fl2Args& a) {
  DevScalars* sc = a.sc;
  const Fl2Cfg& cfg = a.cfg;
  const double tol2 = cfg.tol * cfg.tol;
  const int it = sc->iteration + 1;
  sc->iteration = it;
  const size_t stride = (size_t)cfg.maxit + 1;
  if (cfg.xmode == XR_NONE) { for (int c = 0; c < 3; c++) a.hist[c * stride + it] = sc->alpha * s[4 + c]; }
  else if (cfg.xmode == XR_ONLYDIR) a.hist[cfg.shift * stride + it] = s[4];
  else { for (int c = 0; c < 3; c++) a.hist[c * stride + it] = s[4 + c]; }
  bool cont;
  if (!cfg.minres) {  // pcg2.cu:163-185
    sc->delta_old = sc->delta;
    sc->delta = s[0];
    if (cfg.norm == NORM_L2) {
      sc->metric = sqrt(fabs(s[0]) / fabs(sc->delta0));
      cont = fabs(s[0]) > tol2 * fabs(sc->delta0);
      sc->found = !cont;
    } else if (cfg.norm == NORM_INF) {
      sc->metric = s[1] / sc->res0;
      cont = sc->metric > cfg.tol;
      sc->found = !cont;
    } else {
      // the largest |x| held: the accumulator (1 without one, as the MINRES2 form uses)
      sc->metric = fabs(sc->alpha) * s[2] / (cfg.xmode == XR_NONE ? 1.0 : s[3]);
      cont = !((sc->metric <= cfg.tol) || !(fabs(s[0]) > tol2 * fabs(sc->delta0)));
      sc->found = sc->metric <= cfg.tol;
    }
    sc->beta = sc->delta / sc->delta_old;
  } else {  // pminres2.cu:168-184: the test is on r; delta comes from the F2_ZAZ pass
    if (cfg.norm == NORM_L2) {
      cont = fabs(s[0]) > tol2 * fabs(sc->res0);
      sc->metric = sqrt(fabs(s[0]) / fabs(sc->res0));
    } else if (cfg.norm == NORM_INF) {
      sc->metric = s[1] / sc->res0;
      cont = sc->metric > cfg.tol;
    } else {
      sc->metric = fabs(sc->alpha) * s[2];
      cont = sc->metric > cfg.tol;
    }
    sc->found = sc->metric <= cfg.tol;
  }
  if (!cont || it >= cfg.maxit) sc->done = 1;
}

template <int MODE, int DIM = 3>
__global__ void __launch_bounds__(FL_NT) k_fl2_apply(Fl2Args a) {
  __shared__ double sred[FL_NT / 32];
  if (a.sc->done) return;
  const long nV = a.nV, nT = a.nV + a.nB;
  const bool pre = a.cfg.precond != 0;
  const double alpha = (MODE == F2_UPD) ? a.sc->alpha : (MODE == F2_X0 ? 1.0 : 0.0);
  const int xmode = a.cfg.xmode, shift = a.cfg.shift;
  double acc = 0.0, mr = 0.0, md = 0.0, mx = 0.0, xs0 = 0.0, xs1 = 0.0, xs2 = 0.0;
  for (long t = blockIdx.x * (long)FL_NT + threadIdx.x; t < nT; t += (long)gridDim.x * FL_NT) {
    double out[4];
    unsigned fk;
    fl2_rows<MODE == F2_ZAZ, DIM>(a, t, pre, out, fk);
    const bool pore = t < nV;
    const int cnt = pore ? DIM + 1 : 1;
    for (int k = 0; k < cnt; k++) {
      const long j = pore ? (k < DIM ? DIM * t + k : DIM * nV + t) : DIM * nV + t;
      const double y = pore ? out[k] : out[0];
      const double iv = pre ? (pore ? c_fldiag.pore[k] : c_fldiag.border[fk]) : 1.0;
      if (MODE == F2_DAD) acc += a.in[j] * y;
      if (MODE == F2_AMA) acc += y * y * iv;
      if (MODE == F2_ZAZ) acc += a.in[j] * iv * y;
      if (MODE == F2_UPD || MODE == F2_X0) {
        const double rn = a.r[j] - alpha * y;
        a.r[j] = rn;
        acc += rn * rn * iv;
        mr = fmax(mr, fabs(rn));
        if (pore && k < DIM) {  // velocity rows: the reduced solution
          const double dv = a.d[j];
          if (MODE == F2_UPD) md = fmax(md, fabs(dv));
          double xv = dv;  // F2_X0: the guess itself
          if (xmode == XR_FULL) {
            if (MODE == F2_UPD) xv = a.xa[j] + alpha * dv;
            a.xa[j] = xv;
            mx = fmax(mx, fabs(xv));
          } else if (xmode == XR_ONLYDIR && k == shift) {
            if (MODE == F2_UPD) xv = a.xa[t] + alpha * dv;
            a.xa[t] = xv;
            mx = fmax(mx, fabs(xv));
          }
          // the per-component sums: of the guess (F2_X0); of d (NONE, alpha applied by the
          // finisher), of the accumulator (FULL), of the loaded component into slot 0 (ONLYDIR)
          if (MODE == F2_UPD && xmode == XR_ONLYDIR) { if (k == shift) xs0 += xv; }
          else if (k == 0) xs0 += xv;
          else if (k == 1) xs1 += xv;
          else xs2 += xv;
        }
      }
    }
  }
  if (MODE == F2_UPD || MODE == F2_X0) {
    const double vals[7] = {acc, mr, md, mx, xs0, xs1, xs2};
    const bool ismax[7] = {false, true, true, true, false, false, false};
    double o[7];
    if (grid_reduce<FL_NT, 7>(vals, ismax, a.rc, blockIdx.x, o, sred) && threadIdx.x == 0) {
      for (int k = 0; k < 6; k++) a.sc->red[k] = o[k];
      if (MODE == F2_UPD) {
        fl2_step_finish(o, a);
      } else {
        // cg2.cu:131-152: the x0 sums are entry 0 of the reductions; PCG2 tests the guess here,
        // (P)MINRES2 after its F2_ZAZ pass
        const size_t stride = (size_t)a.cfg.maxit + 1;
        for (int c = 0; c < 3; c++) a.hist[c * stride] = o[4 + c];
        if (!a.cfg.minres) {
          a.sc->delta = o[0];
          a.sc->delta_old = o[0];
          a.sc->beta = 0.0;
          const double tol2 = a.cfg.tol * a.cfg.tol;
          if (!(fabs(o[0]) > tol2 * fabs(a.sc->delta0))) {
            a.sc->done = 1; a.sc->found = 1; a.sc->status = 2; a.sc->metric = sqrt(fabs(o[0]) / fabs(a.sc->delta0));
          }
        }
      }
    }
  } else {
    const double vals[1] = {acc};
    const bool ismax[1] = {false};
    double o[1];
    if (grid_reduce<FL_NT, 1>(vals, ismax, a.rc, blockIdx.x, o, sred) && threadIdx.x == 0) {
      DevScalars* sc = a.sc;
      sc->red[0] = o[0];
      if (a.finish == F2F_ALPHA) sc->alpha = sc->delta / o[0];
      else if (a.finish == F2F_ZAZ_INIT) { sc->delta0 = o[0]; sc->delta = o[0]; sc->delta_old = o[0]; }
      else if (a.finish == F2F_ZAZ_X0) {  // pminres2.cu:95-116: the initial-guess test
        sc->delta = o[0]; sc->delta_old = o[0]; sc->beta = 0.0;
        const double tol2 = a.cfg.tol * a.cfg.tol;
        if (!(fabs(o[0]) > tol2 * fabs(sc->delta0))) {
          sc->done = 1; sc->found = 1; sc->status = 2; sc->metric = sqrt(fabs(o[0]) / fabs(sc->delta0));
        }
      } else if (a.finish == F2F_ZAZ_STEP) {
        sc->delta_old = sc->delta;
        sc->delta = o[0];
        sc->beta = sc->delta / sc->delta_old;
      }
    }
  }
}

// Pointwise passes: P2_INIT (the zero-guess references, null-RHS test) and P2_DIR
// (d = M^-1 r + beta d in place; d = M^-1 r in the first step, where d is not read).
enum Fl2Pw : int { P2_INIT = 0, P2_DIR = 1 };

template <int MODE, int DIM = 3>
__global__ void __launch_bounds__(PW_NT) k_fl2_point(Fl2Args a, double* d) {
  __shared__ double sred[PW_NT / 32];
  if (MODE == P2_DIR && a.sc->done) return;
  const long nV = a.nV, n = (DIM + 1) * a.nV + a.nB;
  const bool pre = a.cfg.precond != 0;
  const bool first = (MODE == P2_DIR) && a.sc->iteration == 0;
  const double beta = (MODE == P2_DIR && !first) ? a.sc->beta : 0.0;
  double s = 0.0, mr = 0.0;
  for (long j = blockIdx.x * (long)PW_NT + threadIdx.x; j < n; j += (long)gridDim.x * PW_NT) {
    const double iv = pre ? fl2_inv<DIM>(j, nV, a.bkeys) : 1.0;
    const double rv = a.r[j];
    if (MODE == P2_DIR) {
      d[j] = first ? rv * iv : fma(beta, d[j], rv * iv);
    } else {
      s += rv * rv * iv;
      mr = fmax(mr, fabs(rv));
    }
  }
  if (MODE == P2_DIR) return;
  const double vals[2] = {s, mr};
  const bool ismax[2] = {false, true};
  double o[2];
  if (grid_reduce<PW_NT, 2>(vals, ismax, a.rc, blockIdx.x, o, sred) && threadIdx.x == 0) {
    // pcg2.cu:60-80 / pminres2.cu:73-91: delta0 (PCG2) and the stopping reference res0
    DevScalars* sc = a.sc;
    sc->iteration = 0; sc->alpha = 0.0; sc->beta = 0.0; sc->found = 0; sc->status = 0; sc->done = 0;
    sc->res0 = (a.cfg.norm == NORM_INF) ? o[1] : o[0];
    sc->metric = 1.0;
    if (!a.cfg.minres) { sc->delta0 = o[0]; sc->delta = o[0]; sc->delta_old = o[0]; }
    if (fabs(sc->res0) < 1e-12) { sc->done = 1; sc->found = 1; sc->metric = 0.0; sc->status = 1; }
  }
}

}  // namespace chfem
