// pointwise.cuh -- fused vector updates of the Krylov loops with their FP64 reductions.
//
// One pass per step instead of the reference's chain of BLAS-1 kernels, each followed by a
// multi-pass reduction and a device->host copy (chfem/src/femhmg/cudapcg/solvers/pcg.cu:
// 163-208, kernels/wrappers.cu:40-60, :247-250).  The scalars of the recurrence (alpha,
// beta, delta, the stopping test) are finished on the device by the last CTA of each pass,
// so an iteration issues no host synchronisation.
//
// The Jacobi diagonal is recomputed from the node key like the reference does
// (matrix_free.cu:167-188 thermal, :388-408 elastic): diag = sum over the node's 8 voxels of
// the diagonal entry of local node e in that voxel's element matrix.
#pragma once
#include "common.cuh"

namespace chfem {

constexpr int PW_NT = 256;

enum PwMode : int {
  PW_INIT = 0,     // s = M^-1 r; delta0 = r.s (zero-guess reference); null-RHS guard
  PW_X0 = 1,       // r -= q (q = A x0); s = M^-1 r; delta = r.s; initial-guess test
  PW_PCG = 2,      // x += a d; r -= a q; s = M^-1 r; delta = r.s; stopping test
  PW_DIR = 3,      // d_new = s + beta d_old (no reduction)
  PW_REPL = 4,     // after a residual replacement: s = M^-1 r; delta = r.s; beta = delta/delta_old
  PW_X0R = 5,      // r already holds b - A x0 (FP64 apply): s = M^-1 r; delta = r.s; initial-guess test
  PW_CHECK = 6,    // r holds the true residual b - A x at an apparent convergence: confirm or restart
};

enum ResNorm : int { NORM_L2 = 0, NORM_INF = 1, NORM_ERR = 2 };

struct SolveCfg {
  double tol;
  int maxit;
  int norm;        // ResNorm
  int precond;     // 0: plain CG, s = r
  long nhmg;       // entries checked by the error norm (the leading velocity DOFs for Stokes)
};

// Finisher shared by every physics.  sums: [0] r.s, [1] max|r|, [2] max|d| over nhmg, [3] max|x| over nhmg.
__device__ inline void pcg_finish(int mode, const double* s, DevScalars* sc, const SolveCfg& cfg) {
  const double tol2 = cfg.tol * cfg.tol;
  if (mode == PW_INIT) {
    sc->delta0 = s[0];
    sc->res0 = (cfg.norm == NORM_INF) ? s[1] : s[0];
    sc->iteration = 0;
    sc->alpha = 0.0;
    sc->beta = 0.0;
    sc->found = 0;
    if (fabs(sc->res0) < 1e-12) {  // pcg.cu:75-81: null solution satisfies the system
      sc->done = 1; sc->found = 1; sc->metric = 0.0; sc->status = 1;
    } else {
      sc->done = 0; sc->delta = s[0]; sc->delta_old = s[0]; sc->metric = 1.0; sc->status = 0;
    }
  } else if (mode == PW_X0 || mode == PW_X0R) {
    sc->delta = s[0];
    sc->delta_old = s[0];
    sc->beta = 0.0;
    if (!(fabs(s[0]) > tol2 * fabs(sc->delta0))) {  // pcg.cu:84-96: initial guess already good
      sc->done = 1; sc->found = 1; sc->status = 2;
      sc->metric = sqrt(fabs(s[0]) / fabs(sc->delta0));
    }
  } else if (mode == PW_PCG) {
    sc->iteration += 1;
    sc->delta_old = sc->delta;
    sc->delta = s[0];
    bool cont;
    if (cfg.norm == NORM_L2) {
      sc->metric = sqrt(fabs(s[0]) / fabs(sc->delta0));
      cont = fabs(s[0]) > tol2 * fabs(sc->delta0);
      sc->found = !cont;
    } else if (cfg.norm == NORM_INF) {
      sc->metric = s[1] / sc->res0;
      cont = sc->metric > cfg.tol;
      sc->found = !cont;
    } else {
      sc->metric = fabs(sc->alpha) * s[2] / s[3];
      cont = !((sc->metric <= cfg.tol) || !(fabs(s[0]) > tol2 * fabs(sc->delta0)));
      sc->found = sc->metric <= cfg.tol;
    }
    sc->beta = sc->delta / sc->delta_old;
    if (!cont || sc->iteration >= cfg.maxit) sc->done = 1;
  } else if (mode == PW_REPL) {
    // The true residual replaces the recursive one.  While the two agree the direction is kept
    // (beta from the true delta); once they have drifted apart the old direction no longer
    // fits the new residual and the iteration restarts from it (beta = 0).
    const double rec = sc->delta;
    sc->delta = s[0];
    if (fabs(s[0]) > 4.0 * fabs(rec) || fabs(s[0]) < 0.25 * fabs(rec)) { sc->beta = 0.0; sc->delta_old = s[0]; }
    else sc->beta = sc->delta / sc->delta_old;
  } else if (mode == PW_CHECK) {
    // Mixed precision: the recursive residual may have drifted below the tolerance while the
    // true one has not.  Confirm on the true residual, or restart the direction (beta = 0).
    sc->delta = s[0];
    sc->metric = sqrt(fabs(s[0]) / fabs(sc->delta0));
    if (!(fabs(s[0]) > tol2 * fabs(sc->delta0))) { sc->done = 1; sc->found = 1; }
    else if (sc->iteration >= cfg.maxit) { sc->done = 1; sc->found = 0; }
    else { sc->done = 0; sc->found = 0; sc->beta = 0.0; sc->delta_old = s[0]; }
  }
}

// ---------------------------------------------------------------------------------------
// Thermal / elastic: one thread per node, ND components per node.
// x (the solution) is FP64 in every precision mode: it accumulates the periodic fluctuation
// plus the macroscopic ramp, whose magnitude reaches the cell size.
template <int ND, typename T>
struct TePw {
  double* x; T* d; T* r; const T* q; T* s; const T* dold;
  const uint16_t* keys;
  const T* Kd; int nmat;
  long N;
  DevScalars* sc;
  RedCtl rc;
  SolveCfg cfg;
  const double* invd = nullptr;  // precomputed inverse Jacobi diagonal (scalar density field)
};

template <int ND, typename T, int MODE>
__global__ void __launch_bounds__(PW_NT) k_te_point(TePw<ND, T> a) {
  constexpr int ED = 8 * ND;
  __shared__ double sred[PW_NT / 32];
  __shared__ T sD[4 * 8 * ND];
  if (MODE != PW_INIT && MODE != PW_CHECK && a.sc->done) return;
  const int tid = threadIdx.x;
  for (int i = tid; i < 4 * 8 * ND; i += PW_NT) {
    const int m = i / (8 * ND), k = i % (8 * ND);
    sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)k * ED + k] : T(1);
  }
  __syncthreads();
  const double alpha64 = (MODE == PW_PCG) ? a.sc->alpha : 0.0;
  const T alpha = T(alpha64);
  const T beta = (MODE == PW_DIR) ? T(a.sc->beta) : T(0);
  double sum = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  for (long i = blockIdx.x * (long)PW_NT + tid; i < a.N; i += (long)gridDim.x * PW_NT) {
    if (MODE == PW_DIR) {
#pragma unroll
      for (int c = 0; c < ND; c++) a.d[i * ND + c] = fma(beta, a.dold[i * ND + c], a.s[i * ND + c]);
      continue;
    }
    T inv[ND];
    if (a.cfg.precond && a.invd) {
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(a.invd[i * ND + c]);
    } else if (a.cfg.precond) {
      const unsigned key = a.keys[i];
      T dg[ND];
#pragma unroll
      for (int c = 0; c < ND; c++) dg[c] = T(0);
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const T* D = sD + ((key >> (2 * e)) & 3u) * 8 * ND + e * ND;
#pragma unroll
        for (int c = 0; c < ND; c++) dg[c] += D[c];
      }
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(1) / dg[c];
    } else {
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(1);
    }
#pragma unroll
    for (int c = 0; c < ND; c++) {
      const long j = i * ND + c;
      T rv = a.r[j];
      if (MODE == PW_X0) { rv -= a.q[j]; a.r[j] = rv; }
      if (MODE == PW_PCG) {
        const T dv = a.d[j];
        const double xv = fma(alpha64, (double)dv, a.x[j]);
        a.x[j] = xv;
        rv = fma(-alpha, a.q[j], rv);
        a.r[j] = rv;
        md = fmax(md, fabs((double)dv));
        mx = fmax(mx, fabs((double)xv));
      }
      const T sv = rv * inv[c];
      if (a.s) a.s[j] = sv;  // thermal / elastic PCG keeps no s (formed from r where it is used)
      sum += (double)rv * (double)sv;
      mr = fmax(mr, fabs((double)rv));
    }
  }
  if (MODE == PW_DIR) return;
  const double vals[4] = {sum, mr, md, mx};
  const bool ismax[4] = {false, true, true, true};
  double out[4];
  if (grid_reduce<PW_NT, 4>(vals, ismax, a.rc, blockIdx.x, out, sred) && tid == 0) {
    for (int k = 0; k < 4; k++) a.sc->red[k] = out[k];
    pcg_finish(MODE, out, a.sc, a.cfg);
  }
}

// Plain vector helpers.
template <typename T>
__global__ void k_fill(T* v, T val, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] = val;
}
template <typename Ts, typename Td>
__global__ void k_convert(const Ts* a, Td* b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) b[i] = (Td)a[i];
}

}  // namespace chfem
