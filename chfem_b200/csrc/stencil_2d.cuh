// stencil_2d.cuh -- matrix-free operator pass for 2D thermal (1 DOF/node) and elastic (2 DOF/node)
// homogenization on pixel images, node by node like the reference
// (chfem/src/femhmg/cudapcg/kernels/matrix_free.cu:70-95 thermal, :353-385 elastic): node i is
// local node e of the pixel at (row - drow(e) - 1, col - dcol(e)), e = 0..3, and the row block of
// local node e of that pixel's element matrix multiplies the pixel's 4 nodal values.  The node key
// holds the pixel's material in bits [4e, 4e + 4) (16 materials; femhmg_2D.c:14-46).
//
// B200 design: a CTA owns tiles of 32 (rows) x 8 (cols) nodes in turn (persistent grid); the
// tile's formed input with its one-node periodic halo is staged in shared memory once, next to
// the element matrices of up to 16 materials.  The Jacobi diagonal comes precomputed (a.invd,
// FP64 per unknown).  Under a scalar density field (a.sdf) each pixel's row block is scaled by
// the pixel's density (the reference's element-by-element density operators,
// matrix_free.cu:1832-1880, :2788-2850).  Modes, outputs and finishers are those of k_te_apply
// (stencil_te.cuh).
#pragma once
#include "common.cuh"
#include "stencil_te.cuh"

namespace chfem {

constexpr int T2_TR = 32, T2_TC = 8, T2_NT = T2_TR * T2_TC;
constexpr int T2_PR = T2_TR + 2, T2_PP = T2_PR * (T2_TC + 2);
constexpr int T2_NMAT = 16;

template <int ND, typename T>
inline size_t t2_smem_bytes() {
  return ((size_t)T2_NMAT * 16 * ND * ND + (size_t)T2_PP * ND) * sizeof(T) + 16;
}

template <int ND, typename T, int MODE>
__global__ void __launch_bounds__(T2_NT) k_2d_apply(TeArgs<ND, T> a) {
  constexpr int ED = 4 * ND;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[T2_NT / 32];
  if (a.skip_if_done && a.sc->done) return;
  T* sK = reinterpret_cast<T*>(smem_raw);  // [16][ED][ED]
  T* sP = sK + T2_NMAT * ED * ED;          // [T2_PP][ND]
  const int tid = threadIdx.x + T2_TR * threadIdx.y;
  for (int i = tid; i < T2_NMAT * ED * ED; i += T2_NT) sK[i] = (i < a.nmat * ED * ED) ? a.Kd[i] : T(0);
  const T beta = (MODE == TE_PCG || MODE == TE_DIRDOT) ? T(a.sc->beta) : T(0);
  const T alpha = (MODE == TE_MR && mr_steps(a.finish)) ? T(a.sc->alpha) : T(0);
  const double alpha64 = (MODE == TE_UPD) ? a.sc->alpha : 0.0;
  const bool pre = a.cfg.precond != 0;
  const int R = a.R, C = a.C;
  const int tiles_r = (R + T2_TR - 1) / T2_TR;
  const long tiles = (long)tiles_r * ((C + T2_TC - 1) / T2_TC);
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * T2_PR;
  double acc = 0.0, acc_rz = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  for (long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int r0 = (int)(t % tiles_r) * T2_TR, c0 = (int)(t / tiles_r) * T2_TC;
    __syncthreads();  // the previous tile's reads are done (and the matrices are in place)
    for (int p = tid; p < T2_PP; p += T2_NT) {
      const size_t node = (size_t)wrap(r0 + p % T2_PR - 1, R) + (size_t)wrap(c0 + p / T2_PR - 1, C) * R;
#pragma unroll
      for (int c = 0; c < ND; c++) {
        const size_t j = node * ND + c;
        T v = a.in0[j];
        if (MODE == TE_PCG || MODE == TE_DIRDOT || MODE == TE_MR) {
          const T inv = pre ? T(a.invd[j]) : T(1);
          if (MODE == TE_MR) v = fma(-alpha, a.in1[j], v) * inv;
          else v = fma(beta, a.in1[j], v * inv);
        }
        sP[p * ND + c] = v;
      }
    }
    __syncthreads();
    const int r = r0 + threadIdx.x, c = c0 + threadIdx.y;
    if (r >= R || c >= C) continue;
    const size_t node = (size_t)r + (size_t)c * R;
    const unsigned key = a.keys[node];
    T out[ND];
#pragma unroll
    for (int ci = 0; ci < ND; ci++) out[ci] = T(0);
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const T* K = sK + ((key >> (4 * e)) & 15u) * ED * ED + e * ND * ED;
      T pe[ND];  // the row block of pixel e times the pixel's nodal values
#pragma unroll
      for (int ci = 0; ci < ND; ci++) pe[ci] = T(0);
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const T* v = sP + (ctr + (drow(b) - drow(e)) + (dcol(b) - dcol(e)) * T2_PR) * ND;
#pragma unroll
        for (int ci = 0; ci < ND; ci++)
#pragma unroll
          for (int cj = 0; cj < ND; cj++) pe[ci] = fma(K[ci * ED + b * ND + cj], v[cj], pe[ci]);
      }
      if (a.sdf) {  // scalar density field: pixel e's matrix scaled by its density
        const size_t pix = (size_t)wrap(r - drow(e) - 1, R) + (size_t)wrap(c - dcol(e), C) * R;
        const T f = T(a.sdf_min + a.sdf_rng * (double)a.sdf[pix] * (1.0 / 65535.0));
#pragma unroll
        for (int ci = 0; ci < ND; ci++) out[ci] = fma(f, pe[ci], out[ci]);
      } else {
#pragma unroll
        for (int ci = 0; ci < ND; ci++) out[ci] += pe[ci];
      }
    }
#pragma unroll
    for (int cc = 0; cc < ND; cc++) {
      const size_t j = node * ND + cc;
      const T v = sP[ctr * ND + cc];
      if (MODE != TE_DIRDOT && MODE != TE_UPD) a.y[j] = out[cc];
      if (MODE == TE_PCG || MODE == TE_DIRDOT) a.vout[j] = v;
      if (MODE == TE_UPD) {
        const T inv = pre ? T(a.invd[j]) : T(1);
        const T rn = fma(-T(alpha64), out[cc], a.vout[j]);
        a.vout[j] = rn;
        const double xv = fma(alpha64, (double)v, a.x[j]);
        a.x[j] = xv;
        acc_rz += (double)rn * (double)(rn * inv);
        mr = fmax(mr, fabs((double)rn));
        md = fmax(md, fabs((double)v));
        mx = fmax(mx, fabs(xv));
      }
      if (MODE == TE_MR) {
        const T rn = fma(-alpha, a.in1[j], a.in0[j]);
        a.vout[j] = rn;
        const T dv = a.d[j];
        const double xv = fma((double)alpha, (double)dv, a.x[j]);
        a.x[j] = xv;
        acc_rz += (double)rn * (double)v;
        mr = fmax(mr, fabs((double)rn));
        md = fmax(md, fabs((double)dv));
        mx = fmax(mx, fabs((double)xv));
      }
      acc += (double)v * (double)out[cc];
    }
  }
  if (a.finish == FIN_NONE) return;
  if (MODE == TE_UPD) {
    const double vals[4] = {acc_rz, mr, md, mx};
    const bool ismax[4] = {false, true, true, true};
    double res[4];
    if (grid_reduce<T2_NT, 4>(vals, ismax, a.rc, blockIdx.x, res, sred) && tid == 0) {
      for (int k = 0; k < 4; k++) a.sc->red[k] = res[k];
      const SolveCfg cfg{a.cfg.tol, a.cfg.maxit, a.cfg.norm, a.cfg.precond, a.cfg.nhmg};
      pcg_finish(PW_PCG, res, a.sc, cfg);
    }
  } else if (MODE == TE_MR) {
    const double vals[5] = {acc, acc_rz, mr, md, mx};
    const bool ismax[5] = {false, false, true, true, true};
    double res[5];
    if (grid_reduce<T2_NT, 5>(vals, ismax, a.rc, blockIdx.x, res, sred) && tid == 0) {
      for (int k = 0; k < 5; k++) a.sc->red[k] = res[k];
      mr_finish(a.finish, res, a.sc, a.cfg);
    }
  } else {
    const double vals[1] = {acc};
    const bool ismax[1] = {false};
    double res[1];
    if (grid_reduce<T2_NT, 1>(vals, ismax, a.rc, blockIdx.x, res, sred) && tid == 0) {
      a.sc->red[0] = res[0];
      if (a.finish == FIN_ALPHA) a.sc->alpha = a.sc->delta / res[0];
    }
  }
}

// Inverse Jacobi diagonal of a 2D model, per unknown, FP64 (matrix_free.cu:51-68, :325-346);
// under a scalar density field (sdf non-null) each pixel's diagonal term is scaled by its
// density (matrix_free.cu:1350-1365, :1398-1416)
template <int ND>
__global__ void k_2d_invdiag(const uint16_t* keys, const double* Kd, int R, int C, const uint16_t* sdf, double fmin,
                             double frng, double* invd) {
  constexpr int ED = 4 * ND;
  const long N = (long)R * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const unsigned key = keys[i];
    const int r = (int)(i % R), cc = (int)(i / R);
    double f[4] = {1.0, 1.0, 1.0, 1.0};
    if (sdf) {
#pragma unroll
      for (int e = 0; e < 4; e++)
        f[e] = fmin + frng * (double)sdf[(size_t)wrap(r - drow(e) - 1, R) + (size_t)wrap(cc - dcol(e), C) * R] * (1.0 / 65535.0);
    }
#pragma unroll
    for (int c = 0; c < ND; c++) {
      double s = 0.0;
#pragma unroll
      for (int e = 0; e < 4; e++) s += f[e] * Kd[(size_t)((key >> (4 * e)) & 15u) * ED * ED + (e * ND + c) * ED + e * ND + c];
      invd[i * ND + c] = 1.0 / s;
    }
  }
}

// 2D node keys from the per-pixel material map (EBE input, femhmg_2D.c:14-46)
__global__ void k_keys_from_elements_2d(const uint16_t* em, uint16_t* keys, int R, int C) {
  const long N = (long)R * C;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i % R), c = (int)(i / R);
    unsigned k = 0;
#pragma unroll
    for (int e = 0; e < 4; e++) k |= ((unsigned)em[(size_t)wrap(r - drow(e) - 1, R) + (size_t)wrap(c - dcol(e), C) * R] & 15u) << (4 * e);
    keys[i] = (uint16_t)k;
  }
}

}  // namespace chfem
