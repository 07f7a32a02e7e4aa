// minres.cuh -- pointwise pass of the (preconditioned) conjugate-residual recurrence that
// chfem calls MINRES / PMINRES (chfem/src/femhmg/cudapcg/solvers/pminres.cu:163-170,
// minres.cu:174-181):  z = M^-1 r;  d = z + b d;  q = s + b q;  a = delta / (q . M^-1 q).
// The other half of the iteration (x += a d, r -= a q, s = A M^-1 r, delta, stopping test)
// is the TE_MR / fluid MR form of the operator kernels.
//
// Difference from the reference, by design: the reference keeps r in place, turning it into
// M^-1 r and back with the Jacobi inverse (pminres.cu:172-176); for thermal and elastic
// models its inverse-Jacobi is an unimplemented stub (wrappers.cu:635-648), which leaves r
// scaled.  This library keeps r and z = M^-1 r apart, which is the Stokes behaviour of the
// reference up to round-off and the intended recurrence for every physics.
#pragma once
#include "common.cuh"
#include "stencil_te.cuh"
#include "stencil_fluid.cuh"

namespace chfem {

template <int ND, typename T>
struct MrDirTe {
  T* d; T* q; const T* r; const T* s;
  const uint16_t* keys; const T* Kd; int nmat;
  long N;
  DevScalars* sc; RedCtl rc; int precond;
  const double* invd = nullptr;  // precomputed inverse Jacobi diagonal (density field, 2D models)
};

template <int ND, typename T>
__global__ void __launch_bounds__(PW_NT) k_te_mr_dir(MrDirTe<ND, T> a) {
  constexpr int ED = 8 * ND;
  __shared__ double sred[PW_NT / 32];
  __shared__ T sD[4 * 8 * ND];
  if (a.sc->done) return;
  for (int i = threadIdx.x; i < 4 * 8 * ND; i += PW_NT) {
    const int m = i / (8 * ND), k = i % (8 * ND);
    sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)k * ED + k] : T(1);
  }
  __syncthreads();
  const T b = T(a.sc->beta);
  double sum = 0.0;
  for (long i = blockIdx.x * (long)PW_NT + threadIdx.x; i < a.N; i += (long)gridDim.x * PW_NT) {
    T inv[ND];
    if (a.precond && a.invd) {
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(a.invd[i * ND + c]);
    } else if (a.precond) te_invdiag<ND, T>(sD, a.keys[i], inv);
    else {
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(1);
    }
#pragma unroll
    for (int c = 0; c < ND; c++) {
      const long j = i * ND + c;
      const T z = a.r[j] * inv[c];
      a.d[j] = fma(b, a.d[j], z);
      const T qn = fma(b, a.q[j], a.s[j]);
      a.q[j] = qn;
      sum += (double)qn * (double)(qn * inv[c]);
    }
  }
  const double vals[1] = {sum};
  const bool ismax[1] = {false};
  double out[1];
  if (grid_reduce<PW_NT, 1>(vals, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
    a.sc->red[5] = out[0];
    a.sc->alpha = a.sc->delta / out[0];
  }
}

template <typename T>
struct MrDirFl {
  T* d; T* q; const T* r; const T* s;
  const uint8_t* bkeys; long nV, nB;
  DevScalars* sc; RedCtl rc; int precond;
};

template <typename T, int DIM = 3>
__global__ void __launch_bounds__(PW_NT) k_fl_mr_dir(MrDirFl<T> a) {
  __shared__ double sred[PW_NT / 32];
  __shared__ double sbd[256];  // interface-node inverse diagonals by fluid key
  if (a.sc->done) return;
  for (int i = threadIdx.x; i < 256; i += PW_NT) sbd[i] = c_fldiag.border[i];
  __syncthreads();
  const T b = T(a.sc->beta);
  const long nV = a.nV, nT = a.nV + a.nB;
  double sum = 0.0;
  for (long t = blockIdx.x * (long)PW_NT + threadIdx.x; t < nT; t += (long)gridDim.x * PW_NT) {
    const bool pore = t < nV;
    const int cnt = pore ? DIM + 1 : 1;
    for (int k = 0; k < cnt; k++) {
      const long j = pore ? (k < DIM ? DIM * t + k : DIM * nV + t) : DIM * nV + t;
      T inv = T(1);
      if (a.precond) inv = pore ? T(c_fldiag.pore[k]) : T(sbd[a.bkeys[t - nV]]);
      const T z = a.r[j] * inv;
      a.d[j] = fma(b, a.d[j], z);
      const T qn = fma(b, a.q[j], a.s[j]);
      a.q[j] = qn;
      sum += (double)qn * (double)(qn * inv);
    }
  }
  const double vals[1] = {sum};
  const bool ismax[1] = {false};
  double out[1];
  if (grid_reduce<PW_NT, 1>(vals, ismax, a.rc, blockIdx.x, out, sred) && threadIdx.x == 0) {
    a.sc->red[5] = out[0];
    a.sc->alpha = a.sc->delta / out[0];
  }
}

template <typename T>
__global__ void k_sub_inplace(T* r, const T* y, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) r[i] -= y[i];
}

}  // namespace chfem
