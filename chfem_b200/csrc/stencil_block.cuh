// stencil_block.cuh -- block multi-RHS form of the thermal/elastic PCG passes: the load
// cases of one model (3 thermal, 6 elastic) advance together, so each pass reads the node keys
// and element matrices once for all of them.
//
// The reference solves the load cases one after the other
// (chfem/src/femhmg/femhmg.c:1017-1119), each apply re-reading the image and re-loading every
// element-matrix coefficient.  Here one CTA applies the operator to NR fields at once: it
// loops over the 27 neighbours of a node, loads each neighbour's NR field values once, and
// reuses every (broadcast) element-matrix coefficient for all NR fields -- the single-field
// kernel issues one shared-memory load per FMA, this one NR FMAs per coefficient load.  Every
// right-hand side keeps its own PCG scalars and stopping test (one DevScalars record each) and
// follows the single-solve recurrence; only the summation order of the operator differs
// (neighbour by neighbour instead of element by element).
#pragma once
#include <type_traits>
#include <utility>
#include "common.cuh"
#include "stencil_te.cuh"
#include "pointwise.cuh"

namespace chfem {

constexpr int BLK_MAX = 6;

template <int ND, typename T>
struct BlkArgs {
  const T* s;       // [NR][n]: r_k (the direction is formed from M^-1 r_k, M^-1 from the keys)
  const T* dold;    // [NR][n]
  T* dnew;          // [NR][n]
  T* q;             // [NR][n]
  const uint16_t* keys;
  const T* Kd;
  int nmat;
  int R, C, L;
  long n;           // unknowns per right-hand side
  DevScalars* sc;   // [NR]
  RedCtl rc;
  int precond;      // 0: M = I (plain CG, and the bare operator apply)
};

// point stride in the staged planes: NR*ND values padded to an odd count (conflict-free
// per-lane access for 32- and 64-bit words)
template <int ND, int NR>
__host__ __device__ constexpr int blk_ps() { return (NR * ND) % 2 ? NR * ND : NR * ND + 1; }

// Element matrices in shared memory.  FP32 elastic: "quad" layout, the 3 columns of one
// (row, local node b) block padded to 4 so one 16-byte load brings all three; a material's
// 24 x 8 quads are followed by 4 padding words, which puts the 4 materials' copies of a quad
// in different banks.  Otherwise row-major ED x ED per material plus one padding word.
template <int ND, typename T>
__host__ __device__ constexpr bool blk_quad() { return ND == 3 && std::is_same<T, float>::value; }
template <int ND, typename T>
__host__ __device__ constexpr int blk_kstride() { return blk_quad<ND, T>() ? 24 * 8 * 4 + 4 : 64 * ND * ND + 1; }

template <int ND, typename T, int NR>
inline size_t blk_smem_bytes() {
  return (size_t)4 * blk_kstride<ND, T>() * sizeof(T) + (size_t)3 * TE_PP * blk_ps<ND, NR>() * sizeof(T) + 16;
}

// The (voxel e, local node b) pairs of the node-centred operator, ordered by the neighbour
// node they reach, as compile-time constants: neighbour o = (drow+1) + 3 (dcol+1) + 9 (dlay+1)
// of node b relative to node e.  The conduction matrix has no coupling between nodes that share
// an element edge, so those pairs are dropped for one DOF per node.
__host__ __device__ constexpr int pair_nbr(int e, int b) {
  return (drow(b) - drow(e) + 1) + 3 * (dcol(b) - dcol(e) + 1) + 9 * (dlay(b) - dlay(e) + 1);
}
template <int ND>
__host__ __device__ constexpr bool pair_used(int e, int b) { return !(ND == 1 && shares_edge(e, b)); }
template <int ND>
__host__ __device__ constexpr int pair_count() {
  int n = 0;
  for (int e = 0; e < 8; e++)
    for (int b = 0; b < 8; b++) n += pair_used<ND>(e, b) ? 1 : 0;
  return n;
}
// pair number P in neighbour order, encoded 8 e + b (-1 past the end)
template <int ND>
__host__ __device__ constexpr int pair_at(int P) {
  int n = 0;
  for (int o = 0; o < 27; o++)
    for (int e = 0; e < 8; e++)
      for (int b = 0; b < 8; b++)
        if (pair_used<ND>(e, b) && pair_nbr(e, b) == o) {
          if (n == P) return 8 * e + b;
          n++;
        }
  return -1;
}

// One pair: load the neighbour's values for all right-hand sides when the pair is the first one
// reaching that neighbour, then out_k += K_e(rows of node e, columns of node b) v_k.
template <int ND, typename T, int NR, int P>
__device__ __forceinline__ void blk_pair_step(const T* pl0, const T* pl1, const T* pl2, int ctr, const T* const (&kb)[8],
                                              T (&v)[NR][ND], T (&out)[NR][ND]) {
  constexpr int ED = 8 * ND;
  constexpr int PS = blk_ps<ND, NR>();
  constexpr int eb = pair_at<ND>(P);
  constexpr int e = eb >> 3, b = eb & 7;
  constexpr int o = pair_nbr(e, b);
  constexpr bool first = (P == 0) || (pair_nbr(pair_at<ND>(P - 1) >> 3, pair_at<ND>(P - 1) & 7) != o);
  if constexpr (first) {
    constexpr int orr = o % 3 - 1, occ = (o / 3) % 3 - 1, oll = o / 9 - 1;
    const T* pb = (oll < 0 ? pl0 : (oll == 0 ? pl1 : pl2)) + (ctr + orr + occ * TE_PR) * PS;
#pragma unroll
    for (int k = 0; k < NR; k++)
#pragma unroll
      for (int cj = 0; cj < ND; cj++) v[k][cj] = pb[k * ND + cj];
  }
  const T* K = kb[e] + e * ND * ED + b * ND;
#pragma unroll
  for (int ci = 0; ci < ND; ci++) {
    [[maybe_unused]] float4 kq;
    if constexpr (blk_quad<ND, T>()) kq = *reinterpret_cast<const float4*>(kb[e] + ((e * ND + ci) * 8 + b) * 4);
#pragma unroll
    for (int cj = 0; cj < ND; cj++) {
      T kv;
      if constexpr (blk_quad<ND, T>()) kv = cj == 0 ? kq.x : (cj == 1 ? kq.y : kq.z);
      else kv = K[ci * ED + cj];
      if constexpr (std::is_same<T, float>::value && NR >= 2) {
        // two right-hand sides per instruction (packed FP32 FMA of sm_100): the same rounding
        // as two scalar FMAs, half the issue slots of the FMA stream; an odd last one alone
        const float2 kk = make_float2(kv, kv);
#pragma unroll
        for (int k = 0; k + 1 < NR; k += 2) {
          const float2 o = __ffma2_rn(kk, make_float2(v[k][cj], v[k + 1][cj]), make_float2(out[k][ci], out[k + 1][ci]));
          out[k][ci] = o.x;
          out[k + 1][ci] = o.y;
        }
        if constexpr (NR % 2) out[NR - 1][ci] = fma(kv, v[NR - 1][cj], out[NR - 1][ci]);
      } else {
#pragma unroll
        for (int k = 0; k < NR; k++) out[k][ci] = fma(kv, v[k][cj], out[k][ci]);
      }
    }
  }
}
template <int ND, typename T, int NR, int... Ps>
__device__ __forceinline__ void blk_all_pairs(std::integer_sequence<int, Ps...>, const T* pl0, const T* pl1, const T* pl2, int ctr,
                                              const T* const (&kb)[8], T (&out)[NR][ND]) {
  T v[NR][ND];
  (blk_pair_step<ND, T, NR, Ps>(pl0, pl1, pl2, ctr, kb, v, out), ...);
}

template <int ND, typename T, int NR>
__global__ void __launch_bounds__(TE_NT) k_blk_apply(BlkArgs<ND, T> a) {
  constexpr int ED = 8 * ND;
  constexpr int PS = blk_ps<ND, NR>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[TE_NT / 32];
  __shared__ T sbeta[NR];
  __shared__ int sdone[NR];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < NR; k++) all_done = all_done && a.sc[k].done;
  if (all_done) return;
  T* sK = reinterpret_cast<T*>(smem_raw);
  constexpr int kstride = blk_kstride<ND, T>();
  T* sP = sK + 4 * kstride;
  const int tid = threadIdx.x + TE_TR * threadIdx.y;
  if constexpr (blk_quad<ND, T>()) {
    for (int q = tid; q < 4 * kstride; q += TE_NT) {
      const int mat = q / kstride, w = q % kstride, row = w / 32, b = (w / 4) % 8, cj = w % 4;
      const bool used = w < 24 * 8 * 4 && cj < 3 && mat < a.nmat;
      sK[q] = used ? a.Kd[(size_t)mat * ED * ED + row * ED + b * 3 + cj] : T(0);
    }
  } else {
    for (int i = tid; i < 4 * ED * ED; i += TE_NT) sK[(i / (ED * ED)) * kstride + i % (ED * ED)] = (i < a.nmat * ED * ED) ? a.Kd[i] : T(0);
  }
  __shared__ T sD[4 * 8 * ND];
  for (int i = tid; i < 4 * 8 * ND; i += TE_NT) {
    const int m = i / (8 * ND), kk = i % (8 * ND);
    sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)kk * ED + kk] : T(1);
  }
  if (tid < NR) { sbeta[tid] = T(a.sc[tid].beta); sdone[tid] = a.sc[tid].done; }
  __syncthreads();
  const int R = a.R, C = a.C, L = a.L;
  const size_t RC = (size_t)R * C;
  int r0 = 0, c0 = 0;  // column tile of the current run
  const long n = a.n;
  const bool pre = a.precond != 0;
  auto slot_of = [&](int l) { return ((l % 3) + 3) % 3; };
  auto load_plane = [&](int l) {
    const int lw = wrap(l, L);
    T* dst = sP + slot_of(l) * TE_PP * PS;
    for (int p = tid; p < TE_PP; p += TE_NT) {
      const int hr = p % TE_PR, hc = p / TE_PR;
      const int gr = wrap(r0 + hr - 1, R), gc = wrap(c0 + hc - 1, C);
      const size_t node = (size_t)gr + (size_t)gc * R + (size_t)lw * RC;
      T inv[ND];
      if (pre) te_invdiag<ND, T>(sD, a.keys[node], inv);
      else {
#pragma unroll
        for (int c = 0; c < ND; c++) inv[c] = T(1);
      }
#pragma unroll
      for (int k = 0; k < NR; k++)
#pragma unroll
        for (int c = 0; c < ND; c++) {
          const size_t j = (size_t)k * n + node * ND + c;
          dst[p * PS + k * ND + c] = fma(sbeta[k], a.dold[j], a.s[j] * inv[c]);
        }
    }
  };
  double acc[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) acc[k] = 0.0;
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * TE_PR;
  const TeWork wk(R, C, L);
  for (long w = wk.begin(), w_end = wk.end(); w < w_end;) {
  int l0, l1;
  wk.run(w, w_end, r0, c0, l0, l1);
  const int r = r0 + threadIdx.x, c = c0 + threadIdx.y;
  const bool active = (r < R) && (c < C);
  __syncthreads();
  load_plane(l0 - 1);
  load_plane(l0);
  for (int l = l0; l < l1; l++) {
    load_plane(l + 1);
    __syncthreads();
    if (active) {
      const size_t node = (size_t)r + (size_t)c * R + (size_t)l * RC;
      const unsigned key = a.keys[node];
      const T* pl0 = sP + slot_of(l - 1) * TE_PP * PS;
      const T* pl1 = sP + slot_of(l) * TE_PP * PS;
      const T* pl2 = sP + slot_of(l + 1) * TE_PP * PS;
      const T* kb[8];
#pragma unroll
      for (int e = 0; e < 8; e++) kb[e] = sK + ((key >> (2 * e)) & 3u) * kstride;
      T out[NR][ND];
#pragma unroll
      for (int k = 0; k < NR; k++)
#pragma unroll
        for (int ci = 0; ci < ND; ci++) out[k][ci] = T(0);
      blk_all_pairs<ND, T, NR>(std::make_integer_sequence<int, pair_count<ND>()>{}, pl0, pl1, pl2, ctr, kb, out);
      const T* pc = pl1 + ctr * PS;
#pragma unroll
      for (int k = 0; k < NR; k++)
#pragma unroll
        for (int ci = 0; ci < ND; ci++) {
          const size_t j = (size_t)k * n + node * ND + ci;
          const T vv = pc[k * ND + ci];
          a.q[j] = out[k][ci];
          a.dnew[j] = vv;
          acc[k] += (double)vv * (double)out[k][ci];
        }
    }
    __syncthreads();
  }
  w += l1 - l0;
  }
  const bool ismax[NR] = {};
  double res[NR];
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (grid_reduce<TE_NT, NR>(acc, ismax, a.rc, bid, res, sred) && tid == 0) {
#pragma unroll
    for (int k = 0; k < NR; k++)
      if (!sdone[k]) { a.sc[k].red[0] = res[k]; a.sc[k].alpha = a.sc[k].delta / res[k]; }
  }
}

// Pointwise pass for all right-hand sides: x_k += a_k d_k, r_k -= a_k q_k, s_k = M^-1 r_k (not
// stored when a.s is null: the operator pass forms it), delta_k and the max-norms, then each
// right-hand side's own finisher (pcg_finish).
template <int ND, typename T>
struct BlkPw {
  double* x; const T* d; T* r; const T* q; T* s;   // [NR][n]
  const uint16_t* keys;
  const T* Kd; int nmat;
  long N, n;
  DevScalars* sc;  // [NR]
  RedCtl rc;
  SolveCfg cfg;
};

// MAXN: the stopping test needs the max-norms (infinity / error norm); the L2 test needs the
// sums r.M^-1 r only, which keeps the per-thread accumulators to NR.
template <int ND, typename T, int NR, bool MAXN>
__global__ void __launch_bounds__(PW_NT) k_blk_point(BlkPw<ND, T> a) {
  constexpr int ED = 8 * ND;
  constexpr int NV = MAXN ? 4 : 1;  // reduced values per right-hand side
  __shared__ double sred[PW_NT / 32];
  __shared__ T sD[4 * 8 * ND];
  __shared__ double salpha[NR];
  __shared__ int sdone[NR];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < NR; k++) all_done = all_done && a.sc[k].done;
  if (all_done) return;
  const int tid = threadIdx.x;
  for (int i = tid; i < 4 * 8 * ND; i += PW_NT) {
    const int m = i / (8 * ND), kk = i % (8 * ND);
    sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)kk * ED + kk] : T(1);
  }
  if (tid < NR) { salpha[tid] = a.sc[tid].alpha; sdone[tid] = a.sc[tid].done; }
  __syncthreads();
  double vals[NV * NR];
#pragma unroll
  for (int k = 0; k < NV * NR; k++) vals[k] = 0.0;
  for (long i = blockIdx.x * (long)PW_NT + tid; i < a.N; i += (long)gridDim.x * PW_NT) {
    T inv[ND];
    if (a.cfg.precond) te_invdiag<ND, T>(sD, a.keys[i], inv);
    else {
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(1);
    }
#pragma unroll
    for (int k = 0; k < NR; k++) {
      if (sdone[k]) continue;
      const double al64 = salpha[k];
      const T al = T(al64);
#pragma unroll
      for (int c = 0; c < ND; c++) {
        const long j = (long)k * a.n + i * ND + c;
        const T dv = a.d[j];
        const double xv = fma(al64, (double)dv, a.x[j]);
        a.x[j] = xv;
        const T rv = fma(-al, a.q[j], a.r[j]);
        a.r[j] = rv;
        const T sv = rv * inv[c];
        if (a.s) a.s[j] = sv;
        vals[NV * k] += (double)rv * (double)sv;
        if constexpr (MAXN) {
          vals[NV * k + 1] = fmax(vals[NV * k + 1], fabs((double)rv));
          vals[NV * k + 2] = fmax(vals[NV * k + 2], fabs((double)dv));
          vals[NV * k + 3] = fmax(vals[NV * k + 3], fabs(xv));
        }
      }
    }
  }
  bool ismax[NV * NR];
#pragma unroll
  for (int k = 0; k < NV * NR; k++) ismax[k] = (k % NV) != 0;
  double out[NV * NR];
  if (grid_reduce<PW_NT, NV * NR>(vals, ismax, a.rc, blockIdx.x, out, sred) && tid == 0) {
#pragma unroll
    for (int k = 0; k < NR; k++) {
      if (sdone[k]) continue;
      double s4[4] = {out[NV * k], 0.0, 0.0, 0.0};
      if constexpr (MAXN) { s4[1] = out[NV * k + 1]; s4[2] = out[NV * k + 2]; s4[3] = out[NV * k + 3]; }
      for (int t = 0; t < 4; t++) a.sc[k].red[t] = s4[t];
      pcg_finish(PW_PCG, s4, a.sc + k, a.cfg);
    }
  }
}

// The same pass with each thread on 4 consecutive unknowns of every right-hand side (16-byte
// vector loads and stores of whole warps' contiguous 512-byte runs) instead of one node's ND
// unknowns at a stride of ND words, which made each warp access touch ND times the sectors it
// used.  The Jacobi diagonal of the (at most two) nodes the 4 unknowns belong to comes from
// their keys.  Requires n % 4 == 0 (every right-hand side's vectors start 16-byte aligned).
template <typename T>
__device__ __forceinline__ void blk_ld4(const T* p, T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p)), b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}
template <typename T>
__device__ __forceinline__ void blk_st4(T* p, const T (&v)[4]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
  }
}

template <int ND, typename T, int NR, bool MAXN>
__global__ void __launch_bounds__(PW_NT) k_blk_point4(BlkPw<ND, T> a) {
  constexpr int ED = 8 * ND;
  constexpr int NV = MAXN ? 4 : 1;
  __shared__ double sred[PW_NT / 32];
  __shared__ T sD[4 * 8 * ND];
  __shared__ double salpha[NR];
  __shared__ int sdone[NR];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < NR; k++) all_done = all_done && a.sc[k].done;
  if (all_done) return;
  const int tid = threadIdx.x;
  for (int i = tid; i < 4 * 8 * ND; i += PW_NT) {
    const int m = i / (8 * ND), kk = i % (8 * ND);
    sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)kk * ED + kk] : T(1);
  }
  if (tid < NR) { salpha[tid] = a.sc[tid].alpha; sdone[tid] = a.sc[tid].done; }
  __syncthreads();
  double vals[NV * NR];
#pragma unroll
  for (int k = 0; k < NV * NR; k++) vals[k] = 0.0;
  const long n4 = a.n / 4;
  for (long t = blockIdx.x * (long)PW_NT + tid; t < n4; t += (long)gridDim.x * PW_NT) {
    const long j0 = 4 * t;
    T inv[4];
    if (a.cfg.precond) {
      // the 4 unknowns span nodes j0 / ND .. (j0 + 3) / ND (at most 2 for ND = 3, 4 for ND = 1)
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const long node = (j0 + i) / ND;
        const int c = (int)(j0 + i - node * ND);
        if (ND == 1 || i == 0 || c == 0) {  // first unknown of a node in this chunk: its diagonal
          T iv[ND];
          te_invdiag<ND, T>(sD, a.keys[node], iv);
#pragma unroll
          for (int q = i; q < 4; q++) {
            const int cq = (int)(j0 + q - node * ND);
            if (cq < ND) inv[q] = iv[cq];
          }
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 4; i++) inv[i] = T(1);
    }
#pragma unroll
    for (int k = 0; k < NR; k++) {
      if (sdone[k]) continue;
      const double al64 = salpha[k];
      const T al = T(al64);
      const long j = (long)k * a.n + j0;
      T dv[4], qv[4], rv[4], sv[4];
      blk_ld4(a.d + j, dv);
      blk_ld4(a.q + j, qv);
      blk_ld4(a.r + j, rv);
      const double2 x01 = __ldcs(reinterpret_cast<const double2*>(a.x + j)), x23 = __ldcs(reinterpret_cast<const double2*>(a.x + j) + 1);
      double xv[4] = {x01.x, x01.y, x23.x, x23.y};
#pragma unroll
      for (int i = 0; i < 4; i++) {
        xv[i] = fma(al64, (double)dv[i], xv[i]);
        rv[i] = fma(-al, qv[i], rv[i]);
        sv[i] = rv[i] * inv[i];
        vals[NV * k] += (double)rv[i] * (double)sv[i];
        if constexpr (MAXN) {
          vals[NV * k + 1] = fmax(vals[NV * k + 1], fabs((double)rv[i]));
          vals[NV * k + 2] = fmax(vals[NV * k + 2], fabs((double)dv[i]));
          vals[NV * k + 3] = fmax(vals[NV * k + 3], fabs(xv[i]));
        }
      }
      reinterpret_cast<double2*>(a.x + j)[0] = make_double2(xv[0], xv[1]);
      reinterpret_cast<double2*>(a.x + j)[1] = make_double2(xv[2], xv[3]);
      blk_st4(a.r + j, rv);
      if (a.s) blk_st4(a.s + j, sv);
    }
  }
  bool ismax[NV * NR];
#pragma unroll
  for (int k = 0; k < NV * NR; k++) ismax[k] = (k % NV) != 0;
  double out[NV * NR];
  if (grid_reduce<PW_NT, NV * NR>(vals, ismax, a.rc, blockIdx.x, out, sred) && tid == 0) {
#pragma unroll
    for (int k = 0; k < NR; k++) {
      if (sdone[k]) continue;
      double s4[4] = {out[NV * k], 0.0, 0.0, 0.0};
      if constexpr (MAXN) { s4[1] = out[NV * k + 1]; s4[2] = out[NV * k + 2]; s4[3] = out[NV * k + 3]; }
      for (int t = 0; t < 4; t++) a.sc[k].red[t] = s4[t];
      pcg_finish(PW_PCG, s4, a.sc + k, a.cfg);
    }
  }
}

}  // namespace chfem
