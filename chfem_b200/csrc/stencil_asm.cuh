// stencil_asm.cuh -- block operator pass for images of at most two materials, with each node's
// 27-neighbour stencil assembled from the table of per-material-configuration blocks
// (asm_table.cuh).
//
// Each thread computes ZB nodes stacked along the layers, so the values of the neighbour planes
// the ZB nodes share are read from shared memory once for all of them.
#pragma once
#include <algorithm>
#include <type_traits>
#include <utility>
#include "common.cuh"
#include "asm_table.cuh"
#include "stencil_te.cuh"
#include "stencil_block.cuh"

namespace chfem {

// RING: staged planes in the shared-memory ring, ZB + 2 (the planes one step reads) or 2 ZB + 2
// (those plus the ZB planes the next step needs, staged while this step computes)
template <int ND, typename T, int NR, int TC, int ZB, int RING = ZB + 2>
inline size_t asm_smem_bytes() {
  using Lo = AsmLayout<ND, T, NR>;
  const size_t pp = (size_t)(TE_TR + 2) * (TC + 2);
  return ((size_t)asm_table_words(ND, Lo::BS) + (size_t)RING * pp * Lo::PS) * sizeof(T);
}


// does any of the ZB nodes use the neighbour position (Q plane, DR row, DC column)?
template <int ND, int ZB>
__host__ __device__ constexpr bool asm_pos_used(int Q, int DR, int DC) {
  for (int z = 0; z < ZB; z++) {
    const int dl = Q - z;
    if (dl >= -1 && dl <= 1 && asm_used<ND>((DR + 1) + 3 * (DC + 1) + 9 * (dl + 1))) return true;
  }
  return false;
}

template <int ND, typename T, int NR, int ZB, int Q, int DR, int DC, int Z>
__device__ __forceinline__ void asm_to_node(const T* __restrict__ sT, const unsigned (&m)[ZB],
                                            const typename AsmLayout<ND, T, NR>::V (&val)[ND][AsmLayout<ND, T, NR>::NW],
                                            typename AsmLayout<ND, T, NR>::V (&out)[ZB][ND][AsmLayout<ND, T, NR>::NW]) {
  constexpr int DL = Q - Z;
  if constexpr (DL >= -1 && DL <= 1) asm_block<ND, T, (DR + 1) + 3 * (DC + 1) + 9 * (DL + 1)>(sT, m[Z], val, out[Z]);
}
template <int ND, typename T, int NR, int ZB, int Q, int DR, int DC, int... Zs>
__device__ __forceinline__ void asm_to_nodes(std::integer_sequence<int, Zs...>, const T* __restrict__ sT, const unsigned (&m)[ZB],
                                             const typename AsmLayout<ND, T, NR>::V (&val)[ND][AsmLayout<ND, T, NR>::NW],
                                             typename AsmLayout<ND, T, NR>::V (&out)[ZB][ND][AsmLayout<ND, T, NR>::NW]) {
  (asm_to_node<ND, T, NR, ZB, Q, DR, DC, Zs>(sT, m, val, out), ...);
}

// Position P of the (ZB + 2) x 3 x 3 neighbour positions: plane Q = P / 9 - 1 relative to the
// first node's layer, row DR = P % 3 - 1, column DC = (P / 3) % 3 - 1.  Loads the position's
// values for every right-hand side once and adds them into each node that reaches it.
template <int ND, typename T, int NR, int ZB, int P>
__device__ __forceinline__ void asm_position(const T* const (&pl)[ZB + 2], int ctr, const T* __restrict__ sT, const unsigned (&m)[ZB],
                                             typename AsmLayout<ND, T, NR>::V (&out)[ZB][ND][AsmLayout<ND, T, NR>::NW]) {
  constexpr int Q = P / 9 - 1, DR = P % 3 - 1, DC = (P / 3) % 3 - 1;
  if constexpr (asm_pos_used<ND, ZB>(Q, DR, DC)) {
    using Lo = AsmLayout<ND, T, NR>;
    using V = typename Lo::V;
    const V* pv = reinterpret_cast<const V*>(pl[Q + 1] + (ctr + DR + DC * TE_PR) * Lo::PS);
    V val[ND][Lo::NW];
#pragma unroll
    for (int cj = 0; cj < ND; cj++)
#pragma unroll
      for (int w = 0; w < Lo::NW; w++) val[cj][w] = pv[cj * Lo::NW + w];
    asm_to_nodes<ND, T, NR, ZB, Q, DR, DC>(std::make_integer_sequence<int, ZB>{}, sT, m, val, out);
  }
}
template <int ND, typename T, int NR, int ZB, int... Ps>
__device__ __forceinline__ void asm_positions(std::integer_sequence<int, Ps...>, const T* const (&pl)[ZB + 2], int ctr,
                                              const T* __restrict__ sT, const unsigned (&m)[ZB],
                                              typename AsmLayout<ND, T, NR>::V (&out)[ZB][ND][AsmLayout<ND, T, NR>::NW]) {
  (asm_position<ND, T, NR, ZB, Ps>(pl, ctr, sT, m, out), ...);
}

// The block PCG operator pass: d_new_k = M^-1 r_k + beta_k d_old_k (the Jacobi diagonal from
// the node keys; a.s holds r), q_k = A d_new_k, and per right-hand side the sum d_new_k . q_k
// reduced over the grid, whose last CTA sets alpha_k = delta_k / (d_new_k . q_k).  A CTA owns a
// 32 x TC column of nodes and marches through its run of layers ZB at a time, with ZB + 2
// halo'd planes of d_new staged in shared memory (d_new is formed while staging).  At the start
// of a step the CTA asks L2 to prefetch (bulk prefetch, one request per contiguous column
// segment of every input vector) the planes it stages after the step, so that those loads find
// them in L2.  MINB: CTAs per SM the registers are capped for.  RING = 2 ZB + 2: the ring also
// holds the next step's planes, which are staged before this step's arithmetic (into slots
// that step does not read), so a step ends with one barrier instead of two and a warp's
// staging loads overlap the other warps' arithmetic.  Requires node keys of materials 0 and 1
// only.
template <int ND, typename T, int NR, int TC, int ZB, int MINB = 1, int RING = ZB + 2>
__global__ void __launch_bounds__(TE_TR * TC, MINB) k_asm_apply(BlkArgs<ND, T> a, const T* __restrict__ tab) {
  static_assert(RING == ZB + 2 || RING == 2 * ZB + 2, "plane ring: ZB + 2 or 2 ZB + 2 slots");
  constexpr bool AHEAD = RING == 2 * ZB + 2;
  using Lo = AsmLayout<ND, T, NR>;
  using V = typename Lo::V;
  constexpr int NW = Lo::NW;
  constexpr int NT = TE_TR * TC;
  constexpr int PS = Lo::PS;
  constexpr int PP = TE_PR * (TC + 2);
  constexpr int NPL = ZB + 2;
  constexpr int PPT = (PP + NT - 1) / NT;  // staged points per thread and plane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[NT / 32];
  __shared__ T sbeta[NR];
  __shared__ int sdone[NR];
  bool all_done = true;
#pragma unroll
  for (int k = 0; k < NR; k++) all_done = all_done && a.sc[k].done;
  if (all_done) return;
  constexpr int TW = asm_table_words(ND, Lo::BS);  // a multiple of 4 words: 16-byte alignment kept
  T* sT = reinterpret_cast<T*>(smem_raw);
  const T* sInv = sT + ASM_NBLK * Lo::BS;  // inverse Jacobi diagonal by node configuration
  T* sP = sT + TW;
  const int tid = threadIdx.x + TE_TR * threadIdx.y;
  for (int i = tid; i < TW; i += NT) sT[i] = tab[i];
  if (tid < NR) { sbeta[tid] = T(a.sc[tid].beta); sdone[tid] = a.sc[tid].done; }
  __syncthreads();
  const int R = a.R, C = a.C, L = a.L;
  const size_t RC = (size_t)R * C;
  const long n = a.n;
  const bool pre = a.precond != 0;
  T beta[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) beta[k] = sbeta[k];
  int r0 = 0, c0 = 0;
  size_t poff[PPT];  // in-layer node index of this thread's staged points (for the current tile)
  auto slot_of = [&](int l) { return ((l % RING) + RING) % RING; };
  auto load_plane = [&](int l) {
    const size_t lo = (size_t)wrap(l, L) * RC;
    T* dst = sP + slot_of(l) * PP * PS;
#pragma unroll
    for (int i = 0; i < PPT; i++) {
      const int p = tid + i * NT;
      if (PP % NT == 0 || p < PP) {
        const size_t node = poff[i] + lo;
        T inv[ND];
        if (pre) {
          const unsigned m = asm_config(a.keys[node]);
#pragma unroll
          for (int c = 0; c < ND; c++) inv[c] = sInv[m * ND + c];
        } else {
#pragma unroll
          for (int c = 0; c < ND; c++) inv[c] = T(1);
        }
#pragma unroll
        for (int k = 0; k < NR; k++)
#pragma unroll
          for (int c = 0; c < ND; c++) {
            const size_t j = (size_t)k * n + node * ND + c;
            dst[p * PS + c * NR + k] = fma(beta[k], a.dold[j], a.s[j] * inv[c]);
          }
      }
    }
  };
  // L2 prefetch of plane l of the current tile: per input vector and tile column, the rows of
  // the tile and its halo that are contiguous in memory (a wrapped halo row is left out)
  auto prefetch_plane = [&](int l) {
    const size_t lo = (size_t)wrap(l, L) * RC;
    const int ra = max(r0 - 1, 0), rb = min(r0 + TE_TR, R - 1);
    for (int i = tid; i < 2 * NR * (TC + 2); i += NT) {
      const int k = i % NR, arr = (i / NR) % 2, hc = i / (2 * NR);
      const size_t node = (size_t)ra + (size_t)wrap(c0 + hc - 1, C) * R + lo;
      const T* base = (arr ? a.dold : a.s) + (size_t)k * n + node * ND;
      asm_prefetch_l2(base, (size_t)(rb - ra + 1) * ND * sizeof(T));
    }
  };
  double acc[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) acc[k] = 0.0;
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * TE_PR;
  const TeWork wk(R, C, L, TC);
  for (long w = wk.begin(), w_end = wk.end(); w < w_end;) {
    int l0, l1;
    wk.run(w, w_end, r0, c0, l0, l1);
    const int r = r0 + threadIdx.x, c = c0 + threadIdx.y;
    const bool active = (r < R) && (c < C);
#pragma unroll
    for (int i = 0; i < PPT; i++) {
      const int p = min(tid + i * NT, PP - 1);
      const int gr = wrap(r0 + p % TE_PR - 1, R), gc = wrap(c0 + p / TE_PR - 1, C);
      poff[i] = (size_t)gr + (size_t)gc * R;
    }
    // node keys are fetched one step ahead, so their global-memory latency overlaps the
    // staging and the previous step's arithmetic; past the run any valid node of the column
    // stands in (its result is not stored)
    const size_t col = active ? (size_t)r + (size_t)c * R : 0;
    unsigned kc[ZB];
#pragma unroll
    for (int z = 0; z < ZB; z++) kc[z] = a.keys[col + (size_t)(l0 + z < l1 ? l0 + z : l0) * RC];
    __syncthreads();  // the previous run's planes are no longer read
#pragma unroll
    for (int q = -1; q <= ZB; q++) load_plane(l0 + q);
    __syncthreads();
    for (int l = l0; l < l1; l += ZB) {
      if (l + ZB < l1) {
#pragma unroll
        for (int q = 1; q <= ZB; q++) prefetch_plane(l + ZB + q);
      }
      unsigned kn[ZB];
#pragma unroll
      for (int z = 0; z < ZB; z++) kn[z] = a.keys[col + (size_t)(l + ZB + z < l1 ? l + ZB + z : l) * RC];
      if constexpr (AHEAD) {
        // planes l + ZB + 1 .. l + 2 ZB into the slots of l - ZB - 1 .. l - 2, read by the
        // previous step only (done before its closing barrier)
        if (l + ZB < l1) {
#pragma unroll
          for (int q = 1; q <= ZB; q++) load_plane(l + ZB + q);
        }
      }
      if (active) {
        const T* pl[NPL];
#pragma unroll
        for (int q = 0; q < NPL; q++) pl[q] = sP + slot_of(l - 1 + q) * PP * PS;
        unsigned m[ZB];
#pragma unroll
        for (int z = 0; z < ZB; z++) m[z] = asm_config(kc[z]);
        V out[ZB][ND][NW];
#pragma unroll
        for (int z = 0; z < ZB; z++)
#pragma unroll
          for (int ci = 0; ci < ND; ci++)
#pragma unroll
            for (int ww = 0; ww < NW; ww++) {
              if constexpr (Lo::PAIRS) out[z][ci][ww] = make_float2(0.f, 0.f);
              else out[z][ci][ww] = T(0);
            }
        asm_positions<ND, T, NR, ZB>(std::make_integer_sequence<int, 9 * (ZB + 2)>{}, pl, ctr, sT, m, out);
#pragma unroll
        for (int z = 0; z < ZB; z++) {
          if (l + z >= l1) break;
          const size_t node = (size_t)r + (size_t)c * R + (size_t)(l + z) * RC;
          const T* pc = pl[z + 1] + ctr * PS;
#pragma unroll
          for (int ci = 0; ci < ND; ci++)
#pragma unroll
            for (int k = 0; k < NR; k++) {
              T qv;
              if constexpr (Lo::PAIRS) qv = (k & 1) ? out[z][ci][k >> 1].y : out[z][ci][k >> 1].x;
              else qv = out[z][ci][k];
              const size_t j = (size_t)k * n + node * ND + ci;
              const T vv = pc[ci * NR + k];
              a.q[j] = qv;
              a.dnew[j] = vv;
              acc[k] += (double)vv * (double)qv;
            }
        }
      }
#pragma unroll
      for (int z = 0; z < ZB; z++) kc[z] = kn[z];
      if (l + ZB < l1) {
        if constexpr (AHEAD) {
          __syncthreads();  // the next step's planes are in place; this step's are no longer read
        } else {
          __syncthreads();  // planes l - 1 .. l + ZB - 2 are no longer read
#pragma unroll
          for (int q = 1; q <= ZB; q++) load_plane(l + ZB + q);
          __syncthreads();
        }
      }
    }
    w += l1 - l0;
  }
  const bool ismax[NR] = {};
  double res[NR];
  if (grid_reduce<NT, NR>(acc, ismax, a.rc, blockIdx.x, res, sred) && tid == 0) {
#pragma unroll
    for (int k = 0; k < NR; k++)
      if (!sdone[k]) { a.sc[k].red[0] = res[k]; a.sc[k].alpha = a.sc[k].delta / res[k]; }
  }
}

}  // namespace chfem
