// stencil_th.cuh -- the thermal operator pass written for the structure of the Q1 conduction
// matrix, for thermal models whose element matrices are cubic-symmetric (a cube of one
// conductivity per voxel: the reference's and this library's thermal models).
//
// Within a voxel of material m the Q1 conduction matrix has one value d_m on the diagonal, 0
// between nodes that share an edge, f_m between nodes across a face diagonal and c_m between
// nodes across the body diagonal (the table of chfem/src/femhmg/physical_phenomena/
// femhmg_thermal_3D.c:42-120).  The reference applies it voxel by voxel (matrix_free.cu:191-323);
// here the node's row is taken voxel by voxel too, but only through the 4 nodes of each voxel
// that couple to the node: for the voxel at position p (the side of the node it lies on along
// rows, columns and layers),
//   y += d_p v0 + f_p (v(dr, dc, 0) + v(dr, 0, dl) + v(0, dc, dl)) + c_p v(dr, dc, dl),
// where (dr, dc, dl) = +-1 point into the voxel; the 6 face neighbours have no coupling.  The
// coefficients of a voxel come from its material (2 bits of the node's 16-bit key) through a
// 4-entry table, and sum_p d_p from the counts of the materials among the 8 voxels (popcounts
// of the key) through a second table, which also holds the inverse Jacobi diagonal.
//
// B200 design: a CTA owns a 32 x TC column of nodes and marches through a run of layers.  Each
// layer's plane of the formed input (with its one-node halo) goes through a 3-slot shared-memory
// ring; the global loads of the plane after it are issued before the current node is computed
// and held in registers until their slot is free.  Each thread reads the 9 values around its
// column of a plane once into registers and adds them into the node below (th_finish), at and
// above (th_start) them, so a node costs 9 shared-memory loads and two planes live in registers.
// All per-node index arithmetic is incremental (no division in the layer loop).  Modes, outputs
// and finishers are those of k_te_apply (stencil_te.cuh).
#pragma once
#include "common.cuh"
#include "stencil_te.cuh"

namespace chfem {

// table: [0, 8) (f_m, c_m) of materials 0..3; then sum_p d_p and its inverse by material
// counts, index n1 + 9 n2 + 81 n3 (n_m: voxels of material m among the node's 8)
constexpr int TH_NCOUNT = 729;
constexpr int TH_DIAG = 8;
constexpr int TH_INV = TH_DIAG + TH_NCOUNT;
constexpr int TH_WORDS = TH_INV + TH_NCOUNT;

// index of the material counts of a key (2 bits per voxel)
__device__ __forceinline__ int th_count_index(unsigned key) {
  const unsigned lo = key & 0x5555u, hi = (key >> 1) & 0x5555u;
  const int n3 = __popc(lo & hi);
  return (__popc(lo) - n3) + 9 * (__popc(hi) - n3) + 81 * n3;
}

// key slot (local index e) of the voxel at position p (bit 0: the voxel spans rows {0,+1} around
// the node, bit 1 columns, bit 2 layers; asm_table.cuh)
__host__ __device__ constexpr int th_slot(int p) {
  int e = 0;
  while (asm_epos(e) != p) e++;
  return e;
}

template <int TC>
struct ThGeom {
  static constexpr int PR = TE_TR + 2, PC = TC + 2, PP = PR * PC, NT = TE_TR * TC;
  static constexpr int PER = (PP + NT - 1) / NT;  // staged points per thread
};

template <typename T, int TC>
inline size_t th_smem_bytes() {
  return ((size_t)TH_WORDS + (size_t)3 * ThGeom<TC>::PP) * sizeof(T) + 16;
}

// value index 3 (dc + 1) + (dr + 1) of the 9 values around a column in one plane
__device__ __forceinline__ constexpr int th_at(int dr, int dc) { return 3 * (dc + 1) + (dr + 1); }

// The node's row in two halves, so that only two planes of values are live at a time.  th_start,
// when the node's own plane (v0) arrives: the diagonal, the four voxels below the node (with the
// plane below, vm) in full, and the in-plane terms of the four voxels above; their coefficients
// for the plane above stay in up[8] (f, c of each).  th_finish, when that plane (vp) arrives.
template <typename T>
__device__ __forceinline__ T th_start(const T* __restrict__ sTab, unsigned key, const T (&vm)[9], const T (&v0)[9], T (&up)[8]) {
  constexpr int SLOT[8] = {th_slot(0), th_slot(1), th_slot(2), th_slot(3), th_slot(4), th_slot(5), th_slot(6), th_slot(7)};
  T y = sTab[TH_DIAG + th_count_index(key)] * v0[th_at(0, 0)];
#pragma unroll
  for (int p = 0; p < 8; p++) {
    const int dr = (p & 1) ? 1 : -1, dc = (p & 2) ? 1 : -1;
    const unsigned m = (key >> (2 * SLOT[p])) & 3u;
    const T f = sTab[2 * m], c = sTab[2 * m + 1];
    y = fma(f, v0[th_at(dr, dc)], y);
    if (p < 4) {
      y = fma(f, vm[th_at(dr, 0)] + vm[th_at(0, dc)], y);
      y = fma(c, vm[th_at(dr, dc)], y);
    } else {
      up[2 * (p - 4)] = f;
      up[2 * (p - 4) + 1] = c;
    }
  }
  return y;
}
template <typename T>
__device__ __forceinline__ T th_finish(T y, const T (&up)[8], const T (&vp)[9]) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int dr = (q & 1) ? 1 : -1, dc = (q & 2) ? 1 : -1;
    y = fma(up[2 * q], vp[th_at(dr, 0)] + vp[th_at(0, dc)], y);
    y = fma(up[2 * q + 1], vp[th_at(dr, dc)], y);
  }
  return y;
}

template <typename T, int MODE, int TC>
__global__ void __launch_bounds__(TE_TR * TC, sizeof(T) == 8 ? 2 : 3) k_th_apply(TeArgs<1, T> a, const T* __restrict__ tab) {
  using G = ThGeom<TC>;
  constexpr int NT = G::NT, PR = G::PR, PP = G::PP, PER = G::PER;
  constexpr bool TWO_IN = (MODE == TE_PCG || MODE == TE_DIRDOT || MODE == TE_MR);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[NT / 32];
  if (a.skip_if_done && a.sc->done) return;
  T* sTab = reinterpret_cast<T*>(smem_raw);
  T* sV = sTab + TH_WORDS;  // [3][PP] formed input
  const int tid = threadIdx.x + TE_TR * threadIdx.y;
  for (int i = tid; i < TH_WORDS; i += NT) sTab[i] = tab[i];
  const T beta = (MODE == TE_PCG || MODE == TE_DIRDOT) ? T(a.sc->beta) : T(0);
  const T alpha = (MODE == TE_MR && mr_steps(a.finish)) ? T(a.sc->alpha) : T(0);
  const double alpha64 = (MODE == TE_UPD) ? a.sc->alpha : 0.0;
  const bool pre = a.cfg.precond != 0;
  const int R = a.R, C = a.C, L = a.L;
  const size_t RC = (size_t)R * C;
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * PR;

  double acc = 0.0, acc_rz = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  size_t pofs[PER];  // column offsets of this thread's staged points in the current tile
  T g0[PER], g1[PER];  // loads of the next plane to stage
  unsigned gk[PER];

  auto load = [&](size_t lofs) {
#pragma unroll
    for (int k = 0; k < PER; k++) {
      if (PER * NT == PP || tid + k * NT < PP) {
        const size_t node = pofs[k] + lofs;
        g0[k] = a.in0[node];
        if (TWO_IN) { g1[k] = a.in1[node]; gk[k] = a.keys[node]; }
      }
    }
  };
  auto commit = [&](T* dv) {
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int p = tid + k * NT;
      if (PER * NT == PP || p < PP) {
        T v = g0[k];
        if (TWO_IN) {
          const T inv = pre ? sTab[TH_INV + th_count_index(gk[k])] : T(1);
          if (MODE == TE_MR) v = fma(-alpha, g1[k], v) * inv;
          else v = fma(beta, g1[k], v * inv);
        }
        dv[p] = v;
      }
    }
  };
  auto gather = [&](const T* s, T (&v)[9]) {
#pragma unroll
    for (int dc = -1; dc <= 1; dc++)
#pragma unroll
      for (int dr = -1; dr <= 1; dr++) v[th_at(dr, dc)] = s[ctr + dr + dc * PR];
  };
  auto layer_ofs = [&](int l) {  // periodic layer l >= -1 of a run, without a division
    while (l < 0) l += L;
    while (l >= L) l -= L;
    return (size_t)l * RC;
  };

  T va[9], vb[9], up[8];
  const TeWork wk(R, C, L, TC);
  for (long w = wk.begin(), w_end = wk.end(); w < w_end;) {
    int l0, l1, r0, c0;
    wk.run(w, w_end, r0, c0, l0, l1);
#pragma unroll
    for (int k = 0; k < PER; k++) {
      const int p = min(tid + k * NT, PP - 1);
      const int hr = p % PR, hc = p / PR;
      pofs[k] = (size_t)wrap(r0 + hr - 1, R) + (size_t)wrap(c0 + hc - 1, C) * R;
    }
    const int r = r0 + threadIdx.x, c = c0 + threadIdx.y;
    const bool active = (r < R) && (c < C);
    const size_t col = active ? (size_t)r + (size_t)c * R : 0;
    // ring slots of the planes below, at and above the current node
    T* s_m = sV;
    T* s_0 = sV + PP;
    T* s_p = sV + 2 * PP;
    __syncthreads();  // the previous run's reads of the ring are done
    load(layer_ofs(l0 - 1));
    commit(s_m);
    load(layer_ofs(l0));
    commit(s_0);
    size_t lofs_next = layer_ofs(l0 + 1);
    load(lofs_next);
    unsigned key = a.keys[col + layer_ofs(l0)];
    unsigned key_next = a.keys[col + lofs_next];
    __syncthreads();
    gather(s_m, va);
    gather(s_0, vb);
    T y = th_start<T>(sTab, key, va, vb, up);
    size_t j = col + (size_t)l0 * RC;
    // node l: its plane in v0 and its partial row in y; the loaded plane l + 1 is committed into
    // the free slot, plane l + 2 loaded, plane l + 1 gathered into vn (which held plane l - 1),
    // node l finished and node l + 1 started
    auto step = [&](int l, const T (&v0)[9], T (&vn)[9]) {
      commit(s_p);
      const bool more = l + 1 < l1;
      if (more) {
        lofs_next += RC;
        if (lofs_next >= (size_t)L * RC) lofs_next -= (size_t)L * RC;
        load(lofs_next);
      }
      __syncthreads();
      gather(s_p, vn);
      const T yl = th_finish<T>(y, up, vn);
      const unsigned kl = key;
      if (more) {
        key = key_next;
        if (active) key_next = a.keys[col + lofs_next];
        y = th_start<T>(sTab, key, v0, vn, up);
      }
      T* t = s_m; s_m = s_0; s_0 = s_p; s_p = t;
      if (active) {
        const T v = v0[th_at(0, 0)];
        if (MODE != TE_DIRDOT && MODE != TE_UPD) a.y[j] = yl;
        if (MODE == TE_PCG || MODE == TE_DIRDOT) a.vout[j] = v;
        if (MODE == TE_UPD) {
          const T inv = pre ? sTab[TH_INV + th_count_index(kl)] : T(1);
          const T rn = fma(-T(alpha64), yl, a.vout[j]);
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
        acc += (double)v * (double)yl;
      }
      j += RC;
    };
    // two register sets take turns as the node's plane and the next one
    for (int l = l0; l < l1; l += 2) {
      step(l, vb, va);
      if (l + 1 < l1) step(l + 1, va, vb);
    }
    w += l1 - l0;
  }
  if (a.finish == FIN_NONE) return;
  const int bid = blockIdx.x;
  if (MODE == TE_UPD) {
    const double vals[4] = {acc_rz, mr, md, mx};
    const bool ismax[4] = {false, true, true, true};
    double out[4];
    if (grid_reduce<NT, 4>(vals, ismax, a.rc, bid, out, sred) && tid == 0) {
      for (int k = 0; k < 4; k++) a.sc->red[k] = out[k];
      const SolveCfg cfg{a.cfg.tol, a.cfg.maxit, a.cfg.norm, a.cfg.precond, a.cfg.nhmg};
      pcg_finish(PW_PCG, out, a.sc, cfg);
    }
  } else if (MODE == TE_MR) {
    const double vals[5] = {acc, acc_rz, mr, md, mx};
    const bool ismax[5] = {false, false, true, true, true};
    double out[5];
    if (grid_reduce<NT, 5>(vals, ismax, a.rc, bid, out, sred) && tid == 0) {
      for (int k = 0; k < 5; k++) a.sc->red[k] = out[k];
      mr_finish(a.finish, out, a.sc, a.cfg);
    }
  } else {
    const double vals[1] = {acc};
    const bool ismax[1] = {false};
    double out[1];
    if (grid_reduce<NT, 1>(vals, ismax, a.rc, bid, out, sred) && tid == 0) {
      a.sc->red[0] = out[0];
      if (a.finish == FIN_ALPHA) a.sc->alpha = a.sc->delta / out[0];
    }
  }
}

}  // namespace chfem
