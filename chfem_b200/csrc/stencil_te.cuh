// stencil_te.cuh -- matrix-free voxel operator for 3D thermal (1 DOF/node) and elastic
// (3 DOF/node) homogenization, applied node by node like the reference
// (chfem/src/femhmg/cudapcg/kernels/matrix_free.cu:191-323 thermal SparseQ1, :410-459
// elastic): for node i and each of its 8 voxels e (in which i is local node e), the row
// block of local node e of the element matrix of that voxel's material multiplies the
// element's 8 nodal values.
//
// B200 design: one CTA owns a 32 (rows) x 8 (cols) column of nodes and marches through a
// chunk of layers, keeping three layers of the input field (with a one-node periodic halo)
// in shared memory, so every field value is read from HBM about once per apply.  The
// element matrices of all materials sit in shared memory (a warp touching up to 4
// materials reads up to 4 distinct addresses per load instead of serialising on the
// constant cache).  The input field is formed while it is staged, which fuses the vector
// update that precedes the operator in each Krylov recurrence:
//   TE_PLAIN  v = in0                                  (plain apply)
//   TE_PCG    v = M^-1 in0 + beta*in1 = M^-1 r + beta d_old   (PCG direction; written once;
//             the preconditioned residual s = M^-1 r is formed here and never stored)
//   TE_MR     r' = in0 - alpha*in1 = r - alpha q, v = M^-1 r'   (PMINRES; r', x updated)
#pragma once
#include <utility>
#include "common.cuh"
#include "asm_table.cuh"
#include "pointwise.cuh"

namespace chfem {

constexpr int TE_TR = 32;              // rows per CTA (fastest dimension, coalesced)
constexpr int TE_TC = 8;               // cols per CTA
constexpr int TE_NT = TE_TR * TE_TC;   // threads per CTA
constexpr int TE_PR = TE_TR + 2;       // plane pitch (rows incl. halo)
constexpr int TE_PC = TE_TC + 2;
constexpr int TE_PP = TE_PR * TE_PC;   // points per plane incl. halo

// TE_DIRDOT and TE_UPD are the two passes of the 3-vector PCG (x, r and the direction's two
// buffers; chfem/src/femhmg/cudapcg/solvers/pcg3.cu:28-227 keeps the same vectors and applies
// the operator twice per iteration):
//   TE_DIRDOT  v = M^-1 in0 + beta in1 = M^-1 r + beta d_old, written to vout; d.Ad -> alpha
//   TE_UPD     v = in0 = d; r (vout) -= alpha A v, x += alpha v; r.M^-1 r, max-norms -> the
//              PCG finisher (delta, beta, stopping test) -- A v itself is never stored
enum TeMode : int { TE_PLAIN = 0, TE_PCG = 1, TE_MR = 2, TE_DIRDOT = 3, TE_UPD = 4 };
// Finishers run by the last CTA on the grid-reduced sums.
enum TeFinish : int {
  FIN_NONE = 0, FIN_ALPHA = 1, FIN_STORE = 2, FIN_MR_INIT = 3, FIN_MR_X0 = 4, FIN_MR_STEP = 5,
  FIN_MR_REPL = 6,   // mixed precision: r holds b - A x (FP64 apply); pass with alpha = 0
  FIN_MR_CHECK = 7   // mixed precision: same, at an apparent convergence: confirm or restart
};
// alpha of a (P)MINRES operator pass: the replacement and check passes evaluate the current
// residual without a step
__device__ __forceinline__ bool mr_steps(int fin) { return fin != FIN_MR_REPL && fin != FIN_MR_CHECK; }

struct MrCfg {
  double tol;
  int maxit;
  int norm;
  int precond;
  long nhmg;
};

// Work schedule of a stencil pass.  The work is every (column tile of TE_TR x TE_TC nodes,
// layer) unit; a 1D grid of P CTAs -- as many as fit on the GPU at once -- takes equal slices of
// one line of those units, so the pass runs in a single wave of equal shares.  The line is
// ordered chunk by chunk: layer chunks of lc = ceil(L tiles / P) layers, within a chunk tile by
// tile, within a tile layer by layer.  A CTA's slice is then about one (tile, chunk) run, and the
// CTAs that run at the same time cover neighbouring tiles over the same layers, so the halo
// planes they share are read from L2 rather than DRAM.
constexpr int TE_MIN_RUN = 4;  // layers per CTA at least (halo restaging overhead)
struct TeWork {
  int tiles_r, L, lc, nc, tc;
  long tiles, W;
  __device__ TeWork(int R, int C, int L_, int tc_ = TE_TC) : tiles_r((R + TE_TR - 1) / TE_TR), L(L_), tc(tc_) {
    tiles = (long)tiles_r * ((C + tc - 1) / tc);
    W = tiles * L;
    const long P = gridDim.x;
    lc = (int)min((long)L, max(1L, (W + P - 1) / P));
    nc = (L + lc - 1) / lc;
  }
  __device__ long begin() const { return (long)blockIdx.x * W / gridDim.x; }
  __device__ long end() const { return ((long)blockIdx.x + 1) * W / gridDim.x; }
  // the run starting at unit w: tile origin (r0, c0) and layers [l0, l1), not past unit w_end
  __device__ void run(long w, long w_end, int& r0, int& c0, int& l0, int& l1) const {
    const long per_full = (long)lc * tiles;
    const int c = (int)min((long)nc - 1, w / per_full);
    const int size = min(lc, L - c * lc);  // layers in this chunk
    const long rem = w - (long)c * per_full;
    const long tile = rem / size;
    l0 = c * lc + (int)(rem % size);
    l1 = (int)min((long)c * lc + size, (long)l0 + (w_end - w));
    r0 = (int)(tile % tiles_r) * TE_TR;
    c0 = (int)(tile / tiles_r) * tc;
  }
};

template <int ND, typename T>
struct TeArgs {
  const T* in0;        // s (PCG) | r (MR) | field to apply
  const T* in1;        // d_old (PCG) | q (MR)
  T* vout;             // PCG: formed direction; MR: updated residual r'
  T* y;                // y = A v
  double* x;           // MR: x += alpha d (FP64 in every precision mode)
  const T* d;          // MR
  const uint16_t* keys;
  const T* Kd;         // dense element matrices [nmat][8ND][8ND]
  int nmat;
  int R, C, L;
  DevScalars* sc;
  RedCtl rc;
  int finish;          // TeFinish
  int skip_if_done;
  MrCfg cfg;
  // scalar density field: voxel v's element matrix scaled by sdf_min + sdf_rng sdf[v] / 65535
  // (cudapcg.cu:327-334); and then the node's inverse Jacobi diagonal, precomputed (FP64)
  const uint16_t* sdf = nullptr;
  double sdf_min = 0.0, sdf_rng = 0.0;
  const double* invd = nullptr;
};

// Index of the voxel in which node (r, c, l) is local node e: (r - drow(e) - 1, c - dcol(e),
// l - dlay(e)), periodic (the 8 voxels around a node in the order of
// matrix_free.cu:2283-2295).
__device__ __forceinline__ size_t te_voxel(int r, int c, int l, int e, int R, int C, int L) {
  return (size_t)wrap(r - drow(e) - 1, R) + (size_t)wrap(c - dcol(e), C) * R + (size_t)wrap(l - dlay(e), L) * R * C;
}

template <int ND, typename T>
__device__ __forceinline__ void te_node(const T* __restrict__ sK, int kstride, unsigned key,
                                        const T* pm, const T* p0, const T* pp, int ctr, T (&out)[ND], const T* scl = nullptr) {
  constexpr int ED = 8 * ND;
#pragma unroll
  for (int c = 0; c < ND; c++) out[c] = T(0);
#pragma unroll
  for (int e = 0; e < 8; e++) {
    const T* K = sK + ((key >> (2 * e)) & 3u) * kstride + e * ND * ED;
    T oe[ND];
#pragma unroll
    for (int ci = 0; ci < ND; ci++) oe[ci] = T(0);
#pragma unroll
    for (int b = 0; b < 8; b++) {
      if (ND == 1 && shares_edge(e, b)) continue;  // structural zero of the Q1 conductivity matrix
      const int dr = drow(b) - drow(e), dc = dcol(b) - dcol(e), dl = dlay(b) - dlay(e);
      const T* P = dl < 0 ? pm : (dl == 0 ? p0 : pp);
      const T* v = P + (ctr + dr + dc * TE_PR) * ND;
#pragma unroll
      for (int ci = 0; ci < ND; ci++) {
        T s = scl ? oe[ci] : out[ci];
#pragma unroll
        for (int cj = 0; cj < ND; cj++) s = fma(K[ci * ED + b * ND + cj], v[cj], s);
        if (scl) oe[ci] = s;
        else out[ci] = s;
      }
    }
    if (scl) {
#pragma unroll
      for (int ci = 0; ci < ND; ci++) out[ci] = fma(scl[e], oe[ci], out[ci]);
    }
  }
}

// Jacobi inverse diagonal of a node from its key (matrix_free.cu:167-188, :388-408).
template <int ND, typename T>
__device__ __forceinline__ void te_invdiag(const T* sD, unsigned key, T (&inv)[ND]) {
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
}

__device__ inline void mr_finish(int fin, const double* s, DevScalars* sc, const MrCfg& cfg) {
  // s: [0] z.Az (delta), [1] r'.z (r' M^-1 r'), [2] max|r'|, [3] max|d| (nhmg), [4] max|x| (nhmg)
  const double tol2 = cfg.tol * cfg.tol;
  if (fin == FIN_MR_INIT) {  // pminres.cu:58-79
    sc->delta0 = s[0];
    sc->res0 = (cfg.norm == 1) ? s[2] : s[1];
    sc->iteration = 0; sc->alpha = 0.0; sc->beta = 0.0; sc->found = 0;
    if (fabs(sc->res0) < 1e-12) { sc->done = 1; sc->found = 1; sc->metric = 0.0; sc->status = 1; }
    else { sc->done = 0; sc->status = 0; sc->delta = s[0]; sc->delta_old = s[0]; sc->metric = 1.0; }
  } else if (fin == FIN_MR_X0) {  // pminres.cu:81-98
    sc->delta = s[0]; sc->delta_old = s[0]; sc->beta = 0.0;
    if (!(fabs(s[0]) > tol2 * fabs(sc->delta0))) {
      sc->done = 1; sc->found = 1; sc->status = 2; sc->metric = sqrt(fabs(s[0]) / fabs(sc->delta0));
    }
  } else if (fin == FIN_MR_STEP) {  // pminres.cu:130-160, :166-204
    sc->iteration += 1;
    sc->delta_old = sc->delta;
    sc->delta = s[0];
    bool cont;
    if (cfg.norm == 0) { cont = fabs(s[1]) > tol2 * fabs(sc->res0); sc->metric = sqrt(fabs(s[1]) / fabs(sc->res0)); }
    else if (cfg.norm == 1) { sc->metric = s[2] / sc->res0; cont = sc->metric > cfg.tol; }
    else { sc->metric = fabs(sc->alpha) * s[3] / s[4]; cont = sc->metric > cfg.tol; }
    sc->found = sc->metric <= cfg.tol;
    sc->beta = sc->delta / sc->delta_old;
    if (!cont || sc->iteration >= cfg.maxit) sc->done = 1;
  } else if (fin == FIN_MR_REPL || fin == FIN_MR_CHECK) {
    // The true residual replaces the recursive one (mixed precision).
    double m;
    bool cont;
    if (cfg.norm == 1) { m = s[2] / sc->res0; cont = m > cfg.tol; }
    else { m = sqrt(fabs(s[1]) / fabs(sc->res0)); cont = fabs(s[1]) > tol2 * fabs(sc->res0); }
    const double m_rec = sc->metric;
    sc->delta = s[0];
    sc->metric = m;
    if (fin == FIN_MR_REPL) {
      // keep the direction while the two residuals agree, else restart from the true one
      if (m > 2.0 * m_rec || m < 0.5 * m_rec) { sc->beta = 0.0; sc->delta_old = s[0]; }
      else sc->beta = sc->delta / sc->delta_old;
    } else {
      if (!cont) { sc->done = 1; sc->found = 1; }
      else if (sc->iteration >= cfg.maxit) { sc->done = 1; sc->found = 0; }
      else { sc->done = 0; sc->found = 0; sc->beta = 0.0; sc->delta_old = s[0]; }
    }
  }
}

// The node's row as 27 assembled neighbour blocks (asm_table.cuh; models of at most two
// materials): out = sum over neighbours o of A(n, n+o) v(n+o).
template <int ND, typename T, int O>
__device__ __forceinline__ void asm_te_offset(const T* __restrict__ sT, unsigned m, const T* pm, const T* p0, const T* pp, int ctr,
                                              T (&out)[ND][1]) {
  if constexpr (asm_used<ND>(O)) {
    constexpr int dr = O % 3 - 1, dc = (O / 3) % 3 - 1, dl = O / 9 - 1;
    const T* v = (dl < 0 ? pm : (dl == 0 ? p0 : pp)) + (ctr + dr + dc * TE_PR) * ND;
    T val[ND][1];
#pragma unroll
    for (int c = 0; c < ND; c++) val[c][0] = v[c];
    asm_block<ND, T, O>(sT, m, val, out);
  }
}
template <int ND, typename T, int... Os>
__device__ __forceinline__ void asm_te_node(std::integer_sequence<int, Os...>, const T* __restrict__ sT, unsigned key, const T* pm,
                                            const T* p0, const T* pp, int ctr, T (&out)[ND]) {
  T o[ND][1];
#pragma unroll
  for (int c = 0; c < ND; c++) o[c][0] = T(0);
  const unsigned m = asm_config(key);
  (asm_te_offset<ND, T, Os>(sT, m, pm, p0, pp, ctr, o), ...);
#pragma unroll
  for (int c = 0; c < ND; c++) out[c] = o[c][0];
}

// ASM: the operator from the assembled neighbour blocks (a.Kd still supplies the Jacobi
// diagonal); the shared-memory head then holds the table instead of the element matrices.
template <int ND, typename T, int MODE, bool ASM = false>
__global__ void __launch_bounds__(TE_NT) k_te_apply(TeArgs<ND, T> a, const T* __restrict__ tab = nullptr) {
  constexpr int ED = 8 * ND;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[TE_NT / 32];
  __shared__ T sD[4 * 8 * ND];
  if (a.skip_if_done && a.sc->done) return;
  T* sK = reinterpret_cast<T*>(smem_raw);
  const int kstride = ED * ED + 1;  // padded material stride spreads materials over banks
  constexpr int TAB = asm_table_words(ND, AsmLayout<ND, T, 1>::BS);
  T* sP = sK + (ASM ? TAB : 4 * kstride);
  // ASM: the inverse Jacobi diagonal by node configuration follows the blocks
  [[maybe_unused]] const T* sInv = sK + ASM_NBLK * AsmLayout<ND, T, 1>::BS;
  auto invdiag = [&](size_t node, unsigned key, T (&inv)[ND]) {
    if (a.invd) {
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = T(a.invd[node * ND + c]);
      return;
    }
    if constexpr (ASM) {
      const unsigned m = asm_config(key);
#pragma unroll
      for (int c = 0; c < ND; c++) inv[c] = sInv[m * ND + c];
    } else {
      te_invdiag<ND, T>(sD, key, inv);
    }
  };
  const int tid = threadIdx.x + TE_TR * threadIdx.y;
  if constexpr (ASM) {
    for (int i = tid; i < TAB; i += TE_NT) sK[i] = tab[i];
  } else {
    // 4 material slots always (keys carry 2 bits per voxel); slots past nmat are zero.
    for (int i = tid; i < 4 * ED * ED; i += TE_NT) sK[(i / (ED * ED)) * kstride + i % (ED * ED)] = (i < a.nmat * ED * ED) ? a.Kd[i] : T(0);
  }
  if (MODE == TE_MR || MODE == TE_PCG || MODE == TE_DIRDOT || MODE == TE_UPD) {
    for (int i = tid; i < 4 * 8 * ND; i += TE_NT) {
      const int m = i / (8 * ND), k = i % (8 * ND);
      sD[i] = (m < a.nmat) ? a.Kd[(size_t)m * ED * ED + (size_t)k * ED + k] : T(1);
    }
    __syncthreads();
  }
  const T beta = (MODE == TE_PCG || MODE == TE_DIRDOT) ? T(a.sc->beta) : T(0);
  const T alpha = (MODE == TE_MR && mr_steps(a.finish)) ? T(a.sc->alpha) : T(0);
  const double alpha64 = (MODE == TE_UPD) ? a.sc->alpha : 0.0;
  const bool pre = a.cfg.precond != 0;
  const int R = a.R, C = a.C, L = a.L;
  const size_t RC = (size_t)R * C;
  int r0 = 0, c0 = 0;  // column tile of the current run

  auto slot_of = [&](int l) { return ((l % 3) + 3) % 3; };
  auto load_plane = [&](int l) {
    const int lw = wrap(l, L);
    T* dst = sP + slot_of(l) * TE_PP * ND;
    for (int p = tid; p < TE_PP; p += TE_NT) {
      const int hr = p % TE_PR, hc = p / TE_PR;
      const int gr = wrap(r0 + hr - 1, R), gc = wrap(c0 + hc - 1, C);
      const size_t node = (size_t)gr + (size_t)gc * R + (size_t)lw * RC;
      T inv[ND];
      if (MODE == TE_MR || MODE == TE_PCG || MODE == TE_DIRDOT) {
        if (pre) invdiag(node, a.invd ? 0u : (unsigned)a.keys[node], inv);
        else {
#pragma unroll
          for (int c = 0; c < ND; c++) inv[c] = T(1);
        }
      }
#pragma unroll
      for (int c = 0; c < ND; c++) {
        T v = a.in0[node * ND + c];
        if (MODE == TE_PCG) v = fma(beta, a.in1[node * ND + c], v * inv[c]);
        if (MODE == TE_MR) v = fma(-alpha, a.in1[node * ND + c], v) * inv[c];
        if (MODE == TE_DIRDOT) v = fma(beta, a.in1[node * ND + c], v * inv[c]);
        dst[p * ND + c] = v;
      }
    }
  };

  double acc = 0.0, acc_rz = 0.0, mr = 0.0, md = 0.0, mx = 0.0;
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * TE_PR;
  const TeWork wk(R, C, L);
  for (long w = wk.begin(), w_end = wk.end(); w < w_end;) {
  int l0, l1;
  wk.run(w, w_end, r0, c0, l0, l1);
  const int r = r0 + threadIdx.x, c = c0 + threadIdx.y;
  const bool active = (r < R) && (c < C);
  // the node key is fetched one layer ahead (its latency overlaps the previous layer's work)
  const size_t col = active ? (size_t)r + (size_t)c * R : 0;
  unsigned key_next = a.keys[col + (size_t)l0 * RC];
  __syncthreads();
  load_plane(l0 - 1);
  load_plane(l0);
  for (int l = l0; l < l1; l++) {
    const unsigned key = key_next;
    key_next = a.keys[col + (size_t)(l + 1 < l1 ? l + 1 : l) * RC];
    load_plane(l + 1);
    __syncthreads();
    if (active) {
      const size_t node = (size_t)r + (size_t)c * R + (size_t)l * RC;
      const T* pm = sP + slot_of(l - 1) * TE_PP * ND;
      const T* p0 = sP + slot_of(l) * TE_PP * ND;
      const T* pp = sP + slot_of(l + 1) * TE_PP * ND;
      T out[ND];
      if constexpr (ASM) {
        asm_te_node<ND, T>(std::make_integer_sequence<int, 27>{}, sK, key, pm, p0, pp, ctr, out);
      } else if (a.sdf) {
        T scl[8];
#pragma unroll
        for (int e = 0; e < 8; e++) scl[e] = T(a.sdf_min + a.sdf_rng * (double)a.sdf[te_voxel(r, c, l, e, R, C, L)] * (1.0 / 65535.0));
        te_node<ND, T>(sK, kstride, key, pm, p0, pp, ctr, out, scl);
      } else {
        te_node<ND, T>(sK, kstride, key, pm, p0, pp, ctr, out);
      }
      [[maybe_unused]] T own_inv[ND];
      if constexpr (MODE == TE_UPD) {
        if (pre) invdiag(node, key, own_inv);
        else {
#pragma unroll
          for (int cc = 0; cc < ND; cc++) own_inv[cc] = T(1);
        }
      }
#pragma unroll
      for (int cc = 0; cc < ND; cc++) {
        const size_t j = node * ND + cc;
        const T v = p0[ctr * ND + cc];
        if (MODE != TE_DIRDOT && MODE != TE_UPD) a.y[j] = out[cc];
        if (MODE == TE_PCG || MODE == TE_DIRDOT) a.vout[j] = v;
        if (MODE == TE_UPD) {
          const T rn = fma(-T(alpha64), out[cc], a.vout[j]);
          a.vout[j] = rn;
          const double xv = fma(alpha64, (double)v, a.x[j]);
          a.x[j] = xv;
          acc_rz += (double)rn * (double)(rn * own_inv[cc]);
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
    __syncthreads();
  }
  w += l1 - l0;
  }
  if (a.finish == FIN_NONE) return;
  const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (MODE == TE_UPD) {
    const double vals[4] = {acc_rz, mr, md, mx};
    const bool ismax[4] = {false, true, true, true};
    double out[4];
    if (grid_reduce<TE_NT, 4>(vals, ismax, a.rc, bid, out, sred) && tid == 0) {
      for (int k = 0; k < 4; k++) a.sc->red[k] = out[k];
      const SolveCfg cfg{a.cfg.tol, a.cfg.maxit, a.cfg.norm, a.cfg.precond, a.cfg.nhmg};
      pcg_finish(PW_PCG, out, a.sc, cfg);
    }
  } else if (MODE == TE_MR) {
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

template <int ND, typename T>
inline size_t te_asm_smem_bytes() {
  return (size_t)asm_table_words(ND, AsmLayout<ND, T, 1>::BS) * sizeof(T) + (size_t)3 * TE_PP * ND * sizeof(T) + 16;
}

template <int ND, typename T>
inline size_t te_smem_bytes(int nmat) {
  const int ED = 8 * ND;
  (void)nmat;
  return (size_t)4 * (ED * ED + 1) * sizeof(T) + (size_t)3 * TE_PP * ND * sizeof(T) + 16;
}

}  // namespace chfem
