// batch_thermal.cuh -- many independent thermal homogenizations solved together.
//
// The reference homogenizes one image per process run (chfem/src/main.c:53-147): every
// sample pays its own model set-up, and small images leave most of the GPU idle.  Here a
// batch of samples of any sizes, each with its own materials, is one problem: all samples and
// their 3 load cases (X, Y, Z) advance together through the same two passes per iteration,
// each load case of each sample with its own PCG scalars and stopping test (the recurrence of
// pcg.cu:100-224).
//
// Work distribution.  The column tiles (32 x TC nodes) times the layers of every still-active
// sample form one work line, rebuilt on the device at the start of each graph chunk
// (k_bt_schedule), so samples that have converged drop out without the host.  A 1D grid of as
// many CTAs as fit on the GPU takes equal slices of the line (k_bt_apply); the pointwise pass
// does the same over the line of nodes (k_bt_point).  A CTA's slice crosses sample boundaries:
// it reduces each sample it touches into its own partial slot, number (CTA index + active
// sample index) -- unique, and in work order -- and the last CTA sums each sample's partials in
// CTA order, so every reduction is deterministic.
//
// Mixed precision (FP32 fields): the solution x and the right-hand side stay FP64; the
// residual-replacement and convergence-check decisions of the single-model solver are taken
// on the device by the pointwise finisher, which marks the load case pending; the next two
// passes (k_bt_apply<..., RES> with the FP64 operator on the FP64 x, then k_bt_point<..., REPL>)
// serve pending load cases and do nothing otherwise, so the whole loop stays graph-captured.
#pragma once
#include <type_traits>
#include <utility>
#include "common.cuh"
#include "pointwise.cuh"
#include "stencil_te.cuh"
#include "stencil_block.cuh"
#include "loadcase.cuh"

namespace chfem {

constexpr int BT_NR = 3;  // load cases per sample (thermal X, Y, Z)
// Every load case of every sample iterates in lockstep (one iteration per pass pair), so
// replacements are decided only at multiples of this period: the FP64 residual pass then serves
// all the load cases that are due at once instead of a few at nearly every iteration.
constexpr int BT_REPL_PERIOD = 10;
enum BtPending : int { BT_NONE = 0, BT_REPL = 1, BT_CHECK = 2 };

struct BtCtl {
  int pending;
  int next_replace;
  int checks;
  int pad;
  double ref;  // delta at the last replacement
};

struct BtSched {
  int n_act;  // active samples
  int pending;  // a load case awaits replacement or a check (mixed precision)
  long W;     // work units (tile, layer) over the active samples
  long Nn;    // nodes over the active samples
};

// Everything the batch passes read; device pointers.
template <typename TV>
struct BtData {
  int n;                     // samples
  const int* dims;           // [n][3]: R (rows, y), C (cols, x), L (layers, z)
  const long* noff;          // [n+1] node offsets; vectors of sample s: base 3 noff[s], case k at + k N_s
  const uint16_t* keys;      // [noff[n]]
  const TV* K;               // [n][4][64] dense conductivity matrices (slots past nmat zero)
  const double* K64;         // same in FP64 (replacement operator, right-hand sides)
  DevScalars* sc;            // [n][3]
  BtCtl* ctl;                // [n][3]
  const BtSched* sch;
  const int* act;            // [n] active sample ids
  const long* wpre;          // [n+1] work prefix over active samples
  const long* npre;          // [n+1] node prefix over active samples
  double* part;              // [(P + n) * 3] partials
  unsigned* ticket;
  int* pending;              // &BtSched::pending: raised by the pointwise finisher, cleared by the replacement pass
  SolveCfg cfg;
  int mixed;
  int replace_every;
  double replace_drop;
};

__device__ __forceinline__ long bt_nodes(const int* dims, int s) { return (long)dims[3 * s] * dims[3 * s + 1] * dims[3 * s + 2]; }
template <int TC>
__device__ __forceinline__ long bt_tiles(const int* dims, int s) {
  return (long)((dims[3 * s] + TE_TR - 1) / TE_TR) * ((dims[3 * s + 1] + TC - 1) / TC);
}
// index of the last prefix entry <= v (prefix[0] = 0 <= v < prefix[m])
__device__ __forceinline__ int bt_find(const long* prefix, int m, long v) {
  int lo = 0, hi = m;  // prefix[lo] <= v < prefix[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= v) lo = mid; else hi = mid;
  }
  return lo;
}
// the CTA (of P over a line of W units) whose slice [b W / P, (b+1) W / P) holds unit w
__device__ __forceinline__ int bt_cta_of(long w, long W, int P) {
  long b = (w * P) / W;
  while (b + 1 < P && ((b + 1) * W) / P <= w) b++;
  while (b > 0 && (b * W) / P > w) b--;
  return (int)b;
}

// whether CTA b's slice is non-empty (when the line is shorter than the grid some are not, and
// they write no partials)
__device__ __forceinline__ bool bt_nonempty(int b, long W, int P) { return ((long)(b + 1) * W) / P > ((long)b * W) / P; }

// Active list: samples with a load case still iterating (or pending a check), with prefix
// sums of their work units and nodes.  One CTA of 1024 threads.
template <int TC>
__global__ void __launch_bounds__(1024) k_bt_schedule(int n, const int* dims, const DevScalars* sc, const BtCtl* ctl, BtSched* sch,
                                                       int* act, long* wpre, long* npre) {
  __shared__ long sw[1024], sn[1024];
  __shared__ int sf[1024];
  __shared__ long cw, cn;
  __shared__ int ca;
  const int tid = threadIdx.x;
  if (tid == 0) { cw = 0; cn = 0; ca = 0; }
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int i = base + tid;
    bool on = false;
    if (i < n)
      for (int k = 0; k < BT_NR; k++) on = on || !sc[BT_NR * i + k].done || ctl[BT_NR * i + k].pending != BT_NONE;
    const long w = on ? bt_tiles<TC>(dims, i) * dims[3 * i + 2] : 0;
    const long nn = on ? bt_nodes(dims, i) : 0;
    sw[tid] = w; sn[tid] = nn; sf[tid] = on ? 1 : 0;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // inclusive scans
      long aw = 0, an = 0;
      int af = 0;
      if (tid >= o) { aw = sw[tid - o]; an = sn[tid - o]; af = sf[tid - o]; }
      __syncthreads();
      sw[tid] += aw; sn[tid] += an; sf[tid] += af;
      __syncthreads();
    }
    if (on) {
      const int pos = ca + sf[tid] - 1;
      act[pos] = i;
      wpre[pos] = cw + sw[tid] - w;
      npre[pos] = cn + sn[tid] - nn;
    }
    __syncthreads();
    if (tid == 1023) { cw += sw[1023]; cn += sn[1023]; ca += sf[1023]; }
    __syncthreads();
  }
  if (tid == 0) {
    wpre[ca] = cw; npre[ca] = cn;
    sch->n_act = ca; sch->W = cw; sch->Nn = cn;
  }
}

// Operator pass over the work line.  RES = false: the block PCG pass, v_k = s_k + beta_k d_k
// formed while staging, q_k = A v_k, d_k <- v_k, alpha_k finished per load case.  RES = true:
// r_k = b_k - A x_k with the FP64 operator on the FP64 x, for pending load cases only.
template <int TC, typename TV, bool RES>
__global__ void __launch_bounds__(TE_TR * TC) k_bt_apply(BtData<TV> a, const TV* sv, const TV* dold, TV* dnew, TV* q, const double* x,
                                                         const double* b64, TV* r) {
  using TS = std::conditional_t<RES, double, TV>;  // staging / compute type
  constexpr int NT = TE_TR * TC, PR = TE_PR, PC = TC + 2, PP = PR * PC, PS = BT_NR;
  __shared__ TS sK[4 * 65];
  __shared__ TS sP[3 * PP * PS];
  __shared__ double sred[NT / 32];
  __shared__ TS sbeta[BT_NR];
  __shared__ int son[BT_NR];  // load case served by this pass
  const BtSched sch = *a.sch;
  if (sch.n_act == 0 || (RES && !sch.pending)) return;
  const int P = gridDim.x, bid = blockIdx.x, tid = threadIdx.x + TE_TR * threadIdx.y;
  const long W = sch.W, w0 = (long)bid * W / P, w1 = ((long)bid + 1) * W / P;
  const int ctr = (threadIdx.x + 1) + (threadIdx.y + 1) * PR;
  double acc[BT_NR] = {0.0, 0.0, 0.0};
  int cur = -1, s = 0, R = 1, C = 1, L = 1, tiles_r = 1;
  long nbase = 0, vbase = 0, Ns = 0;
  bool any_on = false;
  auto flush = [&](int i) {
    if constexpr (!RES) {
#pragma unroll
      for (int k = 0; k < BT_NR; k++) {
        const double t = block_sum<NT>(acc[k], sred);
        if (tid == 0) a.part[((long)bid + i) * BT_NR + k] = t;
        acc[k] = 0.0;
      }
    }
  };
  int i = (w0 < w1) ? bt_find(a.wpre, sch.n_act, w0) : 0;
  for (long w = w0; w < w1;) {
    while (w >= a.wpre[i + 1]) i++;
    if (i != cur) {
      if (cur >= 0) flush(cur);
      cur = i;
      s = a.act[i];
      R = a.dims[3 * s]; C = a.dims[3 * s + 1]; L = a.dims[3 * s + 2];
      tiles_r = (R + TE_TR - 1) / TE_TR;
      nbase = a.noff[s]; Ns = (long)R * C * L; vbase = BT_NR * nbase;
      __syncthreads();
      const double* K64 = a.K64 + (size_t)s * 256;
      const TV* Kv = a.K + (size_t)s * 256;
      for (int t = tid; t < 256; t += NT) sK[(t >> 6) * 65 + (t & 63)] = RES ? TS(K64[t]) : TS(Kv[t]);
      if (tid < BT_NR) {
        const DevScalars& scs = a.sc[BT_NR * s + tid];
        if (RES) son[tid] = a.ctl[BT_NR * s + tid].pending != BT_NONE;
        else son[tid] = !scs.done;
        sbeta[tid] = RES ? TS(0) : TS(scs.beta);
      }
      __syncthreads();
      any_on = son[0] || son[1] || son[2];
    }
    const long u = w - a.wpre[i];
    const int tile = (int)(u / L), l0 = (int)(u % L);
    const int l1 = (int)min((long)L, (long)l0 + (min(w1, a.wpre[i + 1]) - w));
    w += l1 - l0;
    if (!any_on) continue;
    const int r0 = (tile % tiles_r) * TE_TR, c0 = (tile / tiles_r) * TC;
    const size_t RC = (size_t)R * C;
    auto slot = [&](int l) { return ((l % 3) + 3) % 3; };
    auto load_plane = [&](int l) {
      const int lw = wrap(l, L);
      TS* dst = sP + slot(l) * PP * PS;
      for (int p = tid; p < PP; p += NT) {
        const int hr = p % PR, hc = p / PR;
        const int gr = wrap(r0 + hr - 1, R), gc = wrap(c0 + hc - 1, C);
        const size_t node = (size_t)gr + (size_t)gc * R + (size_t)lw * RC;
#pragma unroll
        for (int k = 0; k < BT_NR; k++) {
          const size_t j = vbase + k * Ns + node;
          TS v;
          if (RES) v = son[k] ? TS(x[j]) : TS(0);
          else v = fma(sbeta[k], dold[j], sv[j]);
          dst[p * PS + k] = v;
        }
      }
    };
    __syncthreads();
    load_plane(l0 - 1);
    load_plane(l0);
    const int rr = r0 + threadIdx.x, cc = c0 + threadIdx.y;
    const bool active = rr < R && cc < C;
    for (int l = l0; l < l1; l++) {
      load_plane(l + 1);
      __syncthreads();
      if (active) {
        const size_t node = (size_t)rr + (size_t)cc * R + (size_t)l * RC;
        const unsigned key = a.keys[nbase + node];
        const TS* kb[8];
#pragma unroll
        for (int e = 0; e < 8; e++) kb[e] = sK + ((key >> (2 * e)) & 3u) * 65;
        TS out[BT_NR][1];
#pragma unroll
        for (int k = 0; k < BT_NR; k++) out[k][0] = TS(0);
        // same compile-time pair list as the block operator, with this tile's plane pitch
        blk_all_pairs<1, TS, BT_NR>(std::make_integer_sequence<int, pair_count<1>()>{}, sP + slot(l - 1) * PP * PS,
                                    sP + slot(l) * PP * PS, sP + slot(l + 1) * PP * PS, ctr, kb, out);
        const TS* pc = sP + slot(l) * PP * PS + ctr * PS;
#pragma unroll
        for (int k = 0; k < BT_NR; k++) {
          const size_t j = vbase + k * Ns + node;
          if (RES) {
            if (son[k]) r[j] = TV(b64[j] - (double)out[k][0]);
          } else {
            const TS v = pc[k];
            q[j] = TV(out[k][0]);
            dnew[j] = TV(v);
            acc[k] += (double)v * (double)out[k][0];
          }
        }
      }
      __syncthreads();
    }
  }
  if (RES) return;
  if (cur >= 0) flush(cur);
  // the last CTA finishes alpha_k = delta_k / (d_k . A d_k) per active sample
  __shared__ bool s_last;
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(a.ticket, 1u) == (unsigned)P - 1u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int ii = tid; ii < sch.n_act; ii += NT) {
    const int b0 = bt_cta_of(a.wpre[ii], W, P), b1 = bt_cta_of(a.wpre[ii + 1] - 1, W, P);
    const int ss = a.act[ii];
#pragma unroll
    for (int k = 0; k < BT_NR; k++) {
      DevScalars& sc = a.sc[BT_NR * ss + k];
      if (sc.done) continue;
      double sum = 0.0;
      for (int b = b0; b <= b1; b++)
        if (bt_nonempty(b, W, P)) sum += __ldcg(a.part + ((long)b + ii) * BT_NR + k);
      sc.red[0] = sum;
      sc.alpha = sc.delta / sum;
    }
  }
  if (tid == 0) *a.ticket = 0u;
}

// Pointwise pass over the node line of the active samples.
//   PW_INIT: s = M^-1 r, delta0 (zero guess); PW_PCG: x += a d, r -= a q, s = M^-1 r, delta,
//   stopping test (and, mixed, the replacement / check decisions); PW_REPL: for pending load
//   cases, s = M^-1 r from the true residual, then the replacement or check finisher.
template <typename TV, int MODE>
__global__ void __launch_bounds__(PW_NT) k_bt_point(BtData<TV> a, double* x, const TV* d, TV* r, const TV* q, TV* sv) {
  __shared__ double sred[PW_NT / 32];
  __shared__ TV sD[32];
  __shared__ double salpha[BT_NR];
  __shared__ int son[BT_NR];
  const BtSched sch = *a.sch;
  if (sch.n_act == 0 || (MODE == PW_REPL && !sch.pending)) return;
  const int P = gridDim.x, bid = blockIdx.x, tid = threadIdx.x;
  const long Nn = sch.Nn, n0 = (long)bid * Nn / P, n1 = ((long)bid + 1) * Nn / P;
  double acc[BT_NR] = {0.0, 0.0, 0.0};
  int cur = -1;
  auto flush = [&](int i) {
#pragma unroll
    for (int k = 0; k < BT_NR; k++) {
      const double t = block_sum<PW_NT>(acc[k], sred);
      if (tid == 0) a.part[((long)bid + i) * BT_NR + k] = t;
      acc[k] = 0.0;
    }
  };
  int i = (n0 < n1) ? bt_find(a.npre, sch.n_act, n0) : 0;
  for (long v0 = n0; v0 < n1;) {
    while (v0 >= a.npre[i + 1]) i++;
    if (i != cur) {
      if (cur >= 0) flush(cur);
      cur = i;
      const int s = a.act[i];
      __syncthreads();
      for (int t = tid; t < 32; t += PW_NT) {
        const int m = t >> 3, k = t & 7;
        const TV dv = a.K[(size_t)s * 256 + m * 64 + k * 9];
        sD[t] = (dv != TV(0)) ? dv : TV(1);
      }
      if (tid < BT_NR) {
        const DevScalars& scs = a.sc[BT_NR * s + tid];
        if (MODE == PW_REPL) son[tid] = a.ctl[BT_NR * s + tid].pending != BT_NONE;
        else if (MODE == PW_INIT) son[tid] = 1;
        else son[tid] = !scs.done;
        salpha[tid] = (MODE == PW_PCG) ? scs.alpha : 0.0;
      }
      __syncthreads();
    }
    const int s = a.act[i];
    const long Ns = bt_nodes(a.dims, s), nbase = a.noff[s], vbase = BT_NR * nbase;
    const long seg_end = min(n1, a.npre[i + 1]);
    const long loc0 = v0 - a.npre[i];
    const long cnt = seg_end - v0;
    if (son[0] || son[1] || son[2]) {
      for (long t = tid; t < cnt; t += PW_NT) {
        const long node = loc0 + t;
        TV inv[1];
        if (a.cfg.precond) te_invdiag<1, TV>(sD, a.keys[nbase + node], inv);
        else inv[0] = TV(1);
#pragma unroll
        for (int k = 0; k < BT_NR; k++) {
          if (!son[k]) continue;
          const size_t j = vbase + k * Ns + node;
          TV rv = r[j];
          if (MODE == PW_PCG) {
            const double al = salpha[k];
            const TV dv = d[j];
            x[j] = fma(al, (double)dv, x[j]);
            rv = fma(-TV(al), q[j], rv);
            r[j] = rv;
          }
          const TV s_ = rv * inv[0];
          sv[j] = s_;
          acc[k] += (double)rv * (double)s_;
        }
      }
    }
    v0 = seg_end;
  }
  if (cur >= 0) flush(cur);
  __shared__ bool s_last;
  if (tid == 0) {
    __threadfence();
    s_last = atomicAdd(a.ticket, 1u) == (unsigned)P - 1u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int ii = tid; ii < sch.n_act; ii += PW_NT) {
    const int b0 = bt_cta_of(a.npre[ii], Nn, P), b1 = bt_cta_of(a.npre[ii + 1] - 1, Nn, P);
    const int ss = a.act[ii];
    for (int k = 0; k < BT_NR; k++) {
      DevScalars* sc = a.sc + BT_NR * ss + k;
      BtCtl* ct = a.ctl + BT_NR * ss + k;
      const bool served = (MODE == PW_REPL) ? ct->pending != BT_NONE : (MODE == PW_INIT ? true : !sc->done);
      if (!served) continue;
      double sum = 0.0;
      for (int b = b0; b <= b1; b++)
        if (bt_nonempty(b, Nn, P)) sum += __ldcg(a.part + ((long)b + ii) * BT_NR + k);
      double s4[4] = {sum, 0.0, 0.0, 0.0};
      sc->red[0] = sum;
      if (MODE == PW_INIT) {
        pcg_finish(PW_INIT, s4, sc, a.cfg);
        ct->pending = BT_NONE; ct->next_replace = a.replace_every; ct->checks = 0; ct->ref = fabs(sc->delta0);
      } else if (MODE == PW_PCG) {
        pcg_finish(PW_PCG, s4, sc, a.cfg);
        if (a.mixed) {
          if (sc->done) {
            if (sc->status == 0 && sc->found && ct->checks < 32) ct->pending = BT_CHECK;
          } else if (sc->iteration % BT_REPL_PERIOD == 0 &&
                     ((a.replace_every > 0 && sc->iteration >= ct->next_replace) || fabs(sc->delta) < a.replace_drop * ct->ref)) {
            ct->pending = BT_REPL;
          }
          if (ct->pending != BT_NONE) *a.pending = 1;
        }
      } else {  // PW_REPL
        if (ct->pending == BT_REPL) {
          pcg_finish(PW_REPL, s4, sc, a.cfg);
        } else {
          ct->checks++;
          pcg_finish(PW_CHECK, s4, sc, a.cfg);
        }
        ct->next_replace = sc->iteration + a.replace_every;
        ct->ref = fabs(sc->delta);
        ct->pending = BT_NONE;
      }
    }
  }
  if (tid == 0) {
    *a.ticket = 0u;
    if (MODE == PW_REPL) *a.pending = 0;
  }
}

// Right-hand sides of the three load cases of every sample (the thermal case of
// k_rhs_load_case): b_k = -jump_k * sum of the +k face columns over boundary voxels.
template <typename TV>
__global__ void k_bt_rhs(int n, const int* dims, const long* noff, const uint16_t* keys, const double* K64, double* b64, TV* r) {
  const long Ntot = noff[n];
  for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < Ntot; g += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n;
    while (hi - lo > 1) { const int mid = (lo + hi) >> 1; if (noff[mid] <= g) lo = mid; else hi = mid; }
    const int s = lo;
    const int R = dims[3 * s], C = dims[3 * s + 1], L = dims[3 * s + 2];
    const long node = g - noff[s], Ns = (long)R * C * L;
    const int rr = (int)(node % R), cc = (int)((node / R) % C), ll = (int)(node / ((long)R * C));
    const unsigned key = keys[g];
    const double* Ks = K64 + (size_t)s * 256;
#pragma unroll
    for (int axis = 0; axis < BT_NR; axis++) {
      const double jump = axis == 0 ? C : (axis == 1 ? R : L);
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int er = wrap(rr - drow(k) - 1, R), ec = wrap(cc - dcol(k), C), el = wrap(ll - dlay(k), L);
        const bool boundary = axis == 0 ? ec == C - 1 : (axis == 1 ? er == 0 : el == 0);
        if (!boundary) continue;
        const double* Km = Ks + ((key >> (2 * k)) & 3u) * 64;
        double t = 0.0;
        for (int f = 0; f < 4; f++) t += Km[k * 8 + face_node(axis, f)];
        v -= t * jump;
      }
      const size_t j = BT_NR * noff[s] + axis * Ns + node;
      b64[j] = v;
      r[j] = TV(v);
    }
  }
}

// Volume term of the effective tensor per sample and load case: one CTA per sample,
// moments[s][k][row] = sum_n sum_e CB[mat_e(n)][row][e] x_k[n]   (CB: [n][4][3][8]).
static __global__ void __launch_bounds__(PW_NT) k_bt_moments(const int* dims, const long* noff, const uint16_t* keys, const double* CB,
                                                      const double* x, double* moments) {
  __shared__ double sCB[4 * 24];
  __shared__ double sred[PW_NT / 32];
  const int s = blockIdx.x;
  for (int t = threadIdx.x; t < 96; t += PW_NT) sCB[t] = CB[(size_t)s * 96 + t];
  __syncthreads();
  const long Ns = bt_nodes(dims, s), nbase = noff[s];
  double acc[BT_NR * 3];
#pragma unroll
  for (int t = 0; t < BT_NR * 3; t++) acc[t] = 0.0;
  for (long node = threadIdx.x; node < Ns; node += PW_NT) {
    const unsigned key = keys[nbase + node];
    double w[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const double* cb = sCB + ((key >> (2 * e)) & 3u) * 24 + e;
#pragma unroll
      for (int row = 0; row < 3; row++) w[row] += cb[row * 8];
    }
#pragma unroll
    for (int k = 0; k < BT_NR; k++) {
      const double xv = x[BT_NR * nbase + k * Ns + node];
#pragma unroll
      for (int row = 0; row < 3; row++) acc[3 * k + row] = fma(w[row], xv, acc[3 * k + row]);
    }
  }
#pragma unroll
  for (int t = 0; t < BT_NR * 3; t++) {
    const double v = block_sum<PW_NT>(acc[t], sred);
    if (threadIdx.x == 0) moments[(size_t)s * 9 + t] = v;
  }
}

}  // namespace chfem
