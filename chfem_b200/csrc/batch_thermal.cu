// batch_thermal.cu -- host driver of the batched thermal homogenization
// (cudapcgB200SolveThermalBatch, include/cudapcg_b200.h).  The passes are in
// batch_thermal.cuh; this file uploads the batch, picks the tile shape with a short timing of
// each candidate (cached per batch signature), captures the iteration loop as a CUDA graph and
// replays it until every load case of every sample has stopped.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/cudapcg_b200.h"
#include "batch_thermal.cuh"
#include "loadcase.cuh"

using namespace chfem;

namespace {

std::string g_err;
#define BT_CK(call)                                                      \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) { g_err = std::string(#call) + ": " + cudaGetErrorString(e_); return false; } \
  } while (0)

// tile width chosen per batch signature (sizes histogram, precision)
std::map<std::string, int> g_tile_cache;

struct DevBuf {
  std::vector<void*> ptrs;
  template <typename T>
  bool alloc(T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) { g_err = "cudaMalloc failed (batch too large?)"; return false; }
    ptrs.push_back(q);
    *p = (T*)q;
    return true;
  }
  ~DevBuf() { for (void* p : ptrs) cudaFree(p); }
};

int num_sms() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}
template <typename K>
int resident_ctas(K kernel, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
  return per_sm * num_sms();
}

struct Inputs {
  unsigned n;
  const unsigned* dims;
  const uint16_t* const* keys;
  const unsigned* nmat;
  const double* const* K;
  const double* const* CB;
  double tol;
  unsigned maxit;
  int precond;
  int replace_every;
};

template <typename TV>
struct Batch {
  Inputs in;
  DevBuf buf;
  cudaStream_t st = nullptr;
  int* d_dims = nullptr;
  long* d_noff = nullptr;
  uint16_t* d_keys = nullptr;
  TV* d_K = nullptr;
  double *d_K64 = nullptr, *d_CB = nullptr, *d_x = nullptr, *d_b = nullptr, *d_part = nullptr, *d_mom = nullptr;
  TV *d_r = nullptr, *d_s = nullptr, *d_d0 = nullptr, *d_d1 = nullptr, *d_q = nullptr;
  DevScalars* d_sc = nullptr;
  BtCtl* d_ctl = nullptr;
  BtSched* d_sch = nullptr;
  BtSched* h_sch = nullptr;
  int* d_act = nullptr;
  long *d_wpre = nullptr, *d_npre = nullptr;
  unsigned* d_ticket = nullptr;
  long Ntot = 0;
  unsigned long long launches = 0;

  ~Batch() {
    if (h_sch) cudaFreeHost(h_sch);
    if (st) cudaStreamDestroy(st);
  }

  BtData<TV> data(bool mixed) const {
    BtData<TV> a;
    a.n = (int)in.n; a.dims = d_dims; a.noff = d_noff; a.keys = d_keys; a.K = d_K; a.K64 = d_K64;
    a.sc = d_sc; a.ctl = d_ctl; a.sch = d_sch; a.act = d_act; a.wpre = d_wpre; a.npre = d_npre;
    a.part = d_part; a.ticket = d_ticket; a.pending = &d_sch->pending;
    a.cfg.tol = in.tol; a.cfg.maxit = (int)std::min<unsigned>(in.maxit, 0x7fffffffu); a.cfg.norm = NORM_L2;
    a.cfg.precond = in.precond; a.cfg.nhmg = 0;
    a.mixed = mixed ? 1 : 0;
    a.replace_every = in.replace_every;
    a.replace_drop = 1e-4;
    return a;
  }

  bool setup() {
    const unsigned n = in.n;
    BT_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::vector<int> dims(3 * n);
    std::vector<long> noff(n + 1, 0);
    for (unsigned s = 0; s < n; s++) {
      for (int t = 0; t < 3; t++) dims[3 * s + t] = (int)in.dims[3 * s + t];
      noff[s + 1] = noff[s] + (long)in.dims[3 * s] * in.dims[3 * s + 1] * in.dims[3 * s + 2];
    }
    Ntot = noff[n];
    std::vector<double> K64((size_t)n * 256, 0.0), CB((size_t)n * 96, 0.0);
    std::vector<TV> Kv((size_t)n * 256, TV(0));
    for (unsigned s = 0; s < n; s++) {
      for (unsigned t = 0; t < 64 * in.nmat[s]; t++) { K64[(size_t)s * 256 + t] = in.K[s][t]; Kv[(size_t)s * 256 + t] = TV(in.K[s][t]); }
      for (unsigned t = 0; t < 24 * in.nmat[s]; t++) CB[(size_t)s * 96 + t] = in.CB[s][t];
    }
    const size_t nv = (size_t)BT_NR * Ntot;
    if (!buf.alloc(&d_dims, 3 * n) || !buf.alloc(&d_noff, n + 1) || !buf.alloc(&d_keys, Ntot) || !buf.alloc(&d_K, (size_t)n * 256) ||
        !buf.alloc(&d_K64, (size_t)n * 256) || !buf.alloc(&d_CB, (size_t)n * 96) || !buf.alloc(&d_x, nv) || !buf.alloc(&d_b, nv) ||
        !buf.alloc(&d_r, nv) || !buf.alloc(&d_s, nv) || !buf.alloc(&d_d0, nv) || !buf.alloc(&d_d1, nv) || !buf.alloc(&d_q, nv) ||
        !buf.alloc(&d_sc, (size_t)BT_NR * n) || !buf.alloc(&d_ctl, (size_t)BT_NR * n) || !buf.alloc(&d_sch, 1) ||
        !buf.alloc(&d_act, n) || !buf.alloc(&d_wpre, n + 1) || !buf.alloc(&d_npre, n + 1) || !buf.alloc(&d_ticket, 1) ||
        !buf.alloc(&d_mom, (size_t)n * 9))
      return false;
    const int pmax = 32 * num_sms();  // at most 32 resident CTAs per SM
    if (!buf.alloc(&d_part, ((size_t)pmax + n) * BT_NR)) return false;
    BT_CK(cudaMallocHost(&h_sch, sizeof(BtSched)));
    BT_CK(cudaMemcpyAsync(d_dims, dims.data(), dims.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    BT_CK(cudaMemcpyAsync(d_noff, noff.data(), noff.size() * sizeof(long), cudaMemcpyHostToDevice, st));
    for (unsigned s = 0; s < n; s++)
      BT_CK(cudaMemcpyAsync(d_keys + noff[s], in.keys[s], (noff[s + 1] - noff[s]) * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
    BT_CK(cudaMemcpyAsync(d_K64, K64.data(), K64.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    BT_CK(cudaMemcpyAsync(d_K, Kv.data(), Kv.size() * sizeof(TV), cudaMemcpyHostToDevice, st));
    BT_CK(cudaMemcpyAsync(d_CB, CB.data(), CB.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    BT_CK(cudaMemsetAsync(d_ticket, 0, sizeof(unsigned), st));
    k_bt_rhs<TV><<<8 * num_sms(), 256, 0, st>>>((int)n, d_dims, d_noff, d_keys, d_K64, d_b, d_r);
    launches++;
    BT_CK(cudaPeekAtLastError());
    // host buffers must stay valid until the uploads are done
    BT_CK(cudaStreamSynchronize(st));
    return true;
  }

  bool reset_state() {
    const size_t nv = (size_t)BT_NR * Ntot;
    BT_CK(cudaMemsetAsync(d_x, 0, nv * sizeof(double), st));
    BT_CK(cudaMemsetAsync(d_s, 0, nv * sizeof(TV), st));
    BT_CK(cudaMemsetAsync(d_d0, 0, nv * sizeof(TV), st));
    BT_CK(cudaMemsetAsync(d_d1, 0, nv * sizeof(TV), st));
    BT_CK(cudaMemsetAsync(d_q, 0, nv * sizeof(TV), st));
    BT_CK(cudaMemsetAsync(d_sc, 0, (size_t)BT_NR * in.n * sizeof(DevScalars), st));
    BT_CK(cudaMemsetAsync(d_ctl, 0, (size_t)BT_NR * in.n * sizeof(BtCtl), st));
    BT_CK(cudaMemsetAsync(d_sch, 0, sizeof(BtSched), st));
    return true;
  }

  template <int TC>
  bool enqueue_schedule() {
    k_bt_schedule<TC><<<1, 1024, 0, st>>>((int)in.n, d_dims, d_sc, d_ctl, d_sch, d_act, d_wpre, d_npre);
    launches++;
    BT_CK(cudaPeekAtLastError());
    return true;
  }
  template <int TC>
  bool enqueue_iteration(int parity, bool mixed, int p_apply, int p_point) {
    TV* dold = parity ? d_d1 : d_d0;
    TV* dnew = parity ? d_d0 : d_d1;
    const BtData<TV> a = data(mixed);
    const dim3 blk(TE_TR, TC);
    k_bt_apply<TC, TV, false><<<p_apply, blk, 0, st>>>(a, d_s, dold, dnew, d_q, d_x, d_b, d_r);
    k_bt_point<TV, PW_PCG><<<p_point, PW_NT, 0, st>>>(a, d_x, dnew, d_r, d_q, d_s);
    launches += 2;
    if (mixed) {
      k_bt_apply<TC, TV, true><<<p_apply, blk, 0, st>>>(a, d_s, dold, dnew, d_q, d_x, d_b, d_r);
      k_bt_point<TV, PW_REPL><<<p_point, PW_NT, 0, st>>>(a, d_x, dnew, d_r, d_q, d_s);
      launches += 2;
    }
    BT_CK(cudaPeekAtLastError());
    return true;
  }

  // mean device time of the operator pass with tile width TC, from the initial state
  template <int TC>
  double time_apply() {
    const int p = resident_ctas(k_bt_apply<TC, TV, false>, TE_TR * TC);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    bool ok = reset_state() && enqueue_schedule<TC>();
    for (int rep = 0; ok && rep < 4; rep++) {
      cudaEventRecord(e0, st);
      k_bt_apply<TC, TV, false><<<p, dim3(TE_TR, TC), 0, st>>>(data(false), d_s, d_d0, d_d1, d_q, d_x, d_b, d_r);
      cudaEventRecord(e1, st);
      ok = cudaEventSynchronize(e1) == cudaSuccess;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) best = std::min(best, ms);
    }
    launches += 4;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ok ? best : 1e30;
  }

  template <int TC>
  bool solve(bool mixed, cudapcgB200BatchStats* stats) {
    const int p_apply = resident_ctas(k_bt_apply<TC, TV, false>, TE_TR * TC);
    const int p_point = resident_ctas(k_bt_point<TV, PW_PCG>, PW_NT);
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
    bool ok = reset_state();
    cudaEventRecord(e0, st);
    ok = ok && enqueue_schedule<TC>();
    if (ok) {
      k_bt_point<TV, PW_INIT><<<p_point, PW_NT, 0, st>>>(data(mixed), d_x, d_d0, d_r, d_q, d_s);
      launches++;
      ok = cudaPeekAtLastError() == cudaSuccess;
    }
    cudaEventRecord(e1, st);
    // one graph: the schedule, then an even number of iterations
    const int chunk = 16;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t gx = nullptr;
    if (ok) {
      const unsigned long long l0 = launches;
      ok = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      bool cap = ok && enqueue_schedule<TC>();
      for (int it = 0; cap && it < chunk; it++) cap = enqueue_iteration<TC>(it & 1, mixed, p_apply, p_point);
      const unsigned long long per_graph = launches - l0;
      launches = l0;
      ok = (cudaStreamEndCapture(st, &g) == cudaSuccess) && cap;
      ok = ok && cudaGraphInstantiate(&gx, g, 0) == cudaSuccess;
      const long max_chunks = (long)in.maxit / chunk + 40;  // the check restarts may add a few chunks
      for (long c = 0; ok && c < max_chunks; c++) {
        ok = cudaGraphLaunch(gx, st) == cudaSuccess;
        launches += per_graph;
        ok = ok && cudaMemcpyAsync(h_sch, d_sch, sizeof(BtSched), cudaMemcpyDeviceToHost, st) == cudaSuccess;
        ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
        if (ok && h_sch->n_act == 0) break;
      }
    }
    if (!ok && g_err.empty()) g_err = std::string("batch solve: ") + cudaGetErrorString(cudaGetLastError());
    if (ok) {
      k_bt_moments<<<in.n, PW_NT, 0, st>>>(d_dims, d_noff, d_keys, d_CB, d_x, d_mom);
      launches++;
      ok = cudaPeekAtLastError() == cudaSuccess;
    }
    cudaEventRecord(e2, st);
    ok = ok && cudaEventSynchronize(e2) == cudaSuccess;
    float ms1 = 0, ms2 = 0;
    cudaEventElapsedTime(&ms1, e0, e1);
    cudaEventElapsedTime(&ms2, e1, e2);
    if (stats) {
      stats->setup_seconds = ms1 * 1e-3;
      stats->solve_seconds = ms2 * 1e-3;
      stats->tile_cols = TC;
      stats->ctas_operator = p_apply;
      stats->ctas_pointwise = p_point;
    }
    if (gx) cudaGraphExecDestroy(gx);
    if (g) cudaGraphDestroy(g);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    return ok;
  }

  bool results(double* moments, unsigned* iterations, double* residuals, cudapcgB200BatchStats* stats) {
    const unsigned n = in.n;
    std::vector<DevScalars> sc((size_t)BT_NR * n);
    BT_CK(cudaMemcpyAsync(moments, d_mom, (size_t)n * 9 * sizeof(double), cudaMemcpyDeviceToHost, st));
    BT_CK(cudaMemcpyAsync(sc.data(), d_sc, sc.size() * sizeof(DevScalars), cudaMemcpyDeviceToHost, st));
    BT_CK(cudaStreamSynchronize(st));
    unsigned maxit = 0, found = 0;
    for (size_t t = 0; t < sc.size(); t++) {
      const DevScalars& h = sc[t];
      double res = h.status == 1 ? 0.0 : std::sqrt(std::fabs(h.delta) / std::fabs(h.delta0));
      if (iterations) iterations[t] = (unsigned)h.iteration;
      if (residuals) residuals[t] = res;
      maxit = std::max(maxit, (unsigned)h.iteration);
      found += (h.status == 1 || !(std::fabs(h.delta) > in.tol * in.tol * std::fabs(h.delta0))) ? 1u : 0u;
    }
    if (stats) { stats->max_iterations = maxit; stats->converged = found; stats->kernel_launches = launches; }
    return found == sc.size();
  }
};

template <typename TV>
int run_batch(const Inputs& in, bool mixed, double* moments, unsigned* iterations, double* residuals, cudapcgB200BatchStats* stats) {
  Batch<TV> b;
  b.in = in;
  if (!b.setup()) return 0;
  // tile shape: cached per batch signature, else timed once
  std::string sig = std::string(mixed ? "m" : "d") + std::to_string(in.n) + (in.precond ? "p" : "c");
  {
    std::map<std::string, int> hist;
    for (unsigned s = 0; s < in.n; s++) hist[std::to_string(in.dims[3 * s]) + "x" + std::to_string(in.dims[3 * s + 1]) + "x" + std::to_string(in.dims[3 * s + 2])]++;
    for (auto& kv : hist) sig += ":" + kv.first + "*" + std::to_string(kv.second);
  }
  int tc;
  auto it = g_tile_cache.find(sig);
  if (it != g_tile_cache.end()) tc = it->second;
  else {
    const double t4 = b.template time_apply<4>(), t8 = b.template time_apply<8>(), t16 = b.template time_apply<16>();
    tc = (t4 <= t8 && t4 <= t16) ? 4 : (t8 <= t16 ? 8 : 16);
    if (stats) { stats->tile_ms[0] = t4; stats->tile_ms[1] = t8; stats->tile_ms[2] = t16; }
    g_tile_cache[sig] = tc;
  }
  bool ok = tc == 4 ? b.template solve<4>(mixed, stats) : (tc == 8 ? b.template solve<8>(mixed, stats) : b.template solve<16>(mixed, stats));
  if (!ok) return 0;
  return b.results(moments, iterations, residuals, stats) ? 1 : 2;
}

}  // namespace

extern "C" int cudapcgB200SolveThermalBatch(unsigned int nsamples, const unsigned int* dims, const uint16_t* const* keys,
                                            const unsigned int* nmat, const double* const* Kdense, const double* const* CB,
                                            double tol, unsigned int maxit, int precision, int precondition, double* moments,
                                            unsigned int* iterations, double* residuals, cudapcgB200BatchStats* stats) {
  g_err.clear();
  if (stats) memset(stats, 0, sizeof(*stats));
  if (!nsamples || !dims || !keys || !nmat || !Kdense || !CB || !moments) { g_err = "null argument"; return 0; }
  for (unsigned s = 0; s < nsamples; s++) {
    if (!dims[3 * s] || !dims[3 * s + 1] || !dims[3 * s + 2]) { g_err = "empty sample " + std::to_string(s); return 0; }
    if (nmat[s] < 1 || nmat[s] > 4) { g_err = "1 to 4 materials per sample (16-bit node keys)"; return 0; }
    if (!keys[s] || !Kdense[s] || !CB[s]) { g_err = "null array of sample " + std::to_string(s); return 0; }
  }
  if (!(tol > 0.0)) { g_err = "tolerance must be positive"; return 0; }
  if (precision != CHFEM_B200_FP64 && precision != CHFEM_B200_MIXED) { g_err = "precision must be CHFEM_B200_FP64 or CHFEM_B200_MIXED"; return 0; }
  const Inputs in{nsamples, dims, keys, nmat, Kdense, CB, tol, maxit, precondition ? 1 : 0, 50};
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = (precision == CHFEM_B200_MIXED) ? run_batch<float>(in, true, moments, iterations, residuals, stats)
                                                  : run_batch<double>(in, false, moments, iterations, residuals, stats);
  if (stats) stats->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

extern "C" const char* cudapcgB200BatchLastError(void) { return g_err.c_str(); }
