// cudapcg_b200.cu -- the cudapcg C ABI on B200: model upload, device-resident Krylov loops
// captured in CUDA graphs, precision modes.
//
// Reference counterparts: chfem/src/femhmg/cudapcg/cudapcg.cu (API object and dispatch),
// solvers/pcg.cu, cg.cu, pminres.cu, minres.cu (iteration recurrences),
// kernels/wrappers.cu (launches).  The recurrences, stopping tests and special cases are
// the reference's; the execution is not: each iteration is two fused passes whose scalars
// are finished on the device, and chunks of iterations replay as one CUDA graph.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <chrono>

#include "../../include/cudapcg_b200.h"
#include "common.cuh"
#include "stencil_te.cuh"
#include "pointwise.cuh"
#include "stencil_fluid.cuh"
#include "stencil_fluid2.cuh"
#include "stencil_block.cuh"
#include "stencil_asm.cuh"
#include "asm_apply.h"
#include "th_apply.h"
#include "stencil_2d.cuh"
#include "pore_maps.h"
#include "stencil_fluid_block.cuh"
#include "loadcase.cuh"
#include "fields.cuh"
#include "minres.cuh"

using namespace chfem;

// ---------------------------------------------------------------------------------------
// Errors: recorded, never fatal to the process, never reset the device.
static std::string g_err;
static void set_err(const char* where, const char* what) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s", where, what);
  g_err = buf;
  fprintf(stderr, "chfem_b200 error: %s\n", buf);
}
#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) {                                       \
      set_err(#call, cudaGetErrorString(e_));                      \
      return CUDAPCG_FALSE;                                        \
    }                                                              \
  } while (0)
#define CKV(call)                                                  \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) { set_err(#call, cudaGetErrorString(e_)); return false; } \
  } while (0)

static int g_num_sms = 0;
static int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

// ---------------------------------------------------------------------------------------
// Dense element matrices from the reference's local-matrix formats (cudapcgSetLclMtxs).
// Thermal: 40 stored non-zeros per material, rows 0..7 in ascending column order, the
// zeros being the pairs of nodes that share an edge (femhmg_thermal_3D.c:42-120).
static void sparseq1_to_dense(const double* sp, double* dense) {
  int p = 0;
  for (int a = 0; a < 8; a++)
    for (int b = 0; b < 8; b++) dense[a * 8 + b] = shares_edge(a, b) ? 0.0 : sp[p++];
}

// ---------------------------------------------------------------------------------------
struct Solver {
  // configuration (cudapcg.cu:108-183 defaults)
  int analysis = 0, par = 0;
  bool dim2 = false;  // 2D thermal / elastic (pixel images, one layer, 4-bit key fields)
  bool fluid = false; // Stokes (FLUID_3D or FLUID_2D)
  int fdim = 3;       // Stokes: 3 (voxels) or 2 (pixels, one layer)
  double tol = 0.00001;
  unsigned maxit = 100000;
  int solver_flag = CUDAPCG_CG_SOLVER;
  int precond = 1;
  int resnorm = CUDAPCG_L2_NORM;
  std::string header;
  int precision = CHFEM_B200_FP64;
  unsigned replace_every = 50;
  // mixed precision: also replace once delta = r.M^-1 r has fallen by this factor since the last
  // replacement, before the FP32 recursive residual drifts away from b - A x
  double replace_drop = 1e-4;
  unsigned iters_per_launch = 16;
  // model
  cudapcgModel_t* model = nullptr;
  int R = 0, C = 0, L = 0;
  long N = 0, nvars = 0, nV = 0, nB = 0;
  int nmat = 0, nd = 1;
  std::vector<double> Kd;   // dense element matrices (host copy)
  bool have_K = false, have_keys = false, have_maps = false;
  // image pore map (CUDAPCG_POREMAP_IMG): the per-node fluid keys handed over by
  // cudapcgSetPoreMap, kept until the node->DOF map is there too
  bool poremap_img = false, have_img_keys = false;
  uint8_t* d_img_fkeys = nullptr;
  uint16_t* d_keys = nullptr;
  uint32_t* d_dof_of_node = nullptr;
  uint32_t* d_node_of_dof = nullptr;
  uint8_t* d_bkeys = nullptr;
  double* d_K64 = nullptr;  // dense element matrices, FP64 (FP64 solves, residual replacement)
  float* d_K32 = nullptr;   // dense element matrices, FP32 (mixed-precision iterations)
  // assembled neighbour blocks of a two-material model (stencil_asm.cuh), per precision
  double* d_tab64 = nullptr;
  float* d_tab32 = nullptr;
  // thermal models with cubic-symmetric element matrices: the table of the thermal pass
  // (stencil_th.cuh), per precision; th_state 0 not checked yet, 1 applies, -1 does not
  double* d_th64 = nullptr;
  float* d_th32 = nullptr;
  int th_state = 0;
  // scalar density field (cudapcgSetParametricDensityField): 16-bit code per voxel and its
  // range; the inverse Jacobi diagonal it implies, per unknown (FP64, built at solve set-up)
  uint16_t* d_sdf = nullptr;
  double sdf_min = 0.0, sdf_max = 0.0;
  double* d_invd = nullptr;
  // Krylov work vectors, typed for the precision in use
  int vec_prec = -1;
  int vec_layout = -1;  // which work vectors ensure_vectors allocated (precision, solver kind)
  void* r = nullptr; void* r2 = nullptr; void* d0 = nullptr; void* d1 = nullptr;
  void* q = nullptr; void* s = nullptr; void* q2 = nullptr;
  // FP64 in every mode: the solution, the right-hand side, an operator output and staging
  double* x = nullptr;
  double* b64 = nullptr;
  double* y64 = nullptr;
  double* x64 = nullptr;
  bool arrays_alloc = false, user_arrays = false;
  bool x0_set = false, rhs_set = false;
  // device scalars and reductions
  DevScalars* d_sc = nullptr;
  DevScalars* h_sc = nullptr;  // pinned
  DevScalars* cur_sc = nullptr;  // record the launch helpers target (d_sc, or one of a block's)
  double* d_part = nullptr;
  unsigned* d_ticket = nullptr;
  int part_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  // graph cache
  cudaGraphExec_t gexec = nullptr;
  int graph_key = -1;
  // results
  unsigned iteration = 0;
  double residual = 1.0;
  int found = 0;
  double total_time = 0.0, mean_time = 0.0;
  double solve_dev_s = 0.0, setup_dev_s = 0.0;
  unsigned long long launches = 0;
  unsigned long count = 0;
  // 2-vector solvers (cudapcg.cu:154-156 defaults): reduction of the solution, the loaded
  // velocity component, the scale of the reduced sums; their device accumulators
  unsigned xr_mode = CUDAPCG_XREDUCE_FULL, xr_shift = 0;
  double xr_scale = 1.0;
  double* d_xa = nullptr;
  double* d_hist = nullptr;
  // one-by-one path on the device: element averaging matrices and the reduced volume term
  double* d_vt = nullptr;
  size_t xa_cap = 0, hist_cap = 0;
};

static Solver* S = nullptr;
static cudapcgFlag_t (*g_ctor)(cudapcgModel_t**, const void*) = nullptr;

static cudapcgFlag_t ctor_simple(cudapcgModel_t** ptr, const void* data) {
  if (!data) return CUDAPCG_FALSE;
  *ptr = (cudapcgModel_t*)data;
  return CUDAPCG_TRUE;
}

template <typename T> static int prec_of() { return sizeof(T) == 8 ? CHFEM_B200_FP64 : CHFEM_B200_MIXED; }

// Device memory of the solver comes from the device's default stream-ordered pool, whose
// release threshold is raised (to a quarter of the device's memory) so that what one model
// frees stays mapped for the next: repeated
// solves (one compute_property call after another) then skip the driver's unmapping and
// mapping, which cost 0.006 to 0.47 s per 128^3 elastic call on different B200 boxes.
// cudapcgB200TrimMemory hands the kept blocks back.  Allocations are made on the legacy stream
// and waited for; a free first waits for the solver's stream, so it follows every launch that
// may read the block.
static void pool_keep() {
  static bool kept[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || kept[dev]) return;
  cudaMemPool_t pool;
  size_t free_b = 0, total_b = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
    // kept at most: a quarter of the device's memory, or CHFEM_B200_POOL_KEEP_BYTES
    uint64_t threshold = total_b / 4;
    if (const char* e = getenv("CHFEM_B200_POOL_KEEP_BYTES")) threshold = strtoull(e, nullptr, 10);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  kept[dev] = true;
}
template <typename P>
static cudaError_t dev_malloc(P** p, size_t bytes) {
  pool_keep();
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), bytes, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  return e;
}
static cudaError_t dev_free(void* p) {
  if (!p) return cudaSuccess;
  if (S && S->stream) cudaStreamSynchronize(S->stream);
  return cudaFreeAsync(p, 0);
}
static void free_ptr(void* p) { dev_free(p); }

static void block_invalidate();
static void block_free();
static void invalidate_graphs() {
  if (S && S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; S->graph_key = -1; }
  block_invalidate();
}

static void free_work_vectors() {
  if (!S) return;
  free_ptr(S->r); free_ptr(S->r2); free_ptr(S->d0); free_ptr(S->d1);
  free_ptr(S->q); free_ptr(S->s); free_ptr(S->q2);
  S->r = S->r2 = S->d0 = S->d1 = S->q = S->s = S->q2 = nullptr;
  S->vec_prec = -1;
  S->vec_layout = -1;
  if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; S->graph_key = -1; }
}
static void free_vectors() {
  if (!S) return;
  free_work_vectors();
  free_ptr(S->x); free_ptr(S->b64); free_ptr(S->y64); free_ptr(S->x64);
  S->x = S->b64 = S->y64 = S->x64 = nullptr;
  free_ptr(S->d_xa); free_ptr(S->d_hist);
  S->d_xa = S->d_hist = nullptr;
  S->xa_cap = S->hist_cap = 0;
  S->arrays_alloc = false;
}

static void free_model_dev() {
  if (!S) return;
  free_ptr(S->d_keys); free_ptr(S->d_dof_of_node); free_ptr(S->d_node_of_dof); free_ptr(S->d_bkeys);
  free_ptr(S->d_K64); free_ptr(S->d_K32); free_ptr(S->d_tab64); free_ptr(S->d_tab32);
  free_ptr(S->d_th64); free_ptr(S->d_th32);
  free_ptr(S->d_sdf); free_ptr(S->d_invd); free_ptr(S->d_img_fkeys);
  S->d_img_fkeys = nullptr; S->have_img_keys = false;
  S->d_keys = nullptr; S->d_dof_of_node = S->d_node_of_dof = nullptr; S->d_bkeys = nullptr;
  S->d_K64 = nullptr; S->d_K32 = nullptr; S->d_tab64 = nullptr; S->d_tab32 = nullptr;
  S->d_th64 = nullptr; S->d_th32 = nullptr; S->th_state = 0;
  S->d_sdf = nullptr; S->d_invd = nullptr;
  S->have_K = S->have_keys = S->have_maps = false;
}

// any 2D model (thermal, elastic or Stokes): the block, field, device load-case and
// device-numbering entry points are 3D only
static bool is2d() { return S->dim2 || (S->fluid && S->fdim == 2); }
static bool minres_solver() { return S->solver_flag == CUDAPCG_MINRES_SOLVER || S->solver_flag == CUDAPCG_MINRES3_SOLVER; }
// CG3 on thermal / elastic models: the 3-vector PCG (x, r and the direction's two buffers)
static bool pcg3_solver() { return S->solver_flag == CUDAPCG_CG3_SOLVER && !S->fluid; }

// An FP64 vector of nvars entries allocated on first use (staging and scratch; never called
// while a stream capture is open).
static bool ensure_scratch64(double*& p) {
  if (p) return true;
  CKV(dev_malloc(&p, std::max<size_t>((size_t)S->nvars, 1) * 8));
  return true;
}

// Work vectors for precision T, as many as the selected solver reads:
//   every solver      x (FP64), r, the direction's two buffers d0 / d1
//   PCG / MINRES      q = A d
//   Stokes, MINRES    s (Stokes PCG reads a stored M^-1 r; (P)MINRES keeps A M^-1 r)
//   MINRES            r2, q2 (the residual's second buffer, the q recursion)
//   b64 (FP64 right-hand side): kept except for FP64 PCG3, whose r is the only copy of b (as
//   in the reference's 3-vector solvers, chfem/src/femhmg/cudapcg/solvers/pcg3.cu:28-60)
// The right-hand side is carried across a change of precision or solver.
template <typename T>
static bool ensure_vectors() {
  const int p = prec_of<T>();
  const size_t n = std::max<size_t>((size_t)S->nvars, 1);
  const int layout = p | (minres_solver() ? 0x10 : 0) | (pcg3_solver() ? 0x20 : 0) | (S->fluid ? 0x40 : 0);
  const bool want_b64 = !(pcg3_solver() && p == CHFEM_B200_FP64);
  if (!S->x) {
    CKV(dev_malloc(&S->x, n * 8));
    CKV(cudaMemsetAsync(S->x, 0, n * 8, S->stream));
    S->arrays_alloc = true;
  }
  if (S->vec_prec == p && S->r && S->vec_layout == layout && (S->b64 != nullptr) == want_b64) return true;
  // the right-hand side: from b64, or from an FP64 r that is its only copy
  if (S->rhs_set && !S->b64 && S->r && S->vec_prec == CHFEM_B200_FP64) {
    CKV(dev_malloc(&S->b64, n * 8));
    CKV(cudaMemcpyAsync(S->b64, S->r, n * 8, cudaMemcpyDeviceToDevice, S->stream));
  }
  if (want_b64 && !S->b64) {
    CKV(dev_malloc(&S->b64, n * 8));
    CKV(cudaMemsetAsync(S->b64, 0, n * 8, S->stream));
  }
  free_work_vectors();
  std::vector<void**> vs = {&S->r, &S->d0, &S->d1};
  if (!pcg3_solver()) vs.push_back(&S->q);
  if (S->fluid || minres_solver()) vs.push_back(&S->s);
  if (minres_solver()) { vs.push_back(&S->r2); vs.push_back(&S->q2); }
  for (void** v : vs) {
    CKV(dev_malloc(v, n * sizeof(T)));
    CKV(cudaMemsetAsync(*v, 0, n * sizeof(T), S->stream));
  }
  S->vec_prec = p;
  S->vec_layout = layout;
  if (S->rhs_set && S->b64) {  // re-derive the working right-hand side from its FP64 copy
    if (sizeof(T) == 8) CKV(cudaMemcpyAsync(S->r, S->b64, n * 8, cudaMemcpyDeviceToDevice, S->stream));
    else k_convert<double, float><<<std::max<long>(1, std::min<long>((n + 255) / 256, 8 * 148)), 256, 0, S->stream>>>(S->b64, (float*)S->r, (long)n);
  }
  if (!want_b64 && S->b64) { CKV(cudaStreamSynchronize(S->stream)); free_ptr(S->b64); S->b64 = nullptr; }
  if (p == CHFEM_B200_MIXED && !ensure_scratch64(S->y64)) return false;  // residual replacement
  if (getenv("CHFEM_B200_TRACE"))
    fprintf(stderr, "[vectors] precision %d layout 0x%x: r %d r2 %d d0 %d d1 %d q %d s %d q2 %d | x %d b64 %d y64 %d x64 %d\n", p, layout,
            !!S->r, !!S->r2, !!S->d0, !!S->d1, !!S->q, !!S->s, !!S->q2, !!S->x, !!S->b64, !!S->y64, !!S->x64);
  return true;
}

// Assembled neighbour blocks (stencil_asm.cuh) of a thermal/elastic model of at most two
// materials; CHFEM_B200_BLOCK_OP=element keeps the element-by-element block operator.
static bool asm_applies() {
  if (S->fluid || S->dim2 || S->nmat > 2 || S->d_sdf) return false;
  const char* e = getenv("CHFEM_B200_BLOCK_OP");
  return !(e && !strcmp(e, "element"));
}
template <typename T> static T*& tabdev();
template <> double*& tabdev<double>() { return S->d_tab64; }
template <> float*& tabdev<float>() { return S->d_tab32; }
template <typename T>
static bool ensure_tab() {
  if (tabdev<T>()) return true;
  if (!S->have_K) { set_err("solve", "local matrices were not set (cudapcgSetLclMtxs)"); return false; }
  const int bs = S->nd == 1 ? 1 : (sizeof(T) == 4 ? 12 : 9);  // AsmLayout<ND, T, NR>::BS
  std::vector<double> t64((size_t)asm_table_words(S->nd, bs));
  asm_build_table(S->nd, S->nmat, S->Kd.data(), bs, t64.data());
  std::vector<T> t(t64.begin(), t64.end());
  T* d = nullptr;
  CKV(dev_malloc(&d, t.size() * sizeof(T)));
  CKV(cudaMemcpy(d, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice));
  tabdev<T>() = d;
  return true;
}

// The thermal pass of stencil_th.cuh: 3D thermal models without a density field whose element
// matrices have the cubic structure it relies on (checked once per model);
// CHFEM_B200_THERMAL_OP=generic keeps the generic pass.
static bool th_applies() {
  if (S->analysis != CUDAPCG_THERMAL_3D || S->d_sdf || S->nmat > 4 || !S->have_K) return false;
  const char* e = getenv("CHFEM_B200_THERMAL_OP");
  if (e && !strcmp(e, "generic")) return false;
  if (S->th_state == 0) {
    std::vector<double> t((size_t)th_table_words());
    S->th_state = th_build_table((int)S->nmat, S->Kd.data(), t.data()) ? 1 : -1;
  }
  return S->th_state == 1;
}
template <typename T> static T*& thdev();
template <> double*& thdev<double>() { return S->d_th64; }
template <> float*& thdev<float>() { return S->d_th32; }
template <typename T>
static bool ensure_th() {
  if (thdev<T>()) return true;
  std::vector<double> t64((size_t)th_table_words());
  if (!th_build_table((int)S->nmat, S->Kd.data(), t64.data())) { set_err("solve", "thermal table"); return false; }
  std::vector<T> t(t64.begin(), t64.end());
  T* d = nullptr;
  CKV(dev_malloc(&d, t.size() * sizeof(T)));
  CKV(cudaMemcpy(d, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice));
  thdev<T>() = d;
  return true;
}

// Inverse Jacobi diagonal under a scalar density field: sum over the node's 8 voxels of the
// scaled diagonal of its element matrix (matrix_free.cu:2270-2306 and the elastic counterpart
// compute it per application; here once per model).
template <int ND>
__global__ void k_sdf_invdiag(const uint16_t* keys, const uint16_t* sdf, double fmin, double frng, const double* Kd, int R, int C,
                              int L, double* invd) {
  constexpr int ED = 8 * ND;
  const long N = (long)R * C * L;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    const unsigned key = keys[i];
    double d[ND];
#pragma unroll
    for (int cc = 0; cc < ND; cc++) d[cc] = 0.0;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const double f = fmin + frng * (double)sdf[te_voxel(r, c, l, e, R, C, L)] * (1.0 / 65535.0);
      const double* K = Kd + (size_t)((key >> (2 * e)) & 3u) * ED * ED;
#pragma unroll
      for (int cc = 0; cc < ND; cc++) d[cc] += f * K[(e * ND + cc) * ED + e * ND + cc];
    }
#pragma unroll
    for (int cc = 0; cc < ND; cc++) invd[i * ND + cc] = 1.0 / d[cc];
  }
}
static bool ensure_K64_only();
static bool ensure_invd() {
  if (S->d_invd || !(S->d_sdf || S->dim2)) return true;
  if (!ensure_K64_only()) return false;
  CKV(dev_malloc(&S->d_invd, sizeof(double) * S->N * S->nd));
  const long g = std::max(1L, std::min<long>((S->N + 255) / 256, 8L * num_sms()));
  if (S->dim2) {
    const double fr = S->sdf_max - S->sdf_min;
    if (S->nd == 1) k_2d_invdiag<1><<<(int)g, 256, 0, S->stream>>>(S->d_keys, S->d_K64, S->R, S->C, S->d_sdf, S->sdf_min, fr, S->d_invd);
    else k_2d_invdiag<2><<<(int)g, 256, 0, S->stream>>>(S->d_keys, S->d_K64, S->R, S->C, S->d_sdf, S->sdf_min, fr, S->d_invd);
  } else if (S->nd == 1) k_sdf_invdiag<1><<<(int)g, 256, 0, S->stream>>>(S->d_keys, S->d_sdf, S->sdf_min, S->sdf_max - S->sdf_min, S->d_K64, S->R, S->C, S->L, S->d_invd);
  else k_sdf_invdiag<3><<<(int)g, 256, 0, S->stream>>>(S->d_keys, S->d_sdf, S->sdf_min, S->sdf_max - S->sdf_min, S->d_K64, S->R, S->C, S->L, S->d_invd);
  CKV(cudaGetLastError());
  return true;
}
// the scalar-density-field arguments of a thermal / elastic operator pass
template <int ND, typename T>
static void sdf_args(TeArgs<ND, T>& a) {
  a.sdf = S->d_sdf;
  a.sdf_min = S->sdf_min;
  a.sdf_rng = S->sdf_max - S->sdf_min;
  a.invd = S->d_invd;
}

template <typename T> static T* Kdev();
template <> double* Kdev<double>() { return S->d_K64; }
template <> float* Kdev<float>() { return S->d_K32; }

template <typename T>
static bool ensure_K() {
  if (Kdev<T>()) {  // the derived tables may have been dropped since (new density field, new model)
    if (th_applies() && !ensure_th<T>()) return false;
    if (asm_applies() && !ensure_tab<T>()) return false;
    if ((S->d_sdf || S->dim2) && !ensure_invd()) return false;
    return true;
  }
  if (!S->have_K) { set_err("solve", "local matrices were not set (cudapcgSetLclMtxs)"); return false; }
  std::vector<T> kt(S->Kd.size());
  for (size_t i = 0; i < kt.size(); i++) kt[i] = (T)S->Kd[i];
  T* dk = nullptr;
  CKV(dev_malloc(&dk, kt.size() * sizeof(T)));
  CKV(cudaMemcpy(dk, kt.data(), kt.size() * sizeof(T), cudaMemcpyHostToDevice));
  if (sizeof(T) == 8) S->d_K64 = (double*)dk; else S->d_K32 = (float*)dk;
  if (th_applies() && !ensure_th<T>()) return false;
  if (asm_applies() && !ensure_tab<T>()) return false;
  if ((S->d_sdf || S->dim2) && !ensure_invd()) return false;
  if (S->fluid) {
    if (sizeof(T) == 8) CKV(cudaMemcpyToSymbol(c_flK64, kt.data(), kt.size() * sizeof(double)));
    else CKV(cudaMemcpyToSymbol(c_flK32, kt.data(), kt.size() * sizeof(float)));
  }
  return true;
}

static bool ensure_K64_only() {
  if (S->d_K64) return true;
  if (!S->have_K) { set_err("solve", "local matrices were not set (cudapcgSetLclMtxs)"); return false; }
  CKV(dev_malloc(&S->d_K64, S->Kd.size() * sizeof(double)));
  CKV(cudaMemcpy(S->d_K64, S->Kd.data(), S->Kd.size() * sizeof(double), cudaMemcpyHostToDevice));
  return true;
}

static bool ensure_reduction(int nblocks) {
  if (nblocks <= S->part_cap && S->d_part) return true;
  free_ptr(S->d_part);
  S->part_cap = std::max(nblocks, 4096);
  CKV(dev_malloc(&S->d_part, sizeof(double) * 32 * S->part_cap));
  return true;
}

// ---------------------------------------------------------------------------------------
// Launch helpers.
// CTAs of a persistent stencil pass (see TeWork): as many as fit on the GPU at once for this
// kernel and shared-memory size, but no fewer than TE_MIN_RUN layers of work each.
static long te_work() {
  return (long)((S->R + TE_TR - 1) / TE_TR) * ((S->C + TE_TC - 1) / TE_TC) * S->L;
}
template <typename K>
static int te_ctas(K kernel, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, TE_NT, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  const long resident = (long)per_sm * num_sms();
  return (int)std::max(1L, std::min(resident, te_work() / TE_MIN_RUN));
}
static int pw_grid(long n) {
  long g = (n + PW_NT - 1) / PW_NT;
  const long cap = 8L * num_sms();
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}
// Largest grid any pass of the current model launches (reduction partials are sized once,
// before graph capture, which must not allocate).
static int needed_blocks() {
  long nb = pw_grid(S->fluid ? S->nV + S->nB : S->N);
  // stencil passes: at most 8 resident CTAs of TE_NT = 256 threads per SM
  if (!S->fluid) nb = std::max<long>(nb, 8L * num_sms());
  return (int)nb;
}
static RedCtl redctl(int nblocks) { return RedCtl{S->d_part, S->d_ticket, nblocks}; }
static SolveCfg solvecfg() {
  SolveCfg c;
  c.tol = S->tol; c.maxit = (int)std::min<unsigned>(S->maxit, 0x7fffffffu); c.norm = S->resnorm; c.precond = S->precond;
  c.nhmg = (S->fluid) ? (long)S->fdim * S->nV : S->nvars;
  return c;
}

// y = A v (+ fused direction form and dot finisher).  in1/vout only with fuse.
// CTAs of a 2D operator pass: the tiles, at most 8 per SM
static int d2_ctas() {
  const long tiles = (long)((S->R + T2_TR - 1) / T2_TR) * ((S->C + T2_TC - 1) / T2_TC);
  return (int)std::max(1L, std::min(tiles, 8L * num_sms()));
}

template <typename T>
static bool launch_apply(const T* in0, const T* in1, T* vout, T* y, bool fuse, int finish, bool skip_if_done) {
  if (S->fluid) {
    FlArgs<T> a;
    a.v = in0; a.vd = in1; a.vout = vout; a.y = y; a.x = nullptr; a.d = nullptr;
    a.dof_of_node = S->d_dof_of_node; a.node_of_dof = S->d_node_of_dof; a.bkeys = S->d_bkeys;
    a.R = S->R; a.C = S->C; a.L = S->L; a.nV = S->nV; a.nB = S->nB;
    a.sc = S->cur_sc; a.finish = finish; a.skip_if_done = skip_if_done;
    a.cfg = MrCfg{S->tol, 0, S->resnorm, S->precond, 0};
    const int g = pw_grid(S->nV + S->nB);
    if (!ensure_reduction(g)) return false;
    a.rc = redctl(g);
    if (S->fdim == 2) {
      if (fuse) k_fl_apply<T, TE_PCG, 2><<<g, FL_NT, 0, S->stream>>>(a);
      else k_fl_apply<T, TE_PLAIN, 2><<<g, FL_NT, 0, S->stream>>>(a);
    } else {
      if (fuse) k_fl_apply<T, TE_PCG><<<g, FL_NT, 0, S->stream>>>(a);
      else k_fl_apply<T, TE_PLAIN><<<g, FL_NT, 0, S->stream>>>(a);
    }
  } else if (S->dim2) {
    const int nb = d2_ctas();
    if (!ensure_reduction(nb)) return false;
    const MrCfg cfg{S->tol, 0, S->resnorm, S->precond, 0};
    if (S->nd == 1) {
      TeArgs<1, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, 1, S->cur_sc, redctl(nb), finish, skip_if_done, cfg};
      sdf_args(a);
      if (fuse) k_2d_apply<1, T, TE_PCG><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<1, T>(), S->stream>>>(a);
      else k_2d_apply<1, T, TE_PLAIN><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<1, T>(), S->stream>>>(a);
    } else {
      TeArgs<2, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, 1, S->cur_sc, redctl(nb), finish, skip_if_done, cfg};
      sdf_args(a);
      if (fuse) k_2d_apply<2, T, TE_PCG><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<2, T>(), S->stream>>>(a);
      else k_2d_apply<2, T, TE_PLAIN><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<2, T>(), S->stream>>>(a);
    }
  } else if (th_applies()) {
    const int nb = fuse ? th_ctas<T, TE_PCG>(S->R, S->C, S->L, num_sms()) : th_ctas<T, TE_PLAIN>(S->R, S->C, S->L, num_sms());
    if (nb < 1 || !ensure_reduction(nb)) return false;
    TeArgs<1, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, skip_if_done, MrCfg{S->tol, 0, S->resnorm, S->precond, 0}};
    const cudaError_t e = fuse ? th_launch<T, TE_PCG>(a, thdev<T>(), nb, S->stream) : th_launch<T, TE_PLAIN>(a, thdev<T>(), nb, S->stream);
    S->launches++;
    if (e != cudaSuccess) { set_err("operator pass", cudaGetErrorString(e)); return false; }
    return true;
  } else if (asm_applies()) {
    int nb;
    cudaError_t e;
    if (S->nd == 1) {
      nb = fuse ? asm_te_ctas<1, T, TE_PCG>(S->R, S->C, S->L, num_sms()) : asm_te_ctas<1, T, TE_PLAIN>(S->R, S->C, S->L, num_sms());
      if (nb < 1 || !ensure_reduction(nb)) return false;
      TeArgs<1, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, skip_if_done, MrCfg{S->tol, 0, S->resnorm, S->precond, 0}};
      e = fuse ? asm_te_launch<1, T, TE_PCG>(a, tabdev<T>(), nb, S->stream) : asm_te_launch<1, T, TE_PLAIN>(a, tabdev<T>(), nb, S->stream);
    } else {
      nb = fuse ? asm_te_ctas<3, T, TE_PCG>(S->R, S->C, S->L, num_sms()) : asm_te_ctas<3, T, TE_PLAIN>(S->R, S->C, S->L, num_sms());
      if (nb < 1 || !ensure_reduction(nb)) return false;
      TeArgs<3, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, skip_if_done, MrCfg{S->tol, 0, S->resnorm, S->precond, 0}};
      e = fuse ? asm_te_launch<3, T, TE_PCG>(a, tabdev<T>(), nb, S->stream) : asm_te_launch<3, T, TE_PLAIN>(a, tabdev<T>(), nb, S->stream);
    }
    S->launches++;
    if (e != cudaSuccess) { set_err("operator pass", cudaGetErrorString(e)); return false; }
    return true;
  } else {
    const dim3 block(TE_TR, TE_TC);
    if (S->nd == 1) {
      const size_t sm = te_smem_bytes<1, T>(S->nmat);
      const int nb = fuse ? te_ctas(k_te_apply<1, T, TE_PCG>, sm) : te_ctas(k_te_apply<1, T, TE_PLAIN>, sm);
      if (!ensure_reduction(nb)) return false;
      TeArgs<1, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, skip_if_done, MrCfg{S->tol, 0, S->resnorm, S->precond, 0}};
      sdf_args(a);
      if (fuse) k_te_apply<1, T, TE_PCG><<<nb, block, sm, S->stream>>>(a);
      else k_te_apply<1, T, TE_PLAIN><<<nb, block, sm, S->stream>>>(a);
    } else {
      const size_t sm = te_smem_bytes<3, T>(S->nmat);
      const int nb = fuse ? te_ctas(k_te_apply<3, T, TE_PCG>, sm) : te_ctas(k_te_apply<3, T, TE_PLAIN>, sm);
      if (!ensure_reduction(nb)) return false;
      TeArgs<3, T> a{in0, in1, vout, y, nullptr, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, skip_if_done, MrCfg{S->tol, 0, S->resnorm, S->precond, 0}};
      sdf_args(a);
      if (fuse) k_te_apply<3, T, TE_PCG><<<nb, block, sm, S->stream>>>(a);
      else k_te_apply<3, T, TE_PLAIN><<<nb, block, sm, S->stream>>>(a);
    }
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

// Pointwise PCG pass.
template <typename T, int MODE>
static bool launch_point(double* x, T* d, T* r, const T* q, T* s, const T* dold) {
  const SolveCfg cfg = solvecfg();
  if (S->fluid) {
    const int g = pw_grid(S->nV + S->nB);
    if (!ensure_reduction(g)) return false;
    FlPw<T> a{x, d, r, q, s, dold, S->d_bkeys, S->nV, S->nB, S->cur_sc, redctl(g), cfg};
    if (S->fdim == 2) k_fl_point<T, MODE, 2><<<g, PW_NT, 0, S->stream>>>(a);
    else k_fl_point<T, MODE><<<g, PW_NT, 0, S->stream>>>(a);
  } else {
    const int g = pw_grid(S->N);
    if (!ensure_reduction(g)) return false;
    if (S->dim2 && S->nd == 2) {  // 2D elastic: the Jacobi diagonal from invd only
      TePw<2, T> a{x, d, r, q, s, dold, S->d_keys, Kdev<T>(), 0, S->N, S->cur_sc, redctl(g), cfg, S->d_invd};
      k_te_point<2, T, MODE><<<g, PW_NT, 0, S->stream>>>(a);
    } else if (S->nd == 1) {
      TePw<1, T> a{x, d, r, q, s, dold, S->d_keys, Kdev<T>(), S->dim2 ? 0 : S->nmat, S->N, S->cur_sc, redctl(g), cfg, S->d_invd};
      k_te_point<1, T, MODE><<<g, PW_NT, 0, S->stream>>>(a);
    } else {
      TePw<3, T> a{x, d, r, q, s, dold, S->d_keys, Kdev<T>(), S->nmat, S->N, S->cur_sc, redctl(g), cfg, S->d_invd};
      k_te_point<3, T, MODE><<<g, PW_NT, 0, S->stream>>>(a);
    }
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

template <typename T>
static bool enqueue_minres_iteration(int parity);
template <typename T>
static bool launch_mr_op(const T* rin, T* rout, int fin, bool skip_if_done);

// ---------------------------------------------------------------------------------------
// One PCG / CG iteration: pass 1 forms d_new = s + beta d_old on the fly, applies A and
// finishes alpha = delta / (d_new . A d_new); pass 2 updates x, r, s and finishes delta,
// beta and the stopping test.  Buffers: d_old/d_new alternate, so a chunk has an even
// number of iterations.
// Thermal / elastic PCG forms s = M^-1 r inside the operator pass from r and the node keys and
// stores no s; the Stokes operator (a gather through the DOF map) reads a stored s.
static bool keeps_s() { return S->fluid; }
template <typename T> static T* s_or_null() { return keeps_s() ? (T*)S->s : nullptr; }
template <typename T> static const T* pcg_dir_in() { return keeps_s() ? (const T*)S->s : (const T*)S->r; }

// A thermal / elastic operator pass of the given mode (TE_DIRDOT, TE_UPD: the 3-vector PCG)
// on the model, with the assembled blocks where they apply.
template <typename T, int MODE>
static bool launch_te_mode(const T* in0, const T* in1, T* vout, double* x, int finish) {
  const SolveCfg sc = solvecfg();
  const MrCfg cfg{sc.tol, sc.maxit, sc.norm, sc.precond, sc.nhmg};
  cudaError_t e = cudaSuccess;
  if (S->dim2) {
    const int nb = d2_ctas();
    if (!ensure_reduction(nb)) return false;
    if (S->nd == 1) {
      TeArgs<1, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, 1, S->cur_sc, redctl(nb), finish, 1, cfg};
      sdf_args(a);
      k_2d_apply<1, T, MODE><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<1, T>(), S->stream>>>(a);
    } else {
      TeArgs<2, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, 1, S->cur_sc, redctl(nb), finish, 1, cfg};
      sdf_args(a);
      k_2d_apply<2, T, MODE><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<2, T>(), S->stream>>>(a);
    }
    e = cudaGetLastError();
  } else if (th_applies()) {
    const int nb = th_ctas<T, MODE>(S->R, S->C, S->L, num_sms());
    if (nb < 1 || !ensure_reduction(nb)) return false;
    TeArgs<1, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, 1, cfg};
    e = th_launch<T, MODE>(a, thdev<T>(), nb, S->stream);
  } else if (asm_applies()) {
    if (S->nd == 1) {
      const int nb = asm_te_ctas<1, T, MODE>(S->R, S->C, S->L, num_sms());
      if (nb < 1 || !ensure_reduction(nb)) return false;
      TeArgs<1, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, 1, cfg};
      e = asm_te_launch<1, T, MODE>(a, tabdev<T>(), nb, S->stream);
    } else {
      const int nb = asm_te_ctas<3, T, MODE>(S->R, S->C, S->L, num_sms());
      if (nb < 1 || !ensure_reduction(nb)) return false;
      TeArgs<3, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, 1, cfg};
      e = asm_te_launch<3, T, MODE>(a, tabdev<T>(), nb, S->stream);
    }
  } else {
    const dim3 block(TE_TR, TE_TC);
    if (S->nd == 1) {
      const size_t sm = te_smem_bytes<1, T>(S->nmat);
      const int nb = te_ctas(k_te_apply<1, T, MODE>, sm);
      if (!ensure_reduction(nb)) return false;
      TeArgs<1, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, 1, cfg};
      sdf_args(a);
      k_te_apply<1, T, MODE><<<nb, block, sm, S->stream>>>(a);
    } else {
      const size_t sm = te_smem_bytes<3, T>(S->nmat);
      const int nb = te_ctas(k_te_apply<3, T, MODE>, sm);
      if (!ensure_reduction(nb)) return false;
      TeArgs<3, T> a{in0, in1, vout, nullptr, x, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), finish, 1, cfg};
      sdf_args(a);
      k_te_apply<3, T, MODE><<<nb, block, sm, S->stream>>>(a);
    }
    e = cudaGetLastError();
  }
  S->launches++;
  if (e != cudaSuccess) { set_err("operator pass", cudaGetErrorString(e)); return false; }
  return true;
}

// One 3-vector PCG iteration (CG3 on thermal / elastic models; pcg3.cu:163-208 applies the
// operator twice per iteration on x, r, d): pass 1 forms d_new = M^-1 r + beta d_old and
// finishes alpha = delta / (d_new . A d_new); pass 2 applies A to d_new again and updates
// r -= alpha A d_new, x += alpha d_new, then finishes delta, beta and the stopping test.
template <typename T>
static bool enqueue_pcg3_iteration(int parity) {
  T* dold = (T*)(parity ? S->d1 : S->d0);
  T* dnew = (T*)(parity ? S->d0 : S->d1);
  return launch_te_mode<T, TE_DIRDOT>((const T*)S->r, dold, dnew, nullptr, FIN_ALPHA) &&
         launch_te_mode<T, TE_UPD>(dnew, nullptr, (T*)S->r, S->x, FIN_STORE);
}

template <typename T>
static bool enqueue_pcg_iteration(int parity) {
  T* dold = (T*)(parity ? S->d1 : S->d0);
  T* dnew = (T*)(parity ? S->d0 : S->d1);
  if (!launch_apply<T>(pcg_dir_in<T>(), dold, dnew, (T*)S->q, true, FIN_ALPHA, true)) return false;
  return launch_point<T, PW_PCG>(S->x, dnew, (T*)S->r, (const T*)S->q, s_or_null<T>(), nullptr);
}

// r = b - A x with the operator applied in FP64 to the FP64 solution (initial guesses and
// the mixed-mode residual replacement), rounded once into the working precision.
template <typename T>
__global__ void k_residual_replace(const double* b, const double* Ax, T* r, long n);
template <typename T>
static bool residual_from_x(bool skip_if_done = true, double* x = nullptr, const double* b = nullptr, T* r = nullptr) {
  if (!x) { x = S->x; b = S->b64; r = (T*)S->r; }
  if (!b) b = (const double*)r;  // FP64 without a copy of b: r still holds it (set-up only)
  if (!ensure_K<double>() || !ensure_scratch64(S->y64)) return false;
  if (!launch_apply<double>(x, nullptr, nullptr, S->y64, false, FIN_NONE, skip_if_done)) return false;
  const long n = S->nvars;
  k_residual_replace<T><<<pw_grid(n), PW_NT, 0, S->stream>>>(b, S->y64, r, n);
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}
// Mixed mode: true residual r = b - A x with FP64 accumulation of the subtraction.
template <typename T>
__global__ void k_residual_replace(const double* b, const double* Ax, T* r, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    r[i] = (T)(b[i] - Ax[i]);
}
template <typename T>
__global__ void k_skip_if_done_copy(const DevScalars* sc, int* flag) { if (threadIdx.x == 0 && blockIdx.x == 0) *flag = sc->done; }

template <typename T>
static bool build_graph(int key, int chunk, bool minres) {
  if (S->gexec && S->graph_key == key) return true;
  if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; }
  cudaGraph_t g;
  CKV(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  bool ok = true;
  const unsigned long long l0 = S->launches;
  for (int it = 0; it < chunk && ok; it++) {
    if (minres) ok = enqueue_minres_iteration<T>(it & 1);
    else if (pcg3_solver()) ok = enqueue_pcg3_iteration<T>(it & 1);
    else ok = enqueue_pcg_iteration<T>(it & 1);
  }
  S->launches = l0;
  cudaError_t e = cudaStreamEndCapture(S->stream, &g);
  if (!ok || e != cudaSuccess) { set_err("graph capture", cudaGetErrorString(e)); return false; }
  e = cudaGraphInstantiate(&S->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { set_err("graph instantiate", cudaGetErrorString(e)); return false; }
  S->graph_key = key;
  return true;
}

static bool read_scalars() {
  CKV(cudaMemcpyAsync(S->h_sc, S->d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, S->stream));
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}

// Device loop driver shared by PCG and MINRES: launch graph chunks until the device flags
// completion.  Between chunks the host reads 1 record of scalars.
template <typename T>
static bool run_chunks(bool minres) {
  const int chunk = std::max(2u, S->iters_per_launch & ~1u);
  const int key = (prec_of<T>() << 8) | (minres ? 0x80 : 0) | (chunk & 0x7f) | (S->resnorm << 16) | (S->precond << 20) |
                  (pcg3_solver() ? 1 << 24 : 0);
  if (!build_graph<T>(key, chunk, minres)) return false;
  const bool mixed = sizeof(T) == 4 && S->replace_every > 0;
  unsigned next_replace = S->replace_every;
  // progress measure for the replacement trigger: delta = r.M^-1 r (CG), squared relative
  // residual metric ((P)MINRES); its value at the last replacement
  auto progress = [&]() { return minres ? S->h_sc->metric * S->h_sc->metric : fabs(S->h_sc->delta); };
  double repl_ref = -1.0;
  int checks = 0;
  const bool trace = getenv("CHFEM_B200_TRACE") != nullptr;
  // the (P)MINRES error-norm stop is a step-size test, with no residual to confirm
  const bool can_check = !minres || S->resnorm != CUDAPCG_ERROR_NORM;
  for (;;) {
    if (!read_scalars()) return false;
    if (trace)
      fprintf(stderr, "[single] it %d delta %.6e delta0 %.6e alpha %.6e beta %.6e metric %.6e done %d found %d status %d\n", S->h_sc->iteration,
              S->h_sc->delta, S->h_sc->delta0, S->h_sc->alpha, S->h_sc->beta, S->h_sc->metric, S->h_sc->done, S->h_sc->found, S->h_sc->status);
    if (S->h_sc->status >= 3) break;
    if (S->h_sc->done) {
      // Mixed precision: an apparent convergence is confirmed on the true residual b - A x
      // (FP64 operator, FP64 x); if it does not hold, the iteration restarts from it.
      if (mixed && can_check && S->h_sc->status == 0 && S->h_sc->found && checks < 32) {
        checks++;
        if (!residual_from_x<T>(false)) return false;
        if (minres) { if (!launch_mr_op<T>((const T*)S->r, (T*)S->r2, FIN_MR_CHECK, false)) return false; }
        else if (!launch_point<T, PW_CHECK>(S->x, nullptr, (T*)S->r, nullptr, s_or_null<T>(), nullptr)) return false;
        if (!read_scalars()) return false;
        if (trace) fprintf(stderr, "[single] true-residual check %d: done %d metric %.6e\n", checks, S->h_sc->done, S->h_sc->metric);
        if (S->h_sc->done) break;
        next_replace = (unsigned)S->h_sc->iteration + S->replace_every;
        repl_ref = progress();
      } else {
        break;
      }
    }
    if (repl_ref < 0) repl_ref = minres ? 1.0 : fabs(S->h_sc->delta0);
    if (mixed && ((unsigned)S->h_sc->iteration >= next_replace || progress() < S->replace_drop * repl_ref)) {
      // residual replacement: r = b - A x, then the preconditioned residual and its scalars
      // (keeps the direction unless the recursive residual had drifted, then restarts)
      if (!residual_from_x<T>()) return false;
      if (minres) {
        // (P)MINRES carries q = A d as a recursion (q = s + beta q) that drifts in FP32 like r:
        // both are refreshed, q by an apply of the current direction
        if (!launch_mr_op<T>((const T*)S->r, (T*)S->r2, FIN_MR_REPL, true)) return false;
        if (!launch_apply<T>((const T*)S->d0, nullptr, nullptr, (T*)S->q, false, FIN_NONE, true)) return false;
      } else if (!launch_point<T, PW_REPL>(S->x, nullptr, (T*)S->r, nullptr, s_or_null<T>(), nullptr)) return false;
      next_replace = (unsigned)S->h_sc->iteration + S->replace_every;
      repl_ref = progress();
      if (trace) fprintf(stderr, "[single] residual replacement at %d\n", S->h_sc->iteration);
    }
    CKV(cudaGraphLaunch(S->gexec, S->stream));
    S->launches += (unsigned long long)chunk * 2;
  }
  return true;
}

// ---------------------------------------------------------------------------------------
// Solve on the device; x0 (if set) is in S->x, the RHS in S->r (and S->b64).
template <typename T>
static bool solve_pcg_device() {
  if (!ensure_reduction(needed_blocks())) return false;
  CKV(cudaMemsetAsync(S->d_ticket, 0, sizeof(unsigned), S->stream));
  CKV(cudaMemsetAsync(S->d_sc, 0, sizeof(DevScalars), S->stream));
  const size_t n = (size_t)S->nvars;
  if (!S->x0_set) CKV(cudaMemsetAsync(S->x, 0, n * 8, S->stream));
  if (S->q) CKV(cudaMemsetAsync(S->q, 0, n * sizeof(T), S->stream));
  CKV(cudaMemsetAsync(S->d0, 0, n * sizeof(T), S->stream));
  CKV(cudaMemsetAsync(S->d1, 0, n * sizeof(T), S->stream));
  CKV(cudaEventRecord(S->ev0, S->stream));
  // zero-guess reference: s = M^-1 r, delta0 = r.s   (pcg.cu:61-81)
  if (!launch_point<T, PW_INIT>(S->x, nullptr, (T*)S->r, nullptr, s_or_null<T>(), nullptr)) return false;
  if (S->x0_set) {  // pcg.cu:83-99: r = b - A x0 (FP64 apply), then the initial-guess test
    if (!residual_from_x<T>()) return false;
    if (!launch_point<T, PW_X0R>(S->x, nullptr, (T*)S->r, nullptr, s_or_null<T>(), nullptr)) return false;
  }
  CKV(cudaEventRecord(S->ev1, S->stream));
  if (!run_chunks<T>(false)) return false;
  CKV(cudaEventRecord(S->ev2, S->stream));
  CKV(cudaEventSynchronize(S->ev2));
  float ms1 = 0, ms2 = 0;
  cudaEventElapsedTime(&ms1, S->ev0, S->ev1);
  cudaEventElapsedTime(&ms2, S->ev1, S->ev2);
  S->setup_dev_s = ms1 * 1e-3;
  S->solve_dev_s = ms2 * 1e-3;
  return true;
}

#include "minres_driver.inl"
static bool interp_into(const double* coarse_host, double* target);
#include "block_driver.inl"

// ---------------------------------------------------------------------------------------
// Results: residual / found semantics of pcg.cu:226-233 and pminres.cu:225-227.
static void collect_results(bool minres) {
  const DevScalars& h = *S->h_sc;
  S->iteration = (unsigned)h.iteration;
  if (h.status == 1) { S->residual = 0.0; S->found = 1; return; }
  if (h.status == 2) { S->residual = h.metric; S->found = 1; return; }
  if (!minres && S->resnorm == CUDAPCG_L2_NORM) {
    S->residual = sqrt(fabs(h.delta) / fabs(h.delta0));
    S->found = !(fabs(h.delta) > S->tol * S->tol * fabs(h.delta0));
  } else {
    S->residual = h.metric;
    S->found = S->residual <= S->tol;
  }
}

template <typename T>
static bool copy_x_to_host(double* res_x) {
  const size_t n = (size_t)S->nvars;
  CKV(cudaMemcpyAsync(res_x, S->x, n * 8, cudaMemcpyDeviceToHost, S->stream));
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}

#include "two_vector_driver.inl"

template <typename T>
static bool solve_T(double* res_x) {
  if (!ensure_vectors<T>() || !ensure_K<T>()) return false;
  const bool minres = (S->solver_flag == CUDAPCG_MINRES_SOLVER || S->solver_flag == CUDAPCG_MINRES3_SOLVER);
  bool ok = minres ? solve_minres_device<T>() : solve_pcg_device<T>();
  if (!ok) return false;
  collect_results(minres);
  if (S->h_sc->status == 1 && minres) CKV(cudaMemsetAsync(S->x, 0, S->nvars * 8, S->stream));
  return res_x ? copy_x_to_host<T>(res_x) : true;  // NULL: the solution stays on the device
}

// =======================================================================================
// C ABI
extern "C" {

const char* cudapcgB200LastError(void) { return g_err.c_str(); }

// The stream, its three events and the pinned scalar record outlive a solver: cudapcgEnd keeps
// them for the next cudapcgInit on the same device (destroying and re-creating them cost up to
// 0.7 s per model on some B200 boxes).  A solver on another device gets new ones.
struct KeptHandles {
  int dev = -1;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  DevScalars* h_sc = nullptr;
};
static KeptHandles g_kept;
static void keep_handles() {
  int dev = -1;
  if (S->stream) cudaStreamSynchronize(S->stream);
  if (cudaGetDevice(&dev) == cudaSuccess && S->stream && S->ev0 && S->ev1 && S->ev2 && S->h_sc && !g_kept.stream) {
    g_kept.dev = dev; g_kept.stream = S->stream; g_kept.ev[0] = S->ev0; g_kept.ev[1] = S->ev1; g_kept.ev[2] = S->ev2;
    g_kept.h_sc = S->h_sc;
    return;
  }
  if (S->h_sc) cudaFreeHost(S->h_sc);
  if (S->ev0) cudaEventDestroy(S->ev0);
  if (S->ev1) cudaEventDestroy(S->ev1);
  if (S->ev2) cudaEventDestroy(S->ev2);
  if (S->stream) cudaStreamDestroy(S->stream);
}
static bool take_kept_handles() {
  int dev = -1;
  if (!g_kept.stream || cudaGetDevice(&dev) != cudaSuccess || dev != g_kept.dev) return false;
  S->stream = g_kept.stream; S->ev0 = g_kept.ev[0]; S->ev1 = g_kept.ev[1]; S->ev2 = g_kept.ev[2]; S->h_sc = g_kept.h_sc;
  g_kept = KeptHandles();
  return true;
}

cudapcgFlag_t cudapcgEnd(void) {
  if (!S) return CUDAPCG_FALSE;
  const bool trace = getenv("CHFEM_B200_TRACE") != nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  auto since = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
  block_free();
  const double t_block = since();
  free_vectors();
  free_model_dev();
  free_ptr(S->d_sc); free_ptr(S->d_part); free_ptr(S->d_ticket); free_ptr(S->d_vt);
  const double t_dev = since();
  keep_handles();
  if (trace) fprintf(stderr, "[end] block buffers %.4f s, other device buffers %.4f s, stream and events %.4f s\n", t_block, t_dev - t_block, since() - t_dev);
  if (S->model && S->model->freeAllowed_flag) { free(S->model->name); free(S->model); }
  delete S;
  S = nullptr;
  return CUDAPCG_TRUE;  // no device reset: other contexts on a shared GPU are left alone
}

cudapcgFlag_t cudapcgInit(cudapcgFlag_t analysis_flag, cudapcgFlag_t parStrategy_flag) {
  cudapcgEnd();
  g_err.clear();
  if (analysis_flag > CUDAPCG_FLUID_3D) { set_err("cudapcgInit", "invalid analysis flag"); return CUDAPCG_FALSE; }
  if ((analysis_flag == CUDAPCG_FLUID_3D || analysis_flag == CUDAPCG_FLUID_2D) && parStrategy_flag != CUDAPCG_NBN) {
    printf("ERROR: EBE solver is unavailable for FLUID analysis.\n");
    set_err("cudapcgInit", "EBE is unavailable for FLUID analysis");
    return CUDAPCG_FALSE;
  }
  S = new Solver();
  S->analysis = analysis_flag;
  S->par = parStrategy_flag;
  S->dim2 = analysis_flag == CUDAPCG_THERMAL_2D || analysis_flag == CUDAPCG_ELASTIC_2D;
  S->fluid = analysis_flag == CUDAPCG_FLUID_3D || analysis_flag == CUDAPCG_FLUID_2D;
  S->fdim = analysis_flag == CUDAPCG_FLUID_2D ? 2 : 3;
  S->nd = (analysis_flag == CUDAPCG_ELASTIC_3D) ? 3 : (analysis_flag == CUDAPCG_ELASTIC_2D ? 2 : 1);
  if (const char* e = getenv("CHFEM_B200_PRECISION")) cudapcgB200SetPrecision((!strcmp(e, "mixed") || !strcmp(e, "fp32")) ? CHFEM_B200_MIXED : CHFEM_B200_FP64);
  if (!g_ctor) g_ctor = ctor_simple;
  if (!take_kept_handles()) {
    CK(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&S->ev0)); CK(cudaEventCreate(&S->ev1)); CK(cudaEventCreate(&S->ev2));
    CK(cudaMallocHost(&S->h_sc, sizeof(DevScalars)));
  }
  CK(dev_malloc(&S->d_sc, sizeof(DevScalars)));
  S->cur_sc = S->d_sc;
  CK(dev_malloc(&S->d_ticket, sizeof(unsigned)));
  CK(cudaMemset(S->d_ticket, 0, sizeof(unsigned)));
  memset(S->h_sc, 0, sizeof(DevScalars));
  return CUDAPCG_TRUE;
}

cudapcgModel_t* cudapcgNewModel(void) {
  cudapcgModel_t* m = (cudapcgModel_t*)calloc(1, sizeof(cudapcgModel_t));
  if (!m) return nullptr;
  m->freeAllowed_flag = CUDAPCG_TRUE;
  m->parStrategy_flag = CUDAPCG_NBN;
  m->poremap_flag = CUDAPCG_POREMAP_NUM;
  return m;
}

static cudapcgFlag_t adopt_model() {
  cudapcgModel_t* m = S->model;
  if (S->fluid && m->poremap_flag != CUDAPCG_POREMAP_NUM && m->poremap_flag != CUDAPCG_POREMAP_IMG) {
    set_err("model", "unknown pore map flag");
    return CUDAPCG_FALSE;
  }
  free_vectors();
  free_model_dev();
  S->poremap_img = S->fluid && m->poremap_flag == CUDAPCG_POREMAP_IMG;
  block_free();
  S->R = (int)m->nrows; S->C = (int)m->ncols; S->L = std::max(1, (int)m->nlayers);  // 2D: one layer
  S->N = (long)S->R * S->C * S->L;
  S->nvars = m->nvars; S->nV = m->nporenodes; S->nB = m->nbordernodes;
  S->nmat = (int)m->nkeys;
  if (S->N <= 0 || S->nvars <= 0) { set_err("model", "empty model"); return CUDAPCG_FALSE; }
  if (!S->fluid && (S->nmat < 1 || S->nmat > (S->dim2 ? T2_NMAT : 4))) {
    set_err("model", S->dim2 ? "1 to 16 materials are supported with 16-bit 2D keys" : "1 to 4 materials are supported with 16-bit keys");
    return CUDAPCG_FALSE;
  }
  if (S->fluid) {
    CK(dev_malloc(&S->d_dof_of_node, sizeof(uint32_t) * S->N));
    CK(dev_malloc(&S->d_node_of_dof, sizeof(uint32_t) * std::max<long>(1, S->nV + S->nB)));
    CK(dev_malloc(&S->d_bkeys, std::max<long>(1, S->nB)));
  } else {
    CK(dev_malloc(&S->d_keys, sizeof(uint16_t) * S->N));
  }
  S->x0_set = false;
  return CUDAPCG_TRUE;
}

cudapcgFlag_t cudapcgSetModel(cudapcgModel_t* model) {
  if (!S || !model) return CUDAPCG_FALSE;
  if (S->model && S->model != model && S->model->freeAllowed_flag) { free(S->model->name); free(S->model); }
  S->model = model;
  return adopt_model();
}

cudapcgFlag_t cudapcgSetModelConstructorFcn(cudapcgFlag_t (*fcn)(cudapcgModel_t**, const void*)) {
  if (!fcn) return CUDAPCG_FALSE;
  g_ctor = fcn;
  return CUDAPCG_TRUE;
}

cudapcgFlag_t cudapcgBuildModel(const void* data) {
  if (!S) return CUDAPCG_FALSE;
  if (!S->model) S->model = cudapcgNewModel();
  else if (S->model->freeAllowed_flag) { free(S->model->name); free(S->model); S->model = cudapcgNewModel(); }
  if (!g_ctor(&S->model, data)) return CUDAPCG_FALSE;
  // Device pointers of this library are kept in the Solver, not in the caller's struct.
  return adopt_model();
}

cudapcgFlag_t cudapcgSetNumTol(cudapcgTol_t t) { if (!S) return CUDAPCG_FALSE; S->tol = t; return CUDAPCG_TRUE; }
cudapcgFlag_t cudapcgSetMaxIterations(unsigned int n) { if (!S) return CUDAPCG_FALSE; S->maxit = n; return CUDAPCG_TRUE; }
cudapcgFlag_t cudapcgSetXReduceMode(cudapcgFlag_t flag) {
  if (!S) return CUDAPCG_FALSE;
  S->xr_mode = flag <= CUDAPCG_XREDUCE_FULL ? flag : CUDAPCG_XREDUCE_FULL;
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgSetXReduceShift(unsigned int shift) { if (!S) return CUDAPCG_FALSE; S->xr_shift = shift; return CUDAPCG_TRUE; }
cudapcgFlag_t cudapcgSetXReduceScale(double scl) { if (!S) return CUDAPCG_FALSE; S->xr_scale = scl; return CUDAPCG_TRUE; }
// The reference rescales the terms of its NONE-mode sums by max|d| x this factor before adding
// them (xreduce.cu:8-13) to protect FP32 accumulation; the sums here are FP64 in a fixed order,
// so the factor is accepted and has no effect on the result.
cudapcgFlag_t cudapcgSetReduceStabFactor(double) { return S ? CUDAPCG_TRUE : CUDAPCG_FALSE; }
cudapcgFlag_t cudapcgSetSolver(cudapcgFlag_t flag) {
  if (!S) return CUDAPCG_FALSE;
  if (flag > CUDAPCG_MINRES2_SOLVER) { printf("ERROR: Invalid \"solverFlag\" (%d).\n", flag); return CUDAPCG_FALSE; }
  // the 2-vector solvers keep another set of device vectors: a switch drops the old set
  if ((flag >= CUDAPCG_CG2_SOLVER) != (S->solver_flag >= CUDAPCG_CG2_SOLVER) && S->r) {
    free_vectors();
    S->rhs_set = false;
    S->x0_set = false;
  }
  // CG3 on thermal / elastic models: the 3-vector PCG (same iterates as CG, two operator passes
  // per iteration, no q); MINRES3 runs the iterates of MINRES
  S->solver_flag = flag;
  if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; S->graph_key = -1; }
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgSetPreconditioner(cudapcgFlag_t flag) { if (!S) return CUDAPCG_FALSE; S->precond = flag > 0; return CUDAPCG_TRUE; }
cudapcgFlag_t cudapcgSetResNorm(cudapcgFlag_t flag) { if (!S) return CUDAPCG_FALSE; S->resnorm = flag > CUDAPCG_ERROR_NORM ? CUDAPCG_L2_NORM : flag; return CUDAPCG_TRUE; }
unsigned int cudapcgGetNumIterations(void) { return S ? S->iteration : 0; }
unsigned int cudapcgGetMaxNumIterations(void) { return S ? S->maxit : 0; }
cudapcgVar_t cudapcgGetResidual(void) { return S ? S->residual : 0; }

cudapcgFlag_t cudapcgAllocateArrays(void) {
  if (!S || !S->model) return CUDAPCG_FALSE;
  bool ok = lean_solver() ? ensure_lean_vectors() : (S->precision == CHFEM_B200_FP64) ? ensure_vectors<double>() : ensure_vectors<float>();
  if (ok) S->user_arrays = true;
  return ok ? CUDAPCG_TRUE : CUDAPCG_FALSE;
}
cudapcgFlag_t cudapcgFreeArrays(void) {
  if (!S) return CUDAPCG_FALSE;
  if (!S->x0_set) { free_vectors(); }
  S->user_arrays = false;
  return CUDAPCG_TRUE;
}

static bool upload_vec(const double* host, void* dst_T) {
  const size_t n = (size_t)S->nvars;
  if (S->vec_prec == CHFEM_B200_FP64) {
    CKV(cudaMemcpyAsync(dst_T, host, n * 8, cudaMemcpyHostToDevice, S->stream));
  } else {
    // staged in FP64 scratch: the residual-replacement scratch of mixed mode when it exists
    double*& stage = S->y64 ? S->y64 : S->x64;
    if (!ensure_scratch64(stage)) return false;
    CKV(cudaMemcpyAsync(stage, host, n * 8, cudaMemcpyHostToDevice, S->stream));
    k_convert<double, float><<<pw_grid(n), PW_NT, 0, S->stream>>>(stage, (float*)dst_T, n);
  }
  return true;
}

static bool ensure_vectors_current() {
  if (lean_solver()) return ensure_lean_vectors();
  return (S->precision == CHFEM_B200_FP64) ? ensure_vectors<double>() : ensure_vectors<float>();
}

cudapcgFlag_t cudapcgSetRHS(cudapcgVar_t* RHS) {
  if (!S || !S->model || !RHS) return CUDAPCG_FALSE;
  if (!ensure_vectors_current()) return CUDAPCG_FALSE;
  if (lean_solver()) {  // the 2-vector solvers consume r in place; no other copy is kept
    CK(cudaMemcpy(S->r, RHS, S->nvars * 8, cudaMemcpyHostToDevice));
    S->rhs_set = true;
    return CUDAPCG_TRUE;
  }
  if (!upload_vec(RHS, S->r)) return CUDAPCG_FALSE;
  if (S->b64) CK(cudaMemcpyAsync(S->b64, RHS, S->nvars * 8, cudaMemcpyHostToDevice, S->stream));
  CK(cudaStreamSynchronize(S->stream));
  S->rhs_set = true;
  return CUDAPCG_TRUE;
}

// Coarse-to-fine prolongation for recursive initial guesses (kernels/image.cu:20-123,
// wrappers.cu:290-303): x2 injection at even nodes, then periodic midpoint fill along rows,
// columns and layers, in that order.
}  // extern "C"
template <typename T>
__global__ void k_project2(T* res, const double* v, int rows, int cols, int lays, int nd) {
  const int rc = rows / 2, cc = cols / 2, lc = lays / 2;
  const long nco = (long)rc * cc * (lc + (lc < 1));
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nco; i += (long)gridDim.x * blockDim.x) {
    const long ii = i % rc, jj = (i % ((long)cc * rc)) / rc, kk = i / ((long)cc * rc);
    const long idx = 2 * ii + 2 * jj * rows + 2 * kk * (long)rows * cols;
    for (int j = 0; j < nd; j++) res[nd * idx + j] = (T)(2.0 * v[nd * i + j]);
  }
}
extern "C" {
}  // extern "C"
template <typename T>
__global__ void k_interp_pass(T* v, int rows, int cols, int lays, int nd, int pass) {
  const long RC = (long)rows * cols, n = RC * lays;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const long ii = i % rows, jj = (i % RC) / rows, kk = i / RC;
    long a, b;
    if (pass == 0) {
      if (!((ii & 1) && !(jj & 1) && !(kk & 1))) continue;
      a = i - 1 + rows * (!(i % rows)); b = i + 1 - rows * (!((i + 1) % rows));
    } else if (pass == 1) {
      if (!((jj & 1) && !(kk & 1))) continue;
      const long il = i % RC;
      a = (il + (RC - rows)) % RC + kk * RC; b = (il + rows) % RC + kk * RC;
    } else {
      if (!(kk & 1)) continue;
      a = (i + (n - RC)) % n; b = (i + RC) % n;
    }
    for (int j = 0; j < nd; j++) v[nd * i + j] = (T)(0.5 * (double)v[nd * a + j] + 0.5 * (double)v[nd * b + j]);
  }
}
extern "C" {

}  // extern "C"
// Prolongs a coarse solution (host, nd x (cols/2)(rows/2)(lays/2) values) into the device
// vector `target` of the current model; S->x64 stages the coarse values.
static bool interp_into(const double* coarse_host, double* target) {
  const int rows = S->R, cols = S->C, lays = S->L, nd = (int)(S->nvars / S->N);
  const size_t ncoarse = (size_t)nd * (cols / 2) * (rows / 2) * (lays / 2 + (lays < 2));
  if (!ensure_scratch64(S->x64)) return false;
  CKV(cudaMemcpyAsync(S->x64, coarse_host, ncoarse * 8, cudaMemcpyHostToDevice, S->stream));
  CKV(cudaMemsetAsync(target, 0, S->nvars * 8, S->stream));
  const int g = pw_grid(S->N);
  k_project2<double><<<g, PW_NT, 0, S->stream>>>(target, S->x64, rows, cols, lays, nd);
  for (int p = 0; p < 3; p++) k_interp_pass<double><<<g, PW_NT, 0, S->stream>>>(target, rows, cols, lays, nd, p);
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}
template <typename T>
static bool interp_x0(const double* coarse_host) { return interp_into(coarse_host, S->x); }
extern "C" {

cudapcgFlag_t cudapcgB200SetX0Device(const double* x0) {
  if (!S || !S->model || !x0) return CUDAPCG_FALSE;
  if (!ensure_vectors_current()) return CUDAPCG_FALSE;
  CK(cudaMemcpy(lean_solver() ? (double*)S->d0 : S->x, x0, S->nvars * 8, cudaMemcpyDeviceToDevice));
  S->x0_set = true;
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgSetX0(cudapcgVar_t* x0, cudapcgFlag_t mustInterpolate) {
  if (!S || !S->model) return CUDAPCG_FALSE;
  if (!x0) {  // cudapcg.cu:298-309
    if (!S->x0_set) return CUDAPCG_TRUE;
    S->x0_set = false;
    if (S->x) CK(cudaMemset(S->x, 0, S->nvars * 8));
    return CUDAPCG_TRUE;
  }
  if (!ensure_vectors_current()) return CUDAPCG_FALSE;
  if (lean_solver()) {  // the 2-vector solvers hold x0 in d (cudapcg.cu:302)
    if (mustInterpolate) { set_err("cudapcgSetX0", "coarse-grid guesses are not provided for Stokes"); return CUDAPCG_FALSE; }
    CK(cudaMemcpy(S->d0, x0, S->nvars * 8, cudaMemcpyHostToDevice));
    S->x0_set = true;
    return CUDAPCG_TRUE;
  }
  bool ok;
  if (mustInterpolate) ok = (S->vec_prec == CHFEM_B200_FP64) ? interp_x0<double>(x0) : interp_x0<float>(x0);
  else { ok = cudaMemcpy(S->x, x0, S->nvars * 8, cudaMemcpyHostToDevice) == cudaSuccess; }
  if (!ok) return CUDAPCG_FALSE;
  S->x0_set = true;
  return CUDAPCG_TRUE;
}

// Node keys from a per-voxel material map (EBE input): voxel v is the element whose local
// node 3 is node v (femhmg_3D.c:45-49), so the element in which node (r,c,l) is local node e
// is voxel (r - drow(e) - 1, c - dcol(e), l - dlay(e)).
}  // extern "C"
__global__ void k_keys_from_elements(const uint16_t* em, uint16_t* keys, int R, int C, int L) {
  const long N = (long)R * C * L;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    unsigned k = 0;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const long v = wrap(r - drow(e) - 1, R) + (long)wrap(c - dcol(e), C) * R + (long)wrap(l - dlay(e), L) * R * C;
      k |= ((unsigned)em[v] & 3u) << (2 * e);
    }
    keys[i] = (uint16_t)k;
  }
}
// Node keys straight from the image's colours: the file holds one byte per voxel with x
// fastest (femhmg.c:1644-1700), each voxel split into ref^3 refined voxels; a colour maps to
// its material index through the .nf material list.  A colour the list lacks raises *bad.
struct ColorMap { int16_t mat[256]; };
__global__ void k_keys_from_colors(const uint8_t* colors, ColorMap cm, uint16_t* keys, int R, int C, int L, int ref, int* bad) {
  const long N = (long)R * C * L;
  const int frows = R / ref, fcols = C / ref;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const int r = (int)(i % R), c = (int)((i / R) % C), l = (int)(i / ((long)R * C));
    unsigned k = 0;
#pragma unroll
    for (int e = 0; e < 8; e++) {
      const int vr = wrap(r - drow(e) - 1, R), vc = wrap(c - dcol(e), C), vl = wrap(l - dlay(e), L);
      const long f = (long)(vl / ref) * frows * fcols + (long)(vr / ref) * fcols + vc / ref;
      const int m = cm.mat[colors[f]];
      if (m < 0) { *bad = 1; continue; }
      k |= ((unsigned)m & 3u) << (2 * e);
    }
    keys[i] = (uint16_t)k;
  }
}
extern "C" {

cudapcgFlag_t cudapcgSetImage(cudapcgMap_t* img) {
  if (!S || !S->model || !img) return CUDAPCG_FALSE;
  if (S->fluid) { set_err("cudapcgSetImage", "not used for FLUID analysis"); return CUDAPCG_FALSE; }
  if (S->par == CUDAPCG_EBE) {
    uint16_t* tmp = nullptr;
    CK(dev_malloc(&tmp, sizeof(uint16_t) * S->N));
    CK(cudaMemcpy(tmp, img, sizeof(uint16_t) * S->N, cudaMemcpyHostToDevice));
    if (S->dim2) k_keys_from_elements_2d<<<pw_grid(S->N), PW_NT, 0, S->stream>>>(tmp, S->d_keys, S->R, S->C);
    else k_keys_from_elements<<<pw_grid(S->N), PW_NT, 0, S->stream>>>(tmp, S->d_keys, S->R, S->C, S->L);
    CK(cudaStreamSynchronize(S->stream));
    dev_free(tmp);
  } else {
    CK(cudaMemcpy(S->d_keys, img, sizeof(uint16_t) * S->N, cudaMemcpyHostToDevice));
  }
  S->have_keys = true;
  if (S->dim2) { free_ptr(S->d_invd); S->d_invd = nullptr; invalidate_graphs(); }  // a 2D Jacobi diagonal follows the keys
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgB200SetImageColors(const uint8_t* colors, unsigned int rows, unsigned int cols, unsigned int slices,
                                         unsigned int refinement, const int* material_of_color) {
  const char* who = "cudapcgB200SetImageColors";
  if (!S || !S->model || !colors || !material_of_color || refinement < 1) { set_err(who, "bad arguments"); return CUDAPCG_FALSE; }
  if (S->fluid) { set_err(who, "not used for FLUID analysis"); return CUDAPCG_FALSE; }
  if (S->dim2) { set_err(who, "2D node keys are set with cudapcgSetImage"); return CUDAPCG_FALSE; }
  if ((long)rows * refinement != S->R || (long)cols * refinement != S->C || (long)slices * refinement != S->L) {
    set_err(who, "image dimensions times refinement differ from the model's");
    return CUDAPCG_FALSE;
  }
  ColorMap cm;
  for (int c = 0; c < 256; c++) {
    const int m = material_of_color[c];
    cm.mat[c] = (int16_t)((m >= 0 && m < 4) ? m : -1);
  }
  const size_t nfile = (size_t)rows * cols * slices;
  uint8_t* d_col = nullptr;
  int* d_bad = nullptr;
  CK(dev_malloc(&d_col, nfile));
  cudaError_t e = dev_malloc(&d_bad, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int), S->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_col, colors, nfile, cudaMemcpyHostToDevice, S->stream);
  if (e == cudaSuccess) {
    k_keys_from_colors<<<pw_grid(S->N), PW_NT, 0, S->stream>>>(d_col, cm, S->d_keys, S->R, S->C, S->L, (int)refinement, d_bad);
    e = cudaPeekAtLastError();
  }
  int bad = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, S->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
  dev_free(d_col);
  if (d_bad) dev_free(d_bad);
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return CUDAPCG_FALSE; }
  if (bad) { set_err(who, "the image holds a colour without a material (or a material index above 3)"); return CUDAPCG_FALSE; }
  S->have_keys = true;
  invalidate_graphs();
  return CUDAPCG_TRUE;
}
// Stokes DOF-number maps built on the device from the image's colours (pore_maps.cu): the
// node -> DOF map, the DOF -> node map and the interface keys, numbered as
// femhmg_fluid_3D.c:370-491 does (pore nodes, then interface nodes, each in node order).  The
// current model's unknown counts (and the caller's model struct) are set from the numbering.
cudapcgFlag_t cudapcgB200SetPoreImageColors(const uint8_t* colors, unsigned int rows, unsigned int cols, unsigned int slices,
                                            unsigned int refinement, const int* material_of_color, unsigned int* npore,
                                            unsigned int* nborder) {
  const char* who = "cudapcgB200SetPoreImageColors";
  if (!S || !S->model || !colors || !material_of_color || refinement < 1) { set_err(who, "bad arguments"); return CUDAPCG_FALSE; }
  if (!S->fluid || is2d()) { set_err(who, "FLUID_3D models only (thermal / elastic: cudapcgB200SetImageColors)"); return CUDAPCG_FALSE; }
  if ((long)rows * refinement != S->R || (long)cols * refinement != S->C || (long)slices * refinement != S->L) {
    set_err(who, "image size times refinement differs from the model's");
    return CUDAPCG_FALSE;
  }
  PoreColorMap cm;
  for (int c = 0; c < 256; c++) cm.mat[c] = (int16_t)(material_of_color[c] < 0 ? -1 : material_of_color[c]);
  const long N = S->N, nchunks = pore_maps_chunks(N);
  const size_t nimg = (size_t)rows * cols * slices;
  uint8_t *d_col = nullptr, *d_fk = nullptr;
  unsigned* d_cnt = nullptr;
  unsigned long long* d_tot = nullptr;
  int* d_bad = nullptr;
  auto cleanup = [&]() { dev_free(d_col); dev_free(d_fk); dev_free(d_cnt); dev_free(d_tot); dev_free(d_bad); };
  cudaError_t e = dev_malloc(&d_col, nimg);
  if (e == cudaSuccess) e = dev_malloc(&d_fk, N);
  if (e == cudaSuccess) e = dev_malloc(&d_cnt, 2 * sizeof(unsigned) * nchunks);
  if (e == cudaSuccess) e = dev_malloc(&d_tot, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = dev_malloc(&d_bad, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_col, colors, nimg, cudaMemcpyHostToDevice, S->stream);
  if (e != cudaSuccess) { cleanup(); set_err(who, cudaGetErrorString(e)); return CUDAPCG_FALSE; }
  unsigned long long nV = 0, nB = 0;
  const char* msg = nullptr;
  if (!pore_maps_count(d_col, cm, S->R, S->C, S->L, (int)refinement, d_fk, d_cnt, d_tot, d_bad, &nV, &nB, S->stream, &msg)) {
    cleanup(); set_err(who, msg); return CUDAPCG_FALSE;
  }
  if (nV + nB >= 0xffffffffull || 4 * nV + nB >= 0xffffffffull) { cleanup(); set_err(who, "too many Stokes unknowns for 32-bit DOF ids"); return CUDAPCG_FALSE; }
  // the maps take the sizes of this numbering
  free_vectors();
  block_free();
  free_ptr(S->d_node_of_dof); free_ptr(S->d_bkeys);
  S->d_node_of_dof = nullptr; S->d_bkeys = nullptr;
  e = dev_malloc(&S->d_node_of_dof, sizeof(uint32_t) * std::max<unsigned long long>(1, nV + nB));
  if (e == cudaSuccess) e = dev_malloc(&S->d_bkeys, std::max<unsigned long long>(1, nB));
  if (e != cudaSuccess) { cleanup(); set_err(who, cudaGetErrorString(e)); return CUDAPCG_FALSE; }
  if (!pore_maps_number(d_fk, S->R, S->C, S->L, d_cnt, (unsigned)nV, S->d_dof_of_node, S->d_node_of_dof, S->d_bkeys, S->stream, &msg)) {
    cleanup(); set_err(who, msg); return CUDAPCG_FALSE;
  }
  e = cudaStreamSynchronize(S->stream);
  cleanup();
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return CUDAPCG_FALSE; }
  S->nV = (long)nV; S->nB = (long)nB; S->nvars = 4 * S->nV + S->nB;
  S->model->nporenodes = (unsigned)nV; S->model->nbordernodes = (unsigned)nB;
  S->model->nvars = (unsigned)S->nvars; S->model->nhmgvars = (unsigned)(3 * nV);
  S->have_maps = true;
  invalidate_graphs();
  if (npore) *npore = (unsigned)nV;
  if (nborder) *nborder = (unsigned)nB;
  return CUDAPCG_TRUE;
}
// The current Stokes model's maps copied to the host (N, nV + nB and nB entries); for tests.
cudapcgFlag_t cudapcgB200GetPoreMaps(uint32_t* dof_of_node, uint32_t* node_of_dof, uint8_t* border_keys) {
  if (!S || !S->model || !S->fluid || !S->have_maps) { set_err("cudapcgB200GetPoreMaps", "no Stokes maps"); return CUDAPCG_FALSE; }
  if (dof_of_node) CK(cudaMemcpy(dof_of_node, S->d_dof_of_node, sizeof(uint32_t) * S->N, cudaMemcpyDeviceToHost));
  if (node_of_dof && S->nV + S->nB) CK(cudaMemcpy(node_of_dof, S->d_node_of_dof, sizeof(uint32_t) * (S->nV + S->nB), cudaMemcpyDeviceToHost));
  if (border_keys && S->nB) CK(cudaMemcpy(border_keys, S->d_bkeys, S->nB, cudaMemcpyDeviceToHost));
  return CUDAPCG_TRUE;
}
// cudapcg.cu:327-334: the density codes of every voxel (row-fastest model order) and their
// range; voxel v's element matrix is then scaled by fmin + (fmax - fmin) field[v] / 65535.  A
// thermal model has one material (femhmg.c:256-262 normalises it): without an image, its keys
// are zero.  PCG / CG and the 3-vector PCG solve such models, one load case at a time.
cudapcgFlag_t cudapcgSetParametricDensityField(parametricScalarField_t* field, double fmin, double fmax) {
  const char* who = "cudapcgSetParametricDensityField";
  if (!S || !S->model || !field) { set_err(who, "bad arguments"); return CUDAPCG_FALSE; }
  if (S->fluid) { set_err(who, "not used for FLUID analysis"); return CUDAPCG_FALSE; }
  if (!S->d_sdf) CK(dev_malloc(&S->d_sdf, sizeof(uint16_t) * S->N));
  CK(cudaMemcpy(S->d_sdf, field, sizeof(uint16_t) * S->N, cudaMemcpyHostToDevice));
  S->sdf_min = fmin;
  S->sdf_max = fmax;
  if (!S->have_keys) {
    CK(cudaMemset(S->d_keys, 0, sizeof(uint16_t) * S->N));
    S->have_keys = true;
  }
  free_ptr(S->d_invd); S->d_invd = nullptr;
  free_ptr(S->d_tab64); free_ptr(S->d_tab32); S->d_tab64 = nullptr; S->d_tab32 = nullptr;
  free_ptr(S->d_th64); free_ptr(S->d_th32); S->d_th64 = nullptr; S->d_th32 = nullptr; S->th_state = 0;
  invalidate_graphs();
  return CUDAPCG_TRUE;
}
// Image pore map (CUDAPCG_POREMAP_IMG; femhmg.c:962-965, cudapcg.cu:336-355): the host hands
// over the node->DOF map and every node's fluid key (bit e set when the node's local voxel e is
// pore; 0 for a node in the solid) instead of the DOF->node map and the interface keys.  The
// reference runs dedicated image-walking kernels on it (matrix_free.cu:4707-4958); here the two
// DOF-number maps are scattered from it once, on the device, and the same Stokes passes run:
// node i with a non-zero key and DOF id d < nV + nB is the node of DOF d, and an interface DOF
// (d >= nV) takes the node's key.
__global__ void k_maps_from_pore_image(const uint8_t* fk, const uint32_t* dof_of_node, long N, uint32_t nV, uint32_t nVB,
                                       uint32_t* node_of_dof, uint8_t* bkeys) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x) {
    const uint8_t k = fk[i];
    if (!k) continue;
    const uint32_t d = dof_of_node[i];
    if (d >= nVB) continue;
    node_of_dof[d] = (uint32_t)i;
    if (d >= nV) bkeys[d - nV] = k;
  }
}
static bool maps_from_pore_image() {
  if (!S->poremap_img || !S->have_img_keys || !S->have_maps) return true;
  const long g = std::max(1L, std::min<long>((S->N + 255) / 256, 8L * num_sms()));
  k_maps_from_pore_image<<<(int)g, 256, 0, S->stream>>>(S->d_img_fkeys, S->d_dof_of_node, S->N, (uint32_t)S->nV,
                                                        (uint32_t)(S->nV + S->nB), S->d_node_of_dof, S->d_bkeys);
  CKV(cudaGetLastError());
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}
cudapcgFlag_t cudapcgSetPoreMap(cudapcgFlag_t* pores) {
  if (!S || !S->model || !pores) return CUDAPCG_FALSE;
  if (!S->fluid) return CUDAPCG_FALSE;
  if (S->poremap_img) {  // one fluid key per node
    if (!S->d_img_fkeys) CK(dev_malloc(&S->d_img_fkeys, S->N));
    CK(cudaMemcpy(S->d_img_fkeys, pores, S->N, cudaMemcpyHostToDevice));
    S->have_img_keys = true;
    return maps_from_pore_image() ? CUDAPCG_TRUE : CUDAPCG_FALSE;
  }
  if (S->nB) CK(cudaMemcpy(S->d_bkeys, pores, S->nB, cudaMemcpyHostToDevice));
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgSetPeriodic2DOFMap(cudapcgIdMap_t* vars) {
  if (!S || !S->model || !vars || !S->fluid) return CUDAPCG_FALSE;
  CK(cudaMemcpy(S->d_dof_of_node, vars, sizeof(uint32_t) * S->N, cudaMemcpyHostToDevice));
  S->have_maps = true;
  return maps_from_pore_image() ? CUDAPCG_TRUE : CUDAPCG_FALSE;
}
cudapcgFlag_t cudapcgSetDOF2PeriodicMap(cudapcgIdMap_t* nodes) {
  if (!S || !S->model || !nodes || !S->fluid) return CUDAPCG_FALSE;
  if (S->poremap_img) { set_err("cudapcgSetDOF2PeriodicMap", "not used with the image pore map"); return CUDAPCG_FALSE; }  // cudapcg.cu:360
  CK(cudaMemcpy(S->d_node_of_dof, nodes, sizeof(uint32_t) * (S->nV + S->nB), cudaMemcpyHostToDevice));
  return CUDAPCG_TRUE;
}

// Stokes Jacobi tables (matrix_free.cu:663-672 pore rows, :912-925 interface rows).
static bool set_fluid_diag() {
  FlDiag dg;
  const double* K = S->Kd.data();
  const int D = S->fdim, NE = 1 << D, ED = (D + 1) * NE, PC = D * NE;
  double dv[3] = {0, 0, 0}, dp = 0.0;
  for (int e = 0; e < NE; e++) {
    for (int c = 0; c < D; c++) dv[c] += K[(D * e + c) * (ED + 1)];
    dp -= K[(PC + e) * (ED + 1)];
  }
  for (int c = 0; c < 4; c++) dg.pore[c] = 0.0;
  for (int c = 0; c < D; c++) dg.pore[c] = 1.0 / dv[c];
  dg.pore[D] = 1.0 / dp;
  for (int k = 0; k < 256; k++) {
    double sum = 0.0;
    for (int e = 0; e < NE; e++) sum -= K[(PC + e) * (ED + 1)] * (double)((k >> e) & 1);
    dg.border[k] = (sum != 0.0) ? 1.0 / sum : 0.0;
  }
  CKV(cudaMemcpyToSymbol(c_fldiag, &dg, sizeof(FlDiag)));
  return true;
}

cudapcgFlag_t cudapcgSetLclMtxs(cudapcgVar_t* Lm) {
  if (!S || !S->model || !Lm) return CUDAPCG_FALSE;
  const int nk = S->fluid ? 1 : S->nmat;
  if (S->dim2) {  // dense (4 nd) x (4 nd) per material (femhmg_thermal_2D.c:42-90, femhmg_elastic_2D.c:56-146)
    S->Kd.assign(Lm, Lm + (size_t)16 * S->nd * S->nd * nk);
  } else if (S->analysis == CUDAPCG_THERMAL_3D) {
    S->Kd.assign((size_t)64 * nk, 0.0);
    for (int k = 0; k < nk; k++) sparseq1_to_dense(Lm + 40 * k, S->Kd.data() + 64 * k);
  } else if (S->analysis == CUDAPCG_ELASTIC_3D) {
    S->Kd.assign(Lm, Lm + (size_t)576 * nk);
  } else {
    S->Kd.assign(Lm, Lm + (S->fdim == 2 ? 144 : 1024));  // one (DIM + 1) 2^DIM square matrix
  }
  S->have_K = true;
  free_ptr(S->d_K64); free_ptr(S->d_K32); S->d_K64 = nullptr; S->d_K32 = nullptr;
  free_ptr(S->d_tab64); free_ptr(S->d_tab32); S->d_tab64 = nullptr; S->d_tab32 = nullptr;
  free_ptr(S->d_th64); free_ptr(S->d_th32); S->d_th64 = nullptr; S->d_th32 = nullptr; S->th_state = 0;
  free_ptr(S->d_invd); S->d_invd = nullptr;
  invalidate_graphs();  // captured launches hold the old matrix pointers
  if (S->fluid && !set_fluid_diag()) return CUDAPCG_FALSE;
  return CUDAPCG_TRUE;
}

cudapcgFlag_t cudapcgSolve(cudapcgVar_t* res_x) {
  if (!S || !S->model || (!res_x && lean_solver())) return CUDAPCG_FALSE;
  if (!S->rhs_set) { set_err("cudapcgSolve", "right-hand side was not set"); return CUDAPCG_FALSE; }
  const auto t0 = std::chrono::steady_clock::now();
  S->count++;
  S->launches = 0;
  bool ok = lean_solver() ? solve_two_vector(res_x) : (S->precision == CHFEM_B200_FP64) ? solve_T<double>(res_x) : solve_T<float>(res_x);
  const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  S->total_time = t;
  S->mean_time = S->iteration ? S->solve_dev_s / S->iteration : 0.0;
  if (!ok) { S->found = 0; return CUDAPCG_FALSE; }
  if (S->h_sc->status == 1) printf("%sNull solution satisfied %s.\n", S->header.c_str(), S->solver_flag & 1 ? "MINRES" : (S->precond ? "PCG" : "CG"));
  else if (S->h_sc->status == 2) printf("%sInitial guess satisfied %s.\n", S->header.c_str(), S->solver_flag & 1 ? "MINRES" : (S->precond ? "PCG" : "CG"));
  else if (!getenv("CHFEM_B200_QUIET")) {
    if (S->resnorm != CUDAPCG_ERROR_NORM) printf("%siteration: %d, residual: %.3e\n", S->header.c_str(), S->iteration, S->residual);
    else printf("%siteration: %d, residual: %.3e, error: %.3e\n", S->header.c_str(), S->iteration, sqrt(fabs(S->h_sc->delta) / fabs(S->h_sc->delta0)), S->residual);
  }
  return (cudapcgFlag_t)S->found;
}

cudapcgFlag_t cudapcgSetHeaderString(char* header) {
  if (!S) return CUDAPCG_FALSE;
  S->header = header ? header : "";
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgPrintSolverMetrics(void) {
  if (!S) return CUDAPCG_FALSE;
  printf("%sMean time per iteration: %.2e s\n", S->header.c_str(), S->mean_time);
  printf("%sElapsed time: %.2e s\n", S->header.c_str(), S->total_time);
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgPrintSolverMetrics2(char* dest) {
  if (!dest || !S) return CUDAPCG_FALSE;
  sprintf(dest, "%sMean time per iteration: %.2e s\n%sElapsed time: %.2e s\n", S->header.c_str(), S->mean_time, S->header.c_str(), S->total_time);
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgPrintSolverReport(void) {
  if (!S) return CUDAPCG_FALSE;
  if (S->found) printf("%sPCG solver found a solution in %d iterations.\n", S->header.c_str(), S->iteration);
  else printf("%sPCG solver did not converge within provided max number of iterations (%d).\n", S->header.c_str(), S->maxit);
  printf("%sResidual: %e\n", S->header.c_str(), S->residual);
  return cudapcgPrintSolverMetrics();
}
cudapcgFlag_t cudapcgPrintSolverReport2(char* dest) {
  if (!dest || !S) return CUDAPCG_FALSE;
  sprintf(dest, "%sPCG solver ran through %d iterations.\n%sResidual: %e\n%sMean time per iteration: %.2e s\n%sElapsed time: %.2e s\n",
          S->header.c_str(), S->iteration, S->header.c_str(), S->residual, S->header.c_str(), S->mean_time, S->header.c_str(), S->total_time);
  return CUDAPCG_TRUE;
}

// ---------------- extensions ----------------
cudapcgFlag_t cudapcgB200SetPrecision(int mode) {
  if (!S || (mode != CHFEM_B200_FP64 && mode != CHFEM_B200_MIXED)) return CUDAPCG_FALSE;
  // Stokes stays FP64: the reference's (P)MINRES recurrence (conjugate residuals with a Jacobi
  // diagonal that is negative on the pressure rows) comes close to breaking down on the
  // indefinite saddle-point system -- z.Az changes sign and beta jumps by orders of magnitude
  // even in FP64 -- and FP32 rounding at those points sends it into stagnation.
  S->precision = (S->fluid) ? CHFEM_B200_FP64 : mode;
  return CUDAPCG_TRUE;
}
cudapcgFlag_t cudapcgB200SetResidualReplacement(unsigned int k) { if (!S) return CUDAPCG_FALSE; S->replace_every = k; return CUDAPCG_TRUE; }
cudapcgFlag_t cudapcgB200SetIterationsPerLaunch(unsigned int k) {
  if (!S || k < 2 || k > 126) return CUDAPCG_FALSE;
  S->iters_per_launch = k & ~1u;
  if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; S->graph_key = -1; }
  return CUDAPCG_TRUE;
}

}  // extern "C"
template <typename T>
static bool apply_host_T(const double* xh, double* yh, bool precond_only) {
  if (!ensure_vectors<T>() || !ensure_K<T>()) return false;
  const size_t n = (size_t)S->nvars;
  // the direction buffers are free between solves: d0 takes the input, d1 the output (the
  // solver state in x and r stays untouched)
  if (!upload_vec(xh, S->d0)) return false;
  if (!ensure_reduction(8 * num_sms())) return false;
  CKV(cudaMemsetAsync(S->d_sc, 0, sizeof(DevScalars), S->stream));
  if (precond_only) {
    // M^-1 d0 via the INIT pass on r <- d0 (r saved in x64 meanwhile, as FP64 bits of n T words)
    if (!ensure_scratch64(S->x64)) return false;
    CKV(cudaMemcpyAsync(S->x64, S->r, n * sizeof(T), cudaMemcpyDeviceToDevice, S->stream));
    CKV(cudaMemcpyAsync(S->r, S->d0, n * sizeof(T), cudaMemcpyDeviceToDevice, S->stream));
    if (!launch_point<T, PW_INIT>(S->x, nullptr, (T*)S->r, nullptr, (T*)S->d1, nullptr)) return false;
    CKV(cudaMemcpyAsync(S->r, S->x64, n * sizeof(T), cudaMemcpyDeviceToDevice, S->stream));
  } else {
    if (!launch_apply<T>((const T*)S->d0, nullptr, nullptr, (T*)S->d1, false, FIN_STORE, false)) return false;
  }
  if (sizeof(T) == 8) {
    CKV(cudaMemcpyAsync(yh, S->d1, n * 8, cudaMemcpyDeviceToHost, S->stream));
  } else {
    if (!ensure_scratch64(S->x64)) return false;
    k_convert<float, double><<<pw_grid(n), PW_NT, 0, S->stream>>>((const float*)S->d1, S->x64, n);
    CKV(cudaMemcpyAsync(yh, S->x64, n * 8, cudaMemcpyDeviceToHost, S->stream));
  }
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}
extern "C" {
cudapcgFlag_t cudapcgB200ApplyOperator(const double* x, double* y) {
  if (!S || !S->model || !x || !y) return CUDAPCG_FALSE;
  bool ok = (S->precision == CHFEM_B200_FP64) ? apply_host_T<double>(x, y, false) : apply_host_T<float>(x, y, false);
  return ok ? CUDAPCG_TRUE : CUDAPCG_FALSE;
}
cudapcgFlag_t cudapcgB200ApplyPreconditioner(const double* x, double* y) {
  if (!S || !S->model || !x || !y) return CUDAPCG_FALSE;
  bool ok = (S->precision == CHFEM_B200_FP64) ? apply_host_T<double>(x, y, true) : apply_host_T<float>(x, y, true);
  return ok ? CUDAPCG_TRUE : CUDAPCG_FALSE;
}
cudapcgFlag_t cudapcgB200GetStats(cudapcgB200Stats* out) {
  if (!S || !out) return CUDAPCG_FALSE;
  out->iterations = S->iteration;
  out->residual = S->residual;
  out->solve_seconds = S->solve_dev_s;
  out->setup_seconds = S->setup_dev_s;
  out->kernel_launches = S->launches;
  out->precision = S->vec_prec;
  out->found = S->found;
  return CUDAPCG_TRUE;
}

}  // extern "C"
template <typename T>
static double time_op_T(unsigned reps) {
  if (!ensure_vectors<T>() || !ensure_K<T>()) return -1.0;
  if (!ensure_reduction(8 * num_sms())) return -1.0;
  cudaMemsetAsync(S->d_sc, 0, sizeof(DevScalars), S->stream);
  for (int w = 0; w < 3; w++) launch_apply<T>((const T*)S->d0, nullptr, nullptr, (T*)S->d1, false, FIN_NONE, false);
  cudaEventRecord(S->ev0, S->stream);
  for (unsigned i = 0; i < reps; i++) launch_apply<T>((const T*)S->d0, nullptr, nullptr, (T*)S->d1, false, FIN_NONE, false);
  cudaEventRecord(S->ev1, S->stream);
  if (cudaEventSynchronize(S->ev1) != cudaSuccess) return -1.0;
  float ms = 0;
  cudaEventElapsedTime(&ms, S->ev0, S->ev1);
  return ms * 1e-3 / std::max(1u, reps);
}
extern "C" {
}  // extern "C"
template <typename T>
static double time_kernel_T(int which, unsigned reps) {
  if (!ensure_vectors<T>() || !ensure_K<T>()) return -1.0;
  if (!S->q || ((which == 3 || which == 4) && !S->r2)) { set_err("cudapcgB200TimeKernel", "kernel not used by the selected solver"); return -1.0; }
  if (!ensure_reduction(needed_blocks())) return -1.0;
  // each repetition resets the scalars (so no pass exits early) and brackets only the launch
  float total = 0.f;
  for (unsigned i = 0; i < reps + 3; i++) {
    DevScalars h{};
    h.delta = 1.0; h.delta0 = 1.0; h.delta_old = 1.0; h.alpha = 1e-3; h.beta = 0.5; h.res0 = 1.0; h.metric = 1.0;
    cudaMemcpyAsync(S->d_sc, &h, sizeof(h), cudaMemcpyHostToDevice, S->stream);
    cudaEventRecord(S->ev0, S->stream);
    bool ok;
    switch (which) {
      case 0: ok = launch_apply<T>((const T*)S->d0, nullptr, nullptr, (T*)S->q, false, FIN_NONE, false); break;
      case 1: ok = launch_apply<T>(pcg_dir_in<T>(), (const T*)S->d0, (T*)S->d1, (T*)S->q, true, FIN_ALPHA, false); break;
      case 2: ok = launch_point<T, PW_PCG>(S->x, (T*)S->d1, (T*)S->r, (const T*)S->q, s_or_null<T>(), nullptr); break;
      case 3: ok = launch_mr_op<T>((const T*)S->r, (T*)S->r2, FIN_MR_STEP, false); break;
      case 4: ok = launch_mr_dir<T>((const T*)S->r); break;
      default: ok = false;
    }
    cudaEventRecord(S->ev1, S->stream);
    if (!ok || cudaEventSynchronize(S->ev1) != cudaSuccess) return -1.0;
    float ms = 0;
    cudaEventElapsedTime(&ms, S->ev0, S->ev1);
    if (i >= 3) total += ms;
  }
  return total * 1e-3 / std::max(1u, reps);
}
extern "C" {
double cudapcgB200TimeKernel(int which, unsigned int reps) {
  if (!S || !S->model) return -1.0;
  if (which == 5 || which == 6) {
    if (S->fluid) return -1.0;
    return (S->precision == CHFEM_B200_FP64) ? time_block_kernel_T<double>(which, reps) : time_block_kernel_T<float>(which, reps);
  }
  return (S->precision == CHFEM_B200_FP64) ? time_kernel_T<double>(which, reps) : time_kernel_T<float>(which, reps);
}
double cudapcgB200TimeOperator(unsigned int reps) {
  if (!S || !S->model) return -1.0;
  return (S->precision == CHFEM_B200_FP64) ? time_op_T<double>(reps) : time_op_T<float>(reps);
}
int cudapcgB200TrimMemory(void) {
  int dev = 0;
  cudaMemPool_t pool;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaDeviceGetDefaultMemPool(&pool, dev);
  if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
  if (e != cudaSuccess) { set_err("cudapcgB200TrimMemory", cudaGetErrorString(e)); return 0; }
  return 1;
}
unsigned long long cudapcgB200DeviceBytes(void) {
  if (!S) return 0;
  const unsigned long long n = (unsigned long long)S->nvars;
  unsigned long long b = 0;
  if (S->vec_prec == VEC_LEAN) {  // the 2-vector solvers: r and d, the accumulator, the per-step sums
    b += 16ull * n + 8ull * (S->xa_cap + S->hist_cap);
  } else {
    const unsigned long long es = S->vec_prec == CHFEM_B200_FP64 ? 8 : 4;
    const void* work[] = {S->r, S->r2, S->d0, S->d1, S->q, S->s, S->q2};
    for (const void* v : work) b += v ? es * n : 0;
    const double* v64[] = {S->x, S->b64, S->y64, S->x64};
    for (const double* v : v64) b += v ? 8ull * n : 0;
  }
  if (B) {  // the block solver's vectors: r, s, d0, d1, q in the work precision, x and b in FP64
    const unsigned long long es = B->prec == CHFEM_B200_FP64 ? 8 : 4, tot = (unsigned long long)B->nr * B->n;
    const void* work[] = {B->r, B->s, B->d0, B->d1, B->q};
    for (const void* v : work) b += v ? es * tot : 0;
    b += (B->x ? 8ull * tot : 0) + (B->b64 ? 8ull * tot : 0);
  }
  if (S->fluid) b += 4ull * S->N + 4ull * (S->nV + S->nB) + S->nB;
  else b += 2ull * S->N;
  return b;
}

}  // extern "C"

extern "C" cudapcgFlag_t cudapcgB200ComputeFields(int block_index, int axis, int comp, double jump, const double* props,
                                                  double* field_out) {
  const char* who = "cudapcgB200ComputeFields";
  if (!S || !S->model || !props || !field_out) { set_err(who, "bad arguments"); return CUDAPCG_FALSE; }
  if (is2d()) { set_err(who, "not provided for 2D models"); return CUDAPCG_FALSE; }
  if (S->fluid) { set_err(who, "Stokes fields are the solution itself (velocity, pressure)"); return CUDAPCG_FALSE; }
  if (axis < 0 || axis > 2 || comp < 0 || comp >= S->nd) { set_err(who, "bad load case"); return CUDAPCG_FALSE; }
  const double* x = nullptr;
  if (block_index < 0) x = S->x;
  else if (B && block_index < B->nr) x = (const double*)B->x + (size_t)block_index * S->nvars;
  if (!x) { set_err(who, "no solution on the device"); return CUDAPCG_FALSE; }
  FieldProps fp{};
  const int np = S->nd == 1 ? S->nmat : 2 * S->nmat;
  for (int i = 0; i < np && i < 8; i++) fp.p[i] = props[i];
  const int nf = S->nd == 1 ? 3 : 6;
  double* d_out = nullptr;
  CK(dev_malloc(&d_out, sizeof(double) * nf * S->N));
  if (S->nd == 1) k_nodal_fields<1><<<pw_grid(S->N), PW_NT, 0, S->stream>>>(S->d_keys, x, S->R, S->C, S->L, axis, comp, jump, fp, d_out);
  else k_nodal_fields<3><<<pw_grid(S->N), PW_NT, 0, S->stream>>>(S->d_keys, x, S->R, S->C, S->L, axis, comp, jump, fp, d_out);
  cudaError_t e = cudaPeekAtLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(field_out, d_out, sizeof(double) * nf * S->N, cudaMemcpyDeviceToHost, S->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
  dev_free(d_out);
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return CUDAPCG_FALSE; }
  return CUDAPCG_TRUE;
}

// ---------------------------------------------------------------------------------------
// The one-by-one path on the device: a load case's right-hand side from the node keys (or, for
// Stokes, the pore map), and the volume term of its tensor column from the solution left on the
// device, so neither the right-hand side nor x crosses PCIe.
template <typename T>
static bool load_case_rhs_T(int axis, int comp, double jump, const double* CB) {
  const long n = S->nvars;
  // the 2-vector solvers and FP64 PCG3 keep no copy of b: their FP64 r is it
  double* b = (lean_solver() || !S->b64) ? (double*)S->r : S->b64;
  if (S->fluid) {
    double w = 0.0;
    for (int a = 0; a < 8; a++) w += CB[72 + a];
    k_fl_rhs<T><<<pw_grid(n), PW_NT, 0, S->stream>>>(S->nV, n, axis, w, b, (T*)S->r);
  } else {
    if (!ensure_K<double>()) return false;
    if (S->nd == 1)
      k_rhs_load_case<1, T><<<pw_grid(S->N), PW_NT, 0, S->stream>>>(S->d_keys, S->d_K64, S->R, S->C, S->L, axis, comp, jump, b, (T*)S->r);
    else
      k_rhs_load_case<3, T><<<pw_grid(S->N), PW_NT, 0, S->stream>>>(S->d_keys, S->d_K64, S->R, S->C, S->L, axis, comp, jump, b, (T*)S->r);
  }
  CKV(cudaPeekAtLastError());
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}

extern "C" cudapcgFlag_t cudapcgB200SetLoadCaseRHS(int axis, int comp, double jump, const double* CB) {
  const char* who = "cudapcgB200SetLoadCaseRHS";
  if (!S || !S->model || axis < 0 || axis > 2) { set_err(who, "bad arguments"); return CUDAPCG_FALSE; }
  if (is2d()) { set_err(who, "not provided for 2D models"); return CUDAPCG_FALSE; }
  const bool fluid = S->fluid;
  if (fluid ? !CB : (comp < 0 || comp >= S->nd)) { set_err(who, "bad load case"); return CUDAPCG_FALSE; }
  if (!fluid && !S->have_keys) { set_err(who, "the model's keys were not set"); return CUDAPCG_FALSE; }
  if (!ensure_vectors_current()) return CUDAPCG_FALSE;
  const bool ok = (S->vec_prec == CHFEM_B200_MIXED) ? load_case_rhs_T<float>(axis, comp, jump, CB) : load_case_rhs_T<double>(axis, comp, jump, CB);
  if (!ok) return CUDAPCG_FALSE;
  S->rhs_set = true;
  return CUDAPCG_TRUE;
}

extern "C" cudapcgFlag_t cudapcgB200VolumeTerm(const double* CB, unsigned int ns, double* moments) {
  const char* who = "cudapcgB200VolumeTerm";
  if (!S || !S->model || !CB || !moments || !S->x) { set_err(who, "bad arguments or no solution on the device"); return CUDAPCG_FALSE; }
  if (is2d()) { set_err(who, "not provided for 2D models"); return CUDAPCG_FALSE; }
  const bool fluid = S->fluid;
  if (ns != (fluid ? 3u : (S->nd == 3 ? 6u : 3u))) { set_err(who, "ns must be 3 (thermal, Stokes) or 6 (elastic)"); return CUDAPCG_FALSE; }
  if (!S->d_vt) CK(dev_malloc(&S->d_vt, (8 + 4 * 6 * 24) * sizeof(double)));
  double* d_cb = S->d_vt + 8;
  const int g = pw_grid(fluid ? S->nV : S->N);
  if (!ensure_reduction(g)) return CUDAPCG_FALSE;
  if (fluid) {
    double w[3] = {0, 0, 0};
    for (int a = 0; a < 8; a++) { w[0] += CB[3 * a]; w[1] += CB[24 + 3 * a + 1]; w[2] += CB[48 + 3 * a + 2]; }
    k_fl_moments<<<g, PW_NT, 0, S->stream>>>(S->x, S->nV, w[0], w[1], w[2], redctl(g), S->d_vt);
  } else {
    const size_t ncb = (size_t)S->nmat * ns * 8 * S->nd;
    CK(cudaMemsetAsync(d_cb, 0, 4 * 6 * 24 * sizeof(double), S->stream));
    CK(cudaMemcpyAsync(d_cb, CB, ncb * sizeof(double), cudaMemcpyHostToDevice, S->stream));
    if (S->nd == 1) k_cb_moments<1, 3><<<g, PW_NT, 0, S->stream>>>(S->d_keys, d_cb, S->x, S->N, redctl(g), S->d_vt);
    else k_cb_moments<3, 6><<<g, PW_NT, 0, S->stream>>>(S->d_keys, d_cb, S->x, S->N, redctl(g), S->d_vt);
  }
  CK(cudaPeekAtLastError());
  CK(cudaMemcpyAsync(moments, S->d_vt, ns * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
  CK(cudaStreamSynchronize(S->stream));
  return CUDAPCG_TRUE;
}

extern "C" cudapcgFlag_t cudapcgB200SolveLoadCases(unsigned int nrhs, const int* axis, const int* comp, const double* jump,
                                                   const double* CB, unsigned int ns, const double* const* x0, int x0_interpolate,
                                                   double* moments, double* const* x_out, unsigned int* iterations,
                                                   double* residuals) {
  const char* who = "cudapcgB200SolveLoadCases";
  if (!S || !S->model || !axis || !CB || !moments || nrhs < 1 || nrhs > BLK_MAX) { set_err(who, "bad arguments"); return CUDAPCG_FALSE; }
  if (is2d()) { set_err(who, "not provided for 2D models"); return CUDAPCG_FALSE; }
  if (lean_solver()) { set_err(who, "block solves run CG/MINRES(3); the 2-vector solvers reduce one load case at a time"); return CUDAPCG_FALSE; }
  const bool fluid = S->fluid;
  if (fluid != ((S->solver_flag & 1) != 0)) {
    set_err(who, "load-case blocks are provided for thermal and elastic CG/PCG and Stokes MINRES/PMINRES");
    return CUDAPCG_FALSE;
  }
  const unsigned ns_expected = fluid ? 3u : (S->nd == 3 ? 6u : 3u);
  if (ns != ns_expected) { set_err(who, "ns must be 3 (thermal, Stokes) or 6 (elastic)"); return CUDAPCG_FALSE; }
  for (unsigned k = 0; k < nrhs; k++) {
    if (axis[k] < 0 || axis[k] > 2) { set_err(who, "axis must be 0, 1 or 2"); return CUDAPCG_FALSE; }
    if (!fluid && (!comp || !jump || comp[k] < 0 || comp[k] >= S->nd)) { set_err(who, "comp must be a DOF component of the node"); return CUDAPCG_FALSE; }
  }
  const auto t0 = std::chrono::steady_clock::now();
  S->count++;
  S->launches = 0;
  const LoadCases lc{axis, comp, jump, CB, ns, moments};
  bool ok = (S->precision == CHFEM_B200_FP64)
                ? solve_block_T<double>((int)nrhs, nullptr, x0, x0_interpolate, x_out, iterations, residuals, &lc)
                : solve_block_T<float>((int)nrhs, nullptr, x0, x0_interpolate, x_out, iterations, residuals, &lc);
  S->total_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  S->mean_time = S->iteration ? S->solve_dev_s / S->iteration : 0.0;
  if (!ok) { S->found = 0; return CUDAPCG_FALSE; }
  return (cudapcgFlag_t)S->found;
}

extern "C" cudapcgFlag_t cudapcgB200ApplyBlockOperator(unsigned int nrhs, const double* const* v, double* const* y) {
  if (!S || !S->model || !v || !y || nrhs < 1 || nrhs > BLK_MAX) { set_err("cudapcgB200ApplyBlockOperator", "bad arguments"); return CUDAPCG_FALSE; }
  if (is2d()) { set_err("cudapcgB200ApplyBlockOperator", "not provided for 2D models"); return CUDAPCG_FALSE; }
  if (S->fluid) { set_err("cudapcgB200ApplyBlockOperator", "thermal and elastic models only"); return CUDAPCG_FALSE; }
  for (unsigned k = 0; k < nrhs; k++) if (!v[k] || !y[k]) { set_err("cudapcgB200ApplyBlockOperator", "null buffer"); return CUDAPCG_FALSE; }
  const bool ok = (S->precision == CHFEM_B200_FP64) ? apply_block_T<double>((int)nrhs, v, y) : apply_block_T<float>((int)nrhs, v, y);
  return ok ? CUDAPCG_TRUE : CUDAPCG_FALSE;
}

extern "C" cudapcgFlag_t cudapcgB200SolveBlock(unsigned int nrhs, const double* const* rhs, const double* const* x0,
                                               int x0_interpolate, double* const* x_out, unsigned int* iterations,
                                               double* residuals) {
  if (!S || !S->model || !rhs || !x_out || nrhs < 1 || nrhs > BLK_MAX) { set_err("cudapcgB200SolveBlock", "bad arguments"); return CUDAPCG_FALSE; }
  if (is2d()) { set_err("cudapcgB200SolveBlock", "not provided for 2D models"); return CUDAPCG_FALSE; }
  if (lean_solver()) { set_err("cudapcgB200SolveBlock", "block solves run CG/MINRES(3), not the 2-vector solvers"); return CUDAPCG_FALSE; }
  const bool fluid = S->fluid;
  if (fluid != ((S->solver_flag & 1) != 0)) {
    set_err("cudapcgB200SolveBlock", "block solves are provided for thermal and elastic CG/PCG and Stokes MINRES/PMINRES");
    return CUDAPCG_FALSE;
  }
  for (unsigned k = 0; k < nrhs; k++) if (!rhs[k] || !x_out[k]) { set_err("cudapcgB200SolveBlock", "null buffer"); return CUDAPCG_FALSE; }
  const auto t0 = std::chrono::steady_clock::now();
  S->count++;
  S->launches = 0;
  bool ok = (S->precision == CHFEM_B200_FP64) ? solve_block_T<double>((int)nrhs, rhs, x0, x0_interpolate, x_out, iterations, residuals)
                                             : solve_block_T<float>((int)nrhs, rhs, x0, x0_interpolate, x_out, iterations, residuals);
  S->total_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  S->mean_time = S->iteration ? S->solve_dev_s / S->iteration : 0.0;
  if (!ok) { S->found = 0; return CUDAPCG_FALSE; }
  return (cudapcgFlag_t)S->found;
}

// =======================================================================================
// Operator apply without allocation.
//
// Some callers cannot allocate device memory: an embedder whose device memory is owned by
// its own allocator or pool (a framework that hands out every buffer itself and budgets the
// GPU), or a caller that must not pay cudaMalloc's implicit device synchronisation inside
// its loop.  For them, this entry point applies the thermal or elastic operator to a caller
// buffer and returns the fused dot product v.Av, taking every input and output from the
// caller and keeping its own scratch (reduction partials, arrival ticket, result record) in
// the file-scope array below.  It calls no cudaMalloc, cudaFree or allocating routine.
//
// The array is a fixed 66 KB that every GPU which loads this library holds until the process
// exits.  Its device address is looked up once per device with cudaGetSymbolAddress, on the
// first call made on that device with it current; that first call should therefore come
// before any stream capture.  All calls share the one array, so calls whose executions
// overlap on the GPU race on it; each call clears the ticket and record it needs before its
// kernel runs (the partials are fully written before they are read).
constexpr int NOALLOC_MAX_BLOCKS = 8192;  // reduction partials: one double per CTA
constexpr size_t NOALLOC_HEADER = 512;    // [0,256) ticket, [256,512) result record
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_HEADER + NOALLOC_MAX_BLOCKS * sizeof(double)];
static_assert(sizeof(DevScalars) <= 256, "result record must fit its slot");
static void* g_noalloc_addr[64] = {nullptr};

__global__ void k_noalloc_store_dot(const DevScalars* sc, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = sc->red[0];
}

extern "C" int cudapcgB200ApplyOperatorNoAlloc(int analysis_flag, unsigned int nrows, unsigned int ncols, unsigned int nlayers,
                                               unsigned int nmat, const uint16_t* keys, const double* Kdense, const double* v,
                                               double* y, double* vAv, void* stream) {
  const char* who = "cudapcgB200ApplyOperatorNoAlloc";
  if (analysis_flag != CUDAPCG_THERMAL_3D && analysis_flag != CUDAPCG_ELASTIC_3D) { set_err(who, "analysis must be THERMAL_3D (1) or ELASTIC_3D (3)"); return 0; }
  if (!nrows || !ncols || !nlayers) { set_err(who, "empty model"); return 0; }
  if (nmat < 1 || nmat > 4) { set_err(who, "1 to 4 materials are supported with 16-bit keys"); return 0; }
  if (!keys || !Kdense || !v || !y || !vAv) { set_err(who, "null device pointer"); return 0; }
  // the kernels index rows, columns and layers with int, and each of the three is stepped
  // past by one halo node
  if (nrows > 0x7ffffff0u || ncols > 0x7ffffff0u || nlayers > 0x7ffffff0u) { set_err(who, "model dimension above 2^31 - 16"); return 0; }
  const bool thermal = analysis_flag == CUDAPCG_THERMAL_3D;
  const size_t nvals = (size_t)nrows * ncols * nlayers * (thermal ? 1 : 3);
  // y is written while other CTAs still read v (halo planes), keys and Kdense: no overlap
  auto overlaps = [](const void* a, size_t na, const void* b, size_t nb_) {
    const char *pa = (const char*)a, *pb = (const char*)b;
    return pa < pb + nb_ && pb < pa + na;
  };
  const size_t ybytes = nvals * sizeof(double), kbytes = (size_t)nmat * (thermal ? 64 : 576) * sizeof(double);
  if (overlaps(y, ybytes, v, ybytes) || overlaps(y, ybytes, keys, nvals / (thermal ? 1 : 3) * sizeof(uint16_t)) ||
      overlaps(y, ybytes, Kdense, kbytes) || overlaps(vAv, sizeof(double), y, ybytes) || overlaps(vAv, sizeof(double), v, ybytes)) {
    set_err(who, "y (and vAv) must not overlap v, keys or Kdense");
    return 0;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return 0; }
  if (dev < 0 || dev >= 64) { set_err(who, "device ordinal out of range"); return 0; }
  cudaStream_t st = (cudaStream_t)stream;
  // The array's device address: looked up again on every call made outside stream capture (a
  // device reset or a new primary context moves it); a captured call uses the address of the
  // last uncaptured call on this device.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return 0; }
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) { set_err(who, e != cudaSuccess ? cudaGetErrorString(e) : "no symbol address"); return 0; }
    g_noalloc_addr[dev] = p;
  } else if (!g_noalloc_addr[dev]) {
    set_err(who, "first call on this device made under stream capture: make one call outside capture first");
    return 0;
  }
  unsigned char* base = (unsigned char*)g_noalloc_addr[dev];
  // grid: the persistent stencil schedule (any number of column tiles), at most
  // NOALLOC_MAX_BLOCKS CTAs, one reduction partial each in the array
  const long R = nrows, C = ncols, L = nlayers;
  const long tiles = ((R + TE_TR - 1) / TE_TR) * ((C + TE_TC - 1) / TE_TC);
  const size_t smem = thermal ? te_smem_bytes<1, double>((int)nmat) : te_smem_bytes<3, double>((int)nmat);
  int per_sm = 0, sms = 0;
  e = thermal ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_te_apply<1, double, TE_PLAIN>, TE_NT, smem)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_te_apply<3, double, TE_PLAIN>, TE_NT, smem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return 0; }
  const long work = tiles * L;
  const int nb = (int)std::max(1L, std::min<long>({(long)std::max(1, per_sm) * sms, work / TE_MIN_RUN, (long)NOALLOC_MAX_BLOCKS}));
  (void)cudaGetLastError();  // an earlier call's pending launch error is not this call's
  e = cudaMemsetAsync(base, 0, NOALLOC_HEADER, st);
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return 0; }
  DevScalars* sc = (DevScalars*)(base + 256);
  RedCtl rc{(double*)(base + NOALLOC_HEADER), (unsigned*)base, nb};
  const dim3 block(TE_TR, TE_TC);
  const MrCfg cfg{0.0, 0, 0, 1, 0};
  if (thermal) {
    TeArgs<1, double> a{v, nullptr, nullptr, y, nullptr, nullptr, keys, Kdense, (int)nmat, (int)R, (int)C, (int)L, sc, rc, FIN_STORE, 0, cfg};
    k_te_apply<1, double, TE_PLAIN><<<nb, block, smem, st>>>(a);
  } else {
    TeArgs<3, double> a{v, nullptr, nullptr, y, nullptr, nullptr, keys, Kdense, (int)nmat, (int)R, (int)C, (int)L, sc, rc, FIN_STORE, 0, cfg};
    k_te_apply<3, double, TE_PLAIN><<<nb, block, smem, st>>>(a);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return 0; }
  k_noalloc_store_dot<<<1, 32, 0, st>>>(sc, vAv);
  e = cudaGetLastError();
  if (e != cudaSuccess) { set_err(who, cudaGetErrorString(e)); return 0; }
  return 1;
}
