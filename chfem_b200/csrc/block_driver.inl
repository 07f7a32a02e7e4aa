// block_driver.inl -- block multi-RHS PCG/CG (thermal, elastic); included by cudapcg_b200.cu.
// Per right-hand side the recurrence, stopping test, initial-guess handling and (mixed
// precision) residual replacement and final true-residual check are those of the single
// solve; the operator and vector passes run once for all right-hand sides.

struct BlockState {
  int nr = 0, prec = -1;
  long n = 0;
  void *r = nullptr, *s = nullptr, *d0 = nullptr, *d1 = nullptr, *q = nullptr;  // [nr][n], work precision
  double *x = nullptr, *b64 = nullptr;                                          // [nr][n], FP64
  DevScalars* sc = nullptr;   // [nr]
  DevScalars* h_sc = nullptr; // pinned [nr]
  double* d_mom = nullptr;    // load-case moments [BLK_MAX][8] + CB staging
  cudaGraphExec_t gexec = nullptr;
  int graph_key = -1;
};
static BlockState* B = nullptr;

static void block_invalidate() {
  if (B && B->gexec) { cudaGraphExecDestroy(B->gexec); B->gexec = nullptr; B->graph_key = -1; }
}

static void block_free() {
  if (!B) return;
  void* ps[] = {B->r, B->s, B->d0, B->d1, B->q, B->x, B->b64, B->sc, B->d_mom};
  for (void* p : ps) free_ptr(p);
  if (B->h_sc) cudaFreeHost(B->h_sc);
  if (B->gexec) cudaGraphExecDestroy(B->gexec);
  delete B;
  B = nullptr;
}

template <typename T>
static bool block_alloc(int nr) {
  const int p = prec_of<T>();
  if (B && B->nr == nr && B->prec == p && B->n == S->nvars) return true;
  block_free();
  B = new BlockState();
  B->nr = nr; B->prec = p; B->n = S->nvars;
  const size_t tot = (size_t)nr * std::max<long>(S->nvars, 1);
  // thermal / elastic: r, the direction's two buffers and q (s = M^-1 r is formed by the
  // operator pass); Stokes (P)MINRES also keeps s
  std::vector<void**> vs = {&B->r, &B->d0, &B->d1, &B->q};
  if (S->fluid) vs.push_back(&B->s);
  for (void** v : vs) { CKV(dev_malloc(v, tot * sizeof(T))); CKV(cudaMemset(*v, 0, tot * sizeof(T))); }
  CKV(dev_malloc(&B->x, tot * 8));
  CKV(dev_malloc(&B->b64, tot * 8));
  CKV(dev_malloc(&B->sc, nr * sizeof(DevScalars)));
  CKV(cudaMallocHost(&B->h_sc, nr * sizeof(DevScalars)));
  return true;
}

template <int ND, typename T, int NR>
static bool blk_prepare() {
  static bool done = false;
  if (!done) {
    CKV(cudaFuncSetAttribute(k_blk_apply<ND, T, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)blk_smem_bytes<ND, T, NR>()));
    done = true;
  }
  return true;
}

// tile of the FP32 elastic assembled operator: CHFEM_B200_ASM_TILE = "8x1", "6x2", "8x2", "4x2"
// (columns x layers per thread), "6x1r" or "7x1r" (one layer per thread, 4-slot plane ring)
static int asm_tile_choice() {
  static int choice = -1;
  if (choice < 0) {
    const char* e = getenv("CHFEM_B200_ASM_TILE");
    choice = ASM_TILE_8x1;
    if (e && !strcmp(e, "6x2")) choice = ASM_TILE_6x2;
    if (e && !strcmp(e, "8x2")) choice = ASM_TILE_8x2;
    if (e && !strcmp(e, "4x2")) choice = ASM_TILE_4x2;
    if (e && !strcmp(e, "6x1r")) choice = ASM_TILE_6x1_RING4;
    if (e && !strcmp(e, "7x1r")) choice = ASM_TILE_7x1_RING4;
  }
  return choice;
}

// The assembled-stencil block operator pass (stencil_asm.cuh, launched from asm_apply.cu), on
// the NR right-hand sides from k0 on (dold / dnew: the direction buffers of right-hand side 0).
template <int ND, typename T, int NR>
static bool launch_asm_block(T* dold, T* dnew, int precond, int k0 = 0) {
  const int tile = asm_tile_choice();
  const int nb = asm_block_ctas<ND, T, NR>(S->R, S->C, S->L, num_sms(), tile);
  if (nb < 1) { set_err("assembled block operator", "launch configuration"); return false; }
  if (!ensure_reduction(nb)) return false;
  const size_t off = (size_t)k0 * S->nvars;
  BlkArgs<ND, T> a{(const T*)B->r + off, dold + off, dnew + off, (T*)B->q + off, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L,
                   S->nvars, B->sc + k0, redctl(nb), precond};
  const cudaError_t e = asm_block_launch<ND, T, NR>(a, tabdev<T>(), nb, tile, S->stream);
  S->launches++;
  if (e != cudaSuccess) { set_err("assembled block operator", cudaGetErrorString(e)); return false; }
  return true;
}

// plain: the bare operator (M = I in the direction), for cudapcgB200ApplyBlockOperator.  k0:
// the first of the NR right-hand sides the pass works on.
template <int ND, typename T, int NR>
static bool launch_blk_apply(int parity, bool plain = false, int k0 = 0) {
  const long n = S->nvars;
  T* dold = (T*)(parity ? B->d1 : B->d0);
  T* dnew = (T*)(parity ? B->d0 : B->d1);
  const int precond = plain ? 0 : S->precond;
  if (asm_applies()) return launch_asm_block<ND, T, NR>(dold, dnew, precond, k0);
  const dim3 block(TE_TR, TE_TC);
  if (!blk_prepare<ND, T, NR>()) return false;
  const int nb = te_ctas(k_blk_apply<ND, T, NR>, blk_smem_bytes<ND, T, NR>());
  if (!ensure_reduction(nb)) return false;
  const size_t off = (size_t)k0 * n;
  BlkArgs<ND, T> a{(const T*)B->r + off, dold + off, dnew + off, (T*)B->q + off, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, n,
                   B->sc + k0, redctl(nb), precond};
  k_blk_apply<ND, T, NR><<<nb, block, blk_smem_bytes<ND, T, NR>(), S->stream>>>(a);
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

template <int ND, typename T, int NR>
static bool launch_blk_point(int parity, int k0 = 0) {
  const long n = S->nvars;
  T* dnew = (T*)(parity ? B->d0 : B->d1);
  // whole 16-byte chunks per thread when every right-hand side's vectors start aligned
  const bool chunks = n % 4 == 0;
  const int g = pw_grid(chunks ? n / 4 : S->N);
  if (!ensure_reduction(g)) return false;
  const size_t off = (size_t)k0 * n;
  BlkPw<ND, T> p{B->x + off, dnew + off, (T*)B->r + off, (const T*)B->q + off, nullptr, S->d_keys, Kdev<T>(), S->nmat, S->N, n,
                 B->sc + k0, redctl(g), solvecfg()};
  if (chunks) {
    if (S->resnorm == CUDAPCG_L2_NORM) k_blk_point4<ND, T, NR, false><<<g, PW_NT, 0, S->stream>>>(p);
    else k_blk_point4<ND, T, NR, true><<<g, PW_NT, 0, S->stream>>>(p);
  } else if (S->resnorm == CUDAPCG_L2_NORM) k_blk_point<ND, T, NR, false><<<g, PW_NT, 0, S->stream>>>(p);
  else k_blk_point<ND, T, NR, true><<<g, PW_NT, 0, S->stream>>>(p);
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

template <int ND, typename T, int NR>
static bool enqueue_blk_iteration(int parity, int k0 = 0) {
  return launch_blk_apply<ND, T, NR>(parity, false, k0) && launch_blk_point<ND, T, NR>(parity, k0);
}

// Device time of one block operator pass (which 5) or one block vector pass (which 6), for the
// model's natural block size (3 thermal, 6 elastic); scalars reset before each launch.
template <typename T>
static double time_block_kernel_T(int which, unsigned reps) {
  const int nr = S->nd == 3 ? 6 : 3;
  if (!ensure_vectors<T>() || !ensure_K<T>() || !block_alloc<T>(nr)) return -1.0;
  if (asm_applies() && !ensure_tab<T>()) return -1.0;
  if (!ensure_reduction(needed_blocks())) return -1.0;
  for (int k = 0; k < nr; k++) {
    DevScalars& h = B->h_sc[k];
    h = DevScalars{};
    h.delta = 1.0; h.delta0 = 1.0; h.delta_old = 1.0; h.alpha = 1e-3; h.beta = 0.5; h.res0 = 1.0; h.metric = 1.0;
  }
  float total = 0.f;
  for (unsigned i = 0; i < reps + 3; i++) {
    cudaMemcpyAsync(B->sc, B->h_sc, nr * sizeof(DevScalars), cudaMemcpyHostToDevice, S->stream);
    cudaEventRecord(S->ev0, S->stream);
    bool ok;
    if (S->nd == 1) ok = which == 5 ? launch_blk_apply<1, T, 3>(0) : launch_blk_point<1, T, 3>(0);
    else ok = which == 5 ? launch_blk_apply<3, T, 6>(0) : launch_blk_point<3, T, 6>(0);
    cudaEventRecord(S->ev1, S->stream);
    if (!ok || cudaEventSynchronize(S->ev1) != cudaSuccess) return -1.0;
    float ms = 0;
    cudaEventElapsedTime(&ms, S->ev0, S->ev1);
    if (i >= 3) total += ms;
  }
  return total * 1e-3 / std::max(1u, reps);
}

template <int ND, typename T, int NR>
static bool blk_build_graph(int chunk, int k0 = 0) {
  const int key = (prec_of<T>() << 12) | (ND << 8) | (NR << 4) | (S->resnorm << 2) | S->precond | (chunk << 16) | (k0 << 28);
  if (B->gexec && B->graph_key == key) return true;
  if (B->gexec) { cudaGraphExecDestroy(B->gexec); B->gexec = nullptr; }
  cudaGraph_t g;
  CKV(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  bool ok = true;
  const unsigned long long l0 = S->launches;
  for (int it = 0; it < chunk && ok; it++) ok = enqueue_blk_iteration<ND, T, NR>(it & 1, k0);
  S->launches = l0;
  cudaError_t e = cudaStreamEndCapture(S->stream, &g);
  if (!ok || e != cudaSuccess) { set_err("block graph capture", cudaGetErrorString(e)); return false; }
  e = cudaGraphInstantiate(&B->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { set_err("block graph instantiate", cudaGetErrorString(e)); return false; }
  B->graph_key = key;
  return true;
}

static bool blk_read() {
  CKV(cudaMemcpyAsync(B->h_sc, B->sc, B->nr * sizeof(DevScalars), cudaMemcpyDeviceToHost, S->stream));
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}

// Per-RHS helpers on slices (single-RHS kernels with the k-th scalar record).
template <typename T>
static T* slice(void* base, int k) { return (T*)base + (size_t)k * S->nvars; }

template <int ND, typename T, int NR>
static bool solve_block_device(const bool* has_x0) {
  const long n = S->nvars;
  const size_t tot = (size_t)NR * n;
  if (!ensure_reduction(needed_blocks())) return false;
  CKV(cudaMemsetAsync(S->d_ticket, 0, sizeof(unsigned), S->stream));
  CKV(cudaMemsetAsync(B->sc, 0, NR * sizeof(DevScalars), S->stream));
  CKV(cudaMemsetAsync(B->q, 0, tot * sizeof(T), S->stream));
  CKV(cudaMemsetAsync(B->d0, 0, tot * sizeof(T), S->stream));
  CKV(cudaMemsetAsync(B->d1, 0, tot * sizeof(T), S->stream));
  CKV(cudaEventRecord(S->ev0, S->stream));
  for (int k = 0; k < NR; k++) {
    S->cur_sc = B->sc + k;
    if (!launch_point<T, PW_INIT>(slice<double>(B->x, k), nullptr, slice<T>(B->r, k), nullptr, nullptr, nullptr)) { S->cur_sc = S->d_sc; return false; }
    if (has_x0[k]) {
      if (!residual_from_x<T>(true, slice<double>(B->x, k), slice<double>(B->b64, k), slice<T>(B->r, k)) ||
          !launch_point<T, PW_X0R>(slice<double>(B->x, k), nullptr, slice<T>(B->r, k), nullptr, nullptr, nullptr)) { S->cur_sc = S->d_sc; return false; }
    }
  }
  S->cur_sc = S->d_sc;
  CKV(cudaEventRecord(S->ev1, S->stream));
  const int chunk = std::max(2u, S->iters_per_launch & ~1u);
  if (!blk_build_graph<ND, T, NR>(chunk)) return false;
  int cur_k0 = 0;  // first right-hand side of the captured passes
  const bool mixed = sizeof(T) == 4 && S->replace_every > 0;
  unsigned next_replace[NR];
  double repl_delta[NR];
  int checks[NR];
  bool verified[NR];
  for (int k = 0; k < NR; k++) { next_replace[k] = S->replace_every; repl_delta[k] = -1.0; checks[k] = 0; verified[k] = false; }
  const bool trace = getenv("CHFEM_B200_TRACE") != nullptr;
  for (;;) {
    if (!blk_read()) return false;
    if (trace)
      for (int k = 0; k < NR; k++)
        fprintf(stderr, "[block] rhs %d it %d delta %.6e delta0 %.6e alpha %.6e beta %.6e done %d found %d status %d\n", k,
                B->h_sc[k].iteration, B->h_sc[k].delta, B->h_sc[k].delta0, B->h_sc[k].alpha, B->h_sc[k].beta, B->h_sc[k].done,
                B->h_sc[k].found, B->h_sc[k].status);
    bool checked[NR];
    bool launched_check = false;
    for (int k = 0; k < NR; k++) {
      checked[k] = false;
      const DevScalars& h = B->h_sc[k];
      if (h.done) {
        // mixed precision: confirm an apparent convergence on the true residual b - A x
        if (mixed && h.status == 0 && h.found && !verified[k] && checks[k] < 32) {
          checks[k]++;
          S->cur_sc = B->sc + k;
          bool ok = residual_from_x<T>(false, slice<double>(B->x, k), slice<double>(B->b64, k), slice<T>(B->r, k)) &&
                    launch_point<T, PW_CHECK>(slice<double>(B->x, k), nullptr, slice<T>(B->r, k), nullptr, nullptr, nullptr);
          S->cur_sc = S->d_sc;
          if (!ok) return false;
          checked[k] = true;
          launched_check = true;
          if (trace) fprintf(stderr, "[block] rhs %d true-residual check %d\n", k, checks[k]);
        }
        continue;
      }
      if (repl_delta[k] < 0) repl_delta[k] = fabs(h.delta0);
      if (mixed && ((unsigned)h.iteration >= next_replace[k] || fabs(h.delta) < S->replace_drop * repl_delta[k])) {
        S->cur_sc = B->sc + k;
        bool ok = residual_from_x<T>(true, slice<double>(B->x, k), slice<double>(B->b64, k), slice<T>(B->r, k)) &&
                  launch_point<T, PW_REPL>(slice<double>(B->x, k), nullptr, slice<T>(B->r, k), nullptr, nullptr, nullptr);
        S->cur_sc = S->d_sc;
        if (!ok) return false;
        next_replace[k] = (unsigned)h.iteration + S->replace_every;
        repl_delta[k] = fabs(h.delta);
        if (trace) fprintf(stderr, "[block] rhs %d residual replacement at %d\n", k, h.iteration);
      }
    }
    if (launched_check) {
      if (!blk_read()) return false;
      for (int k = 0; k < NR; k++)
        if (checked[k]) {
          if (B->h_sc[k].done) verified[k] = true;
          else { next_replace[k] = (unsigned)B->h_sc[k].iteration + S->replace_every; repl_delta[k] = fabs(B->h_sc[k].delta); }
        }
    }
    bool any = false;
    for (int k = 0; k < NR; k++) any = any || !B->h_sc[k].done;
    if (!any) break;
    if constexpr (NR == 6) {
      // once the first three cases (the normal strains, which converge first) are done, the
      // passes run on the last three only (the converged cases' lanes are no longer computed);
      // a true-residual check that reopens one of the first three brings all six back
      bool head_done = true;
      for (int k = 0; k < 3; k++) head_done = head_done && B->h_sc[k].done;
      const int want = head_done ? 3 : 0;
      if (want != cur_k0) {
        if (!(want ? blk_build_graph<ND, T, 3>(chunk, 3) : blk_build_graph<ND, T, NR>(chunk, 0))) return false;
        cur_k0 = want;
        if (trace) fprintf(stderr, "[block] passes on right-hand sides %d..%d\n", want, NR - 1);
      }
    }
    CKV(cudaGraphLaunch(B->gexec, S->stream));
    S->launches += (unsigned long long)chunk * 2;
  }
  CKV(cudaEventRecord(S->ev2, S->stream));
  CKV(cudaEventSynchronize(S->ev2));
  float ms1 = 0, ms2 = 0;
  cudaEventElapsedTime(&ms1, S->ev0, S->ev1);
  cudaEventElapsedTime(&ms2, S->ev1, S->ev2);
  S->setup_dev_s = ms1 * 1e-3;
  S->solve_dev_s = ms2 * 1e-3;
  return true;
}

// ---------------------------------------------------------------------------------------
// Block (P)MINRES for the Stokes flow directions.  Buffers: r and r' alternate between
// B->r and B->d1, the direction is B->d0, q = A d is B->q, s = A M^-1 r is B->s.
template <typename T, int NR>
static bool launch_fl_blk_dir(int parity) {
  const T* rcur = (const T*)(parity ? B->d1 : B->r);
  const int g = pw_grid(S->nV + S->nB);
  if (!ensure_reduction(g)) return false;
  FlBlkDir<T> a{(T*)B->d0, (T*)B->q, rcur, (const T*)B->s, S->d_bkeys, S->nV, S->nB, S->nvars, B->sc, redctl(g), S->precond};
  k_fl_blk_dir<T, NR><<<g, PW_NT, 0, S->stream>>>(a);
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}
template <typename T, int NR>
static bool launch_fl_blk_apply(int parity) {
  const T* rcur = (const T*)(parity ? B->d1 : B->r);
  T* rnext = (T*)(parity ? B->r : B->d1);
  const int g = pw_grid(S->nV + S->nB);
  if (!ensure_reduction(g)) return false;
  FlBlkArgs<T> a{rcur, (const T*)B->q, rnext, (T*)B->s, B->x, (const T*)B->d0, S->d_dof_of_node, S->d_node_of_dof, S->d_bkeys,
                 S->R, S->C, S->L, S->nV, S->nB, S->nvars, B->sc, redctl(g), mrcfg()};
  if (S->resnorm == CUDAPCG_L2_NORM) k_fl_blk_apply<T, NR, false><<<g, FL_NT, 0, S->stream>>>(a);
  else k_fl_blk_apply<T, NR, true><<<g, FL_NT, 0, S->stream>>>(a);
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

template <typename T, int NR>
static bool blk_build_graph_mr(int chunk) {
  const int key = (prec_of<T>() << 12) | (NR << 4) | (S->resnorm << 2) | S->precond | (chunk << 16) | (1 << 30);
  if (B->gexec && B->graph_key == key) return true;
  if (B->gexec) { cudaGraphExecDestroy(B->gexec); B->gexec = nullptr; }
  cudaGraph_t g;
  CKV(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  bool ok = true;
  const unsigned long long l0 = S->launches;
  for (int it = 0; it < chunk && ok; it++) ok = launch_fl_blk_dir<T, NR>(it & 1) && launch_fl_blk_apply<T, NR>(it & 1);
  S->launches = l0;
  cudaError_t e = cudaStreamEndCapture(S->stream, &g);
  if (!ok || e != cudaSuccess) { set_err("block graph capture", cudaGetErrorString(e)); return false; }
  e = cudaGraphInstantiate(&B->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { set_err("block graph instantiate", cudaGetErrorString(e)); return false; }
  B->graph_key = key;
  return true;
}

template <typename T, int NR>
static bool solve_block_minres_device(const bool* has_x0) {
  const long n = S->nvars;
  const size_t tot = (size_t)NR * n;
  if (!ensure_reduction(needed_blocks())) return false;
  CKV(cudaMemsetAsync(S->d_ticket, 0, sizeof(unsigned), S->stream));
  CKV(cudaMemsetAsync(B->sc, 0, NR * sizeof(DevScalars), S->stream));
  CKV(cudaMemsetAsync(B->q, 0, tot * sizeof(T), S->stream));
  CKV(cudaMemsetAsync(B->d0, 0, tot * sizeof(T), S->stream));
  CKV(cudaEventRecord(S->ev0, S->stream));
  auto op_k = [&](int k, int fin, bool skip) {
    return launch_mr_op_buf<T>(slice<T>(B->r, k), slice<T>(B->d1, k), slice<T>(B->q, k), slice<T>(B->s, k),
                               slice<double>(B->x, k), slice<T>(B->d0, k), fin, skip);
  };
  for (int k = 0; k < NR; k++) {  // pminres.cu:58-98 per right-hand side
    S->cur_sc = B->sc + k;
    bool ok = op_k(k, FIN_MR_INIT, false);
    if (ok && has_x0[k])
      ok = residual_from_x<T>(true, slice<double>(B->x, k), slice<double>(B->b64, k), slice<T>(B->r, k)) && op_k(k, FIN_MR_X0, true);
    S->cur_sc = S->d_sc;
    if (!ok) return false;
  }
  CKV(cudaEventRecord(S->ev1, S->stream));
  const int chunk = std::max(2u, S->iters_per_launch & ~1u);
  if (!blk_build_graph_mr<T, NR>(chunk)) return false;
  const bool mixed = sizeof(T) == 4 && S->replace_every > 0;
  const bool can_check = S->resnorm != CUDAPCG_ERROR_NORM;
  const bool trace = getenv("CHFEM_B200_TRACE") != nullptr;
  unsigned next_replace[NR];
  double repl_ref[NR];
  int checks[NR];
  bool verified[NR];
  for (int k = 0; k < NR; k++) { next_replace[k] = S->replace_every; repl_ref[k] = 1.0; checks[k] = 0; verified[k] = false; }
  for (;;) {
    if (!blk_read()) return false;
    if (trace)
      for (int k = 0; k < NR; k++)
        fprintf(stderr, "[block-mr] rhs %d it %d metric %.6e delta %.6e alpha %.6e beta %.6e done %d found %d status %d\n", k,
                B->h_sc[k].iteration, B->h_sc[k].metric, B->h_sc[k].delta, B->h_sc[k].alpha, B->h_sc[k].beta, B->h_sc[k].done,
                B->h_sc[k].found, B->h_sc[k].status);
    bool checked[NR];
    bool launched_check = false;
    for (int k = 0; k < NR; k++) {
      checked[k] = false;
      const DevScalars& h = B->h_sc[k];
      if (h.done) {
        if (mixed && can_check && h.status == 0 && h.found && !verified[k] && checks[k] < 32) {
          checks[k]++;
          S->cur_sc = B->sc + k;
          bool ok = residual_from_x<T>(false, slice<double>(B->x, k), slice<double>(B->b64, k), slice<T>(B->r, k)) &&
                    op_k(k, FIN_MR_CHECK, false);
          S->cur_sc = S->d_sc;
          if (!ok) return false;
          checked[k] = true;
          launched_check = true;
        }
        continue;
      }
      const double prog = h.metric * h.metric;
      if (mixed && ((unsigned)h.iteration >= next_replace[k] || prog < S->replace_drop * repl_ref[k])) {
        S->cur_sc = B->sc + k;
        bool ok = residual_from_x<T>(true, slice<double>(B->x, k), slice<double>(B->b64, k), slice<T>(B->r, k)) &&
                  op_k(k, FIN_MR_REPL, true) &&
                  launch_apply<T>(slice<T>(B->d0, k), nullptr, nullptr, slice<T>(B->q, k), false, FIN_NONE, true);  // q = A d afresh
        S->cur_sc = S->d_sc;
        if (!ok) return false;
        next_replace[k] = (unsigned)h.iteration + S->replace_every;
        repl_ref[k] = prog;
        if (trace) fprintf(stderr, "[block-mr] rhs %d residual replacement at %d\n", k, h.iteration);
      }
    }
    if (launched_check) {
      if (!blk_read()) return false;
      for (int k = 0; k < NR; k++)
        if (checked[k]) {
          if (B->h_sc[k].done) verified[k] = true;
          else { next_replace[k] = (unsigned)B->h_sc[k].iteration + S->replace_every; repl_ref[k] = B->h_sc[k].metric * B->h_sc[k].metric; }
        }
    }
    bool any = false;
    for (int k = 0; k < NR; k++) any = any || !B->h_sc[k].done;
    if (!any) break;
    CKV(cudaGraphLaunch(B->gexec, S->stream));
    S->launches += (unsigned long long)chunk * 2;
  }
  CKV(cudaEventRecord(S->ev2, S->stream));
  CKV(cudaEventSynchronize(S->ev2));
  float ms1 = 0, ms2 = 0;
  cudaEventElapsedTime(&ms1, S->ev0, S->ev1);
  cudaEventElapsedTime(&ms2, S->ev1, S->ev2);
  S->setup_dev_s = ms1 * 1e-3;
  S->solve_dev_s = ms2 * 1e-3;
  return true;
}

// Load cases assembled and reduced on the device (cudapcgB200SolveLoadCases).
struct LoadCases {
  const int* axis; const int* comp; const double* jump;
  const double* CB; unsigned ns;
  double* moments;  // [nr][ns] out
};

template <typename T>
static bool rhs_on_device(const LoadCases& lc, int k) {
  const long n = S->nvars;
  if (S->fluid) {
    double w = 0.0;
    for (int a = 0; a < 8; a++) w += lc.CB[72 + a];
    k_fl_rhs<T><<<pw_grid(n), PW_NT, 0, S->stream>>>(S->nV, n, lc.axis[k], w, slice<double>(B->b64, k), slice<T>(B->r, k));
  } else {
    if (!ensure_K<double>()) return false;
    if (S->nd == 1)
      k_rhs_load_case<1, T><<<pw_grid(S->N), PW_NT, 0, S->stream>>>(S->d_keys, S->d_K64, S->R, S->C, S->L, lc.axis[k], lc.comp[k], lc.jump[k],
                                                                    slice<double>(B->b64, k), slice<T>(B->r, k));
    else
      k_rhs_load_case<3, T><<<pw_grid(S->N), PW_NT, 0, S->stream>>>(S->d_keys, S->d_K64, S->R, S->C, S->L, lc.axis[k], lc.comp[k], lc.jump[k],
                                                                    slice<double>(B->b64, k), slice<T>(B->r, k));
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

// volume term of the effective tensor for every right-hand side into lc.moments (host)
static bool moments_on_device(const LoadCases& lc, int nr) {
  if (!B->d_mom) CKV(dev_malloc(&B->d_mom, (size_t)BLK_MAX * 8 * sizeof(double) + 4 * 6 * 24 * sizeof(double)));
  double* d_cb = B->d_mom + BLK_MAX * 8;
  const int g = pw_grid(S->fluid ? S->nV : S->N);
  if (!ensure_reduction(g)) return false;
  if (S->fluid) {
    double w[3] = {0, 0, 0};
    for (int a = 0; a < 8; a++) { w[0] += lc.CB[3 * a]; w[1] += lc.CB[24 + 3 * a + 1]; w[2] += lc.CB[48 + 3 * a + 2]; }
    for (int k = 0; k < nr; k++) k_fl_moments<<<g, PW_NT, 0, S->stream>>>(slice<double>(B->x, k), S->nV, w[0], w[1], w[2], redctl(g), B->d_mom + 8 * k);
  } else {
    const size_t ncb = (size_t)S->nmat * lc.ns * 8 * S->nd;
    CKV(cudaMemsetAsync(d_cb, 0, 4 * 6 * 24 * sizeof(double), S->stream));
    CKV(cudaMemcpyAsync(d_cb, lc.CB, ncb * sizeof(double), cudaMemcpyHostToDevice, S->stream));
    for (int k = 0; k < nr; k++) {
      if (S->nd == 1) k_cb_moments<1, 3><<<g, PW_NT, 0, S->stream>>>(S->d_keys, d_cb, slice<double>(B->x, k), S->N, redctl(g), B->d_mom + 8 * k);
      else k_cb_moments<3, 6><<<g, PW_NT, 0, S->stream>>>(S->d_keys, d_cb, slice<double>(B->x, k), S->N, redctl(g), B->d_mom + 8 * k);
    }
  }
  S->launches += nr;
  double h[BLK_MAX * 8];
  CKV(cudaMemcpyAsync(h, B->d_mom, (size_t)nr * 8 * sizeof(double), cudaMemcpyDeviceToHost, S->stream));
  CKV(cudaStreamSynchronize(S->stream));
  for (int k = 0; k < nr; k++)
    for (unsigned s = 0; s < lc.ns; s++) lc.moments[k * lc.ns + s] = h[8 * k + s];
  return true;
}

template <typename T>
static bool solve_block_T(int nr, const double* const* rhs, const double* const* x0, int x0_mode, double* const* x_out,
                          unsigned* iters, double* resid, const LoadCases* lc = nullptr) {
  if (S->d_sdf) { set_err("cudapcgB200SolveBlock", "a scalar density field is solved one load case at a time"); return false; }
  if (!ensure_vectors<T>() || !ensure_K<T>() || !block_alloc<T>(nr)) return false;
  if (asm_applies() && !ensure_tab<T>()) return false;
  const long n = S->nvars;
  bool has_x0[BLK_MAX] = {false};
  for (int k = 0; k < nr; k++) {
    if (lc) { if (!rhs_on_device<T>(*lc, k)) return false; }
    else {
      CKV(cudaMemcpyAsync(slice<double>(B->b64, k), rhs[k], n * 8, cudaMemcpyHostToDevice, S->stream));
      if (sizeof(T) == 8) CKV(cudaMemcpyAsync(slice<double>(B->r, k), rhs[k], n * 8, cudaMemcpyHostToDevice, S->stream));
      else k_convert<double, float><<<pw_grid(n), PW_NT, 0, S->stream>>>(slice<double>(B->b64, k), slice<float>(B->r, k), n);
    }
    if (x0 && x0[k]) {
      if (x0_mode == 1) { if (!interp_into(x0[k], slice<double>(B->x, k))) return false; }
      else CKV(cudaMemcpyAsync(slice<double>(B->x, k), x0[k], n * 8, x0_mode == 2 ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, S->stream));
      has_x0[k] = true;
    }
    else CKV(cudaMemsetAsync(slice<double>(B->x, k), 0, n * 8, S->stream));
  }
  bool ok;
  if (S->fluid) {
    if (nr != 3) { set_err("cudapcgB200SolveBlock", "Stokes blocks hold the 3 flow directions"); return false; }
    ok = solve_block_minres_device<T, 3>(has_x0);
  } else if (S->nd == 1 && nr == 3) ok = solve_block_device<1, T, 3>(has_x0);
  else if (S->nd == 3 && nr == 6) ok = solve_block_device<3, T, 6>(has_x0);
  else if (S->nd == 3 && nr == 3) ok = solve_block_device<3, T, 3>(has_x0);
  else { set_err("cudapcgB200SolveBlock", "block sizes are 3 (thermal, elastic) and 6 (elastic)"); return false; }
  if (!ok) return false;
  if (!blk_read()) return false;
  for (int k = 0; k < nr; k++) {
    // a null right-hand side under (P)MINRES returns x = 0 as cudapcgSolve does
    if (S->fluid && B->h_sc[k].status == 1) CKV(cudaMemsetAsync(slice<double>(B->x, k), 0, n * 8, S->stream));
    if (x_out && x_out[k]) CKV(cudaMemcpyAsync(x_out[k], slice<double>(B->x, k), n * 8, cudaMemcpyDeviceToHost, S->stream));
  }
  if (lc && !moments_on_device(*lc, nr)) return false;
  CKV(cudaStreamSynchronize(S->stream));
  unsigned maxit = 0;
  int found_all = 1;
  for (int k = 0; k < nr; k++) {
    const DevScalars& h = B->h_sc[k];
    double res;
    int found;
    if (h.status == 1) { res = 0.0; found = 1; }
    else if (h.status == 2) { res = h.metric; found = 1; }
    else if (S->resnorm == CUDAPCG_L2_NORM && !S->fluid) { res = sqrt(fabs(h.delta) / fabs(h.delta0)); found = !(fabs(h.delta) > S->tol * S->tol * fabs(h.delta0)); }
    else { res = h.metric; found = res <= S->tol; }
    if (iters) iters[k] = (unsigned)h.iteration;
    if (resid) resid[k] = res;
    // per right-hand side, the messages cudapcgSolve prints for a single solve
    const char* name = S->fluid ? "MINRES" : (S->precond ? "PCG" : "CG");
    if (h.status == 1) printf("%s[%d] Null solution satisfied %s.\n", S->header.c_str(), k, name);
    else if (h.status == 2) printf("%s[%d] Initial guess satisfied %s.\n", S->header.c_str(), k, name);
    else if (!getenv("CHFEM_B200_QUIET")) {
      if (S->resnorm != CUDAPCG_ERROR_NORM) printf("%s[%d] iteration: %d, residual: %.3e\n", S->header.c_str(), k, h.iteration, res);
      else printf("%s[%d] iteration: %d, residual: %.3e, error: %.3e\n", S->header.c_str(), k, h.iteration, sqrt(fabs(h.delta) / fabs(h.delta0)), res);
    }
    maxit = std::max(maxit, (unsigned)h.iteration);
    found_all = found_all && found;
  }
  S->iteration = maxit;
  S->found = found_all;
  return true;
}

// y_k = A v_k for nr host vectors through the block operator pass of the block solver (the
// assembled-stencil pass for two-material models): v goes into r, and the direction is formed
// with beta = 0 and M = I, so d_new = v and q = A v.
template <typename T>
static bool apply_block_T(int nr, const double* const* v, double* const* y) {
  if (!ensure_vectors<T>() || !ensure_K<T>() || !block_alloc<T>(nr)) return false;
  if (asm_applies() && !ensure_tab<T>()) return false;
  if (!ensure_reduction(needed_blocks())) return false;
  const long n = S->nvars;
  for (int k = 0; k < nr; k++) {
    CKV(cudaMemcpyAsync(slice<double>(B->b64, k), v[k], n * 8, cudaMemcpyHostToDevice, S->stream));
    if (sizeof(T) == 8) CKV(cudaMemcpyAsync(slice<double>(B->r, k), slice<double>(B->b64, k), n * 8, cudaMemcpyDeviceToDevice, S->stream));
    else k_convert<double, float><<<pw_grid(n), PW_NT, 0, S->stream>>>(slice<double>(B->b64, k), slice<float>(B->r, k), n);
  }
  CKV(cudaMemsetAsync(B->d0, 0, (size_t)nr * n * sizeof(T), S->stream));
  for (int k = 0; k < nr; k++) {
    DevScalars& h = B->h_sc[k];
    h = DevScalars{};
    h.delta = 1.0; h.delta0 = 1.0; h.delta_old = 1.0;
  }
  CKV(cudaMemcpyAsync(B->sc, B->h_sc, nr * sizeof(DevScalars), cudaMemcpyHostToDevice, S->stream));
  CKV(cudaMemsetAsync(S->d_ticket, 0, sizeof(unsigned), S->stream));
  bool ok;
  if (S->nd == 1 && nr == 3) ok = launch_blk_apply<1, T, 3>(0, true);
  else if (S->nd == 3 && nr == 6) ok = launch_blk_apply<3, T, 6>(0, true);
  else if (S->nd == 3 && nr == 3) ok = launch_blk_apply<3, T, 3>(0, true);
  else { set_err("cudapcgB200ApplyBlockOperator", "block sizes are 3 (thermal, elastic) and 6 (elastic)"); return false; }
  if (!ok) { set_err("cudapcgB200ApplyBlockOperator", cudaGetErrorString(cudaGetLastError())); return false; }
  for (int k = 0; k < nr; k++) {
    if (sizeof(T) == 4) k_convert<float, double><<<pw_grid(n), PW_NT, 0, S->stream>>>(slice<float>(B->q, k), slice<double>(B->b64, k), n);
    else CKV(cudaMemcpyAsync(slice<double>(B->b64, k), slice<double>(B->q, k), n * 8, cudaMemcpyDeviceToDevice, S->stream));
    CKV(cudaMemcpyAsync(y[k], slice<double>(B->b64, k), n * 8, cudaMemcpyDeviceToHost, S->stream));
  }
  CKV(cudaStreamSynchronize(S->stream));
  return true;
}
