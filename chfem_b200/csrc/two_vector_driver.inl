// two_vector_driver.inl -- host driver of the 2-vector Stokes solvers (kernels in
// stencil_fluid2.cuh), included by cudapcg_b200.cu.
//
// Device memory of a solve: r and d (FP64, the two vectors), the reduction accumulator of the
// solution's velocity part (FULL: D nV values, ONLYDIR: nV, NONE: none; D = 3, or 2 on a 2D
// image) and the per-step sums (3 x (max iterations + 1)), as in
// chfem/src/femhmg/cudapcg/solvers/pcg2.cu:37-56.  The steps run as CUDA-graph chunks like the
// other solvers; the host reads one scalar record per chunk.  The result is the D velocity sums
// of the solution scaled by the x-reduce scale (the permeability column), and the per-step sums
// of the D components go to <model name>_xreduce_metrics_<n>.bin (xreduce.cu:29-48,
// pcg2.cu:258-280).

static constexpr int VEC_LEAN = 7;  // vec_prec marker of the 2-vector allocation

static bool lean_solver() { return S && S->solver_flag >= CUDAPCG_CG2_SOLVER; }

// r -> S->r, d -> S->d0 (FP64); no other work vector
static bool ensure_lean_vectors() {
  if (S->vec_prec == VEC_LEAN && S->r && S->d0) return true;
  free_vectors();
  const size_t n = std::max<size_t>((size_t)S->nvars, 1);
  CKV(dev_malloc(&S->r, n * 8));
  CKV(dev_malloc(&S->d0, n * 8));
  CKV(cudaMemsetAsync(S->r, 0, n * 8, S->stream));
  CKV(cudaMemsetAsync(S->d0, 0, n * 8, S->stream));
  S->vec_prec = VEC_LEAN;
  S->arrays_alloc = true;
  return true;
}

static bool ensure_lean_work() {
  const size_t nxa = S->xr_mode == CUDAPCG_XREDUCE_FULL ? (size_t)S->fdim * S->nV : (S->xr_mode == CUDAPCG_XREDUCE_ONLYDIR ? (size_t)S->nV : 0);
  const size_t nh = 3 * ((size_t)S->maxit + 1);
  if (nxa > S->xa_cap) {
    free_ptr(S->d_xa);
    S->d_xa = nullptr;
    CKV(dev_malloc(&S->d_xa, nxa * 8));
    S->xa_cap = nxa;
    invalidate_graphs();
  }
  if (nh > S->hist_cap) {
    free_ptr(S->d_hist);
    S->d_hist = nullptr;
    CKV(dev_malloc(&S->d_hist, nh * 8));
    S->hist_cap = nh;
    invalidate_graphs();
  }
  if (nxa) CKV(cudaMemsetAsync(S->d_xa, 0, nxa * 8, S->stream));
  CKV(cudaMemsetAsync(S->d_hist, 0, nh * 8, S->stream));
  return true;
}

static Fl2Args fl2_args(const double* in, int finish) {
  Fl2Args a;
  a.in = in; a.r = (double*)S->r; a.d = (const double*)S->d0; a.xa = S->d_xa; a.hist = S->d_hist;
  a.dof_of_node = S->d_dof_of_node; a.node_of_dof = S->d_node_of_dof; a.bkeys = S->d_bkeys;
  a.R = S->R; a.C = S->C; a.L = S->L; a.nV = S->nV; a.nB = S->nB;
  a.sc = S->d_sc;
  a.finish = finish;
  a.cfg = Fl2Cfg{S->tol, (int)std::min<unsigned>(S->maxit, 0x7fffffffu), S->resnorm, S->precond,
                 S->solver_flag == CUDAPCG_MINRES2_SOLVER ? 1 : 0, (int)S->xr_mode, (int)std::min(S->xr_shift, (unsigned)S->fdim - 1)};
  return a;
}

static bool launch_fl2(int mode, const double* in, int finish) {
  Fl2Args a = fl2_args(in, finish);
  const int g = pw_grid(S->nV + S->nB);
  if (!ensure_reduction(g)) return false;
  a.rc = redctl(g);
  if (S->fdim == 2) {
    switch (mode) {
      case F2_DAD: k_fl2_apply<F2_DAD, 2><<<g, FL_NT, 0, S->stream>>>(a); break;
      case F2_AMA: k_fl2_apply<F2_AMA, 2><<<g, FL_NT, 0, S->stream>>>(a); break;
      case F2_UPD: k_fl2_apply<F2_UPD, 2><<<g, FL_NT, 0, S->stream>>>(a); break;
      case F2_ZAZ: k_fl2_apply<F2_ZAZ, 2><<<g, FL_NT, 0, S->stream>>>(a); break;
      default: k_fl2_apply<F2_X0, 2><<<g, FL_NT, 0, S->stream>>>(a); break;
    }
  } else {
    switch (mode) {
      case F2_DAD: k_fl2_apply<F2_DAD><<<g, FL_NT, 0, S->stream>>>(a); break;
      case F2_AMA: k_fl2_apply<F2_AMA><<<g, FL_NT, 0, S->stream>>>(a); break;
      case F2_UPD: k_fl2_apply<F2_UPD><<<g, FL_NT, 0, S->stream>>>(a); break;
      case F2_ZAZ: k_fl2_apply<F2_ZAZ><<<g, FL_NT, 0, S->stream>>>(a); break;
      default: k_fl2_apply<F2_X0><<<g, FL_NT, 0, S->stream>>>(a); break;
    }
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

static bool launch_fl2_point(int mode) {
  Fl2Args a = fl2_args((const double*)S->r, F2F_NONE);
  const int g = pw_grid((S->fdim + 1) * S->nV + S->nB);
  if (!ensure_reduction(g)) return false;
  a.rc = redctl(g);
  if (S->fdim == 2) {
    if (mode == P2_INIT) k_fl2_point<P2_INIT, 2><<<g, PW_NT, 0, S->stream>>>(a, (double*)S->d0);
    else k_fl2_point<P2_DIR, 2><<<g, PW_NT, 0, S->stream>>>(a, (double*)S->d0);
  } else {
    if (mode == P2_INIT) k_fl2_point<P2_INIT><<<g, PW_NT, 0, S->stream>>>(a, (double*)S->d0);
    else k_fl2_point<P2_DIR><<<g, PW_NT, 0, S->stream>>>(a, (double*)S->d0);
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

// One step: d = M^-1 r + beta d; alpha; r -= alpha A d with the reductions and the stopping
// test; (P)MINRES2 also delta = z.Az (pcg2.cu:210-216, pminres2.cu:188-197).
static bool enqueue_two_vector_step(bool minres) {
  const double* d = (const double*)S->d0;
  if (!launch_fl2_point(P2_DIR)) return false;
  if (!launch_fl2(minres ? F2_AMA : F2_DAD, d, F2F_ALPHA)) return false;
  if (!launch_fl2(F2_UPD, d, F2F_STEP)) return false;
  if (minres && !launch_fl2(F2_ZAZ, (const double*)S->r, F2F_ZAZ_STEP)) return false;
  return true;
}

static bool build_two_vector_graph(int key, int chunk, bool minres) {
  if (S->gexec && S->graph_key == key) return true;
  if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; }
  cudaGraph_t g;
  CKV(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  bool ok = true;
  const unsigned long long l0 = S->launches;
  for (int it = 0; it < chunk && ok; it++) ok = enqueue_two_vector_step(minres);
  S->launches = l0;
  cudaError_t e = cudaStreamEndCapture(S->stream, &g);
  if (!ok || e != cudaSuccess) { set_err("graph capture", cudaGetErrorString(e)); return false; }
  e = cudaGraphInstantiate(&S->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { set_err("graph instantiate", cudaGetErrorString(e)); return false; }
  S->graph_key = key;
  return true;
}

// The reference sums the reduced solution as it goes and only scales at the end: res[c][k] *=
// scale for every step, then NONE adds the steps up, ONLYDIR / FULL take the last one.
static bool finish_two_vector(double* res_x, bool write_metrics) {
  const unsigned it = (unsigned)S->h_sc->iteration;
  const size_t stride = (size_t)S->maxit + 1;
  const int D = S->fdim;
  std::vector<double> h((size_t)D * (it + 1));
  for (int c = 0; c < D; c++)
    CKV(cudaMemcpyAsync(h.data() + (size_t)c * (it + 1), S->d_hist + c * stride, (it + 1) * 8, cudaMemcpyDeviceToHost, S->stream));
  CKV(cudaStreamSynchronize(S->stream));
  for (double& v : h) v *= S->xr_scale;
  const unsigned shift = std::min(S->xr_shift, (unsigned)D - 1);
  if (write_metrics) {
    const std::string fn = std::string(S->model->name ? S->model->name : "") + "_xreduce_metrics_" + std::to_string(S->count) + ".bin";
    FILE* f = fopen(fn.c_str(), "wb");
    if (f) {
      if (S->xr_mode != CUDAPCG_XREDUCE_ONLYDIR) fwrite(h.data(), sizeof(double), h.size(), f);
      else fwrite(h.data() + (size_t)shift * (it + 1), sizeof(double), it + 1, f);
      fclose(f);
    }
  }
  for (int c = 0; c < D; c++) {
    const double* p = h.data() + (size_t)c * (it + 1);
    if (S->xr_mode == CUDAPCG_XREDUCE_NONE) {
      double s = 0.0;
      for (unsigned k = it + 1; k-- > 0;) s += p[k];  // last step first, like the reference
      res_x[c] = s;
    } else if (S->xr_mode == CUDAPCG_XREDUCE_ONLYDIR) {
      res_x[c] = (unsigned)c == shift ? p[it] : 0.0;
    } else {
      res_x[c] = p[it];
    }
  }
  return true;
}

static bool solve_two_vector(double* res_x) {
  if (!S->fluid) {
    set_err("cudapcgSolve", "the 2-vector solvers (CG2/MINRES2) reduce Stokes velocities; use CG3/MINRES3 for other analyses");
    return false;
  }
  if (!ensure_lean_vectors() || !ensure_K<double>() || !ensure_lean_work()) return false;
  const bool minres = S->solver_flag == CUDAPCG_MINRES2_SOLVER;
  S->cur_sc = S->d_sc;
  if (!ensure_reduction(needed_blocks())) return false;
  CKV(cudaMemsetAsync(S->d_ticket, 0, sizeof(unsigned), S->stream));
  CKV(cudaMemsetAsync(S->d_sc, 0, sizeof(DevScalars), S->stream));
  CKV(cudaEventRecord(S->ev0, S->stream));
  // zero-guess references (pcg2.cu:60-80, pminres2.cu:73-91)
  if (!launch_fl2_point(P2_INIT)) return false;
  if (minres && !launch_fl2(F2_ZAZ, (const double*)S->r, F2F_ZAZ_INIT)) return false;
  if (S->x0_set) {  // the guess is in d (cudapcg.cu:302): r -= A x0, its sums, the guess test
    if (!launch_fl2(F2_X0, (const double*)S->d0, F2F_X0)) return false;
    if (minres && !launch_fl2(F2_ZAZ, (const double*)S->r, F2F_ZAZ_X0)) return false;
  }
  CKV(cudaEventRecord(S->ev1, S->stream));
  const int chunk = std::max(2u, S->iters_per_launch & ~1u);
  const int key = 0x40000000 | (minres ? 0x80 : 0) | (chunk & 0x7f) | (S->resnorm << 16) | (S->precond << 20) | ((int)S->xr_mode << 22) |
                  ((int)std::min(S->xr_shift, (unsigned)S->fdim - 1) << 24) | (S->fdim << 26);
  if (!build_two_vector_graph(key, chunk, minres)) return false;
  const bool trace = getenv("CHFEM_B200_TRACE") != nullptr;
  for (;;) {
    if (!read_scalars()) return false;
    if (trace)
      fprintf(stderr, "[2vec] it %d delta %.6e delta0 %.6e alpha %.6e beta %.6e metric %.6e done %d\n", S->h_sc->iteration, S->h_sc->delta,
              S->h_sc->delta0, S->h_sc->alpha, S->h_sc->beta, S->h_sc->metric, S->h_sc->done);
    if (S->h_sc->done || S->h_sc->status >= 3) break;
    CKV(cudaGraphLaunch(S->gexec, S->stream));
    S->launches += (unsigned long long)chunk * (minres ? 4 : 3);
  }
  CKV(cudaEventRecord(S->ev2, S->stream));
  CKV(cudaEventSynchronize(S->ev2));
  float ms1 = 0, ms2 = 0;
  cudaEventElapsedTime(&ms1, S->ev0, S->ev1);
  cudaEventElapsedTime(&ms2, S->ev1, S->ev2);
  S->setup_dev_s = ms1 * 1e-3;
  S->solve_dev_s = ms2 * 1e-3;
  collect_results(minres);
  // a null right-hand side or an initial guess that already satisfies the test ends before the
  // reference writes its metrics file; the result is then the zero (or the guess's) column
  return finish_two_vector(res_x, S->h_sc->status == 0);
}
