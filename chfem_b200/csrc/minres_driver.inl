// minres_driver.inl -- (P)MINRES launch sequence; included by cudapcg_b200.cu.
// Recurrence of chfem/src/femhmg/cudapcg/solvers/pminres.cu:28-247 (and minres.cu:58-260
// without preconditioner).  Per iteration: the pointwise direction pass finishes alpha, the
// operator pass updates x and r, applies A to z = M^-1 r and finishes delta, beta and the
// stopping test.  r alternates between two buffers (read r, write r'), so chunks are even.

static MrCfg mrcfg() {
  MrCfg cfg;
  const SolveCfg sc = solvecfg();
  cfg.tol = sc.tol; cfg.maxit = sc.maxit; cfg.norm = sc.norm; cfg.precond = sc.precond; cfg.nhmg = sc.nhmg;
  return cfg;
}

// Operator pass of (P)MINRES on explicit buffers: r' = r - alpha q into rout, s = A M^-1 r',
// x += alpha d, with the scalars of S->cur_sc.
template <typename T>
static bool launch_mr_op_buf(const T* rin, T* rout, const T* q, T* s, double* x, const T* d, int fin, bool skip_if_done) {
  const MrCfg cfg = mrcfg();
  if (S->fluid) {
    FlArgs<T> a;
    a.v = rin; a.vd = q; a.vout = rout; a.y = s; a.x = x; a.d = d;
    a.dof_of_node = S->d_dof_of_node; a.node_of_dof = S->d_node_of_dof; a.bkeys = S->d_bkeys;
    a.R = S->R; a.C = S->C; a.L = S->L; a.nV = S->nV; a.nB = S->nB;
    a.sc = S->cur_sc; a.finish = fin; a.skip_if_done = skip_if_done; a.cfg = cfg;
    const int g = pw_grid(S->nV + S->nB);
    if (!ensure_reduction(g)) return false;
    a.rc = redctl(g);
    if (S->fdim == 2) k_fl_apply<T, TE_MR, 2><<<g, FL_NT, 0, S->stream>>>(a);
    else k_fl_apply<T, TE_MR><<<g, FL_NT, 0, S->stream>>>(a);
  } else if (S->dim2) {
    const int nb = d2_ctas();
    if (!ensure_reduction(nb)) return false;
    if (S->nd == 1) {
      TeArgs<1, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, 1, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
      sdf_args(a);
      k_2d_apply<1, T, TE_MR><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<1, T>(), S->stream>>>(a);
    } else {
      TeArgs<2, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, 1, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
      sdf_args(a);
      k_2d_apply<2, T, TE_MR><<<nb, dim3(T2_TR, T2_TC), t2_smem_bytes<2, T>(), S->stream>>>(a);
    }
  } else if (th_applies()) {
    const int nb = th_ctas<T, TE_MR>(S->R, S->C, S->L, num_sms());
    if (nb < 1 || !ensure_reduction(nb)) return false;
    TeArgs<1, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
    const cudaError_t e = th_launch<T, TE_MR>(a, thdev<T>(), nb, S->stream);
    S->launches++;
    if (e != cudaSuccess) { set_err("operator pass", cudaGetErrorString(e)); return false; }
    return true;
  } else if (asm_applies()) {
    int nb;
    cudaError_t e;
    if (S->nd == 1) {
      nb = asm_te_ctas<1, T, TE_MR>(S->R, S->C, S->L, num_sms());
      if (nb < 1 || !ensure_reduction(nb)) return false;
      TeArgs<1, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
      e = asm_te_launch<1, T, TE_MR>(a, tabdev<T>(), nb, S->stream);
    } else {
      nb = asm_te_ctas<3, T, TE_MR>(S->R, S->C, S->L, num_sms());
      if (nb < 1 || !ensure_reduction(nb)) return false;
      TeArgs<3, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat, S->R, S->C, S->L, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
      e = asm_te_launch<3, T, TE_MR>(a, tabdev<T>(), nb, S->stream);
    }
    S->launches++;
    if (e != cudaSuccess) { set_err("operator pass", cudaGetErrorString(e)); return false; }
    return true;
  } else {
    const dim3 block(TE_TR, TE_TC);
    if (S->nd == 1) {
      const size_t sm = te_smem_bytes<1, T>(S->nmat);
      const int nb = te_ctas(k_te_apply<1, T, TE_MR>, sm);
      if (!ensure_reduction(nb)) return false;
      TeArgs<1, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat,
                     S->R, S->C, S->L, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
      sdf_args(a);
      k_te_apply<1, T, TE_MR><<<nb, block, sm, S->stream>>>(a);
    } else {
      const size_t sm = te_smem_bytes<3, T>(S->nmat);
      const int nb = te_ctas(k_te_apply<3, T, TE_MR>, sm);
      if (!ensure_reduction(nb)) return false;
      TeArgs<3, T> a{rin, q, rout, s, x, d, S->d_keys, Kdev<T>(), S->nmat,
                     S->R, S->C, S->L, S->cur_sc, redctl(nb), fin, skip_if_done, cfg};
      sdf_args(a);
      k_te_apply<3, T, TE_MR><<<nb, block, sm, S->stream>>>(a);
    }
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}
template <typename T>
static bool launch_mr_op(const T* rin, T* rout, int fin, bool skip_if_done) {
  return launch_mr_op_buf<T>(rin, rout, (const T*)S->q, (T*)S->s, S->x, (const T*)S->d0, fin, skip_if_done);
}

template <typename T>
static bool launch_mr_dir(const T* rcur) {
  if (S->fluid) {
    const int g = pw_grid(S->nV + S->nB);
    if (!ensure_reduction(g)) return false;
    MrDirFl<T> a{(T*)S->d0, (T*)S->q, rcur, (const T*)S->s, S->d_bkeys, S->nV, S->nB, S->cur_sc, redctl(g), S->precond};
    if (S->fdim == 2) k_fl_mr_dir<T, 2><<<g, PW_NT, 0, S->stream>>>(a);
    else k_fl_mr_dir<T><<<g, PW_NT, 0, S->stream>>>(a);
  } else {
    const int g = pw_grid(S->N);
    if (!ensure_reduction(g)) return false;
    if (S->dim2 && S->nd == 2) {  // 2D elastic: the Jacobi diagonal from invd only
      MrDirTe<2, T> a{(T*)S->d0, (T*)S->q, rcur, (const T*)S->s, S->d_keys, Kdev<T>(), 0, S->N, S->cur_sc, redctl(g), S->precond, S->d_invd};
      k_te_mr_dir<2, T><<<g, PW_NT, 0, S->stream>>>(a);
    } else if (S->nd == 1) {
      MrDirTe<1, T> a{(T*)S->d0, (T*)S->q, rcur, (const T*)S->s, S->d_keys, Kdev<T>(), S->dim2 ? 0 : S->nmat, S->N, S->cur_sc, redctl(g), S->precond, S->d_invd};
      k_te_mr_dir<1, T><<<g, PW_NT, 0, S->stream>>>(a);
    } else {
      MrDirTe<3, T> a{(T*)S->d0, (T*)S->q, rcur, (const T*)S->s, S->d_keys, Kdev<T>(), S->nmat, S->N, S->cur_sc, redctl(g), S->precond, S->d_invd};
      k_te_mr_dir<3, T><<<g, PW_NT, 0, S->stream>>>(a);
    }
  }
  S->launches++;
  return cudaPeekAtLastError() == cudaSuccess;
}

template <typename T>
static bool enqueue_minres_iteration(int parity) {
  const T* rcur = (const T*)(parity ? S->r2 : S->r);
  T* rnext = (T*)(parity ? S->r : S->r2);
  return launch_mr_dir<T>(rcur) && launch_mr_op<T>(rcur, rnext, FIN_MR_STEP, true);
}

template <typename T>
static bool solve_minres_device() {
  if (!ensure_reduction(needed_blocks())) return false;
  CKV(cudaMemsetAsync(S->d_ticket, 0, sizeof(unsigned), S->stream));
  CKV(cudaMemsetAsync(S->cur_sc, 0, sizeof(DevScalars), S->stream));
  const size_t n = (size_t)S->nvars;
  if (!S->x0_set) CKV(cudaMemsetAsync(S->x, 0, n * 8, S->stream));
  CKV(cudaMemsetAsync(S->q, 0, n * sizeof(T), S->stream));
  CKV(cudaMemsetAsync(S->d0, 0, n * sizeof(T), S->stream));
  CKV(cudaEventRecord(S->ev0, S->stream));
  // zero-guess reference (pminres.cu:58-79): res0 = r.M^-1 r, s = A M^-1 r, delta0 = z.s.
  // alpha is 0 here, so r' = r and x is unchanged.
  if (!launch_mr_op<T>((const T*)S->r, (T*)S->r2, FIN_MR_INIT, false)) return false;
  if (S->x0_set) {  // pminres.cu:81-98: r = b - A x0 (FP64 apply), then the same evaluation
    if (!residual_from_x<T>()) return false;
    if (!launch_mr_op<T>((const T*)S->r, (T*)S->r2, FIN_MR_X0, true)) return false;
  }
  CKV(cudaEventRecord(S->ev1, S->stream));
  if (!run_chunks<T>(true)) return false;
  CKV(cudaEventRecord(S->ev2, S->stream));
  CKV(cudaEventSynchronize(S->ev2));
  float ms1 = 0, ms2 = 0;
  cudaEventElapsedTime(&ms1, S->ev0, S->ev1);
  cudaEventElapsedTime(&ms2, S->ev1, S->ev2);
  S->setup_dev_s = ms1 * 1e-3;
  S->solve_dev_s = ms2 * 1e-3;
  return true;
}
