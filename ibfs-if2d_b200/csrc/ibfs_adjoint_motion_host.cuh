// ibfs_adjoint_motion_host.cuh -- host driver of the discrete adjoint of
// rigidly pitching bodies (included by ibfs_capi.cu after the stationary
// driver, whose working sets, head and tail programs it reuses).
//
// ibfs_adjoint_pitch_run differentiates, for every case c of a handle whose
// cases all pitch (motion_kind 1, CG force solve, FP64),
// J_c = sum_s sum_b (wx[c,s,b] fx_b^s + wy[c,s,b] fy_b^s) over nsteps advances
// with respect to that case's pitch amplitude. All cases are differentiated
// together, one slot each: the forward pass is the handle's batched advance,
// and every stage of the backward step is one launch over all slots.
//
// The amplitude enters every step through the body positions X_s (the
// regularisation weights of reg, regT and the force sums) and the body
// velocities V_s (rhsf). The forward step treats the CG solve as exact, so its
// adjoint is
//   b-hat = A^-T fb-hat,  A = regT M reg,  A^T = regT M^T reg,
// solved by CG with the same kernels on views of the cases whose right-hand
// side is fb-hat and whose solution is b-hat (warm-started from the previous
// step's b-hat; converged slots idle; preconditioned like the forward solve
// when the case is, the preconditioner being symmetric), A^T applied with the transposed
// operators of the stationary adjoint. The position derivative needs, per
// step, fb_s, the flux q1 + q0 at each force's faces (captured by the forward
// rhsf kernel), u = M reg fb_s (one forward a_times) and v = M^T reg b-hat
// (one more A^T application). Checkpointing as in the stationary driver,
// except that each recomputed segment runs all of its steps (fb_s of a step is
// the next slot's fb) and the last segment is stored by the forward pass.

namespace ibfs {

struct AdjMPlan {
  std::vector<AdjCase> acg;  // per-slot working sets of one A^T application
  AdjCase* d_acg = nullptr;
  AdjGroup gcg;              // the plan's slots over acg
  double* blk_acgW = nullptr;
  size_t n_acgW = 0;
  std::vector<DevCase> vc;   // per-slot CG views: rhsf = aF, fb = aRf
  DevCase* d_vc = nullptr;
  int* d_vit = nullptr;      // [n][2] the views' iterations / active flags
  const int* d_iota = nullptr;
  double* d_acc = nullptr;   // [n] dJ/d(amplitude, radians)
  double** d_uout = nullptr;  // a_times outputs (unused; u is the shadows' level-1 flux)
  const double* const* d_xs_fb = nullptr;
  const double* const* d_xs_d = nullptr;
  double* const* d_out_q = nullptr;
  double* const* d_out_q2 = nullptr;
  const double* const* d_us = nullptr;
  Prog head, tail, tail_first, cg_start, cg_iter, cg_iter50, fwd_u, tables;
  cudaGraphExec_t g_head = nullptr, g_tail = nullptr, g_tailf = nullptr, g_start = nullptr, g_iter = nullptr,
                  g_iter50 = nullptr, g_u = nullptr;
  bool graphs = false;
};

// outs[i] = A^T xs[i] for every slot (outs may be null: then only
// acg.aZ1 = ainv(V^T curl^T reg xs) is formed, from which v = curl0(acg.aZ1)).
static void adjm_add_AT(ProgBuilder& B, ibfs_handle* h, const std::vector<int>& cids, AdjMPlan& M,
                        const double* const* xs, double* const* outs) {
  cudaStream_t st = h->st;
  const AdjGroup g = M.gcg;
  double* w = M.blk_acgW;
  size_t wb = sizeof(double) * M.n_acgW;
  B.add([=]() { cudaMemsetAsync(w, 0, wb, st); });
  B.add([=]() { adjm_reg_in(g, xs, st); }, TAG_CHOL);
  adj_add_v2f(B, h, cids, M.acg, g, 1, 1);
  adj_add_ainv(B, h, cids, M.acg);
  if (outs) B.add([=]() { adjm_regT_curl0(g, outs, st); }, TAG_CHOL);
}

static int adjm_init(ibfs_handle* h, AdjPlan& P, AdjMPlan& M) {
  const std::vector<int>& cids = P.cids;
  const int n = (int)cids.size();
  M.acg.assign(n, AdjCase{});
  auto ns = [](const DevCase& c) { return (size_t)c.ns; };
  auto nsL = [](const DevCase& c) { return (size_t)c.L * c.ns; };
  auto nq = [](const DevCase& c) { return (size_t)c.nq; };
  auto ringL = [](const DevCase& c) { return (size_t)c.L * c.nring; };
  bool ok = true;
  ok = ok && (M.blk_acgW = alloc_family(h, cids, M.acg, &AdjCase::aW, nsL, &M.n_acgW));
  ok = ok && alloc_family(h, cids, M.acg, &AdjCase::aQ1, nq);
  ok = ok && alloc_family(h, cids, M.acg, &AdjCase::aS, nsL);
  ok = ok && alloc_family(h, cids, M.acg, &AdjCase::aSbc, ringL);
  for (double* AdjCase::*f : {&AdjCase::aZ1, &AdjCase::aT1, &AdjCase::aT2}) ok = ok && alloc_family(h, cids, M.acg, f, ns);
  M.d_acg = dupload(h, M.acg);
  M.d_vit = dalloc<int>(h, 2 * n);
  ok = ok && M.d_acg && M.d_vit;
  std::vector<const double*> xs_fb, xs_d, us;
  std::vector<double*> out_q, out_q2, uout;
  std::vector<int> iota;
  M.vc.clear();
  for (int i = 0; i < n && ok; i++) {
    DevCase v = slot_case(h, cids, i);
    v.rhsf = P.a[i].aF;
    v.fb = P.a[i].aRf;
    v.cg_r = dalloc<double>(h, v.nf);
    v.cg_d = dalloc<double>(h, v.nf);
    v.cg_q = dalloc<double>(h, v.nf);
    v.cg_q2 = dalloc<double>(h, v.nf);
    v.cg_z = dalloc<double>(h, v.nf);
    v.cg_y = dalloc<double>(h, v.nf);
    v.cg_sc = dalloc<double>(h, 5);
    v.cg_it = M.d_vit + 2 * i;
    ok = v.cg_r && v.cg_d && v.cg_q && v.cg_q2 && v.cg_z && v.cg_y && v.cg_sc;
    M.vc.push_back(v);
    xs_fb.push_back(v.fb);
    xs_d.push_back(v.cg_d);
    out_q.push_back(v.cg_q);
    out_q2.push_back(v.cg_q2);
    us.push_back(h->shx[i].q);  // the shadows follow the CG cases, here every case in order
    uout.push_back(dalloc<double>(h, v.nf));
    iota.push_back(i);
  }
  if (!ok) return set_error(IBFS_ERR_NOMEM, "adjoint allocation failed (moving body)");
  M.d_vc = dupload(h, M.vc);
  M.d_iota = dupload(h, iota);
  M.d_acc = dalloc<double>(h, n);
  M.d_uout = dupload(h, uout);
  M.d_xs_fb = dupload(h, xs_fb);
  M.d_xs_d = dupload(h, xs_d);
  M.d_out_q = dupload(h, out_q);
  M.d_out_q2 = dupload(h, out_q2);
  M.d_us = dupload(h, us);
  if (!M.d_vc || !M.d_iota || !M.d_acc || !M.d_uout || !M.d_xs_fb || !M.d_xs_d || !M.d_out_q || !M.d_out_q2 || !M.d_us)
    return set_error(IBFS_ERR_NOMEM, "adjoint allocation failed (moving body)");
  M.gcg = make_group(h, cids, P.d_cids, M.d_acg);

  cudaStream_t st = h->st;
  const DevCase* dcases = h->d_cases;
  const DevCase* dvc = M.d_vc;
  const int* dio = M.d_iota;
  const int* dci = P.d_cids;
  {  // forward quantities of the step being differentiated
    ProgBuilder B{h, M.tables};
    int mnb = h->max_nb, mnf = h->max_nf, mpatch = h->max_patch;
    B.add([=]() { launch_move_body(dcases, dci, n, mnb, st); });
    B.add([=]() { launch_setup_reg_moving(dcases, dci, n, mnf, mpatch, st); });
    ProgBuilder Bu{h, M.fwd_u};
    build_atimes(Bu, h, M.d_uout);
  }
  {
    ProgBuilder B{h, M.head};
    adj_build_head(h, P, B);
  }
  {  // CG on A^T (operators.f90:393-441 with A^T for A)
    ProgBuilder Bs{h, M.cg_start};
    adjm_add_AT(Bs, h, cids, M, M.d_xs_fb, M.d_out_q);
    Bs.add([=]() { launch_cg_start(dvc, dio, n, st); }, TAG_CHOL);
    ProgBuilder Bi{h, M.cg_iter};
    adjm_add_AT(Bi, h, cids, M, M.d_xs_d, M.d_out_q);
    Bi.add([=]() { launch_cg_alpha(dvc, dio, n, 0, st); }, TAG_CHOL);
    Bi.add([=]() { launch_cg_beta(dvc, dio, n, st); }, TAG_CHOL);
    ProgBuilder B50{h, M.cg_iter50};
    adjm_add_AT(B50, h, cids, M, M.d_xs_d, M.d_out_q);
    B50.add([=]() { launch_cg_alpha(dvc, dio, n, 1, st); }, TAG_CHOL);
    adjm_add_AT(B50, h, cids, M, M.d_xs_fb, M.d_out_q2);
    B50.add([=]() { launch_cg_resid(dvc, dio, n, st); }, TAG_CHOL);
    B50.add([=]() { launch_cg_beta(dvc, dio, n, st); }, TAG_CHOL);
  }
  for (int first = 0; first < 2; first++) {
    ProgBuilder B{h, first ? M.tail_first : M.tail};
    adjm_add_AT(B, h, cids, M, M.d_xs_fb, nullptr);
    const AdjGroup g = P.g;
    const AdjCase* acg = M.d_acg;
    const double* const* us_ = M.d_us;
    double* acc = M.d_acc;
    B.add([=]() { adjm_position(g, acg, us_, acc, st); });
    adj_build_tail(h, P, B, first);
  }
  int kk = 0;
  M.graphs = capture_one(h, M.head, &M.g_head, &kk) && capture_one(h, M.tail, &M.g_tail, &kk) &&
             capture_one(h, M.tail_first, &M.g_tailf, &kk) && capture_one(h, M.cg_start, &M.g_start, &kk) &&
             capture_one(h, M.cg_iter, &M.g_iter, &kk) && capture_one(h, M.cg_iter50, &M.g_iter50, &kk) &&
             capture_one(h, M.fwd_u, &M.g_u, &kk);
  return IBFS_OK;
}

// b-hat = A^-T fb-hat by CG for every slot, replayed in chunks of four
// iterations like the forward solve until no slot is active; returns the
// largest iteration count.
static int adjm_solve(ibfs_handle* h, AdjMPlan& M, int maxit, int* iters) {
  auto ex = [&](cudaGraphExec_t g) { return M.graphs ? g : nullptr; };
  const int n = (int)M.vc.size();
  int rc = run_prog(h, M.cg_start, ex(M.g_start));
  if (rc) return rc;
  std::vector<int> fl(2 * n);
  auto poll = [&]() -> int {
    IBFS_CUDA_CHECK(cudaMemcpyAsync(fl.data(), M.d_vit, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost, h->st));
    IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
    return IBFS_OK;
  };
  auto any = [&]() {
    for (int i = 0; i < n; i++)
      if (fl[2 * i + 1]) return true;
    return false;
  };
  if ((rc = poll())) return rc;
  int it = 0;
  while (any() && it < maxit) {
    for (int c = 0; c < 4 && it < maxit; c++) {
      it++;
      rc = (it % 50 == 0) ? run_prog(h, M.cg_iter50, ex(M.g_iter50)) : run_prog(h, M.cg_iter, ex(M.g_iter));
      if (rc) return rc;
    }
    if ((rc = poll())) return rc;
  }
  *iters = 0;
  for (int i = 0; i < n; i++) *iters = std::max(*iters, fl[2 * i]);
  return IBFS_OK;
}

static int adjm_run(ibfs_handle* h, int nsteps, int K, const double* wx, const double* wy, double* J,
                    double* dJdA, double* ms_fwd, double* ms_total) {
  const int n = (int)h->cases.size();
  if (h->precision != 0 || !h->cg || (int)h->cg_ids.size() != n)
    return set_error(IBFS_ERR_ARG, "the pitch adjoint needs pitching cases (motion_kind 1) only, in the plain FP64 form");
  for (int i = 0; i < n; i++) {
    const HostCase& c = h->cases[i];
    if (!c.dc.moving || h->cg_ids[i] != i)
      return set_error(IBFS_ERR_ARG, "the pitch adjoint needs pitching cases (motion_kind 1) only, in the plain FP64 form");
    if (c.dc.nact) return set_error(IBFS_ERR_ARG, "the adjoint does not cover actuator jets");
    if (c.itime != h->cases[0].itime) return set_error(IBFS_ERR_ARG, "the pitch adjoint needs every case at the same step");
  }
  if (nsteps < 1 || K < 1 || !wx || !wy || !J || !dJdA) return set_error(IBFS_ERR_ARG, "bad adjoint arguments");
  int rc = precompute(h), warn = IBFS_OK;  // the preconditioners' factors, if any
  if (rc) return rc;
  if (!h->adj) {
    std::vector<int> all(n);
    for (int i = 0; i < n; i++) all[i] = i;
    h->adj = new AdjPlan();
    rc = adj_alloc(h, *h->adj, all);
    if (rc) return rc;
  }
  AdjPlan& P = *h->adj;
  if (!h->adjm) {
    h->adjm = new AdjMPlan();
    rc = adjm_init(h, P, *h->adjm);
    if (rc) return rc;
  }
  AdjMPlan& M = *h->adjm;
  if ((rc = adj_staging(P, K))) return rc;
  // per-slot layout of the weights, the captured fluxes and the outputs
  std::vector<size_t> woff(n), tqoff(n);
  size_t wtot = 0, tqtot = 0;
  for (int i = 0; i < n; i++) {
    const DevCase& c = h->cases[i].dc;
    woff[i] = wtot;
    wtot += 2 * (size_t)c.nbody * nsteps;
    tqoff[i] = tqtot;
    tqtot += (size_t)c.nf * 9;
  }
  const int nck = (nsteps + K - 1) / K;
  const int s0_last = (nck - 1) * K;
  double *ck = nullptr, *seg = nullptr, *fin = nullptr, *w = nullptr, *hist = nullptr, *tqseg = nullptr,
         *tqcap = nullptr;
  int *ck_it = nullptr, *its = nullptr;
  auto cleanup = [&]() {
    cudaFree(ck); cudaFree(seg); cudaFree(fin); cudaFree(w); cudaFree(hist); cudaFree(tqseg); cudaFree(tqcap);
    cudaFree(ck_it); cudaFree(its);
  };
  if (cudaMalloc(&ck, sizeof(double) * P.state * nck) != cudaSuccess ||
      cudaMalloc(&seg, sizeof(double) * P.state * (K + 1)) != cudaSuccess ||
      cudaMalloc(&fin, sizeof(double) * P.state) != cudaSuccess ||
      cudaMalloc(&w, sizeof(double) * wtot) != cudaSuccess ||
      cudaMalloc(&hist, sizeof(double) * h->out_stride * (size_t)nsteps) != cudaSuccess ||
      cudaMalloc(&tqseg, sizeof(double) * tqtot * K) != cudaSuccess ||
      cudaMalloc(&tqcap, sizeof(double) * tqtot) != cudaSuccess ||
      cudaMalloc(&ck_it, sizeof(int) * (nck + 1)) != cudaSuccess ||
      cudaMalloc(&its, sizeof(int) * nsteps) != cudaSuccess) {
    cleanup();
    return set_error(IBFS_ERR_NOMEM, "adjoint checkpoint allocation failed");
  }
  // weights: case-major input [c][s][b] -> device [c][s][fx b | fy b]
  std::vector<double> wh(wtot);
  size_t win = 0;
  for (int i = 0; i < n; i++) {
    const int nb = h->cases[i].dc.nbody;
    for (int s = 0; s < nsteps; s++)
      for (int b = 0; b < nb; b++) {
        wh[woff[i] + (size_t)s * 2 * nb + b] = wx[win + (size_t)s * nb + b];
        wh[woff[i] + (size_t)s * 2 * nb + nb + b] = wy[win + (size_t)s * nb + b];
      }
    win += (size_t)nsteps * nb;
  }
  cudaMemcpy(w, wh.data(), sizeof(double) * wtot, cudaMemcpyHostToDevice);
  const int it0 = h->cases[0].itime;
  std::vector<int> ith(nsteps);
  for (int s = 0; s < nsteps; s++) ith[s] = it0 + s + 1;
  cudaMemcpy(its, ith.data(), sizeof(int) * nsteps, cudaMemcpyHostToDevice);
  // the forward rhsf kernel captures (q1 + q0) at the force faces during this run
  for (int i = 0; i < n; i++) {
    DevCase cap = h->cases[i].dc;
    cap.tq = tqcap + tqoff[i];
    cudaMemcpy(h->d_cases + i, &cap, sizeof(DevCase), cudaMemcpyHostToDevice);
    cudaMemcpy(h->cases[i].dc.itime, &it0, sizeof(int), cudaMemcpyHostToDevice);
  }
  const DevCase& c0 = h->cases[0].dc;  // every case's step counter holds the same value
  auto set_itime = [&](const int* src) {
    for (int i = 0; i < n; i++)
      cudaMemcpyAsync(h->cases[i].dc.itime, src, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
  };
  auto step = [&]() {
    int r = run_step(h);
    if (r == IBFS_ERR_CG_MAXITER) { warn = r; r = IBFS_OK; }
    return r;
  };
  auto keep = [&](int s, int s0) {  // slot s+1-s0 = state after step s; its captured fluxes
    adj_save(h, P, seg + P.state * (s + 1 - s0));
    cudaMemcpyAsync(tqseg + tqtot * (s - s0), tqcap, sizeof(double) * tqtot, cudaMemcpyDeviceToDevice, h->st);
  };
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
  cudaEventRecord(e0, h->st);
  // 1. forward pass with checkpoints; the last segment is kept whole
  for (int s = 0; s < nsteps && rc == IBFS_OK; s++) {
    if (s % K == 0) {
      adj_save(h, P, ck + P.state * (s / K));
      cudaMemcpyAsync(ck_it + s / K, c0.itime, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
    }
    if (s == s0_last) adj_save(h, P, seg);
    rc = step();
    cudaMemcpyAsync(hist + (size_t)s * h->out_stride, h->d_out, sizeof(double) * h->out_stride,
                    cudaMemcpyDeviceToDevice, h->st);
    if (s >= s0_last) keep(s, s0_last);
  }
  adj_save(h, P, fin);
  cudaMemcpyAsync(ck_it + nck, c0.itime, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
  cudaEventRecord(e1, h->st);
  std::vector<double> hh((size_t)h->out_stride * nsteps);
  cudaMemcpyAsync(hh.data(), hist, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, h->st);
  cudaStreamSynchronize(h->st);
  win = 0;
  for (int i = 0; i < n; i++) {
    const HostCase& c = h->cases[i];
    const int nb = c.nbody;
    double jj = 0.0;
    for (int s = 0; s < nsteps; s++)
      for (int b = 0; b < nb; b++)
        jj += wx[win + (size_t)s * nb + b] * hh[(size_t)s * h->out_stride + c.out_off + b] +
              wy[win + (size_t)s * nb + b] * hh[(size_t)s * h->out_stride + c.out_off + nb + b];
    J[i] = jj;
    win += (size_t)nsteps * nb;
  }
  // 2. backward pass
  cudaMemsetAsync(P.blk_W, 0, P.n_W * 8, h->st);
  cudaMemsetAsync(P.blk_P, 0, P.n_W * 8, h->st);
  cudaMemsetAsync(P.blk_Q, 0, P.n_Q * 8, h->st);
  cudaMemsetAsync(P.blk_Grad, 0, P.n_F * 8, h->st);
  cudaMemsetAsync(P.blk_Rf, 0, P.n_F * 8, h->st);
  cudaMemsetAsync(M.d_acc, 0, sizeof(double) * n, h->st);
  auto ex = [&](cudaGraphExec_t g) { return M.graphs ? g : nullptr; };
  int maxit = 0;
  for (auto& c : h->cases) maxit = std::max(maxit, c.p.cg_max_iter);
  int max_adj_iters = 0;
  for (int sg = nck - 1; sg >= 0 && rc == IBFS_OK; sg--) {
    const int s0 = sg * K, s1 = std::min(nsteps, s0 + K);
    cudaStreamSynchronize(h->st);  // the pinned slots of the previous segment are free
    if (sg != nck - 1) {
      cudaMemcpyAsync(seg, ck + P.state * sg, sizeof(double) * P.state, cudaMemcpyDeviceToDevice, h->st);
      adj_restore(h, P, ck + P.state * sg);
      set_itime(ck_it + sg);
      for (int s = s0; s < s1 && rc == IBFS_OK; s++) {
        rc = step();
        keep(s, s0);
      }
    }
    for (int s = s1 - 1; s >= s0 && rc == IBFS_OK; s--) {
      // preconditioner slot, positions, tables, fb and u of step s
      set_itime(its + s);
      rc = ensure_precond(h, 0);
      if (rc) break;
      rc = run_prog(h, M.tables, nullptr);
      if (rc) break;
      const double* after = seg + P.state * (s + 1 - s0);
      for (int i = 0; i < n; i++) {
        const DevCase& c = h->cases[i].dc;
        size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
        cudaMemcpyAsync(c.fb, after + P.soff[i] + 2 * nsL + nqL, sizeof(double) * c.nf, cudaMemcpyDeviceToDevice,
                        h->st);
      }
      rc = run_prog(h, M.fwd_u, ex(M.g_u));
      if (rc) break;
      const double* stp = seg + P.state * (s - s0);
      AdjCase* slots = P.h_a + (size_t)(s - s0) * n;
      for (int i = 0; i < n; i++) {
        const DevCase& c = h->cases[i].dc;
        AdjCase cur = P.a[i];
        cur.fwW = stp + P.soff[i];
        cur.fwQ = cur.fwW + 2 * (size_t)c.L * c.ns;
        cur.wx = w + woff[i] + (size_t)s * 2 * c.nbody;
        cur.wy = cur.wx + c.nbody;
        cur.tq = tqseg + tqtot * (s - s0) + tqoff[i];
        slots[i] = cur;
      }
      cudaMemcpyAsync(P.d_a, slots, sizeof(AdjCase) * n, cudaMemcpyHostToDevice, h->st);
      rc = run_prog(h, M.head, ex(M.g_head));
      if (rc) break;
      int iters = 0;
      rc = adjm_solve(h, M, maxit, &iters);
      if (rc) break;
      max_adj_iters = std::max(max_adj_iters, iters);
      if (iters >= maxit) warn = IBFS_ERR_CG_MAXITER;
      bool first = it0 + s + 1 == 1;
      rc = first ? run_prog(h, M.tail_first, ex(M.g_tailf)) : run_prog(h, M.tail, ex(M.g_tail));
    }
  }
  adj_restore(h, P, fin);
  set_itime(ck_it + nck);
  cudaEventRecord(e2, h->st);
  std::vector<double> acc(n);
  cudaMemcpyAsync(acc.data(), M.d_acc, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  for (int i = 0; i < n; i++)  // capture off
    cudaMemcpy(h->d_cases + i, &h->cases[i].dc, sizeof(DevCase), cudaMemcpyHostToDevice);
  float f1 = 0.f, f2 = 0.f;
  cudaEventElapsedTime(&f1, e0, e1);
  cudaEventElapsedTime(&f2, e0, e2);
  if (ms_fwd) *ms_fwd = f1;
  if (ms_total) *ms_total = f2;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
  cleanup();
  for (auto& c : h->cases) c.itime = it0 + nsteps;
  h->last_cg_iters = max_adj_iters;
  for (int i = 0; i < n; i++) dJdA[i] = acc[i] * (M_PI / 180.0);  // per degree of amplitude
  if (rc) return rc;
  if (e != cudaSuccess) return fail_cuda(e, "pitch adjoint run");
  if (warn) return fail(warn, "WARNING!! CJGR used max iterations!");
  return IBFS_OK;
}

}  // namespace ibfs
