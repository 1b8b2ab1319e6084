// ibfs_adjoint_motion_host.cuh -- host driver of the discrete adjoint of a
// rigidly pitching body (included by ibfs_capi.cu after the stationary
// driver, whose working set, head and tail programs it reuses).
//
// ibfs_adjoint_pitch_run differentiates J = sum_s sum_b (wx[s,b] fx_b^s +
// wy[s,b] fy_b^s) over nsteps advances with respect to the pitch amplitude of
// a single moving case (motion_kind 1, CG force solve, FP64). The amplitude
// enters every step through the body positions X_s (the regularisation
// weights of reg, regT and the force sums) and the body velocities V_s
// (rhsf). The forward step treats the CG solve as exact, so its adjoint is
//   b-hat = A^-T fb-hat,  A = regT M reg,  A^T = regT M^T reg,
// solved by CG with the same kernels on a view of the case whose right-hand
// side is fb-hat and whose solution is b-hat (warm-started from the previous
// step's b-hat), A^T applied with the transposed operators of the stationary
// adjoint. The position derivative needs, per step, fb_s, the flux q1 + q0 at
// each force's faces (captured by the forward rhsf kernel), u = M reg fb_s
// (one forward a_times) and v = M^T reg b-hat (one more A^T application).
// Checkpointing as in the stationary driver, except that each recomputed
// segment runs all of its steps (fb_s of a step is the next slot's fb) and the
// last segment is stored by the forward pass itself.

namespace ibfs {

struct AdjMPlan {
  AdjCase acg{};          // working set of one A^T application
  AdjCase* d_acg = nullptr;
  DevCase vc{};           // the adjoint CG's view of the case: rhsf = aF, fb = aRf
  DevCase* d_vc = nullptr;
  int* d_vit = nullptr;   // the view's iterations / active flag
  const int* d_zero = nullptr;
  double* d_acc = nullptr;    // dJ/d(amplitude, radians)
  double** d_uout = nullptr;  // a_times output (unused; u is the shadow's level-1 flux)
  Prog head, tail, tail_first, cg_start, cg_iter, cg_iter50, fwd_u, tables;
  cudaGraphExec_t g_head = nullptr, g_tail = nullptr, g_tailf = nullptr, g_start = nullptr, g_iter = nullptr,
                  g_iter50 = nullptr, g_u = nullptr;
  bool graphs = false;
};

// out = A^T in (out may be null: then only acg.aZ1 = ainv(M'^T reg in) is
// formed, from which v = curl0(acg.aZ1)).
static void adjm_add_AT(ProgBuilder& B, ibfs_handle* h, AdjMPlan& M, const double* in, double* out) {
  const DevCase& c = h->cases[0].dc;
  const DevCase* dc = h->d_cases;
  const AdjCase& a = M.acg;
  const AdjCase* da = M.d_acg;
  cudaStream_t st = h->st;
  DevCase hc = c;
  double* aW = a.aW;
  size_t wb = sizeof(double) * c.L * c.ns;
  B.add([=]() { cudaMemsetAsync(aW, 0, wb, st); });
  B.add([=]() { adjm_reg_in(dc, da, in, hc, st); }, TAG_CHOL);
  adj_add_v2f(B, dc, da, c, a, 1, 1);
  B.gemm({right_desc(c, a.aW, a.aT1)}, false);
  B.gemm({left_desc(c, a.aT1, a.aT2, EPI_AINV, 1)}, false);
  B.gemm({right_desc(c, a.aT2, a.aT1)}, false);
  B.gemm({left_desc(c, a.aT1, a.aZ1, EPI_STORE, 1)}, false);
  if (out) B.add([=]() { adjm_regT_curl0(dc, da, out, hc, st); }, TAG_CHOL);
}

static int adjm_init(ibfs_handle* h, AdjPlan& P, AdjMPlan& M) {
  const DevCase& c = h->cases[0].dc;
  size_t nsL = (size_t)c.L * c.ns;
  AdjCase& a = M.acg;
  a.aW = dalloc<double>(h, nsL);
  a.aQ1 = dalloc<double>(h, c.nq);
  a.aS = dalloc<double>(h, nsL);
  a.aSbc = dalloc<double>(h, (size_t)c.L * c.nring);
  a.aZ1 = dalloc<double>(h, c.ns);
  a.aT1 = dalloc<double>(h, c.ns);
  a.aT2 = dalloc<double>(h, c.ns);
  M.d_acg = dupload(h, std::vector<AdjCase>{a});
  DevCase& v = M.vc;
  v = c;
  v.rhsf = P.a.aF;
  v.fb = P.a.aRf;
  v.cg_r = dalloc<double>(h, c.nf);
  v.cg_d = dalloc<double>(h, c.nf);
  v.cg_q = dalloc<double>(h, c.nf);
  v.cg_q2 = dalloc<double>(h, c.nf);
  v.cg_sc = dalloc<double>(h, 4);
  M.d_vit = dalloc<int>(h, 2);
  v.cg_it = M.d_vit;
  M.d_vc = dupload(h, std::vector<DevCase>{v});
  M.d_zero = dupload(h, std::vector<int>{0});
  M.d_acc = dalloc<double>(h, 1);
  M.d_uout = dupload(h, std::vector<double*>{dalloc<double>(h, c.nf)});
  if (!a.aW || !a.aQ1 || !a.aS || !a.aSbc || !a.aZ1 || !a.aT1 || !a.aT2 || !M.d_acg || !v.cg_r || !v.cg_d ||
      !v.cg_q || !v.cg_q2 || !v.cg_sc || !M.d_vit || !M.d_vc || !M.d_zero || !M.d_acc || !M.d_uout)
    return set_error(IBFS_ERR_NOMEM, "adjoint allocation failed (moving body)");

  cudaStream_t st = h->st;
  const DevCase* dcases = h->d_cases;
  const DevCase* dvc = M.d_vc;
  const int* d0 = M.d_zero;
  {  // forward quantities of the step being differentiated
    ProgBuilder B{h, M.tables};
    int mnb = h->max_nb, mnf = h->max_nf, mpatch = h->max_patch;
    B.add([=]() { launch_move_body(dcases, d0, 1, mnb, st); });
    B.add([=]() { launch_setup_reg_moving(dcases, d0, 1, mnf, mpatch, st); });
    ProgBuilder Bu{h, M.fwd_u};
    build_atimes(Bu, h, M.d_uout);
  }
  {
    ProgBuilder B{h, M.head};
    adj_build_head(h, P, B);
  }
  {  // CG on A^T (operators.f90:393-441 with A^T for A)
    ProgBuilder Bs{h, M.cg_start};
    adjm_add_AT(Bs, h, M, v.fb, v.cg_q);
    Bs.add([=]() { launch_cg_start(dvc, d0, 1, st); }, TAG_CHOL);
    ProgBuilder Bi{h, M.cg_iter};
    adjm_add_AT(Bi, h, M, v.cg_d, v.cg_q);
    Bi.add([=]() { launch_cg_alpha(dvc, d0, 1, 0, st); }, TAG_CHOL);
    Bi.add([=]() { launch_cg_beta(dvc, d0, 1, st); }, TAG_CHOL);
    ProgBuilder B50{h, M.cg_iter50};
    adjm_add_AT(B50, h, M, v.cg_d, v.cg_q);
    B50.add([=]() { launch_cg_alpha(dvc, d0, 1, 1, st); }, TAG_CHOL);
    adjm_add_AT(B50, h, M, v.fb, v.cg_q2);
    B50.add([=]() { launch_cg_resid(dvc, d0, 1, st); }, TAG_CHOL);
    B50.add([=]() { launch_cg_beta(dvc, d0, 1, st); }, TAG_CHOL);
  }
  for (int first = 0; first < 2; first++) {
    ProgBuilder B{h, first ? M.tail_first : M.tail};
    adjm_add_AT(B, h, M, v.fb, nullptr);
    const AdjCase* da = P.d_a;
    const double* zcg = a.aZ1;
    const double* u = h->shx[0].q;
    double* acc = M.d_acc;
    B.add([=]() { adjm_position(dcases, da, zcg, u, acc, st); });
    adj_build_tail(h, P, B, first);
  }
  int kk = 0;
  M.graphs = capture_one(h, M.head, &M.g_head, &kk) && capture_one(h, M.tail, &M.g_tail, &kk) &&
             capture_one(h, M.tail_first, &M.g_tailf, &kk) && capture_one(h, M.cg_start, &M.g_start, &kk) &&
             capture_one(h, M.cg_iter, &M.g_iter, &kk) && capture_one(h, M.cg_iter50, &M.g_iter50, &kk) &&
             capture_one(h, M.fwd_u, &M.g_u, &kk);
  return IBFS_OK;
}

// b-hat = A^-T fb-hat by CG, replayed in chunks of four iterations like the
// forward solve; returns the iterations used.
static int adjm_solve(ibfs_handle* h, AdjMPlan& M, int maxit, int* iters) {
  auto ex = [&](cudaGraphExec_t g) { return M.graphs ? g : nullptr; };
  int rc = run_prog(h, M.cg_start, ex(M.g_start));
  if (rc) return rc;
  int fl[2] = {0, 0};
  IBFS_CUDA_CHECK(cudaMemcpyAsync(fl, M.d_vit, sizeof(fl), cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  int it = 0;
  while (fl[1] && it < maxit) {
    for (int c = 0; c < 4 && it < maxit; c++) {
      it++;
      rc = (it % 50 == 0) ? run_prog(h, M.cg_iter50, ex(M.g_iter50)) : run_prog(h, M.cg_iter, ex(M.g_iter));
      if (rc) return rc;
    }
    IBFS_CUDA_CHECK(cudaMemcpyAsync(fl, M.d_vit, sizeof(fl), cudaMemcpyDeviceToHost, h->st));
    IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  }
  *iters = fl[0];
  return IBFS_OK;
}

static int adjm_run(ibfs_handle* h, int nsteps, int K, const double* wx, const double* wy, double* J,
                    double* dJdA, double* ms_fwd, double* ms_total) {
  if (h->cases.size() != 1 || !h->cases[0].dc.moving || h->precision != 0 || !h->cg)
    return set_error(IBFS_ERR_ARG, "the pitch adjoint needs a single pitching case (motion_kind 1) in the plain FP64 form");
  if (h->cases[0].dc.nact) return set_error(IBFS_ERR_ARG, "the adjoint does not cover actuator jets");
  if (nsteps < 1 || K < 1 || !wx || !wy || !J || !dJdA) return set_error(IBFS_ERR_ARG, "bad adjoint arguments");
  HostCase& hc = h->cases[0];
  const DevCase& c = hc.dc;
  int rc = IBFS_OK, warn = IBFS_OK;
  if (!h->adj) {
    h->adj = new AdjPlan();
    rc = adj_alloc(h, *h->adj);
    if (rc) return rc;
  }
  AdjPlan& P = *h->adj;
  if (!h->adjm) {
    h->adjm = new AdjMPlan();
    rc = adjm_init(h, P, *h->adjm);
    if (rc) return rc;
  }
  AdjMPlan& M = *h->adjm;
  if (P.h_slots < K) {
    if (P.h_a) cudaFreeHost(P.h_a);
    P.h_a = nullptr;
    if (cudaMallocHost(&P.h_a, sizeof(AdjCase) * K) != cudaSuccess) return set_error(IBFS_ERR_NOMEM, "pinned allocation");
    P.h_slots = K;
  }
  const int nb = c.nbody, nf = c.nf;
  const size_t nf9 = (size_t)nf * 9;
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
      cudaMalloc(&w, sizeof(double) * 2 * nb * (size_t)nsteps) != cudaSuccess ||
      cudaMalloc(&hist, sizeof(double) * h->out_stride * (size_t)nsteps) != cudaSuccess ||
      cudaMalloc(&tqseg, sizeof(double) * nf9 * K) != cudaSuccess ||
      cudaMalloc(&tqcap, sizeof(double) * nf9) != cudaSuccess ||
      cudaMalloc(&ck_it, sizeof(int) * (nck + 1)) != cudaSuccess ||
      cudaMalloc(&its, sizeof(int) * nsteps) != cudaSuccess) {
    cleanup();
    return set_error(IBFS_ERR_NOMEM, "adjoint checkpoint allocation failed");
  }
  std::vector<double> wh(2 * nb * (size_t)nsteps);
  for (int s = 0; s < nsteps; s++)
    for (int b = 0; b < nb; b++) {
      wh[(size_t)s * 2 * nb + b] = wx[(size_t)s * nb + b];
      wh[(size_t)s * 2 * nb + nb + b] = wy[(size_t)s * nb + b];
    }
  cudaMemcpy(w, wh.data(), sizeof(double) * wh.size(), cudaMemcpyHostToDevice);
  const int it0 = hc.itime;
  std::vector<int> ith(nsteps);
  for (int s = 0; s < nsteps; s++) ith[s] = it0 + s + 1;
  cudaMemcpy(its, ith.data(), sizeof(int) * nsteps, cudaMemcpyHostToDevice);
  cudaMemcpy(c.itime, &it0, sizeof(int), cudaMemcpyHostToDevice);
  // the forward rhsf kernel captures (q1 + q0) at the force faces during this run
  DevCase cap = c;
  cap.tq = tqcap;
  cudaMemcpy(h->d_cases, &cap, sizeof(DevCase), cudaMemcpyHostToDevice);
  const size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  auto step = [&]() {
    int r = run_step(h);
    if (r == IBFS_ERR_CG_MAXITER) { warn = r; r = IBFS_OK; }
    return r;
  };
  auto keep = [&](int s, int s0) {  // slot s+1-s0 = state after step s; its captured fluxes
    adj_save(h, seg + P.state * (s + 1 - s0));
    cudaMemcpyAsync(tqseg + nf9 * (s - s0), tqcap, sizeof(double) * nf9, cudaMemcpyDeviceToDevice, h->st);
  };
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
  cudaEventRecord(e0, h->st);
  // 1. forward pass with checkpoints; the last segment is kept whole
  for (int s = 0; s < nsteps && rc == IBFS_OK; s++) {
    if (s % K == 0) {
      adj_save(h, ck + P.state * (s / K));
      cudaMemcpyAsync(ck_it + s / K, c.itime, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
    }
    if (s == s0_last) adj_save(h, seg);
    rc = step();
    cudaMemcpyAsync(hist + (size_t)s * h->out_stride, h->d_out, sizeof(double) * h->out_stride,
                    cudaMemcpyDeviceToDevice, h->st);
    if (s >= s0_last) keep(s, s0_last);
  }
  adj_save(h, fin);
  cudaMemcpyAsync(ck_it + nck, c.itime, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
  cudaEventRecord(e1, h->st);
  std::vector<double> hh((size_t)h->out_stride * nsteps);
  cudaMemcpyAsync(hh.data(), hist, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, h->st);
  cudaStreamSynchronize(h->st);
  double jj = 0.0;
  for (int s = 0; s < nsteps; s++)
    for (int b = 0; b < nb; b++)
      jj += wx[(size_t)s * nb + b] * hh[(size_t)s * h->out_stride + b] +
            wy[(size_t)s * nb + b] * hh[(size_t)s * h->out_stride + nb + b];
  *J = jj;
  // 2. backward pass
  const AdjCase& a = P.a;
  cudaMemsetAsync(a.aW, 0, nsL * 8, h->st);
  cudaMemsetAsync(a.aP, 0, nsL * 8, h->st);
  cudaMemsetAsync(a.aQ, 0, nqL * 8, h->st);
  cudaMemsetAsync(a.aGrad, 0, (size_t)nf * 8, h->st);
  cudaMemsetAsync(a.aRf, 0, (size_t)nf * 8, h->st);
  cudaMemsetAsync(M.d_acc, 0, sizeof(double), h->st);
  auto ex = [&](cudaGraphExec_t g) { return M.graphs ? g : nullptr; };
  const int maxit = hc.p.cg_max_iter;
  int max_adj_iters = 0;
  for (int sg = nck - 1; sg >= 0 && rc == IBFS_OK; sg--) {
    const int s0 = sg * K, s1 = std::min(nsteps, s0 + K);
    cudaStreamSynchronize(h->st);  // the pinned slots of the previous segment are free
    if (sg != nck - 1) {
      cudaMemcpyAsync(seg, ck + P.state * sg, sizeof(double) * P.state, cudaMemcpyDeviceToDevice, h->st);
      adj_restore(h, ck + P.state * sg);
      cudaMemcpyAsync(c.itime, ck_it + sg, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
      for (int s = s0; s < s1 && rc == IBFS_OK; s++) {
        rc = step();
        keep(s, s0);
      }
    }
    for (int s = s1 - 1; s >= s0 && rc == IBFS_OK; s--) {
      // positions, tables, fb and u of step s
      cudaMemcpyAsync(c.itime, its + s, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
      rc = run_prog(h, M.tables, nullptr);
      if (rc) break;
      cudaMemcpyAsync(c.fb, seg + P.state * (s + 1 - s0) + 2 * nsL + nqL, sizeof(double) * nf,
                      cudaMemcpyDeviceToDevice, h->st);
      rc = run_prog(h, M.fwd_u, ex(M.g_u));
      if (rc) break;
      const double* stp = seg + P.state * (s - s0);
      AdjCase cur = a;
      cur.fwW = stp;
      cur.fwQ = stp + 2 * nsL;
      cur.wx = w + (size_t)s * 2 * nb;
      cur.wy = cur.wx + nb;
      cur.tq = tqseg + nf9 * (s - s0);
      AdjCase* slot = P.h_a + (s - s0);
      *slot = cur;
      cudaMemcpyAsync(P.d_a, slot, sizeof(AdjCase), cudaMemcpyHostToDevice, h->st);
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
  adj_restore(h, fin);
  cudaMemcpyAsync(c.itime, ck_it + nck, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
  cudaEventRecord(e2, h->st);
  double acc = 0.0;
  cudaMemcpyAsync(&acc, M.d_acc, sizeof(double), cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  cudaMemcpy(h->d_cases, &c, sizeof(DevCase), cudaMemcpyHostToDevice);  // capture off
  float f1 = 0.f, f2 = 0.f;
  cudaEventElapsedTime(&f1, e0, e1);
  cudaEventElapsedTime(&f2, e0, e2);
  if (ms_fwd) *ms_fwd = f1;
  if (ms_total) *ms_total = f2;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
  cleanup();
  hc.itime = it0 + nsteps;
  h->last_cg_iters = max_adj_iters;
  *dJdA = acc * (M_PI / 180.0);  // per degree of amplitude
  if (rc) return rc;
  if (e != cudaSuccess) return fail_cuda(e, "pitch adjoint run");
  if (warn) return fail(warn, "WARNING!! CJGR used max iterations!");
  return IBFS_OK;
}

}  // namespace ibfs
