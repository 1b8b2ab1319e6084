// ibfs_adjoint_host.cuh -- host driver of the discrete adjoint (included by
// ibfs_capi.cu, whose program-building helpers it uses).
//
// ibfs_adjoint_run differentiates J = sum_s sum_b (wx[s,b] fx_b^s + wy[s,b] fy_b^s)
// over nsteps advances (write_force outputs) with respect to a body-velocity
// vector held constant over the run, for a single stationary case in FP64:
//   1. forward pass from the current state, storing a checkpoint of the state
//      (omega, rhs_old, q, fb, itime) every K steps and the forces of every step;
//   2. backward pass, segment by segment from the last: restore the segment's
//      checkpoint, recompute its K steps storing each step-start state, then
//      run the adjoint step backwards through the segment.
// The adjoint step is one fixed launch program (captured as a CUDA graph);
// per step only the pointers to the stored forward state and the objective
// weights change, uploaded into the device AdjCase before each replay.

namespace ibfs {

struct AdjPlan {
  AdjCase a{};
  AdjCase* d_a = nullptr;
  AdjCase* h_a = nullptr;  // pinned staging of the per-step AdjCase, one slot per segment step
  int h_slots = 0;
  Prog bw, bw_first;
  cudaGraphExec_t g_bw = nullptr, g_bwf = nullptr;
  bool graphs = false;
  size_t state = 0;  // doubles per stored state
};

static void adj_add_ctci(ProgBuilder& B, const DevCase& c, const double* in, double* out, double* t1, double* t2) {
  B.gemm({right_desc(c, in, t1)}, false);
  B.gemm({left_desc(c, t1, t2, EPI_LAMINV, 1)}, false);
  B.gemm({right_desc(c, t2, t1)}, false);
  B.gemm({left_desc(c, t1, out, EPI_STORE, 1)}, false);
}

// Adjoint of vort2flux(vel, omega, nlev) (operators.f90:191-240): incoming
// adjoints of the fluxes (aQ, or aQ1 for nlev = 1) and of the coarsified
// omega (aW); aW becomes the adjoint of the omega passed in.
static void adj_add_v2f(ProgBuilder& B, const DevCase* dc, const AdjCase* da, const DevCase& c, const AdjCase& a,
                        int nlev, int use_q1) {
  cudaStream_t st = B.h->st;
  DevCase hc = c;
  B.add([=]() { adj_curlT(dc, da, hc, nlev, use_q1, st); });
  for (int k = 1; k <= c.L; k++) {
    adj_add_ctci(B, c, a.aS + (size_t)(k - 1) * c.ns, a.aZ1, a.aT1, a.aT2);
    B.add([=]() { adj_v2f_level(dc, da, hc, k, st); });
    if (k < c.L) {
      const double* ring = a.aSbc + (size_t)(k - 1) * c.nring;
      double* dst = a.aS + (size_t)k * c.ns;
      B.add([=]() { adj_getbcT(dc, ring, dst, hc, 1.0, st); });
    }
  }
  for (int k = c.L; k >= 2; k--) B.add([=]() { adj_coarsifyT(dc, da, hc, k, st); });
}

// Adjoint step, first part: steps (7) and (6) of the forward step run
// backwards, ending with the adjoint of fb (aF).
static void adj_build_head(ibfs_handle* h, AdjPlan& P, ProgBuilder& B) {
  const DevCase& c = h->cases[0].dc;
  const DevCase* dc = h->d_cases;
  const AdjCase& a = P.a;
  const AdjCase* da = P.d_a;
  cudaStream_t st = h->st;
  DevCase hc = c;
  double* aLb = a.aLb;
  size_t lbb = sizeof(double) * c.L * c.nring;
  B.add([=]() { cudaMemsetAsync(aLb, 0, lbb, st); });
  // (7) vort2flux(q, omega, L), operators.f90:177
  adj_add_v2f(B, dc, da, c, a, c.L, 0);
  // (6) omega_1 -= ainv(rot(reg(fb))), operators.f90:174
  B.gemm({right_desc(c, a.aW, a.aT1)}, false);
  B.gemm({left_desc(c, a.aT1, a.aT2, EPI_AINV, 1)}, false);
  B.gemm({right_desc(c, a.aT2, a.aT1)}, false);
  B.gemm({left_desc(c, a.aT1, a.aZ1, EPI_STORE, 1)}, false);
  B.add([=]() { adj_force(dc, da, hc, st); });
}

// Adjoint step, last part: from the adjoint of rhsf (aRf) through steps (4)
// to (1).
static void adj_build_tail(ibfs_handle* h, AdjPlan& P, ProgBuilder& B, int first) {
  const DevCase& c = h->cases[0].dc;
  const DevCase* dc = h->d_cases;
  const AdjCase& a = P.a;
  const AdjCase* da = P.d_a;
  cudaStream_t st = h->st;
  DevCase hc = c;
  size_t nsL = (size_t)c.L * c.ns;
  // (4) rhsf = regT(q_1) - motion
  B.add([=]() { adj_rhsf(dc, da, hc, st); });
  // (3) vort2flux(q(:,1), omega, 1), operators.f90:163
  adj_add_v2f(B, dc, da, c, a, 1, 1);
  // (2) level loop k = L..1 run backwards (operators.f90:103-134)
  double* aW2 = a.aW2;
  B.add([=]() { cudaMemsetAsync(aW2, 0, sizeof(double) * nsL, st); });
  for (int k = 1; k <= c.L; k++) {
    double* Wk = a.aW + (size_t)(k - 1) * c.ns;
    B.gemm({right_desc(c, Wk, a.aT1)}, false);
    GemmDesc dd = left_desc(c, a.aT1, a.aZ1, EPI_ADJ_CN, k);
    dd.C2 = a.aZ2;
    B.gemm({dd}, false);
    B.gemm({right_desc(c, a.aZ1, a.aT1), right_desc(c, a.aZ2, a.aT2)}, false);
    B.gemm({left_desc(c, a.aT1, a.aA, EPI_STORE, k), left_desc(c, a.aT2, a.aW2 + (size_t)(k - 1) * c.ns, EPI_ADD, k)},
           false);
    B.add([=]() { adj_level(dc, da, hc, k, first, st); });
    if (k < c.L) {
      const double* ob = a.aObc;
      double* dst = a.aW + (size_t)k * c.ns;
      B.add([=]() { adj_getbcT(dc, ob, dst, hc, 0.25, st); });
    }
    B.add([=]() { adj_nonlinear(dc, da, hc, k, st); });
  }
  // (1) lastbc(:,k) = get_bc(omega(:,:,k+1), 0.25), operators.f90:97-99
  for (int k = 1; k < c.L; k++) {
    const double* ring = a.aLb + (size_t)(k - 1) * c.nring;
    double* dst = a.aW2 + (size_t)k * c.ns;
    B.add([=]() { adj_getbcT(dc, ring, dst, hc, 0.25, st); });
  }
  double* aW = a.aW;
  B.add([=]() { cudaMemcpyAsync(aW, aW2, sizeof(double) * nsL, cudaMemcpyDeviceToDevice, st); });
}

// The whole adjoint step of a stationary body: (5) fb = cholsl(rhsf) is
// symmetric, so its adjoint is the same two triangular solves.
static void adj_build(ibfs_handle* h, AdjPlan& P, Prog& prog, int first) {
  const DevCase& c = h->cases[0].dc;
  const DevCase* dc = h->d_cases;
  const AdjCase& a = P.a;
  cudaStream_t st = h->st;
  ProgBuilder B{h, prog};
  DevCase hc = c;
  adj_build_head(h, P, B);
  double *aF = a.aF, *aTmp = a.aTmp, *aRf = a.aRf;
  B.add([=]() { adj_solve(dc, aF, aTmp, aRf, hc, st); }, TAG_CHOL);
  adj_build_tail(h, P, B, first);
}

// Buffers of the adjoint working set of the handle's single case.
static int adj_alloc(ibfs_handle* h, AdjPlan& P) {
  const DevCase& c = h->cases[0].dc;
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  AdjCase& a = P.a;
  a.aW = dalloc<double>(h, nsL);
  a.aW2 = dalloc<double>(h, nsL);
  a.aP = dalloc<double>(h, nsL);
  a.aQ = dalloc<double>(h, nqL);
  a.aQ1 = dalloc<double>(h, c.nq);
  a.aS = dalloc<double>(h, nsL);
  a.aSbc = dalloc<double>(h, (size_t)c.L * c.nring);
  a.aLb = dalloc<double>(h, (size_t)c.L * c.nring);
  a.aObc = dalloc<double>(h, c.nring);
  a.aA = dalloc<double>(h, c.ns);
  a.aZ1 = dalloc<double>(h, c.ns);
  a.aZ2 = dalloc<double>(h, c.ns);
  a.aR = dalloc<double>(h, c.ns);
  a.aT1 = dalloc<double>(h, c.ns);
  a.aT2 = dalloc<double>(h, c.ns);
  a.aF = dalloc<double>(h, c.nf);
  a.aRf = dalloc<double>(h, c.nf);
  a.aTmp = dalloc<double>(h, c.nf);
  a.aGrad = dalloc<double>(h, c.nf);
  P.d_a = dalloc<AdjCase>(h, 1);
  if (!a.aW || !a.aQ || !a.aS || !a.aGrad || !P.d_a) return set_error(IBFS_ERR_NOMEM, "adjoint allocation failed");
  P.state = 2 * nsL + nqL + c.nf;
  return IBFS_OK;
}

static int adj_init(ibfs_handle* h, AdjPlan& P) {
  int rc = adj_alloc(h, P);
  if (rc) return rc;
  adj_build(h, P, P.bw, 0);
  adj_build(h, P, P.bw_first, 1);
  int kk = 0;
  P.graphs = capture_one(h, P.bw, &P.g_bw, &kk) && capture_one(h, P.bw_first, &P.g_bwf, &kk);
  return IBFS_OK;
}

// state slot <-> case state (omega, rhs_old, q, fb)
static void adj_save(ibfs_handle* h, double* slot) {
  const DevCase& c = h->cases[0].dc;
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  cudaMemcpyAsync(slot, c.omega, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(slot + nsL, c.rhs_old, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(slot + 2 * nsL, c.q, nqL * 8, cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(slot + 2 * nsL + nqL, c.fb, (size_t)c.nf * 8, cudaMemcpyDeviceToDevice, h->st);
}
static void adj_restore(ibfs_handle* h, const double* slot) {
  const DevCase& c = h->cases[0].dc;
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  cudaMemcpyAsync(c.omega, slot, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(c.rhs_old, slot + nsL, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(c.q, slot + 2 * nsL, nqL * 8, cudaMemcpyDeviceToDevice, h->st);
  cudaMemcpyAsync(c.fb, slot + 2 * nsL + nqL, (size_t)c.nf * 8, cudaMemcpyDeviceToDevice, h->st);
}

static int adj_run(ibfs_handle* h, int nsteps, int K, const double* body_vel, const double* wx, const double* wy,
                   double* J, double* grad, double* ms_fwd, double* ms_total) {
  if (h->cases.size() != 1 || !h->cases[0].p.stationary || h->precision != 0)
    return set_error(IBFS_ERR_ARG, "the adjoint needs a single stationary case in the plain FP64 form");
  if (h->cases[0].dc.nact) return set_error(IBFS_ERR_ARG, "the adjoint does not cover actuator jets");
  if (nsteps < 1 || K < 1 || !wx || !wy || !J || !grad) return set_error(IBFS_ERR_ARG, "bad adjoint arguments");
  HostCase& hc = h->cases[0];
  const DevCase& c = hc.dc;
  int rc = precompute(h);
  if (rc) return rc;
  if (!h->adj) {
    h->adj = new AdjPlan();
    rc = adj_init(h, *h->adj);
    if (rc) return rc;
  }
  AdjPlan& P = *h->adj;
  if (P.h_slots < K) {
    if (P.h_a) cudaFreeHost(P.h_a);
    P.h_a = nullptr;
    if (cudaMallocHost(&P.h_a, sizeof(AdjCase) * K) != cudaSuccess) return set_error(IBFS_ERR_NOMEM, "pinned allocation");
    P.h_slots = K;
  }
  int nb = c.nbody;
  int nck = (nsteps + K - 1) / K;
  double *ck = nullptr, *seg = nullptr, *fin = nullptr, *w = nullptr, *hist = nullptr;
  int* ck_it = nullptr;
  auto cleanup = [&]() {
    cudaFree(ck); cudaFree(seg); cudaFree(fin); cudaFree(w); cudaFree(hist); cudaFree(ck_it);
  };
  if (cudaMalloc(&ck, sizeof(double) * P.state * nck) != cudaSuccess ||
      cudaMalloc(&seg, sizeof(double) * P.state * K) != cudaSuccess ||
      cudaMalloc(&fin, sizeof(double) * P.state) != cudaSuccess ||
      cudaMalloc(&w, sizeof(double) * 2 * nb * (size_t)nsteps) != cudaSuccess ||
      cudaMalloc(&hist, sizeof(double) * h->out_stride * (size_t)nsteps) != cudaSuccess ||
      cudaMalloc(&ck_it, sizeof(int) * (nck + 1)) != cudaSuccess) {
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
  if (body_vel) cudaMemcpy(c.bvel, body_vel, sizeof(double) * c.nf, cudaMemcpyHostToDevice);
  else cudaMemset(c.bvel, 0, sizeof(double) * c.nf);
  int it0 = hc.itime;
  cudaMemcpy(c.itime, &it0, sizeof(int), cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
  cudaEventRecord(e0, h->st);
  // 1. forward pass with checkpoints
  for (int s = 0; s < nsteps && rc == IBFS_OK; s++) {
    if (s % K == 0) {
      adj_save(h, ck + P.state * (s / K));
      cudaMemcpyAsync(ck_it + s / K, c.itime, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
    }
    rc = run_step(h);
    cudaMemcpyAsync(hist + (size_t)s * h->out_stride, h->d_out, sizeof(double) * h->out_stride,
                    cudaMemcpyDeviceToDevice, h->st);
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
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  cudaMemsetAsync(a.aW, 0, nsL * 8, h->st);
  cudaMemsetAsync(a.aP, 0, nsL * 8, h->st);
  cudaMemsetAsync(a.aQ, 0, nqL * 8, h->st);
  cudaMemsetAsync(a.aGrad, 0, (size_t)c.nf * 8, h->st);
  for (int sg = nck - 1; sg >= 0 && rc == IBFS_OK; sg--) {
    int s0 = sg * K, s1 = std::min(nsteps, s0 + K);
    cudaStreamSynchronize(h->st);  // the pinned slots of the previous segment are free
    // recompute the segment's step-start states; the first is the checkpoint
    // itself and the last step's result is not needed
    cudaMemcpyAsync(seg, ck + P.state * sg, sizeof(double) * P.state, cudaMemcpyDeviceToDevice, h->st);
    if (s1 - s0 > 1) {
      adj_restore(h, ck + P.state * sg);
      cudaMemcpyAsync(c.itime, ck_it + sg, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
      for (int s = s0; s < s1 - 1 && rc == IBFS_OK; s++) {
        rc = run_step(h);
        adj_save(h, seg + P.state * (s + 1 - s0));
      }
    }
    for (int s = s1 - 1; s >= s0 && rc == IBFS_OK; s--) {
      const double* st = seg + P.state * (s - s0);
      AdjCase cur = a;
      cur.fwW = st;
      cur.fwQ = st + 2 * nsL;
      cur.wx = w + (size_t)s * 2 * nb;
      cur.wy = cur.wx + nb;
      AdjCase* slot = P.h_a + (s - s0);
      *slot = cur;
      cudaMemcpyAsync(P.d_a, slot, sizeof(AdjCase), cudaMemcpyHostToDevice, h->st);
      bool first = it0 + s + 1 == 1;
      Prog& prog = first ? P.bw_first : P.bw;
      cudaGraphExec_t ex = first ? P.g_bwf : P.g_bw;
      rc = run_prog(h, prog, P.graphs ? ex : nullptr);
    }
  }
  adj_restore(h, fin);
  cudaMemcpyAsync(c.itime, ck_it + nck, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
  cudaEventRecord(e2, h->st);
  cudaMemcpyAsync(grad, a.aGrad, sizeof(double) * c.nf, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  float f1 = 0.f, f2 = 0.f;
  cudaEventElapsedTime(&f1, e0, e1);
  cudaEventElapsedTime(&f2, e0, e2);
  if (ms_fwd) *ms_fwd = f1;
  if (ms_total) *ms_total = f2;
  cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
  cleanup();
  hc.itime = it0 + nsteps;
  if (rc) return rc;
  if (e != cudaSuccess) return fail_cuda(e, "adjoint run");
  return IBFS_OK;
}

}  // namespace ibfs
