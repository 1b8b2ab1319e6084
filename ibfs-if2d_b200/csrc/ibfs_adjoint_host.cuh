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
//      run the adjoint step backwards through the segment. The forward pass
//      stores the last segment's step-start states itself, so that segment is
//      not recomputed.
// The adjoint step is one fixed launch program (captured as a CUDA graph);
// per step only the pointers to the stored forward state and the objective
// weights change, uploaded into the device AdjCase array before each replay.
//
// The programs serve a group of slots (one case each, differentiated
// together, as the pitching-body driver does for a batch): every stage is one
// launch over all slots and the sine-transform GEMMs of all slots share one
// grouped launch. Each per-slot buffer family is one contiguous block.

namespace ibfs {

struct AdjPlan {
  std::vector<int> cids;     // case of each slot
  const int* d_cids = nullptr;
  std::vector<AdjCase> a;    // per-slot working sets (host copy of d_a)
  AdjCase* d_a = nullptr;
  AdjGroup g;
  double *blk_W = nullptr, *blk_W2 = nullptr, *blk_Lb = nullptr, *blk_P = nullptr, *blk_Q = nullptr,
         *blk_Grad = nullptr, *blk_Rf = nullptr;
  size_t n_W = 0, n_Lb = 0, n_Q = 0, n_F = 0;  // doubles in the node / ring / face / force blocks
  AdjCase* h_a = nullptr;    // pinned staging of the per-step AdjCase arrays, [h_slots]
  int h_slots = 0;
  Prog bw, bw_first;
  cudaGraphExec_t g_bw = nullptr, g_bwf = nullptr;
  bool graphs = false;
  std::vector<size_t> soff;  // offset of each slot's part of a stored state
  size_t state = 0;          // doubles per stored state (all slots)
};

static const DevCase& slot_case(ibfs_handle* h, const std::vector<int>& cids, int i) {
  return h->cases[cids[i]].dc;
}

static AdjGroup make_group(ibfs_handle* h, const std::vector<int>& cids, const int* d_cids, const AdjCase* da) {
  AdjGroup g;
  g.n = (int)cids.size();
  g.cids = d_cids;
  g.dc = h->d_cases;
  g.da = da;
  for (int c : cids) {
    const DevCase& d = h->cases[c].dc;
    g.max_ns = std::max(g.max_ns, d.ns);
    g.max_nq = std::max(g.max_nq, d.nq);
    g.max_nf = std::max(g.max_nf, d.nf);
    g.max_ring = std::max(g.max_ring, d.nring);
    g.max_L = std::max(g.max_L, d.L);
    g.max_perim = std::max(g.max_perim, 2 * (d.m / 2 + 1) + 2 * (d.n / 2 - 1));
  }
  return g;
}

// One contiguous block per buffer family; slot i's part starts after the
// parts of slots < i. per(c) = doubles slot c needs.
template <class F>
static double* alloc_family(ibfs_handle* h, const std::vector<int>& cids, std::vector<AdjCase>& a,
                            double* AdjCase::*field, F per, size_t* total = nullptr) {
  size_t n = 0;
  for (size_t i = 0; i < cids.size(); i++) n += per(slot_case(h, cids, (int)i));
  double* blk = dalloc<double>(h, std::max<size_t>(n, 1));
  if (!blk) return nullptr;
  size_t o = 0;
  for (size_t i = 0; i < cids.size(); i++) {
    a[i].*field = blk + o;
    o += per(slot_case(h, cids, (int)i));
  }
  if (total) *total = n;
  return blk;
}

// One grouped GEMM launch over the slots whose level count reaches k;
// make(i, case, descs) appends slot i's descriptors.
template <class F>
static void gemm_slots(ProgBuilder& B, ibfs_handle* h, const std::vector<int>& cids, int k, F make) {
  std::vector<GemmDesc> ds;
  for (int i = 0; i < (int)cids.size(); i++)
    if (slot_case(h, cids, i).L >= k) make(i, slot_case(h, cids, i), ds);
  B.gemm(ds, false);
}

// aZ1 = ainv(aW_1) of every slot (ainv, myfft.f90:112-124, is symmetric).
static void adj_add_ainv(ProgBuilder& B, ibfs_handle* h, const std::vector<int>& cids, const std::vector<AdjCase>& a) {
  using V = std::vector<GemmDesc>;
  gemm_slots(B, h, cids, 1, [&](int i, const DevCase& c, V& d) { d.push_back(right_desc(c, a[i].aW, a[i].aT1)); });
  gemm_slots(B, h, cids, 1, [&](int i, const DevCase& c, V& d) { d.push_back(left_desc(c, a[i].aT1, a[i].aT2, EPI_AINV, 1)); });
  gemm_slots(B, h, cids, 1, [&](int i, const DevCase& c, V& d) { d.push_back(right_desc(c, a[i].aT2, a[i].aT1)); });
  gemm_slots(B, h, cids, 1, [&](int i, const DevCase& c, V& d) { d.push_back(left_desc(c, a[i].aT1, a[i].aZ1, EPI_STORE, 1)); });
}

// Adjoint of vort2flux(vel, omega, nlev) (operators.f90:191-240): incoming
// adjoints of the fluxes (aQ, or aQ1 for nlev = 1) and of the coarsified
// omega (aW); aW becomes the adjoint of the omega passed in.
static void adj_add_v2f(ProgBuilder& B, ibfs_handle* h, const std::vector<int>& cids, const std::vector<AdjCase>& a,
                        const AdjGroup& g, int nlev, int use_q1) {
  using V = std::vector<GemmDesc>;
  cudaStream_t st = h->st;
  B.add([=]() { adj_curlT(g, nlev, use_q1, st); });
  for (int k = 1; k <= g.max_L; k++) {
    // aZ1 = ctci(aS_k)
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) { d.push_back(right_desc(c, a[i].aS + (size_t)(k - 1) * c.ns, a[i].aT1)); });
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) { d.push_back(left_desc(c, a[i].aT1, a[i].aT2, EPI_LAMINV, 1)); });
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) { d.push_back(right_desc(c, a[i].aT2, a[i].aT1)); });
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) { d.push_back(left_desc(c, a[i].aT1, a[i].aZ1, EPI_STORE, 1)); });
    B.add([=]() { adj_v2f_level(g, k, st); });
    if (k < g.max_L) B.add([=]() { adj_getbcT(g, GETBC_SBC, k, 1.0, st); });
  }
  for (int k = g.max_L; k >= 2; k--) B.add([=]() { adj_coarsifyT(g, k, st); });
}

// Adjoint step, first part: steps (7) and (6) of the forward step run
// backwards, ending with the adjoint of fb (aF).
static void adj_build_head(ibfs_handle* h, AdjPlan& P, ProgBuilder& B) {
  cudaStream_t st = h->st;
  const AdjGroup g = P.g;
  double* lb = P.blk_Lb;
  size_t lbb = sizeof(double) * P.n_Lb;
  B.add([=]() { cudaMemsetAsync(lb, 0, lbb, st); });
  // (7) vort2flux(q, omega, L), operators.f90:177
  adj_add_v2f(B, h, P.cids, P.a, g, g.max_L, 0);
  // (6) omega_1 -= ainv(rot(reg(fb))), operators.f90:174
  adj_add_ainv(B, h, P.cids, P.a);
  B.add([=]() { adj_force(g, st); });
}

// Adjoint step, last part: from the adjoint of rhsf (aRf) through steps (4)
// to (1).
static void adj_build_tail(ibfs_handle* h, AdjPlan& P, ProgBuilder& B, int first) {
  using V = std::vector<GemmDesc>;
  cudaStream_t st = h->st;
  const AdjGroup g = P.g;
  const std::vector<int>& cids = P.cids;
  const std::vector<AdjCase>& a = P.a;
  // (4) rhsf = regT(q_1) - motion
  B.add([=]() { adj_rhsf(g, st); });
  // (3) vort2flux(q(:,1), omega, 1), operators.f90:163
  adj_add_v2f(B, h, cids, a, g, 1, 1);
  // (2) level loop k = L..1 run backwards (operators.f90:103-134)
  double* w2 = P.blk_W2;
  size_t wb = sizeof(double) * P.n_W;
  B.add([=]() { cudaMemsetAsync(w2, 0, wb, st); });
  for (int k = 1; k <= g.max_L; k++) {
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) { d.push_back(right_desc(c, a[i].aW + (size_t)(k - 1) * c.ns, a[i].aT1)); });
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) {
      GemmDesc dd = left_desc(c, a[i].aT1, a[i].aZ1, EPI_ADJ_CN, k);
      dd.C2 = a[i].aZ2;
      d.push_back(dd);
    });
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) {
      d.push_back(right_desc(c, a[i].aZ1, a[i].aT1));
      d.push_back(right_desc(c, a[i].aZ2, a[i].aT2));
    });
    gemm_slots(B, h, cids, k, [&](int i, const DevCase& c, V& d) {
      d.push_back(left_desc(c, a[i].aT1, a[i].aA, EPI_STORE, k));
      d.push_back(left_desc(c, a[i].aT2, a[i].aW2 + (size_t)(k - 1) * c.ns, EPI_ADD, k));
    });
    B.add([=]() { adj_level(g, k, first, st); });
    if (k < g.max_L) B.add([=]() { adj_getbcT(g, GETBC_OBC, k, 0.25, st); });
    B.add([=]() { adj_nonlinear(g, k, st); });
  }
  // (1) lastbc(:,k) = get_bc(omega(:,:,k+1), 0.25), operators.f90:97-99
  for (int k = 1; k < g.max_L; k++) B.add([=]() { adj_getbcT(g, GETBC_LB, k, 0.25, st); });
  double* w = P.blk_W;
  B.add([=]() { cudaMemcpyAsync(w, w2, wb, cudaMemcpyDeviceToDevice, st); });
}

// The whole adjoint step of a stationary body: (5) fb = cholsl(rhsf) is
// symmetric, so its adjoint is the same two triangular solves.
static void adj_build(ibfs_handle* h, AdjPlan& P, Prog& prog, int first) {
  ProgBuilder B{h, prog};
  const AdjGroup g = P.g;
  cudaStream_t st = h->st;
  adj_build_head(h, P, B);
  B.add([=]() { adj_solve(g, st); }, TAG_CHOL);
  adj_build_tail(h, P, B, first);
}

// Working sets of the slots (cases cids of the handle).
static int adj_alloc(ibfs_handle* h, AdjPlan& P, const std::vector<int>& cids) {
  P.cids = cids;
  const int n = (int)cids.size();
  P.a.assign(n, AdjCase{});
  auto ns = [](const DevCase& c) { return (size_t)c.ns; };
  auto nsL = [](const DevCase& c) { return (size_t)c.L * c.ns; };
  auto nqL = [](const DevCase& c) { return (size_t)c.L * c.nq; };
  auto nq = [](const DevCase& c) { return (size_t)c.nq; };
  auto ringL = [](const DevCase& c) { return (size_t)c.L * c.nring; };
  auto ring = [](const DevCase& c) { return (size_t)c.nring; };
  auto nf = [](const DevCase& c) { return (size_t)c.nf; };
  bool ok = true;
  ok = ok && (P.blk_W = alloc_family(h, cids, P.a, &AdjCase::aW, nsL, &P.n_W));
  ok = ok && (P.blk_W2 = alloc_family(h, cids, P.a, &AdjCase::aW2, nsL));
  ok = ok && (P.blk_P = alloc_family(h, cids, P.a, &AdjCase::aP, nsL));
  ok = ok && (P.blk_Q = alloc_family(h, cids, P.a, &AdjCase::aQ, nqL, &P.n_Q));
  ok = ok && alloc_family(h, cids, P.a, &AdjCase::aQ1, nq);
  ok = ok && alloc_family(h, cids, P.a, &AdjCase::aS, nsL);
  ok = ok && alloc_family(h, cids, P.a, &AdjCase::aSbc, ringL);
  ok = ok && (P.blk_Lb = alloc_family(h, cids, P.a, &AdjCase::aLb, ringL, &P.n_Lb));
  ok = ok && alloc_family(h, cids, P.a, &AdjCase::aObc, ring);
  for (double* AdjCase::*f : {&AdjCase::aA, &AdjCase::aZ1, &AdjCase::aZ2, &AdjCase::aR, &AdjCase::aT1, &AdjCase::aT2})
    ok = ok && alloc_family(h, cids, P.a, f, ns);
  ok = ok && alloc_family(h, cids, P.a, &AdjCase::aF, nf, &P.n_F);
  ok = ok && (P.blk_Rf = alloc_family(h, cids, P.a, &AdjCase::aRf, nf));
  ok = ok && alloc_family(h, cids, P.a, &AdjCase::aTmp, nf);
  ok = ok && (P.blk_Grad = alloc_family(h, cids, P.a, &AdjCase::aGrad, nf));
  P.d_a = dupload(h, P.a);
  P.d_cids = dupload(h, cids);
  if (!ok || !P.d_a || !P.d_cids) return set_error(IBFS_ERR_NOMEM, "adjoint allocation failed");
  P.g = make_group(h, cids, P.d_cids, P.d_a);
  P.soff.clear();
  P.state = 0;
  for (int i = 0; i < n; i++) {
    const DevCase& c = slot_case(h, cids, i);
    P.soff.push_back(P.state);
    P.state += 2 * nsL(c) + nqL(c) + c.nf;
  }
  return IBFS_OK;
}

static int adj_init(ibfs_handle* h, AdjPlan& P) {
  int rc = adj_alloc(h, P, {0});
  if (rc) return rc;
  adj_build(h, P, P.bw, 0);
  adj_build(h, P, P.bw_first, 1);
  int kk = 0;
  P.graphs = capture_one(h, P.bw, &P.g_bw, &kk) && capture_one(h, P.bw_first, &P.g_bwf, &kk);
  return IBFS_OK;
}

// pinned staging for K per-step AdjCase arrays of the plan's slots
static int adj_staging(AdjPlan& P, int K) {
  int need = K * (int)P.cids.size();
  if (P.h_slots >= need) return IBFS_OK;
  if (P.h_a) cudaFreeHost(P.h_a);
  P.h_a = nullptr;
  P.h_slots = 0;
  if (cudaMallocHost(&P.h_a, sizeof(AdjCase) * need) != cudaSuccess) return set_error(IBFS_ERR_NOMEM, "pinned allocation");
  P.h_slots = need;
  return IBFS_OK;
}

// stored state <-> the slots' case states (omega, rhs_old, q, fb)
static void adj_save(ibfs_handle* h, const AdjPlan& P, double* slot) {
  for (size_t i = 0; i < P.cids.size(); i++) {
    const DevCase& c = slot_case(h, P.cids, (int)i);
    size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
    double* s = slot + P.soff[i];
    cudaMemcpyAsync(s, c.omega, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(s + nsL, c.rhs_old, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(s + 2 * nsL, c.q, nqL * 8, cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(s + 2 * nsL + nqL, c.fb, (size_t)c.nf * 8, cudaMemcpyDeviceToDevice, h->st);
  }
}
static void adj_restore(ibfs_handle* h, const AdjPlan& P, const double* slot) {
  for (size_t i = 0; i < P.cids.size(); i++) {
    const DevCase& c = slot_case(h, P.cids, (int)i);
    size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
    const double* s = slot + P.soff[i];
    cudaMemcpyAsync(c.omega, s, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(c.rhs_old, s + nsL, nsL * 8, cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(c.q, s + 2 * nsL, nqL * 8, cudaMemcpyDeviceToDevice, h->st);
    cudaMemcpyAsync(c.fb, s + 2 * nsL + nqL, (size_t)c.nf * 8, cudaMemcpyDeviceToDevice, h->st);
  }
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
  if ((rc = adj_staging(P, K))) return rc;
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
  // 1. forward pass with checkpoints; the last segment's step-start states go
  // straight into the segment buffer, so the backward pass starts without
  // recomputing it
  const int s_last = (nck - 1) * K;
  for (int s = 0; s < nsteps && rc == IBFS_OK; s++) {
    if (s % K == 0) {
      adj_save(h, P, ck + P.state * (s / K));
      cudaMemcpyAsync(ck_it + s / K, c.itime, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
    }
    if (s >= s_last) adj_save(h, P, seg + P.state * (s - s_last));
    rc = run_step(h);
    cudaMemcpyAsync(hist + (size_t)s * h->out_stride, h->d_out, sizeof(double) * h->out_stride,
                    cudaMemcpyDeviceToDevice, h->st);
  }
  adj_save(h, P, fin);
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
  const AdjCase& a = P.a[0];
  size_t nsL = (size_t)c.L * c.ns;
  cudaMemsetAsync(P.blk_W, 0, P.n_W * 8, h->st);
  cudaMemsetAsync(P.blk_P, 0, P.n_W * 8, h->st);
  cudaMemsetAsync(P.blk_Q, 0, P.n_Q * 8, h->st);
  cudaMemsetAsync(P.blk_Grad, 0, P.n_F * 8, h->st);
  for (int sg = nck - 1; sg >= 0 && rc == IBFS_OK; sg--) {
    int s0 = sg * K, s1 = std::min(nsteps, s0 + K);
    cudaStreamSynchronize(h->st);  // the pinned slots of the previous segment are free
    // recompute the segment's step-start states (the last segment's are
    // already there from the forward pass); the first is the checkpoint
    // itself and the last step's result is not needed
    if (sg != nck - 1)
      cudaMemcpyAsync(seg, ck + P.state * sg, sizeof(double) * P.state, cudaMemcpyDeviceToDevice, h->st);
    if (sg != nck - 1 && s1 - s0 > 1) {
      adj_restore(h, P, ck + P.state * sg);
      cudaMemcpyAsync(c.itime, ck_it + sg, sizeof(int), cudaMemcpyDeviceToDevice, h->st);
      for (int s = s0; s < s1 - 1 && rc == IBFS_OK; s++) {
        rc = run_step(h);
        adj_save(h, P, seg + P.state * (s + 1 - s0));
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
  adj_restore(h, P, fin);
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
