// ibfs_capi.cu -- host runtime of the B200 IBFS advance behind include/ibfs_capi.h.
//
// A handle owns one or more cases (the batched form is the same code with
// more items). At creation it builds, once, the whole step as a fixed list of
// grouped launches (the "step program", mirroring advance, operators.f90:62-188)
// and captures it into a CUDA graph that every step replays. Host work per
// step is one graph launch (plus output copies when asked for).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include <mutex>
#include "../../include/ibfs_capi.h"
#include "ibfs_handle.cuh"

namespace ibfs {

static thread_local std::string t_error;

int fail_cuda(cudaError_t e, const char* what) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) at %s", (int)e, cudaGetErrorString(e), what);
  t_error = buf;
  return IBFS_ERR_CUDA;
}

static int fail(int code, const std::string& msg) {
  t_error = msg;
  return code;
}

int set_error(int code, const char* msg) { return fail(code, msg); }

// grid.f90:79: FLOOR(LOG(REAL(MIN(m,n)/2))/LOG(2.d0)) - 1 with single-precision LOG.
static int nlevmax(int m, int n) {
  int mn = std::min(m, n) / 2;
  float lf = logf((float)mn);
  return (int)std::floor((double)lf / std::log(2.0)) - 1;
}

// grid.f90:233-249.
static double deltafnc(double r, double r0, double dr) {
  double d = std::fabs(r - r0);
  if (d <= 0.5 * dr) {
    double t = (r - r0) / dr;
    return (1.0 + std::sqrt(-3.0 * t * t + 1.0)) / (3.0 * dr);
  } else if (d <= 1.5 * dr) {
    double a = std::fabs((r - r0) / dr);
    double u = 1.0 - a;
    return (5.0 - 3.0 * a - std::sqrt(-3.0 * u * u + 1.0)) / (6.0 * dr);
  }
  return 0.0;
}

}  // namespace ibfs

#include "ibfs_handle.cuh"

using namespace ibfs;

namespace ibfs {

template <class T>
static T* dalloc(ibfs_handle* h, size_t count, bool zero = true) {
  void* p = nullptr;
  if (count == 0) count = 1;
  if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
  if (zero) cudaMemset(p, 0, count * sizeof(T));
  h->allocs.push_back(p);
  return (T*)p;
}

template <class T>
static T* dupload(ibfs_handle* h, const std::vector<T>& v) {
  T* p = dalloc<T>(h, v.size(), false);
  if (p && !v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return p;
}

// Host-side setup_reg (grid.f90:142-230): for every face within 1.5*delta of a
// body point (box test), weight delta^2 * d(x-xb) * d(y-yb). Faces near each
// point are enumerated directly instead of scanning all Nq faces; per-face
// entry order stays the reference's (ascending body point), and per-force
// entries are by ascending face index, the order of regT's scatter loop.
static void setup_reg_host(HostCase& c) {
  int m = c.m, n = c.n, nb = c.nb;
  double delta = c.delta, d2 = 0.5 * delta, sup = 3.0 * d2;
  double ox = c.p.offsetx, oy = c.p.offsety;
  struct Ent { int face, force; double w; };
  std::vector<Ent> ents;
  for (int k = 0; k < nb; k++) {
    double xk = c.xb[k], yk = c.yb[k];
    // u faces: x = delta*(i-1)-ox, y = delta*(j-1)-oy+d2
    int i0 = std::max(1, (int)std::floor((xk + ox - sup) / delta) + 1 - 1);
    int i1 = std::min(m + 1, (int)std::ceil((xk + ox + sup) / delta) + 1 + 1);
    int j0 = std::max(1, (int)std::floor((yk + oy - d2 - sup) / delta) + 1 - 1);
    int j1 = std::min(n, (int)std::ceil((yk + oy - d2 + sup) / delta) + 1 + 1);
    for (int i = i0; i <= i1; i++)
      for (int j = j0; j <= j1; j++) {
        double x = delta * (double)(i - 1) - ox;
        double y = delta * (double)(j - 1) - oy + d2;
        if (std::fabs(x - xk) < sup && std::fabs(y - yk) < sup)
          ents.push_back({(i - 1) + (j - 1) * (m + 1), k,
                          (delta * delta) * deltafnc(x, xk, delta) * deltafnc(y, yk, delta)});
      }
    // v faces: x = delta*(i-1)-ox+d2, y = delta*(j-1)-oy
    i0 = std::max(1, (int)std::floor((xk + ox - d2 - sup) / delta) + 1 - 1);
    i1 = std::min(m, (int)std::ceil((xk + ox - d2 + sup) / delta) + 1 + 1);
    j0 = std::max(1, (int)std::floor((yk + oy - sup) / delta) + 1 - 1);
    j1 = std::min(n + 1, (int)std::ceil((yk + oy + sup) / delta) + 1 + 1);
    for (int i = i0; i <= i1; i++)
      for (int j = j0; j <= j1; j++) {
        double x = delta * (double)(i - 1) - ox + d2;
        double y = delta * (double)(j - 1) - oy;
        if (std::fabs(x - xk) < sup && std::fabs(y - yk) < sup)
          ents.push_back({(m + 1) * n + (i - 1) + (j - 1) * m, nb + k,
                          (delta * delta) * deltafnc(x, xk, delta) * deltafnc(y, yk, delta)});
      }
  }
  // CSR by face, entries in ascending body-point order (stable sort by face)
  std::stable_sort(ents.begin(), ents.end(), [](const Ent& a, const Ent& b) { return a.face < b.face; });
  c.face_ptr.assign(c.nq + 1, 0);
  c.face_f.clear();
  c.face_w.clear();
  for (auto& e : ents) c.face_ptr[e.face + 1]++;
  for (int f = 0; f < c.nq; f++) c.face_ptr[f + 1] += c.face_ptr[f];
  for (auto& e : ents) {
    c.face_f.push_back(e.force);
    c.face_w.push_back(e.w);
  }
  // CSR by force, faces ascending (ents is face-sorted; stable by force)
  std::vector<Ent> byf = ents;
  std::stable_sort(byf.begin(), byf.end(), [](const Ent& a, const Ent& b) { return a.force < b.force; });
  c.force_ptr.assign(c.nf + 1, 0);
  c.force_face.clear();
  c.force_w.clear();
  for (auto& e : byf) c.force_ptr[e.force + 1]++;
  for (int f = 0; f < c.nf; f++) c.force_ptr[f + 1] += c.force_ptr[f];
  c.wsum.assign(c.nf, 0.0);
  for (auto& e : byf) {
    c.force_face.push_back(e.face);
    c.force_w.push_back(e.w);
    c.wsum[e.force] += e.w;
  }
}

static double* sine_matrix(ibfs_handle* h, int m) {
  auto it = h->sine.find(m);
  if (it != h->sine.end()) return it->second;
  int N = m - 1;
  std::vector<double> S((size_t)N * N);
  for (int a = 0; a < N; a++)
    for (int b = 0; b < N; b++) {
      long long p = ((long long)(a + 1) * (b + 1)) % (2 * m);
      S[a + (size_t)b * N] = 2.0 * std::sin(M_PI * (double)p / (double)m);
    }
  double* d = dupload(h, S);
  h->sine[m] = d;
  return d;
}

static double* cos_table(ibfs_handle* h, int m) {
  auto it = h->costab.find(m);
  if (it != h->costab.end()) return it->second;
  const double pi = 3.1415926535897932384;
  std::vector<double> c(m - 1);
  for (int i = 1; i <= m - 1; i++) c[i - 1] = std::cos(pi * (double)i / (double)m);
  double* d = dupload(h, c);
  h->costab[m] = d;
  return d;
}

// ---------------------------------------------------------------------------
// Tile autotuner of the FP64 transform GEMMs. A launch group (the GEMMs of one
// step-program entry) with enough tiles to fill the SMs is timed once with each
// of the four unsplit tile shapes -- its outputs redirected to a scratch
// buffer, its inputs read where they lie, so no state changes -- and the
// fastest shape is kept. Results are cached per process and device by the
// group's shape signature, so handles of the same sizes tune once. The
// unsplit shapes do not change the order of any output's K sum: they give
// bit-identical results. Groups with few tiles use a split-K cluster
// variant fixed by their tile count (tune_gemm).
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tuned;

static std::string gemm_signature(const std::vector<GemmDesc>& ds, bool dual) {
  std::vector<std::string> parts;
  for (auto& d : ds) parts.push_back(std::to_string(d.M) + "x" + std::to_string(d.N) + "x" + std::to_string(d.K) + ":" +
                                     std::to_string(d.pro) + "/" + std::to_string(d.epi));
  std::sort(parts.begin(), parts.end());
  int dev = 0;
  cudaGetDevice(&dev);
  std::string key = "dev" + std::to_string(dev) + (dual ? "|dual|" : "|");
  for (auto& p : parts) key += p + ";";
  return key;
}

static int num_sms() {
  static int sms = [] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    return n;
  }();
  return sms;
}

static int tune_gemm(const std::vector<GemmDesc>& ds, bool dual, cudaStream_t st, bool allow_split = true) {
  // A group with few 32x32 tiles (one or a few cases) leaves SMs idle: it gets
  // a split-K cluster configuration, chosen by the tile count alone and never
  // by timing, so that a group shape gets the same configuration -- the same
  // summation order -- in every process and in every grouping of the same
  // cases. Larger groups are timed over the unsplit shapes only, which give
  // bit-identical results, so timing noise never changes a result.
  long tiles32 = 0;
  for (auto& d : ds) tiles32 += gemm_tiles(d.M, d.N, 1);
  if (allow_split && tiles32 < 2L * num_sms()) return tiles32 >= num_sms() / 2 ? 4 : 6;
  const int fallback = [&] {
    long tiles64 = 0;
    for (auto& d : ds) tiles64 += gemm_tiles(d.M, d.N, 0);
    return tiles64 >= 2 * 148 ? 0 : 1;
  }();
  const std::string key = gemm_signature(ds, dual);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(key);
  if (it != g_tuned.end()) return it->second;
  size_t need = 1;
  for (auto& d : ds) need = std::max(need, (size_t)d.ldc * (size_t)d.N);
  std::vector<GemmDesc> t = ds;
  double* scratch = nullptr;
  GemmDesc* dd = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int best = fallback;
  if (cudaMalloc(&scratch, need * sizeof(double)) == cudaSuccess &&
      cudaMalloc(&dd, sizeof(GemmDesc) * t.size()) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
      cudaEventCreate(&e1) == cudaSuccess) {
    for (auto& d : t) {
      d.C = scratch;
      if (d.C2) d.C2 = scratch;
    }
    cudaMemcpy(dd, t.data(), sizeof(GemmDesc) * t.size(), cudaMemcpyHostToDevice);
    float best_ms = 1e30f;
    for (int cfg = 0; cfg < 4; cfg++) {
      int mt = 0;
      for (auto& d : t) mt = std::max(mt, gemm_tiles(d.M, d.N, cfg));
      launch_gemm_f64(dd, (int)t.size(), mt, cfg, dual, st);  // warm-up
      cudaEventRecord(e0, st);
      for (int r = 0; r < 3; r++) launch_gemm_f64(dd, (int)t.size(), mt, cfg, dual, st);
      cudaEventRecord(e1, st);
      float ms = 0.f;
      if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess &&
          ms < best_ms) {
        best_ms = ms;
        best = cfg;
      }
    }
  }
  cudaGetLastError();
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (dd) cudaFree(dd);
  if (scratch) cudaFree(scratch);
  g_tuned[key] = best;
  return best;
}

int tuned_gemm_sites() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return (int)g_tuned.size();
}

// ---------------------------------------------------------------------------
// Step program construction
struct ProgBuilder {
  ibfs_handle* h;
  Prog& P;
  bool allow_split = true;  // split-K tiles for groups with few tiles (not for preprocess, see factor_cases)
  void add(std::function<void()> fn, int tag = TAG_STENCIL, double flops = 0.0) { P.push_back({fn, tag, flops}); }
  void gemm(std::vector<GemmDesc> ds, bool dual) {
    if (ds.empty()) return;
    const int cfg =
        h->tile_cfg >= 0 && h->tile_cfg < kGemmF64Cfgs ? h->tile_cfg : tune_gemm(ds, dual, h->st, allow_split);
    int mt = 0;
    for (auto& d : ds) mt = std::max(mt, gemm_tiles(d.M, d.N, cfg));
    GemmDesc* dd = dupload(h, ds);
    int nd = (int)ds.size();
    cudaStream_t st = h->st;
    double fl = 0.0;
    for (auto& d : ds) fl += 2.0 * d.M * (double)d.N * d.K * (dual ? 2 : 1);
    add([=]() { launch_gemm_f64(dd, nd, mt, cfg, dual, st); }, TAG_GEMM_F64, fl);
  }
  const LevelItem* items(const std::vector<LevelItem>& v) { return dupload(h, v); }
  // block map of a grouped element-wise launch from its items' element counts
  std::pair<const int2*, int> bmap(const std::vector<int>& counts) {
    std::vector<int2> v = block_map(counts);
    return {dupload(h, v), (int)v.size()};
  }
  const int* ints(const std::vector<int>& v) { return dupload(h, v); }
};

static GemmDesc right_desc(const DevCase& c, const double* A, double* C) {
  GemmDesc d{};
  d.A = A; d.B = c.Sn; d.C = C;
  d.M = c.m - 1; d.N = c.n - 1; d.K = c.n - 1;
  d.lda = c.m - 1; d.ldb = c.n - 1; d.ldc = c.m - 1;
  d.m = c.m; d.n = c.n;
  d.cosx = c.cosx; d.cosy = c.cosy;
  d.dt = c.dt; d.re = c.re; d.norm = c.norm;
  return d;
}
static GemmDesc left_desc(const DevCase& c, const double* B, double* C, int epi, int k) {
  GemmDesc d{};
  d.A = c.Sm; d.B = B; d.C = C;
  d.M = c.m - 1; d.N = c.n - 1; d.K = c.m - 1;
  d.lda = c.m - 1; d.ldb = c.m - 1; d.ldc = c.m - 1;
  d.m = c.m; d.n = c.n; d.k = k;
  d.epi = epi;
  d.cosx = c.cosx; d.cosy = c.cosy;
  d.dt = c.dt; d.re = c.re; d.norm = c.norm;
  d.del22 = c.delta * c.delta * std::pow(4.0, k - 1);
  return d;
}

// vort2flux (operators.f90:191-240) over the given cases (host copies + their
// index in the device case array). curl_all: curl on every level (nlev = L),
// else on level 1 only (nlev = 1).
static void build_vort2flux(ProgBuilder& B, const DevCase* dcases, const std::vector<DevCase>& cs,
                            const std::vector<int>& ids, bool curl_all) {
  ibfs_handle* h = B.h;
  cudaStream_t st = h->st;
  int Lmax = 0, mns = 0, mnq = 0;
  for (auto& c : cs) { Lmax = std::max(Lmax, c.L); mns = std::max(mns, c.ns); mnq = std::max(mnq, c.nq); }
  for (int k = 2; k <= Lmax; k++) {
    std::vector<LevelItem> it;
    std::vector<int> cnt;
    for (size_t i = 0; i < cs.size(); i++)
      if (cs[i].L >= k) { it.push_back({ids[i], k}); cnt.push_back(coarsify_count(cs[i].m, cs[i].n)); }
    if (it.empty()) continue;
    const LevelItem* d = B.items(it);
    auto bm = B.bmap(cnt);
    B.add([=]() { launch_coarsify(dcases, d, bm.first, bm.second, st); });
  }
  for (int t = 0; t < Lmax; t++) {
    std::vector<GemmDesc> r1, l1, r2, l2;
    for (size_t i = 0; i < cs.size(); i++) {
      const DevCase& c = cs[i];
      int k = c.L - t;
      if (k < 1) continue;
      double* om = c.omega + (size_t)(k - 1) * c.ns;
      GemmDesc d = right_desc(c, om, c.wa);
      if (k < c.L) { d.pro = PRO_APPLY_BC; d.bcsrc = c.s + (size_t)k * c.ns; }
      r1.push_back(d);
      l1.push_back(left_desc(c, c.wa, c.wb, EPI_LAMINV, k));
      r2.push_back(right_desc(c, c.wb, c.wa));
      l2.push_back(left_desc(c, c.wa, c.s + (size_t)(k - 1) * c.ns, EPI_STORE, k));
    }
    B.gemm(r1, false);
    B.gemm(l1, false);
    B.gemm(r2, false);
    B.gemm(l2, false);
  }
  std::vector<LevelItem> ci;
  std::vector<int> cnt;
  for (size_t i = 0; i < cs.size(); i++)
    for (int k = 1; k <= (curl_all ? cs[i].L : 1); k++) { ci.push_back({ids[i], k}); cnt.push_back(cs[i].nq); }
  const LevelItem* d = B.items(ci);
  auto bm = B.bmap(cnt);
  B.add([=]() { launch_curl(dcases, d, bm.first, bm.second, st); });
}

// ainv(x) on level 1 (myfft.f90:112-124): x in c.vort, result stored (or
// subtracted) into omega level 1.
static void build_ainv(ProgBuilder& B, const std::vector<DevCase>& cs, int final_epi) {
  std::vector<GemmDesc> r1, l1, r2, l2;
  for (auto& c : cs) {
    r1.push_back(right_desc(c, c.vort, c.wa));
    l1.push_back(left_desc(c, c.wa, c.wb, EPI_AINV, 1));
    r2.push_back(right_desc(c, c.wb, c.wa));
    l2.push_back(left_desc(c, c.wa, c.omega, final_epi, 1));
  }
  B.gemm(r1, false);
  B.gemm(l1, false);
  B.gemm(r2, false);
  B.gemm(l2, false);
}

// a_times (operators.f90:444-462) of every CG case in FP64 on its shadow:
// vort(:,:,1) = ainv(rot(reg(x))), other levels zero; vort2flux(vel, vort, 1);
// out = regT(vel). Input x is the shadow's fb (the case's fb for shx, cg_d
// for shd).
static void build_atimes_on(ProgBuilder& B, ibfs_handle* h, const DevCase* dsh, const std::vector<DevCase>& sh,
                            double** d_out) {
  cudaStream_t st = h->st;
  double* om = h->sh_omega;
  size_t ob = h->sh_omega_bytes;
  B.add([=]() { cudaMemsetAsync(om, 0, ob, st); });
  int n = (int)sh.size(), mns = 0, mnf = 0;
  std::vector<int> ids(n);
  for (int i = 0; i < n; i++) { ids[i] = i; mns = std::max(mns, sh[i].ns); mnf = std::max(mnf, sh[i].nf); }
  const int* dids = B.ints(ids);
  std::vector<int> cnt(n);
  for (int i = 0; i < n; i++) cnt[i] = sh[i].ns;
  auto bm = B.bmap(cnt);
  B.add([=]() { launch_regrot(dsh, dids, bm.first, bm.second, st); }, TAG_CHOL);
  build_ainv(B, sh, EPI_STORE);
  build_vort2flux(B, dsh, sh, ids, false);
  B.add([=]() { launch_regT_out(dsh, dids, n, mnf, d_out, st); }, TAG_CHOL);
}
static void build_atimes(ProgBuilder& B, ibfs_handle* h, double** d_out) {
  build_atimes_on(B, h, h->d_shx, h->shx, d_out);
}
static void build_atimes_d(ProgBuilder& B, ibfs_handle* h, double** d_out) {
  build_atimes_on(B, h, h->d_shd, h->shd, d_out);
}

static void build_step_program(ibfs_handle* h) {
  h->prog.clear();
  if (h->prec) precision_reset_tile_choices(h->prec);
  ProgBuilder B{h, h->prog};
  cudaStream_t st = h->st;
  const DevCase* dcases = h->d_cases;
  std::vector<DevCase> cs;
  std::vector<int> ids;
  for (size_t i = 0; i < h->cases.size(); i++) { cs.push_back(h->cases[i].dc); ids.push_back((int)i); }
  int nc = (int)cs.size();
  int Lmax = h->max_L, mnf = h->max_nf, mring = h->max_ring;
  const int* d_ids = B.ints(ids);
  B.add([=]() { launch_step_begin(dcases, nc, st); });
  // move_body + setup_reg for moving bodies (operators.f90:142-144); step 1
  // does not use the regularisation, so doing it first is equivalent
  std::vector<int> mv;
  for (int i = 0; i < nc; i++) if (cs[i].moving) mv.push_back(i);
  if (!mv.empty()) {
    const int* d_mv = B.ints(mv);
    int nmv = (int)mv.size(), mnb = h->max_nb, mpatch = h->max_patch;
    B.add([=]() { launch_move_body(dcases, d_mv, nmv, mnb, st); });
    B.add([=]() { launch_setup_reg_moving(dcases, d_mv, nmv, mnf, mpatch, st); });
  }
  // actuator jets after the body motion (operators.f90:149-151)
  std::vector<int> ac;
  int mact = 0;
  for (int i = 0; i < nc; i++)
    if (cs[i].nact > 0) { ac.push_back(i); mact = std::max(mact, cs[i].nact); }
  if (!ac.empty()) {
    const int* d_ac = B.ints(ac);
    int nac = (int)ac.size();
    B.add([=]() { launch_actuate(dcases, d_ac, nac, mact, st); });
  }
  // STEP 1 (operators.f90:97-134)
  std::vector<LevelItem> all;
  for (int i = 0; i < nc; i++) for (int k = 1; k <= cs[i].L; k++) all.push_back({i, k});
  const LevelItem* d_all = B.items(all);
  int nall = (int)all.size();
  B.add([=]() { launch_lastbc(dcases, d_all, nall, mring, st); });
  if (h->precision == 1) {
    build_precision_step1(h->prec, B.P, dcases, cs, st);
  } else {
    for (int t = 0; t < Lmax; t++) {
      std::vector<LevelItem> it;
      std::vector<int> cnt;
      std::vector<GemmDesc> r1, l1, r2, l2;
      for (int i = 0; i < nc; i++) {
        const DevCase& c = cs[i];
        int k = c.L - t;
        if (k < 1) continue;
        it.push_back({i, k});
        cnt.push_back(c.ns);
        double* om = c.omega + (size_t)(k - 1) * c.ns;
        r1.push_back(right_desc(c, c.rhsA, c.wa));
        r1.push_back(right_desc(c, om, c.wb));
        GemmDesc cn = left_desc(c, c.wa, c.wc, EPI_CN, k);
        cn.B2 = c.wb;
        l1.push_back(cn);
        r2.push_back(right_desc(c, c.wc, c.wa));
        l2.push_back(left_desc(c, c.wa, om, EPI_STORE, k));
      }
      const LevelItem* d = B.items(it);
      auto bm = B.bmap(cnt);
      B.add([=]() { launch_rhs(dcases, d, bm.first, bm.second, 0, st); });
      B.gemm(r1, false);
      B.gemm(l1, true);
      B.gemm(r2, false);
      B.gemm(l2, false);
    }
  }
  // STEP 2 (operators.f90:142-171)
  if (h->precision == 1) build_precision_vort2flux(h->prec, B.P, dcases, cs, ids, false, st);
  else build_vort2flux(B, dcases, cs, ids, false);
  B.add([=]() { launch_rhsf(dcases, d_ids, nc, mnf, st); });
  std::vector<int> chol_ids;
  for (int i = 0; i < nc; i++) if (h->cases[i].p.stationary) chol_ids.push_back(i);
  if (!chol_ids.empty()) {
    const int* d_ch = B.ints(chol_ids);
    int nch = (int)chol_ids.size();
    B.add([=]() { launch_chol_solve(dcases, d_ch, nch, mnf, st); }, TAG_CHOL);
  }
  h->prog_iter.clear();
  h->prog_iter50.clear();
  h->prog_post.clear();
  if (h->cg) {
    const int* d_cg = B.ints(h->cg_ids);
    int ncg = (int)h->cg_ids.size();
    std::vector<double*> oq, oq2;
    for (int i : h->cg_ids) { oq.push_back(cs[i].cg_q); oq2.push_back(cs[i].cg_q2); }
    double** d_oq = dupload(h, oq);
    double** d_oq2 = dupload(h, oq2);
    // r = b - A x, d = r (operators.f90:409-412)
    build_atimes(B, h, d_oq);
    B.add([=]() { launch_cg_start(dcases, d_cg, ncg, st); }, TAG_CHOL);
    ProgBuilder Bi{h, h->prog_iter};
    build_atimes_d(Bi, h, d_oq);
    Bi.add([=]() { launch_cg_alpha(dcases, d_cg, ncg, 0, st); }, TAG_CHOL);
    Bi.add([=]() { launch_cg_beta(dcases, d_cg, ncg, st); }, TAG_CHOL);
    ProgBuilder B50{h, h->prog_iter50};
    build_atimes_d(B50, h, d_oq);
    B50.add([=]() { launch_cg_alpha(dcases, d_cg, ncg, 1, st); }, TAG_CHOL);
    build_atimes(B50, h, d_oq2);
    B50.add([=]() { launch_cg_resid(dcases, d_cg, ncg, st); }, TAG_CHOL);
    B50.add([=]() { launch_cg_beta(dcases, d_cg, ncg, st); }, TAG_CHOL);
  }
  ProgBuilder Bp{h, h->cg ? h->prog_post : h->prog};
  // STEP 3 (operators.f90:174)
  std::vector<int> ns_all(nc);
  for (int i = 0; i < nc; i++) ns_all[i] = cs[i].ns;
  auto bm_all = Bp.bmap(ns_all);
  Bp.add([=]() { launch_regrot(dcases, d_ids, bm_all.first, bm_all.second, st); });
  if (h->precision == 1) build_precision_ainv(h->prec, Bp.P, dcases, cs, EPI_SUBTRACT, st);
  else build_ainv(Bp, cs, EPI_SUBTRACT);
  // STEP 4 (operators.f90:177)
  if (h->precision == 1) build_precision_vort2flux(h->prec, Bp.P, dcases, cs, ids, true, st);
  else build_vort2flux(Bp, dcases, cs, ids, true);
  // outputs (operators.f90:184-186)
  std::vector<int> base;
  int acc = 0;
  for (int i = 0; i < nc; i++) { base.push_back(acc); acc += cs[i].L; }
  const int* d_base = Bp.ints(base);
  double* part = h->d_partial;
  Bp.add([=]() { launch_outputs(dcases, d_all, nall, d_ids, d_base, nc, part, st); });
}

static bool capture_one(ibfs_handle* h, Prog& P, cudaGraphExec_t* ex, int* kernels) {
  if (*ex) { cudaGraphExecDestroy(*ex); *ex = nullptr; }
  cudaGraph_t g;
  if (cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
  for (auto& e : P) e.fn();
  if (cudaStreamEndCapture(h->st, &g) != cudaSuccess) { cudaGetLastError(); return false; }
  size_t nn = 0;
  cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) (*kernels)++;
  }
  bool ok = cudaGraphInstantiate(ex, g, 0) == cudaSuccess;
  if (!ok) cudaGetLastError();
  cudaGraphDestroy(g);
  return ok;
}

static int capture_graph(ibfs_handle* h) {
  h->graph_kernels = 0;
  h->graph_ok = capture_one(h, h->prog, &h->gexec, &h->graph_kernels);
  if (h->cg) {
    int k_iter = 0, k50 = 0;
    h->graph_ok = h->graph_ok && capture_one(h, h->prog_iter, &h->gx_iter, &k_iter) &&
                  capture_one(h, h->prog_iter50, &h->gx_iter50, &k50) &&
                  capture_one(h, h->prog_post, &h->gx_post, &h->graph_kernels);
    h->graph_kernels += k_iter;
  }
  return 0;
}

static int run_prog(ibfs_handle* h, Prog& P, cudaGraphExec_t ex) {
  if (h->graph_ok && ex) IBFS_CUDA_CHECK(cudaGraphLaunch(ex, h->st));
  else for (auto& e : P) e.fn();
  IBFS_CUDA_CHECK(cudaGetLastError());
  return IBFS_OK;
}

// One advance. CG handles replay the iteration graph in chunks of four and
// read the per-case active flags between chunks (converged cases skip work
// inside the CG kernels); returns IBFS_ERR_CG_MAXITER when a case used
// cg_max_iter iterations (the reference warns and carries on, :435-438).
static int ensure_precond(ibfs_handle* h, int offset);

static int run_step(ibfs_handle* h) {
  int rc = ensure_precond(h, 1);
  if (rc) return rc;
  rc = run_prog(h, h->prog, h->gexec);
  if (rc || !h->cg) return rc;
  int maxit = 0;
  for (auto& c : h->cases) maxit = std::max(maxit, c.p.cg_max_iter);
  int nc = (int)h->cases.size();
  int it = 0;
  bool any = true, hit_max = false;
  IBFS_CUDA_CHECK(cudaMemcpyAsync(h->h_cgit.data(), h->d_cgit, sizeof(int) * 2 * nc, cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  any = false;
  for (int c = 0; c < nc; c++) any = any || h->h_cgit[2 * c + 1] != 0;
  while (any && it < maxit) {
    for (int c = 0; c < 4 && it < maxit; c++) {
      it++;
      rc = (it % 50 == 0) ? run_prog(h, h->prog_iter50, h->gx_iter50) : run_prog(h, h->prog_iter, h->gx_iter);
      if (rc) return rc;
    }
    IBFS_CUDA_CHECK(cudaMemcpyAsync(h->h_cgit.data(), h->d_cgit, sizeof(int) * 2 * nc, cudaMemcpyDeviceToHost, h->st));
    IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
    any = false;
    for (int c = 0; c < nc; c++) any = any || h->h_cgit[2 * c + 1] != 0;
  }
  h->last_cg_iters = 0;
  for (int c = 0; c < nc; c++) {
    h->last_cg_iters = std::max(h->last_cg_iters, h->h_cgit[2 * c]);
    if (h->h_cgit[2 * c] >= h->cases[c].p.cg_max_iter) hit_max = true;
  }
  rc = run_prog(h, h->prog_post, h->gx_post);
  if (rc) return rc;
  return hit_max ? fail(IBFS_ERR_CG_MAXITER, "WARNING!! CJGR used max iterations!") : IBFS_OK;
}

// ---------------------------------------------------------------------------
// A stationary body needs the factor of its force operator for the Cholesky
// solve (preconditioned CG cases keep their own factors, ensure_precond).
static bool needs_factor(const HostCase& c) {
  return c.p.stationary && !c.have_chol && c.nf > 0;
}

// preprocess (operators.f90:29-59) for every case lacking a factor:
// the columns a_times(e_j) of all such cases are computed as "shadow cases"
// (one per right-hand side, sharing the real case's grid tables, with private
// scratch), packed from any mix of cases into chunks of a fixed memory budget
// so that small cases share launches; then one CTA per case factors A.
static int factor_cases(ibfs_handle* h, const std::vector<int>& need);

static int precompute(ibfs_handle* h) {
  std::vector<int> need;
  for (size_t i = 0; i < h->cases.size(); i++)
    if (needs_factor(h->cases[i])) need.push_back((int)i);
  if (need.empty()) return IBFS_OK;
  int rc = factor_cases(h, need);
  if (rc) return rc;
  for (int ci : need) h->cases[ci].have_chol = true;
  return IBFS_OK;
}

// The factor of the force operator of each case in need, with the case's
// current regularisation tables: columns a_times(e_j) into cholmat, choldc,
// and the inverse factor into Linv / LinvT.
static int factor_cases(ibfs_handle* h, const std::vector<int>& need) {
  auto per_rhs = [&](const DevCase& c) {
    size_t nsL = (size_t)c.L * c.ns;
    size_t b = sizeof(double) * (2 * nsL + 4 * (size_t)c.ns + c.nq + c.nf);
    return (b + 255) / 256 * 256;
  };
  // column pool: up to 4 GB, at most half of the free device memory (the
  // preconditioner slots are factored in the middle of a run), at least one
  // column of the largest case
  size_t one = 0;
  for (int ci : need) one = std::max(one, per_rhs(h->cases[ci].dc));
  size_t free_b = 0, total_b = 0;
  size_t budget = (size_t)4 << 30;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = std::min(budget, free_b / 2);
  budget = std::max(budget, one);
  char* pool = nullptr;
  if (cudaMalloc(&pool, budget) != cudaSuccess) return fail(IBFS_ERR_NOMEM, "device allocation failed in preprocess");
  struct Rhs { int ci, col; };
  std::vector<Rhs> all;
  for (int ci : need)
    for (int j = 0; j < h->cases[ci].nf; j++) all.push_back({ci, j});
  int rc = IBFS_OK;
  size_t pos = 0;
  while (pos < all.size() && rc == IBFS_OK) {
    // pack right-hand sides until the pool is full
    std::vector<DevCase> sh;
    std::vector<int> cols;
    std::vector<double*> outs;
    size_t used = 0;
    while (pos < all.size()) {
      const DevCase& c = h->cases[all[pos].ci].dc;
      size_t b = per_rhs(c);
      if (used + b > budget && !sh.empty()) break;
      if (b > budget) { rc = fail(IBFS_ERR_NOMEM, "one a_times column exceeds the preprocess pool"); break; }
      DevCase s = c;
      double* p = (double*)(pool + used);
      size_t nsL = (size_t)c.L * c.ns;
      s.omega = p; p += nsL;
      s.s = p; p += nsL;
      s.wa = p; p += c.ns;
      s.wb = p; p += c.ns;
      s.wc = p; p += c.ns;
      s.vort = p; p += c.ns;
      s.q = p; p += c.nq;
      s.fb = p;
      cudaMemsetAsync(s.omega, 0, sizeof(double) * nsL, h->st);
      cols.push_back(all[pos].col);
      outs.push_back(c.chol + (size_t)all[pos].col * c.nf);  // cholmat(:, j) = a_times(e_j)
      sh.push_back(s);
      used += b;
      pos++;
    }
    if (rc) break;
    int nr = (int)sh.size();
    std::vector<int> ids(nr);
    int mnf = 0, mns = 0;
    for (int r = 0; r < nr; r++) { ids[r] = r; mnf = std::max(mnf, sh[r].nf); mns = std::max(mns, sh[r].ns); }
    Prog P;
    ibfs_handle tmp;  // collects this chunk's uploads
    tmp.tile_cfg = h->tile_cfg;
    tmp.st = h->st;
    // the columns are packed into chunks by memory budget, so a case's GEMM
    // groups here depend on what it is batched with: only the unsplit tile
    // shapes (bit-identical to each other) keep its factor the same alone
    // and in any batch
    ProgBuilder B{&tmp, P};
    B.allow_split = false;
    DevCase* dsh = dupload(&tmp, sh);
    const int* dids = B.ints(ids);
    const int* dcols = B.ints(cols);
    double** douts = dupload(&tmp, outs);
    cudaStream_t st = h->st;
    B.add([=]() { launch_unit_fb(dsh, dids, dcols, nr, mnf, st); });
    std::vector<int> cnt(nr);
    for (int r = 0; r < nr; r++) cnt[r] = sh[r].ns;
    auto bm = B.bmap(cnt);
    B.add([=]() { launch_regrot(dsh, dids, bm.first, bm.second, st); });
    // A is always built in FP64 (the force system stays FP64 in every form)
    build_ainv(B, sh, EPI_STORE);
    build_vort2flux(B, dsh, sh, ids, false);
    B.add([=]() { launch_regT_out(dsh, dids, nr, mnf, douts, st); });
    for (auto& f : P) {
      f.fn();
      cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) { rc = fail_cuda(le, "preprocess launch"); break; }
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (rc == IBFS_OK && e != cudaSuccess) rc = fail_cuda(e, "preprocess a_times");
    for (void* p : tmp.allocs) cudaFree(p);
    tmp.allocs.clear();
  }
  cudaFree(pool);
  if (rc) return rc;
  int* dcid = dupload(h, need);
  int nn = (int)need.size();
  IBFS_CUDA_CHECK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->st));
  launch_chol_factor(h->d_cases, dcid, nn, h->d_status, h->st);
  int status = 0;
  IBFS_CUDA_CHECK(cudaMemcpyAsync(&status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  if (status) return fail(IBFS_ERR_CHOL, "choldc failed");
  launch_chol_inverse(h->d_cases, dcid, nn, h->st);
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  return IBFS_OK;
}

// Preconditioned CG cases: the slot of the step at device itime + offset
// (offset 1 before a step, 0 during the adjoint of the step being
// differentiated), the grid angle nearest the step's pitch; slots not yet
// factored are factored first, with the body turned by the slot's angle
// (positions and tables rebuilt there; the step's own move_body restores
// them). The slot index is a function of the step number alone, so every
// recomputation of a step uses the same factor.
#define IBFS_CHECK_OK(x)    \
  do {                      \
    int r_ = (x);           \
    if (r_) return r_;      \
  } while (0)

static int ensure_precond(ibfs_handle* h, int offset) {
  std::vector<int> pc;
  for (size_t i = 0; i < h->cases.size(); i++)
    if (h->cases[i].dc.cg_pre) pc.push_back((int)i);
  if (pc.empty()) return IBFS_OK;
  const int nc = (int)h->cases.size();
  std::vector<int> it(nc);
  IBFS_CUDA_CHECK(cudaMemcpyAsync(it.data(), h->d_itime, sizeof(int) * nc, cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  std::vector<int> todo, slot(nc, 0);
  for (int i : pc) {
    HostCase& hc = h->cases[i];
    const DevCase& d = hc.dc;
    int k = 0;
    if (d.moving) {
      double th = -(d.pitch_amp * std::sin(d.pitch_omega * (d.dt * (double)(it[i] + offset))));
      k = d.pre_k0 + (int)std::lround(th / d.pre_dth);
      k = std::max(0, std::min(k, (int)hc.pre_done.size() - 1));
    }
    slot[i] = k;
    if (!hc.pre_done[k]) todo.push_back(i);
  }
  if (!todo.empty()) {
    std::vector<int> mv;
    for (int i : todo) {
      HostCase& hc = h->cases[i];
      const DevCase& d = hc.dc;
      if (!d.moving) continue;
      // the zero-pitch shape turned by the slot's angle (move_body's rotation)
      const double th = (double)(slot[i] - d.pre_k0) * d.pre_dth, c = std::cos(th), s = std::sin(th);
      std::vector<double> x(hc.nb), y(hc.nb);
      for (int k = 0; k < hc.nb; k++) {
        double rx = hc.xb[k] - d.pivot_x, ry = hc.yb[k] - d.pivot_y;
        x[k] = d.pivot_x + c * rx - s * ry;
        y[k] = d.pivot_y + s * rx + c * ry;
      }
      IBFS_CUDA_CHECK(cudaMemcpy(d.xb, x.data(), sizeof(double) * hc.nb, cudaMemcpyHostToDevice));
      IBFS_CUDA_CHECK(cudaMemcpy(d.yb, y.data(), sizeof(double) * hc.nb, cudaMemcpyHostToDevice));
      mv.push_back(i);
    }
    if (!mv.empty()) {
      int* dmv = dupload(h, mv);
      launch_setup_reg_moving(h->d_cases, dmv, (int)mv.size(), h->max_nf, h->max_patch, h->st);
    }
    int rc = factor_cases(h, todo);
    if (rc) return rc;
    for (int i : todo) {
      HostCase& hc = h->cases[i];
      const DevCase& d = hc.dc;
      size_t nn = (size_t)d.nf * d.nf;
      double* dst = d.pre_fac + (size_t)slot[i] * 2 * nn;
      IBFS_CUDA_CHECK(cudaMemcpyAsync(dst, d.Linv, sizeof(double) * nn, cudaMemcpyDeviceToDevice, h->st));
      IBFS_CUDA_CHECK(cudaMemcpyAsync(dst + nn, d.LinvT, sizeof(double) * nn, cudaMemcpyDeviceToDevice, h->st));
      hc.pre_done[slot[i]] = 1;
    }
  }
  for (int i : pc)
    IBFS_CUDA_CHECK(cudaMemcpyAsync(const_cast<int*>(h->cases[i].dc.pre_idx), &slot[i], sizeof(int),
                                    cudaMemcpyHostToDevice, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));  // slot[] is host stack memory
  return IBFS_OK;
}

static int refresh_inverse(ibfs_handle* h, int ci) {
  std::vector<int> one{ci};
  int* dcid = dupload(h, one);
  launch_chol_inverse(h->d_cases, dcid, 1, h->st);
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  return IBFS_OK;
}

static int setup_case(ibfs_handle* h, HostCase& c, const ibfs_params_c& p, const ibfs_options_c* o, int nb,
                      const double* xb, const double* yb, const int* bdyno) {
  c.p = p;
  if (o) c.o = *o; else { memset(&c.o, 0, sizeof(c.o)); c.o.tile_cfg = -1; }
  if (p.m % 4 != 0 || p.n % 4 != 0 || p.m < 8 || p.n < 8)
    return fail(IBFS_ERR_GRID, "HEY! Grid nodes must be divisible by 4!!");
  c.m = p.m; c.n = p.n;
  c.delta = p.len / (double)p.m;
  int nlm = nlevmax(p.m, p.n);
  c.L = std::max(1, std::min(p.mgridlev, nlm));
  c.p.mgridlev = c.L;
  c.ns = (c.m - 1) * (c.n - 1);
  c.nq = (c.m + 1) * c.n + (c.n + 1) * c.m;
  c.nb = nb; c.nf = 2 * nb;
  c.nring = 2 * (c.m + 1) + 2 * (c.n + 1);
  c.norm = 4.0 * (double)(float)((long long)c.m * c.n);
  c.xb.assign(xb, xb + nb);
  c.yb.assign(yb, yb + nb);
  c.bdyno.assign(nb, 0);
  if (bdyno) c.bdyno.assign(bdyno, bdyno + nb);
  int bmin = 0, bmax = 0;
  for (int k = 0; k < nb; k++) {
    if (k == 0 || c.bdyno[k] < bmin) bmin = c.bdyno[k];
    if (k == 0 || c.bdyno[k] > bmax) bmax = c.bdyno[k];
  }
  c.bmin = bmin;
  c.nbody = nb ? bmax - bmin + 1 : 0;
  if (c.nbody > 64) return fail(IBFS_ERR_ARG, "at most 64 bodies per case");
  c.itime = p.istart;
  setup_reg_host(c);
  DevCase& d = c.dc;
  d.m = c.m; d.n = c.n; d.L = c.L; d.ns = c.ns; d.nq = c.nq; d.nb = c.nb; d.nf = c.nf; d.nring = c.nring;
  d.nbody = c.nbody; d.bmin = c.bmin;
  d.delta = c.delta; d.dt = p.dt; d.re = p.re; d.norm = c.norm;
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  d.omega = dalloc<double>(h, nsL);
  d.rhs_old = dalloc<double>(h, nsL);
  d.q = dalloc<double>(h, nqL);
  d.q0 = dalloc<double>(h, nqL);
  d.fb = dalloc<double>(h, c.nf);
  d.s = dalloc<double>(h, nsL);
  d.lastbc = dalloc<double>(h, (size_t)c.L * c.nring);
  d.rhsA = dalloc<double>(h, c.ns);
  d.wa = dalloc<double>(h, c.ns);
  d.wb = dalloc<double>(h, c.ns);
  d.wc = dalloc<double>(h, c.ns);
  d.wd = dalloc<double>(h, c.ns);
  d.vort = dalloc<double>(h, c.ns);
  d.cosx = cos_table(h, c.m);
  d.cosy = cos_table(h, c.n);
  d.Sm = sine_matrix(h, c.m);
  d.Sn = sine_matrix(h, c.n);
  d.rhsf = dalloc<double>(h, c.nf);
  d.motion = dalloc<double>(h, c.nf);
  d.fwork = dalloc<double>(h, c.nf);
  d.bvel = dalloc<double>(h, c.nf);
  d.face_ptr = dupload(h, c.face_ptr);
  d.face_f = dupload(h, c.face_f);
  d.face_w = dupload(h, c.face_w);
  d.force_ptr = dupload(h, c.force_ptr);
  d.force_face = dupload(h, c.force_face);
  d.force_w = dupload(h, c.force_w);
  d.wsum = dupload(h, c.wsum);
  d.bdyno = dupload(h, c.bdyno);
  d.Linv = dalloc<double>(h, (size_t)c.nf * c.nf);
  d.LinvT = dalloc<double>(h, (size_t)c.nf * c.nf);
  d.chol = dalloc<double>(h, (size_t)c.nf * c.nf + c.nf);
  if (!d.omega || !d.q || !d.s || !d.chol || !d.Sm || !d.Sn) return fail(IBFS_ERR_NOMEM, "device allocation failed");
  d.offx = p.offsetx;
  d.offy = p.offsety;
  d.moving = c.o.motion_kind == 1 ? 1 : 0;
  if (c.o.motion_kind != 0 && c.o.motion_kind != 1) return fail(IBFS_ERR_ARG, "unknown motion_kind");
  if (d.moving) {
    if (p.stationary) return fail(IBFS_ERR_ARG, "a moving body needs stationary = .FALSE. (CG force solve)");
    const double pi = 3.1415926535897932384;
    d.pitch_amp = c.o.pitch_amp_deg * pi / 180.0;
    d.pitch_omega = 2.0 * pi * c.o.pitch_freq;
    d.pivot_x = c.o.pivot_x;
    d.pivot_y = c.o.pivot_y;
    d.xb0 = dupload(h, c.xb);
    d.yb0 = dupload(h, c.yb);
    d.xb = dupload(h, c.xb);
    d.yb = dupload(h, c.yb);
    // patch of faces the body can reach: a disc around the pivot, 3 dx margin
    double R = 0.0;
    for (int k = 0; k < nb; k++)
      R = std::max(R, std::hypot(c.xb[k] - d.pivot_x, c.yb[k] - d.pivot_y));
    double mg = R + 3.0 * c.delta, dx = c.delta, h2 = 0.5 * dx;
    auto lo = [&](double v, double off, int lim) { return std::max(1, (int)std::floor((v + off) / dx) + 1 - 1); };
    auto hi = [&](double v, double off, int lim) { return std::min(lim, (int)std::ceil((v + off) / dx) + 1 + 1); };
    d.pu_i0 = lo(d.pivot_x - mg, p.offsetx, c.m + 1);
    d.pu_w = hi(d.pivot_x + mg, p.offsetx, c.m + 1) - d.pu_i0 + 1;
    d.pu_j0 = lo(d.pivot_y - mg, p.offsety - h2, c.n);
    d.pu_h = hi(d.pivot_y + mg, p.offsety - h2, c.n) - d.pu_j0 + 1;
    d.pv_i0 = lo(d.pivot_x - mg, p.offsetx - h2, c.m);
    d.pv_w = hi(d.pivot_x + mg, p.offsetx - h2, c.m) - d.pv_i0 + 1;
    d.pv_j0 = lo(d.pivot_y - mg, p.offsety, c.n + 1);
    d.pv_h = hi(d.pivot_y + mg, p.offsety, c.n + 1) - d.pv_j0 + 1;
    int np = d.pu_w * d.pu_h + d.pv_w * d.pv_h;
    d.pcnt = dalloc<int>(h, np);
    d.pf = dalloc<int>(h, (size_t)np * kPatchCap);
    d.pw = dalloc<double>(h, (size_t)np * kPatchCap);
    d.tcnt = dalloc<int>(h, c.nf);
    d.tface = dalloc<int>(h, (size_t)c.nf * 9);
    d.tw = dalloc<double>(h, (size_t)c.nf * 9);
    d.twsum = dalloc<double>(h, c.nf);
    h->max_patch = std::max(h->max_patch, np);
  }
  h->max_nb = std::max(h->max_nb, nb);
  if (!p.stationary) {
    d.cg_r = dalloc<double>(h, c.nf);
    d.cg_d = dalloc<double>(h, c.nf);
    d.cg_q = dalloc<double>(h, c.nf);
    d.cg_q2 = dalloc<double>(h, c.nf);
    d.cg_z = dalloc<double>(h, c.nf);
    d.cg_y = dalloc<double>(h, c.nf);
    d.cg_sc = dalloc<double>(h, 5);
    d.cg_pre = c.o.cg_precond ? 1 : 0;
    if (d.cg_pre) {
      // factor slots at a grid of pitch angles covering the amplitude, fine
      // enough that no body point is more than an eighth of a cell from where
      // the nearest slot has it (spacing 0.25 dx / r_max), at most 1 degree
      // and at most 1025 slots
      double rmax = 0.0;
      for (int k = 0; k < nb; k++)
        rmax = std::max(rmax, std::hypot(xb[k] - d.pivot_x, yb[k] - d.pivot_y));
      d.pre_dth = 3.1415926535897932384 / 180.0;
      if (rmax > 0.0) d.pre_dth = std::min(d.pre_dth, 0.25 * c.delta / rmax);
      if (d.moving) d.pre_dth = std::max(d.pre_dth, std::fabs(d.pitch_amp) / 512.0);
      d.pre_k0 = d.moving ? (int)std::ceil(std::fabs(d.pitch_amp) / d.pre_dth) : 0;
      int slots = 2 * d.pre_k0 + 1;
      d.pre_fac = dalloc<double>(h, (size_t)slots * 2 * c.nf * c.nf, false);
      d.pre_idx = dalloc<int>(h, 1);
      c.pre_done.assign(slots, 0);
      if (!d.pre_fac || !d.pre_idx) return fail(IBFS_ERR_NOMEM, "device allocation failed (preconditioner)");
    }
    d.cgtol = p.cgtol;
    d.cg_max_iter = p.cg_max_iter;
    d.cg_rel = c.o.cg_relative;
  }
  // initial state (variables.f90:55-64)
  if (p.unif_flow) {
    std::vector<double> q0(nqL, 0.0);
    for (int k = 1; k <= c.L; k++)
      for (size_t t = 0; t < (size_t)(c.m + 1) * c.n; t++) q0[t + (k - 1) * c.nq] = c.delta * std::pow(2.0, k - 1);
    cudaMemcpy(d.q0, q0.data(), sizeof(double) * nqL, cudaMemcpyHostToDevice);
  }
  d.q0_const = 1;
  d.q0_u1 = p.unif_flow ? c.delta : 0.0;
  return IBFS_OK;
}

// Whether a q0 array (L levels of Nq faces) is q0_u1 * 2^(k-1) on the u-faces
// of every level k and 0 on the v-faces, for q0_u1 = its first value.
static bool q0_closed_form(const HostCase& c, const double* q0, double* u1) {
  const size_t nu = (size_t)(c.m + 1) * c.n;
  *u1 = q0[0];
  for (int k = 1; k <= c.L; k++) {
    const double* lv = q0 + (size_t)(k - 1) * c.nq;
    const double uk = *u1 * std::pow(2.0, k - 1);
    for (size_t t = 0; t < nu; t++)
      if (lv[t] != uk) return false;
    for (size_t t = nu; t < (size_t)c.nq; t++)
      if (lv[t] != 0.0) return false;
  }
  return true;
}

static int finish_create(ibfs_handle* h) {
  gemm_f64_init();
  IBFS_CUDA_CHECK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  IBFS_CUDA_CHECK(cudaEventCreate(&h->ev0));
  IBFS_CUDA_CHECK(cudaEventCreate(&h->ev1));
  int nc = (int)h->cases.size();
  h->d_itime = dalloc<int>(h, nc);
  h->d_status = dalloc<int>(h, 4);
  int off = 0;
  for (int i = 0; i < nc; i++) {
    HostCase& c = h->cases[i];
    c.out_off = off;
    off += 2 * c.nbody + c.L + 1;
    h->max_ns = std::max(h->max_ns, c.ns);
    h->max_nq = std::max(h->max_nq, c.nq);
    h->max_nf = std::max(h->max_nf, c.nf);
    h->max_ring = std::max(h->max_ring, c.nring);
    h->max_L = std::max(h->max_L, c.L);
  }
  h->out_stride = off;
  h->d_out = dalloc<double>(h, off);
  // body velocities of all cases in one array, so that a batched step moves
  // them with one copy
  for (auto& c : h->cases) h->sum_nf += c.nf;
  h->d_bvel = dalloc<double>(h, h->sum_nf);
  if (!h->d_bvel || cudaMallocHost(&h->h_bvel, sizeof(double) * std::max(1, h->sum_nf)) != cudaSuccess)
    return fail(IBFS_ERR_NOMEM, "body velocity buffers");
  for (int i = 0, o = 0; i < nc; i++) {
    h->cases[i].dc.bvel = h->d_bvel + o;
    o += h->cases[i].nf;
  }
  int nitems = 0;
  for (auto& c : h->cases) nitems += c.L;
  h->d_partial = dalloc<double>(h, (size_t)nitems * 32);
  std::vector<int> it0(nc);
  for (int i = 0; i < nc; i++) {
    HostCase& c = h->cases[i];
    c.dc.out = h->d_out + c.out_off;
    c.dc.itime = h->d_itime + i;
    c.dc.status = h->d_status;
    it0[i] = c.itime;
  }
  cudaMemcpy(h->d_itime, it0.data(), sizeof(int) * nc, cudaMemcpyHostToDevice);
  // CG flags for every case; a_times shadows for the CG cases
  h->d_cgit = dalloc<int>(h, 2 * nc);
  h->h_cgit.assign(2 * nc, 0);
  h->cg_ids.clear();
  for (int i = 0; i < nc; i++) {
    h->cases[i].dc.cg_it = h->d_cgit + 2 * i;
    if (!h->cases[i].p.stationary) h->cg_ids.push_back(i);
  }
  h->cg = !h->cg_ids.empty();
  if (h->cg) {
    size_t om = 0, rest = 0;
    for (int i : h->cg_ids) {
      const DevCase& c = h->cases[i].dc;
      om += (size_t)c.L * c.ns;
      rest += (size_t)c.L * c.ns + c.nq + 4 * (size_t)c.ns;
    }
    h->sh_omega = dalloc<double>(h, om);
    double* pr = dalloc<double>(h, rest);
    if (!h->sh_omega || !pr) return fail(IBFS_ERR_NOMEM, "device allocation failed (CG scratch)");
    h->sh_omega_bytes = om * sizeof(double);
    double* po = h->sh_omega;
    for (int i : h->cg_ids) {
      DevCase s = h->cases[i].dc;
      s.omega = po; po += (size_t)s.L * s.ns;
      s.s = pr; pr += (size_t)s.L * s.ns;
      s.q = pr; pr += s.nq;
      s.wa = pr; pr += s.ns;
      s.wb = pr; pr += s.ns;
      s.wc = pr; pr += s.ns;
      s.vort = pr; pr += s.ns;
      h->shx.push_back(s);
      s.fb = h->cases[i].dc.cg_d;
      h->shd.push_back(s);
    }
    h->d_shx = dupload(h, h->shx);
    h->d_shd = dupload(h, h->shd);
  }
  std::vector<DevCase> dcs;
  for (auto& c : h->cases) dcs.push_back(c.dc);
  h->d_cases = dupload(h, dcs);
  if (!h->d_cases || !h->d_out) return fail(IBFS_ERR_NOMEM, "device allocation failed");
  if (cudaMallocHost(&h->h_stage, sizeof(double) * std::max(off, h->max_nf) * 2) != cudaSuccess)
    return fail(IBFS_ERR_NOMEM, "pinned allocation failed");
  if (h->precision == 1) {
    int rc = precision_init(h->prec, h->st, dcs, h->d_cases, [h](size_t bytes) -> void* {
      void* p = nullptr;
      if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
      cudaMemset(p, 0, bytes);
      h->allocs.push_back(p);
      return p;
    });
    if (rc) return fail(rc, precision_error());
    precision_set_tile(h->prec, h->cases[0].o.tc_tile);
    precision_set_refine(h->prec, h->cases[0].o.refine_slices, h->cases[0].o.poisson_sweeps);
  }
  build_step_program(h);
  IBFS_CUDA_CHECK(cudaDeviceSynchronize());
  capture_graph(h);
  IBFS_CUDA_CHECK(cudaGetLastError());
  return IBFS_OK;
}

static void free_adj(ibfs_handle* h);

static void free_handle(ibfs_handle* h) {
  if (!h) return;
  if (h->st) cudaStreamSynchronize(h->st);
  free_adj(h);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->gx_iter) cudaGraphExecDestroy(h->gx_iter);
  if (h->gx_iter50) cudaGraphExecDestroy(h->gx_iter50);
  if (h->gx_post) cudaGraphExecDestroy(h->gx_post);
  for (void* p : h->allocs) cudaFree(p);
  if (h->h_stage) cudaFreeHost(h->h_stage);
  if (h->h_bvel) cudaFreeHost(h->h_bvel);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->st) cudaStreamDestroy(h->st);
  if (h->prec) precision_free(h->prec);
  delete h;
}

static int run_apply_op(ibfs_handle* h, int op, const double* in, double* out);

}  // namespace ibfs

#include "ibfs_adjoint_host.cuh"
#include "ibfs_adjoint_motion_host.cuh"

namespace ibfs {
static void free_adj(ibfs_handle* h) {
  if (h->adjm) {
    for (cudaGraphExec_t g : {h->adjm->g_head, h->adjm->g_tail, h->adjm->g_tailf, h->adjm->g_start,
                              h->adjm->g_iter, h->adjm->g_iter50, h->adjm->g_u})
      if (g) cudaGraphExecDestroy(g);
    delete h->adjm;
    h->adjm = nullptr;
  }
  if (!h->adj) return;
  if (h->adj->g_bw) cudaGraphExecDestroy(h->adj->g_bw);
  if (h->adj->g_bwf) cudaGraphExecDestroy(h->adj->g_bwf);
  if (h->adj->h_a) cudaFreeHost(h->adj->h_a);
  delete h->adj;
  h->adj = nullptr;
}
}  // namespace ibfs

// ===========================================================================
// C-ABI
// Status word of the tensor-core GEMM after a step: bit 2 = a bounded wait
// gave up (status[1..3]: role, block, pipeline step of the first one), bit 4 =
// a drain wait gave up as well. Reads it with the stream synchronised.
static int check_device_waits(ibfs_handle* h) {
  int st4[4] = {0, 0, 0, 0};
  IBFS_CUDA_CHECK(cudaMemcpyAsync(st4, h->d_status, sizeof(st4), cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  if (!(st4[0] & 2)) return IBFS_OK;
  static const char* roles[] = {"?", "producer waiting for a free stage", "MMA waiting for a free accumulator",
                                "MMA waiting for a loaded stage", "epilogue waiting for an accumulator",
                                "probe wait of the timeout test"};
  const int r = (st4[1] >= 1 && st4[1] <= 5) ? st4[1] : 0;
  std::string msg = std::string("a bounded device wait gave up (tensor-core GEMM: ") + roles[r] + ", block " +
                    std::to_string(st4[2]) + ", step " + std::to_string(st4[3]) + ")";
  if (st4[0] & 4) msg += "; a drain of in-flight copies also gave up";
  msg += "; the handle's state is undefined";
  return fail(IBFS_ERR_TIMEOUT, msg);
}

extern "C" {

int ibfs_batch_create(int ncases, const ibfs_params_c* p, const ibfs_options_c* opt, const int* nb,
                      const double* xb, const double* yb, const int* bdyno, ibfs_handle** out) {
  if (!out || !p || !nb || ncases < 1) return fail(IBFS_ERR_ARG, "null argument");
  *out = nullptr;
  ibfs_handle* h = new ibfs_handle();
  h->precision = opt ? opt[0].precision : 0;
  h->tile_cfg = opt ? opt[0].tile_cfg : -1;
  if (opt && opt[0].tile_cfg == 0 && opt[0].precision == 0 && opt[0].cg_relative == 0 && opt[0].motion_kind == 0)
    h->tile_cfg = -1;  // zero-initialised options mean "auto"
  h->cases.resize(ncases);
  size_t off = 0;
  for (int i = 0; i < ncases; i++) {
    int rc = setup_case(h, h->cases[i], p[i], opt ? &opt[i] : nullptr, nb[i], xb + off, yb + off,
                        bdyno ? bdyno + off : nullptr);
    off += nb[i];
    if (rc) { std::string e = t_error; free_handle(h); t_error = e; return rc; }
  }
  int rc = finish_create(h);
  if (rc) { std::string e = t_error; free_handle(h); t_error = e; return rc; }
  *out = h;
  return IBFS_OK;
}

int ibfs_create(const ibfs_params_c* p, const ibfs_options_c* opt, int nb, const double* xb, const double* yb,
                const int* bdyno, ibfs_handle** out) {
  return ibfs_batch_create(1, p, opt, &nb, xb, yb, bdyno, out);
}

int ibfs_destroy(ibfs_handle* h) {
  free_handle(h);
  return IBFS_OK;
}

int ibfs_num_cases(const ibfs_handle* h) { return h ? (int)h->cases.size() : 0; }

int ibfs_case_sizes(const ibfs_handle* h, int icase, int* m, int* n, int* nlev, int* nq, int* nb, int* nbody) {
  if (!h || icase < 0 || icase >= (int)h->cases.size()) return IBFS_ERR_ARG;
  const HostCase& c = h->cases[icase];
  if (m) *m = c.m;
  if (n) *n = c.n;
  if (nlev) *nlev = c.L;
  if (nq) *nq = c.nq;
  if (nb) *nb = c.nb;
  if (nbody) *nbody = c.nbody;
  return IBFS_OK;
}

int ibfs_set_state(ibfs_handle* h, int icase, const double* omega, const double* fb, const double* rhs_old,
                   const double* q, const double* q0) {
  if (!h || icase < 0 || icase >= (int)h->cases.size()) return IBFS_ERR_ARG;
  HostCase& c = h->cases[icase];
  if (q0) {  // the stencils read q0 from the array unless it has the closed form
    double u1 = 0.0;
    const int cf = q0_closed_form(c, q0, &u1) ? 1 : 0;
    if (cf != c.dc.q0_const || (cf && u1 != c.dc.q0_u1)) {
      c.dc.q0_const = cf;
      c.dc.q0_u1 = cf ? u1 : 0.0;
      IBFS_CUDA_CHECK(cudaMemcpyAsync(&h->d_cases[icase].q0_const, &c.dc.q0_const, sizeof(int),
                                      cudaMemcpyHostToDevice, h->st));
      IBFS_CUDA_CHECK(cudaMemcpyAsync(&h->d_cases[icase].q0_u1, &c.dc.q0_u1, sizeof(double),
                                      cudaMemcpyHostToDevice, h->st));
    }
  }
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  auto cp = [&](double* d, const double* s, size_t n) {
    return s ? cudaMemcpyAsync(d, s, n * sizeof(double), cudaMemcpyHostToDevice, h->st) : cudaSuccess;
  };
  IBFS_CUDA_CHECK(cp(c.dc.omega, omega, nsL));
  IBFS_CUDA_CHECK(cp(c.dc.fb, fb, c.nf));
  IBFS_CUDA_CHECK(cp(c.dc.rhs_old, rhs_old, nsL));
  IBFS_CUDA_CHECK(cp(c.dc.q, q, nqL));
  IBFS_CUDA_CHECK(cp(c.dc.q0, q0, nqL));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  return IBFS_OK;
}

int ibfs_get_state(const ibfs_handle* h, int icase, double* omega, double* fb, double* rhs_old, double* q,
                   double* q0) {
  if (!h || icase < 0 || icase >= (int)h->cases.size()) return IBFS_ERR_ARG;
  const HostCase& c = h->cases[icase];
  size_t nsL = (size_t)c.L * c.ns, nqL = (size_t)c.L * c.nq;
  auto cp = [&](double* d, const double* s, size_t n) {
    return d ? cudaMemcpyAsync(d, s, n * sizeof(double), cudaMemcpyDeviceToHost, h->st) : cudaSuccess;
  };
  IBFS_CUDA_CHECK(cp(omega, c.dc.omega, nsL));
  IBFS_CUDA_CHECK(cp(fb, c.dc.fb, c.nf));
  IBFS_CUDA_CHECK(cp(rhs_old, c.dc.rhs_old, nsL));
  IBFS_CUDA_CHECK(cp(q, c.dc.q, nqL));
  IBFS_CUDA_CHECK(cp(q0, c.dc.q0, nqL));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  return IBFS_OK;
}

int ibfs_vertex_fields(ibfs_handle* h, int icase, int level, double* out) {
  if (!h || icase < 0 || icase >= (int)h->cases.size() || !out) return fail(IBFS_ERR_ARG, "null argument or case");
  const HostCase& c = h->cases[icase];
  if (level < 1 || level > c.L) return fail(IBFS_ERR_ARG, "level outside 1..mgridlev");
  if (!h->d_vertex) {
    h->d_vertex = dalloc<double>(h, (size_t)5 * h->max_ns, false);
    if (!h->d_vertex) return fail(IBFS_ERR_NOMEM, "vertex buffer");
  }
  launch_vertex(h->d_cases, icase, level, c.ns, h->d_vertex, h->st);
  IBFS_CUDA_CHECK(cudaGetLastError());
  IBFS_CUDA_CHECK(cudaMemcpyAsync(out, h->d_vertex, sizeof(double) * 5 * (size_t)c.ns, cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  return IBFS_OK;
}

int ibfs_set_cholesky(ibfs_handle* h, int icase, const double* cholmat, const double* cholvec) {
  if (!h || icase < 0 || icase >= (int)h->cases.size() || !cholmat || !cholvec) return IBFS_ERR_ARG;
  HostCase& c = h->cases[icase];
  size_t nf = c.nf;
  IBFS_CUDA_CHECK(cudaMemcpy(c.dc.chol, cholmat, nf * nf * sizeof(double), cudaMemcpyHostToDevice));
  IBFS_CUDA_CHECK(cudaMemcpy(c.dc.chol + nf * nf, cholvec, nf * sizeof(double), cudaMemcpyHostToDevice));
  int rc = refresh_inverse(h, icase);
  if (rc) return rc;
  c.have_chol = true;
  return IBFS_OK;
}

int ibfs_get_cholesky(const ibfs_handle* h, int icase, double* cholmat, double* cholvec) {
  if (!h || icase < 0 || icase >= (int)h->cases.size()) return IBFS_ERR_ARG;
  const HostCase& c = h->cases[icase];
  size_t nf = c.nf;
  if (cholmat) IBFS_CUDA_CHECK(cudaMemcpy(cholmat, c.dc.chol, nf * nf * sizeof(double), cudaMemcpyDeviceToHost));
  if (cholvec) IBFS_CUDA_CHECK(cudaMemcpy(cholvec, c.dc.chol + nf * nf, nf * sizeof(double), cudaMemcpyDeviceToHost));
  return IBFS_OK;
}

int ibfs_precompute(ibfs_handle* h) {
  if (!h) return IBFS_ERR_ARG;
  int rc = precompute(h);
  if (rc) h->err = t_error;
  return rc;
}

int ibfs_advance(ibfs_handle* h, int* itime, const double* body_vel, double* fx, double* fy, double* circ,
                 double* slip) {
  if (!h || !itime || h->cases.size() != 1) return fail(IBFS_ERR_ARG, "ibfs_advance needs a single-case handle");
  HostCase& c = h->cases[0];
  if (*itime != c.itime) {
    c.itime = *itime;
    IBFS_CUDA_CHECK(cudaMemcpyAsync(h->d_itime, itime, sizeof(int), cudaMemcpyHostToDevice, h->st));
  }
  // preprocess at the first step (operators.f90:88-90), unless the caller
  // supplied the factor (the reference reads input/ibfs.chd then, :44-46)
  if (needs_factor(c)) {
    int rc = precompute(h);
    if (rc) { h->err = t_error; return rc; }
  }
  if (body_vel) {
    memcpy(h->h_stage, body_vel, sizeof(double) * c.nf);
    IBFS_CUDA_CHECK(cudaMemcpyAsync(c.dc.bvel, h->h_stage, sizeof(double) * c.nf, cudaMemcpyHostToDevice, h->st));
  } else {
    IBFS_CUDA_CHECK(cudaMemsetAsync(c.dc.bvel, 0, sizeof(double) * c.nf, h->st));
  }
  // IBFS_ERR_CG_MAXITER is the reference's warning (operators.f90:435-438):
  // the step is complete, so its outputs are still returned
  int rc = run_step(h);
  if (rc && rc != IBFS_ERR_CG_MAXITER) { h->err = t_error; return rc; }
  if (rc) h->err = t_error;
  double* o = h->h_stage + c.nf;
  IBFS_CUDA_CHECK(cudaMemcpyAsync(o, h->d_out, sizeof(double) * h->out_stride, cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  {
    int wrc = check_device_waits(h);
    if (wrc) { h->err = t_error; return wrc; }
  }
  *itime += 1;
  c.itime = *itime;
  if (fx) memcpy(fx, o, sizeof(double) * c.nbody);
  if (fy) memcpy(fy, o + c.nbody, sizeof(double) * c.nbody);
  if (circ) memcpy(circ, o + 2 * c.nbody, sizeof(double) * c.L);
  if (slip) *slip = o[2 * c.nbody + c.L];
  return rc;
}

int ibfs_batch_advance(ibfs_handle* h, const double* body_vel, double* out) {
  if (!h) return IBFS_ERR_ARG;
  bool need = false;
  for (auto& c : h->cases) if (needs_factor(c)) need = true;
  if (need) {
    int rc = precompute(h);
    if (rc) { h->err = t_error; return rc; }
  }
  if (body_vel) {
    memcpy(h->h_bvel, body_vel, sizeof(double) * h->sum_nf);
    IBFS_CUDA_CHECK(cudaMemcpyAsync(h->d_bvel, h->h_bvel, sizeof(double) * h->sum_nf, cudaMemcpyHostToDevice, h->st));
  } else {
    IBFS_CUDA_CHECK(cudaMemsetAsync(h->d_bvel, 0, sizeof(double) * h->sum_nf, h->st));
  }
  int rc = run_step(h);
  if (rc && rc != IBFS_ERR_CG_MAXITER) { h->err = t_error; return rc; }
  if (rc) h->err = t_error;
  IBFS_CUDA_CHECK(cudaMemcpyAsync(h->h_stage, h->d_out, sizeof(double) * h->out_stride, cudaMemcpyDeviceToHost, h->st));
  {
    int wrc = check_device_waits(h);
    if (wrc) { h->err = t_error; return wrc; }
  }
  if (out) memcpy(out, h->h_stage, sizeof(double) * h->out_stride);
  for (auto& c : h->cases) c.itime += 1;
  return rc;
}

int ibfs_advance_n(ibfs_handle* h, int nsteps, double* hist) {
  if (!h || nsteps < 0) return IBFS_ERR_ARG;
  bool need = false;
  for (auto& c : h->cases) if (needs_factor(c)) need = true;
  if (need) {
    int rc = precompute(h);
    if (rc) { h->err = t_error; return rc; }
  }
  if (hist && h->hist_steps < nsteps) {
    if (h->d_hist) cudaFree(h->d_hist);
    if (cudaMalloc(&h->d_hist, sizeof(double) * (size_t)nsteps * h->out_stride) != cudaSuccess)
      return fail(IBFS_ERR_NOMEM, "history allocation failed");
    h->hist_steps = nsteps;
  }
  IBFS_CUDA_CHECK(cudaEventRecord(h->ev0, h->st));
  int warn = IBFS_OK;
  for (int s = 0; s < nsteps; s++) {
    int rc = run_step(h);
    if (rc == IBFS_ERR_CG_MAXITER) { h->err = t_error; warn = rc; rc = IBFS_OK; }
    if (rc) { h->err = t_error; return rc; }
    if (hist)
      IBFS_CUDA_CHECK(cudaMemcpyAsync(h->d_hist + (size_t)s * h->out_stride, h->d_out,
                                      sizeof(double) * h->out_stride, cudaMemcpyDeviceToDevice, h->st));
  }
  IBFS_CUDA_CHECK(cudaEventRecord(h->ev1, h->st));
  if (hist)
    IBFS_CUDA_CHECK(cudaMemcpyAsync(hist, h->d_hist, sizeof(double) * (size_t)nsteps * h->out_stride,
                                    cudaMemcpyDeviceToHost, h->st));
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  {
    int wrc = check_device_waits(h);
    if (wrc) { h->err = t_error; return wrc; }
  }
  for (auto& c : h->cases) c.itime += nsteps;
  return warn;
}

int ibfs_output_offset(const ibfs_handle* h, int icase) {
  if (!h || icase < 0 || icase >= (int)h->cases.size()) return -1;
  return h->cases[icase].out_off;
}
int ibfs_output_stride(const ibfs_handle* h) { return h ? h->out_stride : 0; }

int ibfs_kernels_per_step(const ibfs_handle* h) { return h ? h->graph_kernels : -1; }

int ibfs_gemm_tiles(const ibfs_handle* h, int* cfgs, int max) {
  if (!h) return -1;
  if (!h->prec) return 0;
  const std::vector<int>& w = precision_tile_choices(h->prec);
  for (int i = 0; cfgs && i < (int)w.size() && i < max; i++) cfgs[i] = w[i];
  return (int)w.size();
}

int ibfs_last_cg_iterations(const ibfs_handle* h) { return h ? h->last_cg_iters : -1; }

int ibfs_adjoint_run(ibfs_handle* h, int nsteps, int checkpoint_every, const double* body_vel, const double* wx,
                     const double* wy, double* J, double* grad_vel, double* ms_forward, double* ms_total) {
  if (!h) return IBFS_ERR_ARG;
  int rc = adj_run(h, nsteps, checkpoint_every, body_vel, wx, wy, J, grad_vel, ms_forward, ms_total);
  if (rc) h->err = ibfs_last_error(nullptr);
  return rc;
}

int ibfs_set_actuators(ibfs_handle* h, int icase, int n_act, const int* npt, const double* u_j,
                       const double* u_j_osc, const double* omg_j, const double* theta_j) {
  if (!h) return IBFS_ERR_ARG;
  if (icase < 0 || icase >= (int)h->cases.size() || n_act < 0 ||
      (n_act > 0 && (!npt || !u_j || !u_j_osc || !omg_j || !theta_j)))
    return fail(IBFS_ERR_ARG, "ibfs_set_actuators: bad arguments");
  HostCase& c = h->cases[icase];
  std::vector<double> tab;
  const double pi = 3.1415926535897932384;
  for (int a = 0; a < n_act; a++) {
    if (npt[a] < 1) return fail(IBFS_ERR_ARG, "ibfs_set_actuators: an actuator needs at least one point");
    for (int p = 0; p < npt[a]; p++) {
      tab.push_back(u_j[a]);
      tab.push_back(u_j_osc[a]);
      tab.push_back(omg_j[a]);
      tab.push_back(std::cos(pi / 180.0 * theta_j[a]));
      tab.push_back(std::sin(pi / 180.0 * theta_j[a]));
    }
  }
  const int nact = (int)tab.size() / 5;
  if (nact > c.nb) return fail(IBFS_ERR_ARG, "ibfs_set_actuators: more actuator points than body points");
  c.dc.nact = nact;
  c.dc.act = nact ? dupload(h, tab) : nullptr;
  if (nact && !c.dc.act) return fail(IBFS_ERR_NOMEM, "device allocation failed (actuators)");
  IBFS_CUDA_CHECK(cudaMemcpy(h->d_cases + icase, &c.dc, sizeof(DevCase), cudaMemcpyHostToDevice));
  build_step_program(h);
  IBFS_CUDA_CHECK(cudaDeviceSynchronize());
  capture_graph(h);
  IBFS_CUDA_CHECK(cudaGetLastError());
  return IBFS_OK;
}

int ibfs_adjoint_pitch_run(ibfs_handle* h, int nsteps, int checkpoint_every, const double* wx, const double* wy,
                           double* J, double* dJ_damp, double* ms_forward, double* ms_total) {
  if (!h) return IBFS_ERR_ARG;
  int rc = adjm_run(h, nsteps, checkpoint_every, wx, wy, J, dJ_damp, ms_forward, ms_total);
  if (rc) h->err = ibfs_last_error(nullptr);
  return rc;
}

int ibfs_profile_step(ibfs_handle* h, double* ms, int* launches, double* flops) {
  if (!h || !ms || !launches || !flops) return IBFS_ERR_ARG;
  IBFS_CHECK_OK(ensure_precond(h, 1));
  size_t n = h->prog.size();
  std::vector<cudaEvent_t> ev(n + 1);
  for (auto& e : ev) IBFS_CUDA_CHECK(cudaEventCreate(&e));
  for (int t = 0; t < TAG_NTAGS; t++) { ms[t] = 0.0; launches[t] = 0; flops[t] = 0.0; }
  IBFS_CUDA_CHECK(cudaEventRecord(ev[0], h->st));
  for (size_t i = 0; i < n; i++) {
    h->prog[i].fn();
    IBFS_CUDA_CHECK(cudaEventRecord(ev[i + 1], h->st));
  }
  IBFS_CUDA_CHECK(cudaStreamSynchronize(h->st));
  IBFS_CUDA_CHECK(cudaGetLastError());
  for (size_t i = 0; i < n; i++) {
    float t = 0.f;
    cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
    int tag = h->prog[i].tag;
    ms[tag] += t;
    launches[tag] += 1;
    flops[tag] += h->prog[i].flops;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (auto& c : h->cases) c.itime += 1;
  int wrc = check_device_waits(h);
  if (wrc) h->err = t_error;
  return wrc;
}

int ibfs_set_wait_limit(ibfs_handle* h, double seconds, int probe) {
  if (!h || !(seconds >= 0.0) || seconds > 60.0)
    return fail(IBFS_ERR_ARG, "ibfs_set_wait_limit: seconds must be in [0, 60]");
  if (!h->prec) return IBFS_OK;  // plain FP64 handles have no bounded device waits
  int rc = precision_set_wait_limit(h->prec, seconds, probe);
  if (rc) return fail(rc, "ibfs_set_wait_limit: cannot write the limit to the device");
  return IBFS_OK;
}

int ibfs_last_timing(const ibfs_handle* h, double* ms) {
  if (!h || !ms) return IBFS_ERR_ARG;
  *ms = h->last_ms;
  return IBFS_OK;
}

int ibfs_apply_op(ibfs_handle* h, int op, const double* in, double* out) {
  if (!h || !in || !out) return IBFS_ERR_ARG;
  int rc = run_apply_op(h, op, in, out);
  if (rc) h->err = t_error;
  return rc;
}

const char* ibfs_last_error(const ibfs_handle* h) {
  if (h && !h->err.empty()) return h->err.c_str();
  return t_error.c_str();
}

}  // extern "C"

namespace ibfs {

// Single-operator application on case 0 (verification entry point).
static int run_apply_op(ibfs_handle* h, int op, const double* in, double* out) {
  HostCase& hc = h->cases[0];
  DevCase c = hc.dc;
  cudaStream_t st = h->st;
  Prog P;
  ibfs_handle tmp;
  tmp.st = st;
  tmp.tile_cfg = h->tile_cfg;
  ProgBuilder B{&tmp, P};
  size_t ns = c.ns;
  // private scratch so the case state is untouched
  DevCase s = c;
  s.omega = dalloc<double>(&tmp, (size_t)c.L * ns);
  s.s = dalloc<double>(&tmp, (size_t)c.L * ns);
  s.q = dalloc<double>(&tmp, (size_t)c.L * c.nq);
  s.fb = dalloc<double>(&tmp, c.nf);
  s.wa = dalloc<double>(&tmp, ns);
  s.wb = dalloc<double>(&tmp, ns);
  s.wc = dalloc<double>(&tmp, ns);
  s.vort = dalloc<double>(&tmp, ns);
  std::vector<DevCase> sv{s};
  DevCase* ds = dupload(&tmp, sv);
  std::vector<int> ids{0};
  const int* dids = B.ints(ids);
  int rc = IBFS_OK;
  size_t out_n = 0;
  double* dout = nullptr;
  if (op == 0 || op == 1 || op == 2) {
    out_n = ns;
    IBFS_CUDA_CHECK(cudaMemcpy(s.vort, in, ns * sizeof(double), cudaMemcpyHostToDevice));
    if (h->precision == 1) {
      rc = precision_apply_op(h->prec, op, ds, s, st);
      if (rc) rc = fail(rc, precision_error());
      dout = s.omega;
    } else {
      if (op == 0) {
        B.gemm({right_desc(s, s.vort, s.wa)}, false);
        B.gemm({left_desc(s, s.wa, s.omega, EPI_STORE, 1)}, false);
      } else {
        B.gemm({right_desc(s, s.vort, s.wa)}, false);
        B.gemm({left_desc(s, s.wa, s.wb, op == 1 ? EPI_LAMINV : EPI_AINV, 1)}, false);
        B.gemm({right_desc(s, s.wb, s.wa)}, false);
        B.gemm({left_desc(s, s.wa, s.omega, EPI_STORE, 1)}, false);
      }
      dout = s.omega;
    }
  } else if (op == 3) {  // a_times
    out_n = c.nf;
    IBFS_CUDA_CHECK(cudaMemcpy(s.fb, in, c.nf * sizeof(double), cudaMemcpyHostToDevice));
    IBFS_CUDA_CHECK(cudaMemset(s.omega, 0, (size_t)c.L * ns * sizeof(double)));
    auto bm1 = B.bmap({(int)ns});
    B.add([=]() { launch_regrot(ds, dids, bm1.first, bm1.second, st); });
    if (h->precision == 1) build_precision_ainv(h->prec, P, ds, sv, EPI_STORE, st);
    else build_ainv(B, sv, EPI_STORE);
    if (h->precision == 1) build_precision_vort2flux(h->prec, P, ds, sv, ids, false, st);
    else build_vort2flux(B, ds, sv, ids, false);
    double** douts = nullptr;
    std::vector<double*> o1{s.wc};
    douts = dupload(&tmp, o1);
    int nf = c.nf;
    B.add([=]() { launch_regT_out(ds, dids, 1, nf, douts, st); });
    dout = s.wc;
  } else if (op == 4) {  // regT
    out_n = c.nf;
    IBFS_CUDA_CHECK(cudaMemcpy(s.q, in, c.nq * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double*> o1{s.wc};
    double** douts = dupload(&tmp, o1);
    int nf = c.nf;
    B.add([=]() { launch_regT_out(ds, dids, 1, nf, douts, st); });
    dout = s.wc;
  } else if (op == 5) {  // rot(reg(f))
    out_n = ns;
    IBFS_CUDA_CHECK(cudaMemcpy(s.fb, in, c.nf * sizeof(double), cudaMemcpyHostToDevice));
    auto bm1 = B.bmap({(int)ns});
    B.add([=]() { launch_regrot(ds, dids, bm1.first, bm1.second, st); });
    dout = s.vort;
  } else {
    rc = fail(IBFS_ERR_ARG, "unknown op");
  }
  if (rc == IBFS_OK) {
    for (auto& f : P) f.fn();
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = fail_cuda(e, "apply_op");
    else if (cudaMemcpy(out, dout, out_n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = fail(IBFS_ERR_CUDA, "copy out");
  }
  for (void* p : tmp.allocs) cudaFree(p);
  tmp.allocs.clear();
  return rc;
}

}  // namespace ibfs
