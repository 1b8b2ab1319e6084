// ibfs_handle.cuh -- host-side handle of the B200 IBFS advance (shared by
// the C-ABI runtime and the adjoint driver).
#pragma once
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/ibfs_capi.h"
#include "ibfs_common.cuh"
#include "ibfs_kernels.cuh"
#include "ibfs_precision.cuh"
#include "ibfs_adjoint.cuh"

namespace ibfs {

struct AdjPlan;   // adjoint driver state (ibfs_adjoint_host.cuh)
struct AdjMPlan;  // moving-body adjoint state (ibfs_adjoint_motion_host.cuh)

struct HostCase {
  ibfs_params_c p;
  ibfs_options_c o;
  int m, n, L, ns, nq, nb, nf, nring, nbody, bmin;
  double delta, norm;
  std::vector<double> xb, yb;
  std::vector<int> bdyno;
  std::vector<int> face_ptr, face_f, force_ptr, force_face;
  std::vector<double> face_w, force_w, wsum;
  bool have_chol = false;
  std::vector<char> pre_done;  // preconditioner slots already factored (cg_precond)
  int out_off = 0;
  int itime = 0;
  DevCase dc{};
};

}  // namespace ibfs

using namespace ibfs;

struct ibfs_handle {
  std::vector<HostCase> cases;
  std::vector<void*> allocs;
  DevCase* d_cases = nullptr;
  std::map<int, double*> sine;
  std::map<int, double*> costab;
  cudaStream_t st = nullptr;
  Prog prog;                       // whole step (Cholesky handles) or the part before CG
  Prog prog_iter, prog_iter50, prog_post;  // CG handles: one iteration, one with residual refresh, after CG
  cudaGraphExec_t gexec = nullptr, gx_iter = nullptr, gx_iter50 = nullptr, gx_post = nullptr;
  bool graph_ok = false;
  int graph_kernels = 0;  // kernel nodes in the captured step graph(s), one CG iteration counted
  bool cg = false;        // cases solve the force system by CG (stationary = .FALSE.)
  int* d_cgit = nullptr;  // [ncases][2] iterations, active
  // a_times shadows of the CG cases: input fb (x) or cg_d (d), private scratch
  std::vector<DevCase> shx, shd;
  std::vector<int> cg_ids;
  DevCase *d_shx = nullptr, *d_shd = nullptr;
  double* sh_omega = nullptr;
  size_t sh_omega_bytes = 0;
  int max_patch = 0, max_nb = 0;
  std::vector<int> h_cgit;
  int last_cg_iters = 0;
  int* d_status = nullptr;
  int* d_itime = nullptr;
  double* d_out = nullptr;
  double* d_hist = nullptr;
  int hist_steps = 0;
  int out_stride = 0;
  double* d_partial = nullptr;
  std::string err;
  float last_ms = 0.f;
  int tile_cfg = -1;
  int precision = 0;
  PrecisionPlan* prec = nullptr;
  int max_ns = 0, max_nq = 0, max_nf = 0, max_ring = 0, max_L = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double* h_stage = nullptr;  // pinned staging for outputs / body velocities
  double* d_bvel = nullptr;   // every case's body velocities, contiguous in case order
  double* h_bvel = nullptr;   // pinned staging of the same
  int sum_nf = 0;
  double* d_vertex = nullptr;  // 5 x max_ns, vertex fields of the Tecplot export (allocated on first use)
  AdjPlan* adj = nullptr;
  AdjMPlan* adjm = nullptr;
};


namespace ibfs {
int fail_cuda(cudaError_t e, const char* what);
int set_error(int code, const char* msg);
}  // namespace ibfs
