// ibfs_driver.cpp -- host driver of the B200 IBFS advance (program ibfs_gpu).
//
// The reference's PROGRAM main (main.f90:12-63) with the time step on the
// GPU: same run directory, same input files, same output files.
//   input      input/ibfs.inp (&READ_PARAMETERS; written with the defaults if
//              absent, parameters.f90:54-69), optional &B200_OPTIONS group
//   setup      input/geom.inp; else input/geom.spec (the reference's primitives,
//              one per line, written out as geom.inp); else a circle of diameter
//              1 at the origin (grid.f90:252-353); the point spacing is checked
//              against the grid; grid checks and regularisation happen in
//              ibfs_create
//   variables  istart = 0: zero (or uniform) flow; otherwise
//              output/ibfsNNNNNNN.var and, for a stationary body,
//              input/ibfs.chd (variables.f90:28-77)
//   preprocess first step of a stationary body: input/ibfs.chd if present,
//              else ibfs_precompute and write input/ibfs.chd
//              (operators.f90:29-59)
//   advance    ibfs_advance per step; every isave steps and at istop the
//              restart record; force.dat / circ.dat / slip.dat every step
//              (operators.f90:176-188, 549-699)
//   actuators  input/actuator.NNN.inp (&READ_ACT_PARAMETERS) for NNN = 001..100:
//              when geom.inp already holds actuator points (bodyno < 0) their
//              counts come from input/slot.NNN.inp; otherwise each actuator's
//              slot points are appended (actuator_slot, writing slot.dat and
//              slot.NNN.inp) and geom.inp is rewritten (grid.f90:286-325,
//              382-401); the jets (actuation, grid.f90:579-633) then run on
//              the device through ibfs_set_actuators, the namelists read once
//              instead of every step
//
//   ibfs_gpu [-C dir] [--dry-run | --post]
// --dry-run reads and checks the inputs (and a restart record when
// istart > 0) and prints them as JSON without touching the GPU.
// --post is the reference's post-processing program (post.f90): for every
// step istart..istop that has a restart record (it % isave == 0 or istop; the
// initial state for it = 0) it writes post/ibfs_g<level>t<it>_vel.dat for each
// level, the Tecplot files of write_tecplot (operators.f90:702-763).
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "ibfs_io.h"

using namespace ibfs_host;

namespace {

FILE* g_inf = nullptr;

void logline(const std::string& s) {
  if (g_inf) {
    std::fprintf(g_inf, " %s\n", s.c_str());
    std::fflush(g_inf);
  }
}

int stop(const std::string& msg, int code) {
  std::fprintf(stderr, "%s\n", msg.c_str());
  logline(msg);
  if (g_inf) std::fclose(g_inf);
  return code;
}

void append_line(const std::string& path, int it, const std::string& line) {
  // the reference replaces the file at it == 1 and appends otherwise
  // (creating it when missing), operators.f90:564-573
  FILE* f = std::fopen(path.c_str(), it == 1 ? "w" : "a");
  if (!f) return;
  std::fprintf(f, "%s\n", line.c_str());
  std::fclose(f);
}

std::string var_name(int it) {
  char b[64];
  std::snprintf(b, sizeof b, "output/ibfs%07d.var", it);
  return b;
}

}  // namespace

int main(int argc, char** argv) {
  bool dry = false, post = false;
  for (int a = 1; a < argc; a++) {
    if (!std::strcmp(argv[a], "--dry-run")) dry = true;
    else if (!std::strcmp(argv[a], "--post")) post = true;
    else if (!std::strcmp(argv[a], "-C") && a + 1 < argc) {
      if (::chdir(argv[++a]) != 0) return stop(std::string("cannot enter ") + argv[a], 2);
    } else {
      std::fprintf(stderr, "usage: ibfs_gpu [-C dir] [--dry-run | --post]\n");
      return 2;
    }
  }
  ::mkdir("output", 0755);
  ::mkdir("input", 0755);
  auto t0 = std::chrono::steady_clock::now();
  if (!dry) {
    g_inf = std::fopen("output/ibfs.inf", "a");
    logline("===================================");
    logline("|   Welcome to IBFS MGRID v1.0    |");
    logline("|   (GPU time step, B200 build)   |");
    logline("===================================");
    std::time_t now = std::time(nullptr);
    char tb[64];
    std::strftime(tb, sizeof tb, "Executed at time: %H%M%S on date: %Y%m%d", std::localtime(&now));
    logline(tb);
    std::printf("\n=======================================\n|     Welcome to IBFS MGRID v1.0      |\n"
                "|  time step on the GPU (B200 build)  |\n=======================================\n\n%s\n",
                tb);
  }

  // INPUT (parameters.f90:54-69)
  ibfs_params_c p = default_params();
  ibfs_options_c opt{};
  opt.tile_cfg = -1;
  std::string msg;
  if (file_exists("input/ibfs.inp")) {
    bool ok = false;
    std::string text = file_text("input/ibfs.inp", ok);
    if (!ok || !parse_read_parameters(text, p, msg)) return stop("input/ibfs.inp: " + msg, 2);
    if (!parse_b200_options(text, opt, msg)) return stop("input/ibfs.inp: " + msg, 2);
    logline("... Read parameters from ibfs.inp");
  } else {
    if (FILE* f = std::fopen("input/ibfs.inp", "w")) {
      std::fputs(format_read_parameters(p).c_str(), f);
      std::fclose(f);
    }
    logline("... loading default run");
  }
  logline("... Input parameters follow");
  if (g_inf) std::fputs(format_read_parameters(p).c_str(), g_inf);

  // SETUP GEOMETRY (grid.f90:252-353)
  Geometry geo;
  const double ds = p.len / (double)p.m;
  const bool from_inp = file_exists("input/geom.inp");
  bool from_spec = false;
  if (from_inp) {
    if (!read_geometry("input/geom.inp", geo, msg)) return stop(msg, 2);
    logline("Reading geometry from geom.inp");
    if (!dry) std::printf("Reading geometry from geom.inp\n");
  } else if (file_exists("input/geom.spec")) {  // primitives -> geom.inp
    bool ok = false;
    std::string spec = file_text("input/geom.spec", ok);
    if (!ok || !geometry_from_spec(spec, ds, geo, msg)) return stop("input/geom.spec: " + msg, 2);
    from_spec = true;
  } else {
    geo = default_geometry(p);
  }
  // ACTUATORS (grid.f90:286-325, 382-394)
  auto numbered = [](const char* fmt, int i) {
    char b[64];
    std::snprintf(b, sizeof b, fmt, i);
    return std::string(b);
  };
  bool defined = false;
  for (int b : geo.bodyno) defined = defined || b < 0;
  std::vector<Actuator> acts;  // actuators 1..n_act in order, with their point counts
  std::vector<int> act_npt;
  auto read_act = [&](int i, Actuator& a) {
    std::string an = numbered("input/actuator.%03d.inp", i);
    bool ok = false;
    std::string text = file_text(an, ok);
    if (!ok || !parse_act_parameters(text, a, msg)) {
      msg = an + ": " + msg;
      return false;
    }
    return true;
  };
  if (!(from_inp && defined)) {  // append each actuator's slot points
    for (int i = 1; i <= 100; i++) {
      if (!file_exists(numbered("input/actuator.%03d.inp", i))) continue;
      Actuator a;
      if (!read_act(i, a)) return stop(msg, 2);
      int np = actuator_slot(a.x_j, a.y_j, a.h_j, ds, a.theta_j, -i, geo, !dry, msg);
      if (np < 0) return stop(msg, 2);
      acts.push_back(a);
      act_npt.push_back(np);
    }
  } else {  // points already in geom.inp: counts from slot.NNN.inp
    int n = 0;
    for (int i = 1; i <= 100; i++)
      if (file_exists(numbered("input/actuator.%03d.inp", i))) n++;
    for (int i = 1; i <= n; i++) {
      Actuator a;
      if (!read_act(i, a)) return stop(msg, 2);
      std::string sn = numbered("input/slot.%03d.inp", i);
      bool ok = false;
      int np = 0;
      std::string st = file_text(sn, ok);
      if (!ok || std::sscanf(st.c_str(), "%d", &np) != 1 || np < 1)
        return stop("cannot read the point count in " + sn, 2);
      acts.push_back(a);
      act_npt.push_back(np);
    }
  }
  const int n_act = (int)acts.size();
  int n_act_pt = 0;
  for (int np : act_npt) n_act_pt += np;
  if (n_act_pt > (int)geo.x.size()) return stop("the actuators have more points than the geometry", 2);
  if (!dry && (!from_inp || (n_act > 0 && !defined))) {  // geometry written for the next run
    if (!write_geometry("input/geom.inp", geo, msg)) return stop(msg, 2);
    if (from_spec) logline("Generated geometry from primitives (input/geom.spec) into geom.inp");
    if (n_act > 0) logline("...appended actuator info to geom.inp");
  }
  std::vector<double> act_u, act_osc, act_omg, act_theta;
  for (const Actuator& a : acts) {
    act_u.push_back(a.u_j);
    act_osc.push_back(a.u_j_osc);
    act_omg.push_back(a.omg_j);
    act_theta.push_back(a.theta_j);
  }
  for (const std::string& w : spacing_warnings(geo, ds)) {
    std::fprintf(stderr, "%s\n", w.c_str());
    logline(w);
  }
  const int nb = (int)geo.x.size();

  if (dry) {
    std::vector<double> var_sums;
    if (p.istart > 0) {  // check the restart record against the grid
      int L = p.mgridlev;  // the level clamp is applied by ibfs_create; the dry run reads the namelist value
      size_t ns = (size_t)(p.m - 1) * (p.n - 1), nq = (size_t)(p.m + 1) * p.n + (size_t)(p.n + 1) * p.m;
      std::vector<size_t> cnt = {ns * L, (size_t)2 * nb, ns * L, nq * L, nq * L};
      std::vector<std::vector<double>> buf;
      std::vector<double*> parts;
      for (size_t c : cnt) buf.emplace_back(c);
      for (auto& b : buf) parts.push_back(b.data());
      if (!read_record(var_name(p.istart), parts, cnt, msg)) return stop(msg, IBFS_ERR_IO);
      for (auto& b : buf) {
        double s = 0.0;
        for (double v : b) s += v;
        var_sums.push_back(s);
      }
    }
    // the Cholesky record a stationary run would read (variables.f90:110-137)
    int chd_ok = -1;  // -1: no file
    if (p.stationary && file_exists("input/ibfs.chd")) {
      std::vector<double> cm((size_t)4 * nb * nb), cv((size_t)2 * nb);
      if (!read_record("input/ibfs.chd", {cm.data(), cv.data()}, {cm.size(), cv.size()}, msg))
        return stop("input/ibfs.chd: " + msg, IBFS_ERR_IO);
      chd_ok = 1;
    }
    std::printf("{\"istart\": %d, \"istop\": %d, \"isave\": %d, \"m\": %d, \"n\": %d, \"dt\": %.17g, "
                "\"re\": %.17g, \"cgtol\": %.17g, \"cg_max_iter\": %d, \"unif_flow\": %d, \"len\": %.17g, "
                "\"offsetx\": %.17g, \"offsety\": %.17g, \"mgridlev\": %d, \"make_vortex\": %d, "
                "\"stationary\": %d, \"precision\": %d, \"cg_relative\": %d, \"motion_kind\": %d, "
                "\"tile_cfg\": %d, \"cg_precond\": %d, \"tc_tile\": %d, \"nb\": %d, \"x0\": %.17g, \"y0\": %.17g, \"xsum\": %.17g, \"ysum\": %.17g, "
                "\"n_act\": %d, \"n_act_pt\": %d, \"chd_ok\": %d, \"var_sums\": [",
                p.istart, p.istop, p.isave, p.m, p.n, p.dt, p.re, p.cgtol, p.cg_max_iter, p.unif_flow, p.len,
                p.offsetx, p.offsety, p.mgridlev, p.make_vortex, p.stationary, opt.precision, opt.cg_relative,
                opt.motion_kind, opt.tile_cfg, opt.cg_precond, opt.tc_tile, nb, nb ? geo.x[0] : 0.0, nb ? geo.y[0] : 0.0,
                [&] { double t = 0.0; for (double v : geo.x) t += v; return t; }(),
                [&] { double t = 0.0; for (double v : geo.y) t += v; return t; }(), n_act, n_act_pt, chd_ok);
    for (size_t i = 0; i < var_sums.size(); i++) std::printf("%s%.17g", i ? ", " : "", var_sums[i]);
    std::printf("]}\n");
    return 0;
  }

  // SETUP + SETUP_VARIABLES (grid.f90:44-139, variables.f90:28-77)
  ibfs_handle* h = nullptr;
  int rc = ibfs_create(&p, &opt, nb, geo.x.data(), geo.y.data(), geo.bodyno.data(), &h);
  if (rc) return stop(std::string("ibfs_create: ") + ibfs_last_error(h), 10 + rc);
  if (n_act > 0) {
    rc = ibfs_set_actuators(h, 0, n_act, act_npt.data(), act_u.data(), act_osc.data(), act_omg.data(),
                            act_theta.data());
    if (rc) return stop(std::string("ibfs_set_actuators: ") + ibfs_last_error(h), 10 + rc);
  }
  int m, n, L, nq, nbb, nbody;
  ibfs_case_sizes(h, 0, &m, &n, &L, &nq, &nbb, &nbody);
  const size_t ns = (size_t)(m - 1) * (n - 1);
  const int nf = 2 * nbb;
  std::vector<double> omega(ns * L), fb(nf), rhs_old(ns * L), q((size_t)nq * L), q0((size_t)nq * L);
  std::vector<double> cholmat((size_t)nf * nf), cholvec(nf);
  auto read_chd = [&]() -> bool {
    if (!read_record("input/ibfs.chd", {cholmat.data(), cholvec.data()}, {cholmat.size(), cholvec.size()}, msg))
      return false;
    logline("Reading Cholesky decompopsition...");
    std::printf("Reading Cholesky premade decomposition...\n");
    return ibfs_set_cholesky(h, 0, cholmat.data(), cholvec.data()) == IBFS_OK;
  };
  if (post) {  // post.f90: Tecplot files of every saved step
    ::mkdir("post", 0755);
    std::vector<double> fields((size_t)5 * ns);
    for (int it = p.istart; it <= p.istop; it++) {
      if (!(it % p.isave == 0 || it == p.istop)) continue;
      if (it > 0) {
        if (!read_record(var_name(it), {omega.data(), fb.data(), rhs_old.data(), q.data(), q0.data()},
                         {omega.size(), fb.size(), rhs_old.size(), q.size(), q0.size()}, msg))
          return stop(msg, IBFS_ERR_IO);
        rc = ibfs_set_state(h, 0, omega.data(), fb.data(), rhs_old.data(), q.data(), q0.data());
        if (rc) return stop(std::string("ibfs_set_state: ") + ibfs_last_error(h), 10 + rc);
      }
      std::printf(" Post-processing: itime = %12d\n", it);
      for (int k = 1; k <= L; k++) {
        rc = ibfs_vertex_fields(h, 0, k, fields.data());
        if (rc) return stop(std::string("ibfs_vertex_fields: ") + ibfs_last_error(h), 10 + rc);
        char name[96];
        std::snprintf(name, sizeof name, "post/ibfs_g%1dt%07d_vel.dat", k, it);
        if (!write_tecplot(name, it, m, n, (double)(float)(1 << (k - 1)), p.len / (double)p.m, p.len,
                           p.offsetx, p.offsety, fields.data(), msg))
          return stop(msg, IBFS_ERR_IO);
      }
    }
    ibfs_destroy(h);
    if (g_inf) std::fclose(g_inf);
    return 0;
  }
  if (p.istart > 0) {
    if (!read_record(var_name(p.istart), {omega.data(), fb.data(), rhs_old.data(), q.data(), q0.data()},
                     {omega.size(), fb.size(), rhs_old.size(), q.size(), q0.size()}, msg))
      return stop(msg, IBFS_ERR_IO);
    rc = ibfs_set_state(h, 0, omega.data(), fb.data(), rhs_old.data(), q.data(), q0.data());
    if (rc) return stop(std::string("ibfs_set_state: ") + ibfs_last_error(h), 10 + rc);
    logline("Reading restart file at itime= " + std::to_string(p.istart));
    std::printf("Reading restart file at itime = %d\n", p.istart);
    if (p.stationary && !read_chd()) return stop("input/ibfs.chd: " + msg, IBFS_ERR_IO);
  }

  // TIME MARCH (main.f90:45-50)
  std::vector<double> fx(nbody > 0 ? nbody : 1), fy(nbody > 0 ? nbody : 1), circ(L);
  double slip = 0.0;
  int it = p.istart;
  while (it < p.istop) {
    if (it + 1 == 1 && p.stationary) {  // preprocess (operators.f90:88-90)
      if (file_exists("input/ibfs.chd")) {
        if (!read_chd()) return stop("input/ibfs.chd: " + msg, IBFS_ERR_IO);
      } else {
        std::printf("Precomputing body matrix...\n");
        logline("Precomputing body matrix...");
        rc = ibfs_precompute(h);
        if (rc) return stop(std::string("ibfs_precompute: ") + ibfs_last_error(h), 10 + rc);
        ibfs_get_cholesky(h, 0, cholmat.data(), cholvec.data());
        if (!write_record("input/ibfs.chd", {cholmat.data(), cholvec.data()}, {cholmat.size(), cholvec.size()},
                          msg))
          return stop(msg, IBFS_ERR_IO);
        logline("Saving cholesky decomposition...");
      }
    }
    std::printf(" \n-------------------------------------------\n * For itime = %d\n", it + 1);
    logline("...Advancing to itime = " + std::to_string(it + 1));
    rc = ibfs_advance(h, &it, nullptr, fx.data(), fy.data(), circ.data(), &slip);
    if (rc == IBFS_ERR_CG_MAXITER) {  // the reference warns and carries on (operators.f90:435-438)
      logline("WARNING!! CJGR used max iterations!");
      std::printf(" => itmax = %d\n", p.cg_max_iter);
    } else if (rc) {
      return stop(std::string("ibfs_advance: ") + ibfs_last_error(h), 10 + rc);
    }
    if (it % p.isave == 0 || it == p.istop) {  // write_variables (variables.f90:141-155)
      ibfs_get_state(h, 0, omega.data(), fb.data(), rhs_old.data(), q.data(), q0.data());
      if (!write_record(var_name(it), {omega.data(), fb.data(), rhs_old.data(), q.data(), q0.data()},
                        {omega.size(), fb.size(), rhs_old.size(), q.size(), q0.size()}, msg))
        return stop(msg, IBFS_ERR_IO);
      logline("Writing restart file at itime= " + std::to_string(it));
    }
    std::vector<double> fv;
    for (int b = 0; b < nbody; b++) fv.push_back(fx[b]);
    for (int b = 0; b < nbody; b++) fv.push_back(fy[b]);
    append_line("output/force.dat", it, list_directed(it, fv));
    logline("Computed x- & y-forces at itime= " + std::to_string(it));
    append_line("output/circ.dat", it, list_directed(it, circ));
    append_line("output/slip.dat", it, list_directed(it, {slip}));
    std::printf(" SLIP = %.17g\n", slip);
  }
  ibfs_destroy(h);
  double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf(" \n Total run time: %.6f s\n \n", secs);
  logline("Total run time: " + std::to_string(secs) + " s");
  if (g_inf) std::fclose(g_inf);
  return 0;
}
