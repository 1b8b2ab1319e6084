// ibfs_io.cpp -- file formats of the IBFS host driver (see ibfs_io.h).
#include "ibfs_io.h"

#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ibfs_host {

ibfs_params_c default_params() {
  ibfs_params_c p{};
  p.istart = 0;
  p.istop = 400;
  p.isave = 25;
  p.m = 100;
  p.n = 100;
  p.dt = 0.005;
  p.re = 300.0;
  p.cgtol = 1e-7;
  p.cg_max_iter = 3000;
  p.unif_flow = 1;
  p.len = 2.0;
  p.offsetx = 1.0;
  p.offsety = 1.0;
  p.mgridlev = 4;
  p.make_vortex = 0;
  p.stationary = 0;
  return p;
}

namespace {

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// Text of one namelist group: from "&NAME" to the closing "/" (or "&END"),
// comments ("!" to end of line) removed; empty if the group is absent.
std::string group_body(const std::string& text, const std::string& name, bool& found) {
  std::string t;
  t.reserve(text.size());
  bool comment = false, quote = false;
  for (char c : text) {  // drop comments
    if (c == '\n') comment = false;
    if (c == '\'' || c == '"') quote = !quote;
    if (c == '!' && !quote) comment = true;
    if (!comment) t.push_back(c);
  }
  std::string T = upper(t);
  std::string key = "&" + upper(name);
  size_t pos = 0;
  found = false;
  while ((pos = T.find(key, pos)) != std::string::npos) {
    size_t e = pos + key.size();
    if (e >= T.size() || !(std::isalnum((unsigned char)T[e]) || T[e] == '_')) {
      found = true;
      break;
    }
    pos = e;
  }
  if (!found) return "";
  size_t b = pos + key.size();
  size_t end = T.find('/', b);
  size_t amp = T.find('&', b);
  if (amp != std::string::npos && (end == std::string::npos || amp < end)) end = amp;
  if (end == std::string::npos) end = T.size();
  return T.substr(b, end - b);
}

// name=value pairs of a group body (values separated by commas or blanks).
bool pairs(const std::string& body, std::vector<std::pair<std::string, std::string>>& out, std::string& msg) {
  std::string s = body;
  for (auto& c : s)
    if (c == ',' || c == '\n' || c == '\r' || c == '\t') c = ' ';
  // tokens around '='
  std::vector<std::string> tok;
  std::string cur;
  for (char c : s) {
    if (c == '=') {
      if (!cur.empty()) tok.push_back(cur);
      tok.push_back("=");
      cur.clear();
    } else if (c == ' ') {
      if (!cur.empty()) tok.push_back(cur);
      cur.clear();
    } else {
      cur.push_back(c);
    }
  }
  if (!cur.empty()) tok.push_back(cur);
  for (size_t i = 0; i < tok.size();) {
    if (i + 2 >= tok.size()) {
      msg = "incomplete assignment near '" + tok[i] + "'";
      return false;
    }
    if (tok[i + 1] != "=") {
      msg = "expected '=' after '" + tok[i] + "'";
      return false;
    }
    out.push_back({tok[i], tok[i + 2]});
    i += 3;
  }
  return true;
}

bool to_double(const std::string& v, double& d) {
  std::string s = v;
  for (auto& c : s)
    if (c == 'D' || c == 'd') c = 'E';
  char* e = nullptr;
  d = std::strtod(s.c_str(), &e);
  return e && *e == '\0' && !s.empty();
}
bool to_int(const std::string& v, int& i) {
  char* e = nullptr;
  long x = std::strtol(v.c_str(), &e, 10);
  if (!e || *e != '\0' || v.empty()) return false;
  i = (int)x;
  return true;
}
bool to_logical(const std::string& v, int& b) {
  std::string s = upper(v);
  if (!s.empty() && s[0] == '.') s = s.substr(1);
  if (s.empty()) return false;
  if (s[0] == 'T') { b = 1; return true; }
  if (s[0] == 'F') { b = 0; return true; }
  return false;
}

}  // namespace

bool parse_read_parameters(const std::string& text, ibfs_params_c& p, std::string& msg) {
  bool found = false;
  std::string body = group_body(text, "READ_PARAMETERS", found);
  if (!found) {
    msg = "no &READ_PARAMETERS group";
    return false;
  }
  std::vector<std::pair<std::string, std::string>> kv;
  if (!pairs(body, kv, msg)) return false;
  for (auto& [k, v] : kv) {
    bool ok = true;
    if (k == "ISTART") ok = to_int(v, p.istart);
    else if (k == "ISTOP") ok = to_int(v, p.istop);
    else if (k == "ISAVE") ok = to_int(v, p.isave);
    else if (k == "M") ok = to_int(v, p.m);
    else if (k == "N") ok = to_int(v, p.n);
    else if (k == "DT") ok = to_double(v, p.dt);
    else if (k == "RE") ok = to_double(v, p.re);
    else if (k == "CGTOL") ok = to_double(v, p.cgtol);
    else if (k == "CG_MAX_ITER") ok = to_int(v, p.cg_max_iter);
    else if (k == "UNIF_FLOW") ok = to_logical(v, p.unif_flow);
    else if (k == "LEN") ok = to_double(v, p.len);
    else if (k == "OFFSETX") ok = to_double(v, p.offsetx);
    else if (k == "OFFSETY") ok = to_double(v, p.offsety);
    else if (k == "MGRIDLEV") ok = to_int(v, p.mgridlev);
    else if (k == "MAKE_VORTEX") ok = to_logical(v, p.make_vortex);
    else if (k == "STATIONARY") ok = to_logical(v, p.stationary);
    else {
      msg = "unknown namelist item " + k;
      return false;
    }
    if (!ok) {
      msg = "bad value '" + v + "' for " + k;
      return false;
    }
  }
  return true;
}

bool parse_b200_options(const std::string& text, ibfs_options_c& o, std::string& msg) {
  bool found = false;
  std::string body = group_body(text, "B200_OPTIONS", found);
  o = ibfs_options_c{};
  o.tile_cfg = -1;
  if (!found) return true;
  std::vector<std::pair<std::string, std::string>> kv;
  if (!pairs(body, kv, msg)) return false;
  for (auto& [k, v] : kv) {
    bool ok = true;
    if (k == "PRECISION") ok = to_int(v, o.precision);
    else if (k == "CG_RELATIVE") ok = to_logical(v, o.cg_relative) || to_int(v, o.cg_relative);
    else if (k == "MOTION_KIND") ok = to_int(v, o.motion_kind);
    else if (k == "PITCH_AMP_DEG") ok = to_double(v, o.pitch_amp_deg);
    else if (k == "PITCH_FREQ") ok = to_double(v, o.pitch_freq);
    else if (k == "PIVOT_X") ok = to_double(v, o.pivot_x);
    else if (k == "PIVOT_Y") ok = to_double(v, o.pivot_y);
    else if (k == "TILE_CFG") ok = to_int(v, o.tile_cfg);
    else if (k == "CG_PRECOND") ok = to_logical(v, o.cg_precond) || to_int(v, o.cg_precond);
    else if (k == "REFINE_SLICES") ok = to_int(v, o.refine_slices) && (o.refine_slices == 0 || o.refine_slices == 2 || o.refine_slices == 3);
    else if (k == "POISSON_SWEEPS") ok = to_int(v, o.poisson_sweeps) && o.poisson_sweeps >= 0 && o.poisson_sweeps <= 2;
    else if (k == "TC_TILE") ok = to_int(v, o.tc_tile) && o.tc_tile >= 0 && o.tc_tile <= 4;
    else {
      msg = "unknown &B200_OPTIONS item " + k;
      return false;
    }
    if (!ok) {
      msg = "bad value '" + v + "' for " + k;
      return false;
    }
  }
  return true;
}

bool parse_act_parameters(const std::string& text, Actuator& a, std::string& msg) {
  bool found = false;
  std::string body = group_body(text, "READ_ACT_PARAMETERS", found);
  if (!found) {
    msg = "no &READ_ACT_PARAMETERS group";
    return false;
  }
  std::vector<std::pair<std::string, std::string>> kv;
  if (!pairs(body, kv, msg)) return false;
  for (auto& [k, v] : kv) {
    double* dst = k == "X_J" ? &a.x_j : k == "Y_J" ? &a.y_j : k == "H_J" ? &a.h_j : k == "U_J" ? &a.u_j
                : k == "U_J_OSC" ? &a.u_j_osc : k == "THETA_J" ? &a.theta_j : k == "OMG_J" ? &a.omg_j : nullptr;
    if (!dst) {
      msg = "unknown namelist item " + k;
      return false;
    }
    if (!to_double(v, *dst)) {
      msg = "bad value '" + v + "' for " + k;
      return false;
    }
  }
  return true;
}

std::string format_read_parameters(const ibfs_params_c& p) {
  char b[1024];
  auto L = [](int v) { return v ? "T" : "F"; };
  std::snprintf(b, sizeof b,
                "&READ_PARAMETERS\n ISTART=%d,\n ISTOP=%d,\n ISAVE=%d,\n M=%d,\n N=%d,\n DT=%.17g,\n RE=%.17g,\n"
                " CGTOL=%.17g,\n CG_MAX_ITER=%d,\n UNIF_FLOW=%s,\n LEN=%.17g,\n OFFSETX=%.17g,\n OFFSETY=%.17g,\n"
                " MGRIDLEV=%d,\n MAKE_VORTEX=%s,\n STATIONARY=%s,\n /\n",
                p.istart, p.istop, p.isave, p.m, p.n, p.dt, p.re, p.cgtol, p.cg_max_iter, L(p.unif_flow), p.len,
                p.offsetx, p.offsety, p.mgridlev, L(p.make_vortex), L(p.stationary));
  return b;
}

bool read_geometry(const std::string& path, Geometry& g, std::string& msg) {
  std::ifstream f(path);
  if (!f) {
    msg = "cannot open " + path;
    return false;
  }
  long ntot = 0;
  if (!(f >> ntot) || ntot <= 0) {
    msg = "bad point count in " + path;
    return false;
  }
  g.x.resize(ntot);
  g.y.resize(ntot);
  g.bodyno.resize(ntot);
  for (long i = 0; i < ntot; i++) {
    std::string xs, ys;
    if (!(f >> xs >> ys >> g.bodyno[i]) || !to_double(upper(xs), g.x[i]) || !to_double(upper(ys), g.y[i])) {
      msg = "bad point " + std::to_string(i + 1) + " in " + path;
      return false;
    }
  }
  return true;
}

Geometry default_geometry(const ibfs_params_c& p) {
  const double pi = 3.1415926535897932384;
  const double ds = p.len / (double)p.m;
  const int npt = (int)(pi * 1.0 / ds);
  Geometry g;
  for (int i = 1; i <= npt; i++) {
    double a = 2.0 * pi * (double)(float)(i - 1) / (double)(float)npt;
    g.x.push_back(0.0 + 0.5 * 1.0 * std::cos(a));
    g.y.push_back(0.0 + 0.5 * 1.0 * std::sin(a));
    g.bodyno.push_back(0);
  }
  return g;
}

bool geometry_from_spec(const std::string& text, double ds, Geometry& g, std::string& msg) {
  const double pi = 3.1415926535897932384;
  std::istringstream in(text);
  std::string line;
  int ln = 0;
  while (std::getline(in, line)) {
    ln++;
    size_t h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    std::istringstream w(line);
    std::string kind;
    if (!(w >> kind)) continue;
    kind = upper(kind);
    auto bad = [&]() {
      msg = "geometry spec line " + std::to_string(ln) + ": cannot read '" + line + "'";
      return false;
    };
    auto add = [&](double x, double y, int b) {
      g.x.push_back(x);
      g.y.push_back(y);
      g.bodyno.push_back(b);
    };
    if (kind == "VERTEX") {
      double x, y;
      int b;
      if (!(w >> x >> y >> b)) return bad();
      add(x, y, b);
    } else if (kind == "LINE") {  // grid.f90:431-462
      double len, aoa;
      int b;
      if (!(w >> len >> aoa >> b)) return bad();
      const double angle = -aoa * pi / 180.0;
      const double xle = -0.5 * len * std::cos(angle), yle = -0.5 * len * std::sin(angle);
      const int npt = (int)(len / ds);
      for (int i = 1; i <= npt + 1; i++) {
        const double seg = (double)(float)(i - 1) * len / (double)(float)npt;
        add(xle + seg * std::cos(angle), yle + seg * std::sin(angle), b);
      }
    } else if (kind == "SEGMENT") {  // grid.f90:465-493
      double x1, y1, x2, y2;
      int b;
      if (!(w >> x1 >> y1 >> x2 >> y2 >> b)) return bad();
      const double len = std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
      const double angle = std::atan2(y2 - y1, x2 - x1);
      const int npt = (int)(len / ds);
      for (int i = 1; i <= npt - 1; i++) {
        const double seg = (double)(float)i * len / (double)(float)npt;
        add(x1 + seg * std::cos(angle), y1 + seg * std::sin(angle), b);
      }
    } else if (kind == "CIRCLE") {  // grid.f90:496-520
      double dia, x, y;
      int b;
      if (!(w >> dia >> x >> y >> b)) return bad();
      const int npt = (int)(pi * dia / ds);
      for (int i = 1; i <= npt; i++) {
        const double a = 2.0 * pi * (double)(float)(i - 1) / (double)(float)npt;
        add(x + 0.5 * dia * std::cos(a), y + 0.5 * dia * std::sin(a), b);
      }
    } else {
      msg = "geometry spec line " + std::to_string(ln) + ": unknown primitive '" + kind + "'";
      return false;
    }
  }
  if (g.x.empty()) {
    msg = "geometry spec holds no points";
    return false;
  }
  return true;
}

bool write_geometry(const std::string& path, const Geometry& g, std::string& msg) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) {
    msg = "cannot write " + path;
    return false;
  }
  std::fprintf(f, "%12zu\n", g.x.size());
  for (size_t i = 0; i < g.x.size(); i++) std::fprintf(f, " %.17g %.17g %d\n", g.x[i], g.y[i], g.bodyno[i]);
  bool ok = std::fclose(f) == 0;
  if (!ok) msg = "write failed: " + path;
  return ok;
}

std::vector<std::string> spacing_warnings(const Geometry& g, double ds) {
  std::vector<std::string> out;
  std::vector<int> bodies;
  for (int b : g.bodyno)
    if (std::find(bodies.begin(), bodies.end(), b) == bodies.end()) bodies.push_back(b);
  for (int b : bodies) {
    double lo = 1e300, hi = 0.0;
    int prev = -1, n = 0;
    for (size_t i = 0; i < g.x.size(); i++) {
      if (g.bodyno[i] != b) continue;
      n++;
      if (prev >= 0) {
        const double d = std::hypot(g.x[i] - g.x[prev], g.y[i] - g.y[prev]);
        lo = std::min(lo, d);
        hi = std::max(hi, d);
      }
      prev = (int)i;
    }
    if (n < 2) continue;
    if (lo < 0.5 * ds || hi > 2.0 * ds) {
      char m[256];
      std::snprintf(m, sizeof m,
                    "WARNING: body %d point spacing %.4g .. %.4g is outside [0.5, 2] x grid spacing %.4g", b, lo, hi,
                    ds);
      out.push_back(m);
    }
  }
  return out;
}

namespace {
constexpr int64_t kMaxSub = 2147483639;  // gfortran's largest subrecord payload
}

bool write_record(const std::string& path, const std::vector<const double*>& parts,
                  const std::vector<size_t>& counts, std::string& msg) {
  std::vector<char> buf;
  size_t total = 0;
  for (size_t c : counts) total += c * sizeof(double);
  buf.resize(total);
  size_t o = 0;
  for (size_t i = 0; i < parts.size(); i++) {
    std::memcpy(buf.data() + o, parts[i], counts[i] * sizeof(double));
    o += counts[i] * sizeof(double);
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    msg = "cannot write " + path;
    return false;
  }
  int64_t left = (int64_t)total;
  size_t pos = 0;
  bool first = true;
  do {
    int64_t len = left > kMaxSub ? kMaxSub : left;
    bool more = left > kMaxSub;
    int32_t head = (int32_t)(more ? -len : len);
    int32_t tail = (int32_t)(first ? len : -len);
    std::fwrite(&head, 4, 1, f);
    std::fwrite(buf.data() + pos, 1, (size_t)len, f);
    std::fwrite(&tail, 4, 1, f);
    pos += (size_t)len;
    left -= len;
    first = false;
  } while (left > 0);
  bool ok = std::fclose(f) == 0;
  if (!ok) msg = "write failed: " + path;
  return ok;
}

bool read_record(const std::string& path, const std::vector<double*>& parts, const std::vector<size_t>& counts,
                 std::string& msg) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    msg = "cannot open " + path;
    return false;
  }
  std::vector<char> buf;
  for (;;) {  // concatenate the subrecords of the first record
    int32_t head = 0, tail = 0;
    if (std::fread(&head, 4, 1, f) != 1) {
      msg = "truncated record in " + path;
      std::fclose(f);
      return false;
    }
    int64_t len = head < 0 ? -(int64_t)head : head;
    size_t at = buf.size();
    buf.resize(at + (size_t)len);
    if (std::fread(buf.data() + at, 1, (size_t)len, f) != (size_t)len || std::fread(&tail, 4, 1, f) != 1 ||
        (tail < 0 ? -(int64_t)tail : tail) != len) {
      msg = "corrupt record markers in " + path;
      std::fclose(f);
      return false;
    }
    if (head >= 0) break;
  }
  std::fclose(f);
  size_t need = 0;
  for (size_t c : counts) need += c * sizeof(double);
  if (buf.size() < need) {
    msg = path + ": record holds " + std::to_string(buf.size()) + " bytes, the grid needs " +
          std::to_string(need);
    return false;
  }
  size_t o = 0;
  for (size_t i = 0; i < parts.size(); i++) {
    if (parts[i]) std::memcpy(parts[i], buf.data() + o, counts[i] * sizeof(double));
    o += counts[i] * sizeof(double);
  }
  return true;
}

namespace {
std::string real_item(double x) {
  char b[64];
  double ax = std::fabs(x);
  if (x == 0.0) {
    std::snprintf(b, sizeof b, "%25s", "0.0000000000000000     ");
  } else if (ax >= 0.1 && ax < 1e17) {
    int e = (int)std::floor(std::log10(ax)) + 1;  // digits before the point
    int dec = 17 - e;
    if (dec < 0) dec = 0;
    char v[48];
    std::snprintf(v, sizeof v, "%.*f     ", dec, x);
    std::snprintf(b, sizeof b, "%25s", v);
  } else {
    char v[48];
    std::snprintf(v, sizeof v, "%.16E", x);  // d.dddE+xx -> d.dddE+0xx
    std::string s = v;
    size_t p = s.find('E');
    std::string mant = s.substr(0, p), ex = s.substr(p + 1);
    char sign = ex[0];
    std::string digits = ex.substr(1);
    while (digits.size() < 3) digits = "0" + digits;
    std::string t = mant + "E" + sign + digits;
    std::snprintf(b, sizeof b, "%25s", t.c_str());
  }
  return std::string(" ") + b;
}
}  // namespace

int actuator_slot(double x, double y, double hs, double ds, double angle, int num, Geometry& g, bool write_files,
                  std::string& msg) {
  const double pi = 3.1415926535897932384;
  const int npt = (int)(hs / ds);
  if (npt == 0) {
    g.x.push_back(x);
    g.y.push_back(y);
    g.bodyno.push_back(num);
  } else {
    const double a = pi * (angle + 90.0) / 180.0;
    for (int i = 1; i <= npt + 1; i++) {
      const double seg = (double)(float)(i - 1) * hs / (double)(float)npt;
      g.x.push_back(x - hs / 2.0 * std::cos(a) + seg * std::cos(a));
      g.y.push_back(y - hs / 2.0 * std::sin(a) + seg * std::sin(a));
      g.bodyno.push_back(num);
    }
  }
  if (!write_files) return npt + 1;
  char name[64];
  std::snprintf(name, sizeof name, "input/slot.%03d.inp", -num);
  // slot.dat is replaced by the first actuator and appended to by the others;
  // slot.NNN.inp is replaced by actuator 1, appended to otherwise (grid.f90:682-698)
  FILE* f1 = std::fopen("input/slot.dat", num == -1 ? "w" : "a");
  FILE* f2 = std::fopen(name, num == -1 ? "w" : "a");
  if (!f1 || !f2) {
    if (f1) std::fclose(f1);
    if (f2) std::fclose(f2);
    msg = std::string("cannot write input/slot.dat or ") + name;
    return -1;
  }
  std::fprintf(f1, "  ----------- ACTUATOR No. %12d\n", -num);
  std::fprintf(f1, "    o Desired slot width               = %s\n", real_item(hs).c_str());
  std::fprintf(f1, "    o Actual slot width in simulation  = %s\n", real_item(npt == 0 ? ds : hs).c_str());
  std::fprintf(f1, "    o Number of pts used to model slot = %12d\n", npt + 1);
  std::fprintf(f2, "%12d\n", npt + 1);
  bool ok = std::fclose(f1) == 0;
  ok = std::fclose(f2) == 0 && ok;
  if (!ok) {
    msg = std::string("write failed: ") + name;
    return -1;
  }
  return npt + 1;
}

std::string list_directed(int it, const std::vector<double>& v) {
  char b[32];
  std::snprintf(b, sizeof b, "%12d", it);
  std::string s = b;
  for (double x : v) s += real_item(x);
  return s;
}

std::string fortran_E(double x, int w, int d) {
  std::string body;
  if (x == 0.0 || !std::isfinite(x)) {
    if (!std::isfinite(x)) body = std::string(w, '*');
    else body = "0." + std::string(d, '0') + "E+00";
  } else {
    char v[64];
    std::snprintf(v, sizeof v, "%.*E", d - 1, std::fabs(x));  // D.DDDDE+XX, rounded to d digits
    std::string t = v;
    size_t e = t.find('E');
    std::string digits = t.substr(0, 1) + t.substr(2, e - 2);
    int ex = std::atoi(t.c_str() + e + 1) + 1;  // 0.DDDDD x 10^ex
    char eb[16];
    if (std::abs(ex) <= 99) std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    body = std::string(x < 0 ? "-" : "") + "0." + digits + eb;
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

bool write_tecplot(const std::string& path, int it, int m, int n, double fac, double delta, double len,
                   double offsetx, double offsety, const double* f, std::string& msg) {
  FILE* o = std::fopen(path.c_str(), "w");
  if (!o) {
    msg = "cannot write " + path;
    return false;
  }
  const double offx = (fac - 1.0) / 2.0 * len;
  const double offy = (fac - 1.0) / 2.0 * delta * (double)(float)n;
  const size_t ns = (size_t)(m - 1) * (n - 1);
  std::fprintf(o, " TITLE     = \"IBFS V1.0 AT ITIME=%12d\"\n", it);
  std::fprintf(o, " VARIABLES = \"x\"\n \"y\"\n \"u\"\n \"v\"\n \"etfx\"\n \"etfy\"\n \"vort\"\n");
  std::fprintf(o, " ZONE T=\"Rectangular zone\"\n");
  std::fprintf(o, " I=%12d, J=%12d, K=1, ZONETYPE=Ordered\n", m - 1, n - 1);
  std::fprintf(o, " DATAPACKING=POINT\n DT=(SINGLE SINGLE SINGLE SINGLE SINGLE SINGLE SINGLE)\n");
  for (int j = 2; j <= n; j++)
    for (int i = 2; i <= m; i++) {
      const size_t t = (size_t)(i - 2) + (size_t)(j - 2) * (m - 1);
      std::string line = fortran_E(fac * delta * (double)(float)(i - 1) - offx - offsetx, 14, 5) +
                         fortran_E(fac * delta * (double)(float)(j - 1) - offy - offsety, 14, 5);
      for (int k = 0; k < 5; k++) line += fortran_E(f[k * ns + t], 14, 5);
      std::fprintf(o, "%s\n", line.c_str());
    }
  bool ok = std::fclose(o) == 0;
  if (!ok) msg = "write failed: " + path;
  return ok;
}

std::string file_text(const std::string& path, bool& ok) {
  std::ifstream f(path);
  ok = (bool)f;
  if (!ok) return "";
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

bool file_exists(const std::string& path) {
  struct stat st;
  return ::stat(path.c_str(), &st) == 0;
}

}  // namespace ibfs_host
