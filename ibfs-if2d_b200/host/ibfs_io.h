// ibfs_io.h -- host-side file formats of the IBFS driver (no CUDA).
//
// The reference keeps all I/O in its Fortran host code; the B200 driver keeps
// the same files so that a run directory works with either program:
//   input/ibfs.inp   namelist &READ_PARAMETERS (parameters.f90:48-69)
//   input/geom.inp   ntot, then "x y bodyno" per point (grid.f90:270-277)
//   input/ibfs.chd   one unformatted record: cholmat(Nf,Nf), cholvec(Nf) (variables.f90:110-137)
//   output/ibfsNNNNNNN.var  one unformatted record: omega, fb, rhs_old, q, q0 (variables.f90:141-175)
//   output/force.dat, circ.dat, slip.dat  one list-directed line per step (operators.f90:549-699)
//   output/ibfs.inf  run log (main.f90:21-29)
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ibfs_capi.h"

namespace ibfs_host {

// Reference defaults (parameters.f90:12-31).
ibfs_params_c default_params();

// Parses the &READ_PARAMETERS group of a namelist text into p (fields not
// present keep their value). Names are case-insensitive; values may be
// Fortran integers, reals (E or D exponents, trailing '.') or logicals
// (T, F, .TRUE., .FALSE.). Returns false with msg set on a malformed group or
// an unknown name.
bool parse_read_parameters(const std::string& text, ibfs_params_c& p, std::string& msg);

// Optional &B200_OPTIONS group of the same file (precision, cg_relative,
// motion_kind, pitch_amp_deg, pitch_freq, pivot_x, pivot_y, tile_cfg,
// cg_precond, tc_tile, refine_slices, poisson_sweeps); a
// Fortran READ of &READ_PARAMETERS skips it. Returns false on a malformed
// group; absent group = zero-initialised options (reference behaviour).
bool parse_b200_options(const std::string& text, ibfs_options_c& o, std::string& msg);

// &READ_ACT_PARAMETERS of input/actuator.NNN.inp (grid.f90:263-264, 616-623):
// slot centre, width, jet speed, its oscillating part, angle (degrees) and
// angular frequency; absent items stay zero.
struct Actuator {
  double x_j = 0.0, y_j = 0.0, h_j = 0.0, u_j = 0.0, u_j_osc = 0.0, theta_j = 0.0, omg_j = 0.0;
};
bool parse_act_parameters(const std::string& text, Actuator& a, std::string& msg);

// The namelist written when input/ibfs.inp is absent (parameters.f90:64-66).
std::string format_read_parameters(const ibfs_params_c& p);

struct Geometry {
  std::vector<double> x, y;
  std::vector<int> bodyno;
};
bool read_geometry(const std::string& path, Geometry& g, std::string& msg);
// circle(ds, 1, 0, 0) -- the primitive the reference falls back to when
// geom.inp is absent (grid.f90:353, 496-520).
Geometry default_geometry(const ibfs_params_c& p);

// The reference's geometry primitives (grid.f90:408-520), appended to g:
//   vertex x y body                one point
//   line len aoa body              len/ds segments with end points, centred on
//                                  the origin at -aoa degrees (the reference's
//                                  line ignores its x, y arguments)
//   segment x1 y1 x2 y2 body       the len/ds - 1 interior points
//   circle dia x y body            INT(pi dia / ds) points from angle 0
// A spec text holds one primitive per line ('#' starts a comment); ds is the
// grid spacing len/m. Returns false with msg on a malformed line.
bool geometry_from_spec(const std::string& text, double ds, Geometry& g, std::string& msg);
bool write_geometry(const std::string& path, const Geometry& g, std::string& msg);

// actuator_slot (grid.f90:636-718): appends to g the INT(hs/ds)+1 points of a
// slot of width hs centred at (x, y) across the jet angle (degrees), spacing
// hs/INT(hs/ds), or the single point (x, y) when INT(hs/ds) = 0, with body
// number num (-actuator number). With write_files it also writes the user
// summary input/slot.dat and the point count input/slot.NNN.inp as the
// reference does. Returns the point count, or -1 with msg on a write failure.
int actuator_slot(double x, double y, double hs, double ds, double angle, int num, Geometry& g, bool write_files,
                  std::string& msg);

// The check the reference leaves out (grid.f90:280-284): for every body, the
// distance between consecutive points against ds; one message per body whose
// spacing leaves [0.5 ds, 2 ds] (the delta function spans 1.5 ds).
std::vector<std::string> spacing_warnings(const Geometry& g, double ds);

// Fortran unformatted sequential records (gfortran layout: 4-byte
// little-endian length markers around the payload; payloads above
// 2147483639 bytes are split into subrecords, the leading marker negative
// when the record continues, the trailing marker negative when it continued
// from the previous subrecord).
bool write_record(const std::string& path, const std::vector<const double*>& parts,
                  const std::vector<size_t>& counts, std::string& msg);
bool read_record(const std::string& path, const std::vector<double*>& parts, const std::vector<size_t>& counts,
                 std::string& msg);

// One list-directed line "it v1 v2 ..." in the spacing gfortran uses for
// default INTEGER and REAL(8) items (values written with 17 significant
// digits, so they read back exactly).
std::string list_directed(int it, const std::vector<double>& v);

// Fortran Ew.d editing of one value: 0.ddddd mantissa, two-digit exponent
// with its sign (E+ee), or a three-digit exponent without the E.
std::string fortran_E(double x, int w, int d);

// One level's Tecplot file of write_tecplot (operators.f90:702-763): the
// header, then per node (j outer, i inner) x, y and the five fields of
// ibfs_vertex_fields in (8E14.5). fac = 2^(level-1); the offsets follow the
// reference (offx = (fac-1)/2 len, offy = (fac-1)/2 delta n).
bool write_tecplot(const std::string& path, int it, int m, int n, double fac, double delta, double len,
                   double offsetx, double offsety, const double* fields, std::string& msg);

std::string file_text(const std::string& path, bool& ok);
bool file_exists(const std::string& path);

}  // namespace ibfs_host
