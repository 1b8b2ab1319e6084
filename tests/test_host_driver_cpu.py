"""Host driver (ibfs-if2d_b200/ibfs_gpu) without a GPU: the reference's input
files are read the way the Fortran program reads them (namelist
&READ_PARAMETERS, parameters.f90:48-69; geom.inp, grid.f90:270-277; the
unformatted restart record, variables.f90:141-175), checked through
--dry-run, which stops before any CUDA call."""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import PKG

DRIVER = os.path.join(PKG, "ibfs_gpu")

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built (make -C ibfs-if2d_b200)")


def run(d, *args):
    r = subprocess.run([DRIVER, "-C", str(d), "--dry-run", *args], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout, r.stderr


def write_inp(d, text):
    os.makedirs(d / "input", exist_ok=True)
    (d / "input" / "ibfs.inp").write_text(text)


def fortran_record(path, arrays):
    """gfortran sequential unformatted record: 4-byte length, payload, 4-byte length."""
    payload = b"".join(np.ascontiguousarray(a, dtype="<f8").tobytes() for a in arrays)
    with open(path, "wb") as f:
        f.write(struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload)))


def test_namelist_reference_style(tmp_path):
    # list-directed style of the reference's input file: upper case, commas,
    # reals with a trailing '.' and an E exponent, logicals T/F
    write_inp(tmp_path, " &READ_PARAMETERS ISTART = 0, ISTOP = 7, ISAVE = 3, M = 64,\n"
                        " N = 48, DT = 0.0025, RE = 150., CGTOL = 1.E-9, CG_MAX_ITER = 500, \n"
                        " UNIF_FLOW = T, LEN = 4.0, OFFSETX = 2, OFFSETY = 1.5D0, MGRIDLEV = 3, \n"
                        " MAKE_VORTEX = F, STATIONARY = T,\n /\n")
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    p = json.loads(out)
    assert (p["istart"], p["istop"], p["isave"], p["m"], p["n"]) == (0, 7, 3, 64, 48)
    assert (p["dt"], p["re"], p["cgtol"], p["cg_max_iter"]) == (0.0025, 150.0, 1e-9, 500)
    assert (p["unif_flow"], p["len"], p["offsetx"], p["offsety"]) == (1, 4.0, 2.0, 1.5)
    assert (p["mgridlev"], p["make_vortex"], p["stationary"]) == (3, 0, 1)
    assert p["precision"] == 0 and p["tile_cfg"] == -1
    # no geom.inp: circle of diameter 1 at the origin, INT(pi/ds) points (grid.f90:353, 512)
    assert p["nb"] == int(np.pi * 64 / 4.0) and abs(p["x0"] - 0.5) < 1e-15 and p["y0"] == 0.0


def test_options_group_and_geometry(tmp_path):
    write_inp(tmp_path, "&read_parameters m=32, n=32, len=4.0, offsetx=2.0, offsety=2.0, stationary=.true. /\n"
                        "&B200_OPTIONS PRECISION=1, CG_RELATIVE=T, TILE_CFG=2, CG_PRECOND=T /\n")
    (tmp_path / "input" / "geom.inp").write_text("3\n 0.1 0.2 0\n -0.25 0.5E-1 0\n 0.3 -0.1 0\n")
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    p = json.loads(out)
    assert (p["precision"], p["cg_relative"], p["tile_cfg"], p["cg_precond"]) == (1, 1, 2, 1)
    assert (p["nb"], p["x0"], p["y0"]) == (3, 0.1, 0.2)
    # fields not in the file keep the reference defaults (parameters.f90:12-31)
    assert (p["istop"], p["isave"], p["dt"], p["re"], p["mgridlev"]) == (400, 25, 0.005, 300.0, 4)


@pytest.mark.parametrize("tile,ok", [(0, True), (3, True), (4, True), (5, False), (-1, False)])
def test_tensor_core_tile_option(tmp_path, tile, ok):
    """TC_TILE picks the tensor-core GEMM's tile configuration: 0 (the
    autotuner), 1..3 single-CTA tiles, 4 the CTA-pair tile; anything else is
    refused before any CUDA call."""
    write_inp(tmp_path, "&read_parameters m=32, n=32, len=4.0, offsetx=2.0, offsety=2.0 /\n"
                        f"&B200_OPTIONS PRECISION=1, TC_TILE={tile} /\n")
    rc, out, err = run(tmp_path)
    if ok:
        assert rc == 0, err
        assert json.loads(out)["tc_tile"] == tile
    else:
        assert rc != 0 and "TC_TILE" in err


def test_restart_record(tmp_path):
    m = n = 32
    L = 3
    write_inp(tmp_path, f"&READ_PARAMETERS ISTART=12, ISTOP=14, M={m}, N={n}, MGRIDLEV={L}, LEN=4., "
                        "OFFSETX=2., OFFSETY=2., STATIONARY=T /\n")
    (tmp_path / "input" / "geom.inp").write_text("2\n 0.0 0.0 0\n 0.1 0.0 0\n")
    os.makedirs(tmp_path / "output", exist_ok=True)
    ns, nq = (m - 1) * (n - 1), (m + 1) * n + (n + 1) * m
    rng = np.random.default_rng(3)
    parts = [rng.standard_normal(ns * L), rng.standard_normal(4), rng.standard_normal(ns * L),
             rng.standard_normal(nq * L), rng.standard_normal(nq * L)]
    fortran_record(tmp_path / "output" / "ibfs0000012.var", parts)
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    sums = json.loads(out)["var_sums"]
    assert np.allclose(sums, [a.sum() for a in parts], rtol=0, atol=1e-9)
    # a record too short for the grid is refused
    fortran_record(tmp_path / "output" / "ibfs0000012.var", parts[:3])
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO and "record holds" in err


IBFS_ERR_IO = 5  # include/ibfs_capi.h; the driver's exit status for a file it cannot use


def test_truncated_and_corrupt_records_are_io_errors(tmp_path):
    """Restart (.var, variables.f90:141-175) and Cholesky (.chd, :110-137)
    records cut short or with broken record markers stop the driver with
    IBFS_ERR_IO, as the reference's READ would stop on a bad record."""
    m = n = 32
    L = 3
    write_inp(tmp_path, f"&READ_PARAMETERS ISTART=12, ISTOP=14, M={m}, N={n}, MGRIDLEV={L}, LEN=4., "
                        "OFFSETX=2., OFFSETY=2., STATIONARY=T /\n")
    (tmp_path / "input" / "geom.inp").write_text("2\n 0.0 0.0 0\n 0.1 0.0 0\n")
    os.makedirs(tmp_path / "output", exist_ok=True)
    ns, nq, nf = (m - 1) * (n - 1), (m + 1) * n + (n + 1) * m, 4
    rng = np.random.default_rng(4)
    parts = [rng.standard_normal(ns * L), rng.standard_normal(nf), rng.standard_normal(ns * L),
             rng.standard_normal(nq * L), rng.standard_normal(nq * L)]
    var = tmp_path / "output" / "ibfs0000012.var"
    chd = tmp_path / "input" / "ibfs.chd"
    fortran_record(var, parts)
    fortran_record(chd, [rng.standard_normal(nf * nf), rng.standard_normal(nf)])
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    assert json.loads(out)["chd_ok"] == 1
    good_var, good_chd = var.read_bytes(), chd.read_bytes()
    # .var cut in the middle of its payload: the trailing record marker is missing
    var.write_bytes(good_var[:len(good_var) // 2])
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO and "corrupt record markers" in err, (rc, err)
    # .var with only its leading marker
    var.write_bytes(good_var[:4])
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO, (rc, err)
    # empty .var
    var.write_bytes(b"")
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO and "truncated record" in err, (rc, err)
    var.write_bytes(good_var)
    # .chd truncated, then with a trailing marker that disagrees with the leading one
    chd.write_bytes(good_chd[:-12])
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO and "ibfs.chd" in err, (rc, err)
    bad = bytearray(good_chd)
    bad[-4:] = struct.pack("<i", 8)
    chd.write_bytes(bytes(bad))
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO and "corrupt record markers" in err, (rc, err)
    # a .chd record for a smaller body (fewer forces than the geometry has)
    fortran_record(chd, [rng.standard_normal(4), rng.standard_normal(2)])
    rc, out, err = run(tmp_path)
    assert rc == IBFS_ERR_IO and "record holds" in err, (rc, err)


def test_bad_namelist(tmp_path):
    write_inp(tmp_path, "&READ_PARAMETERS M=32, NOSUCH=3 /\n")
    rc, out, err = run(tmp_path)
    assert rc != 0 and "NOSUCH" in err
    write_inp(tmp_path, "&READ_PARAMETERS M=3.5 /\n")
    rc, out, err = run(tmp_path)
    assert rc != 0 and "bad value" in err


def test_geometry_primitives_and_spacing_check(tmp_path):
    """input/geom.spec builds the body from the reference's primitives
    (grid.f90:408-520) with the reference's point placement; the point spacing
    is checked against the grid spacing (the check grid.f90:280-284 asks for)."""
    import workloads as W
    write_inp(tmp_path, "&READ_PARAMETERS M=64, N=64, LEN=4.0, OFFSETX=2.0, OFFSETY=2.0 /\n")
    (tmp_path / "input" / "geom.spec").write_text("# a plate and a cylinder\nline 1.0 30 0\ncircle 0.5 0.2 0.1 1\n")
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    p = json.loads(out)
    xl, yl = W.line(4.0 / 64, 1.0, 30.0)
    xc, yc = W.circle(4.0 / 64, 0.5, 0.2, 0.1)
    assert p["nb"] == len(xl) + len(xc)
    assert abs(p["x0"] - xl[0]) < 1e-15 and abs(p["y0"] - yl[0]) < 1e-15
    assert abs(p["xsum"] - (xl.sum() + xc.sum())) < 1e-12 and abs(p["ysum"] - (yl.sum() + yc.sum())) < 1e-12
    assert "WARNING" not in err
    # points far apart for the grid: warned, not refused
    (tmp_path / "input" / "geom.inp").write_text("3\n 0.0 0.0 0\n 0.5 0.0 0\n 1.0 0.0 0\n")
    rc, out, err = run(tmp_path)
    assert rc == 0 and "WARNING: body 0 point spacing" in err
    (tmp_path / "input" / "geom.inp").unlink()
    (tmp_path / "input" / "geom.spec").write_text("ellipse 1 2 0\n")
    rc, out, err = run(tmp_path)
    assert rc != 0 and "unknown primitive" in err


def test_actuator_slots(tmp_path):
    """input/actuator.NNN.inp (&READ_ACT_PARAMETERS): the slot points are
    appended to the geometry as the reference's actuator_slot makes them
    (grid.f90:636-680, restated in the oracle), one point when the slot is
    narrower than ds; with geom.inp already holding them (bodyno < 0) the
    counts come from slot.NNN.inp (grid.f90:286-301)."""
    import oracle as O
    m = 48
    ds = 4.0 / m
    write_inp(tmp_path, f"&READ_PARAMETERS M = {m}, N = {m}, LEN = 4.0, OFFSETX = 2, OFFSETY = 2, "
                        "STATIONARY = T /\n")
    (tmp_path / "input" / "geom.inp").write_text("2\n 0.5 0.0 0\n -0.5 0.0 0\n")
    acts = [dict(x_j=0.0, y_j=0.75, h_j=0.3, u_j=0.5, u_j_osc=0.2, theta_j=90.0, omg_j=6.283185307179586),
            dict(x_j=0.1, y_j=-0.8, h_j=0.05, u_j=-0.3, u_j_osc=0.1, theta_j=-60.0, omg_j=3.0)]
    for i, a in enumerate(acts):
        body = ", ".join(f"{k.upper()} = {v!r}" for k, v in a.items())
        (tmp_path / "input" / f"actuator.{i + 1:03d}.inp").write_text(f" &READ_ACT_PARAMETERS {body} /\n")
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    p = json.loads(out)
    pts = [O.actuator_slot(a["x_j"], a["y_j"], a["h_j"], ds, a["theta_j"], -(i + 1)) for i, a in enumerate(acts)]
    npt = [len(x) for x, _, _ in pts]
    assert npt == [int(0.3 / ds) + 1, 1]
    assert (p["n_act"], p["n_act_pt"], p["nb"]) == (2, sum(npt), 2 + sum(npt))
    xs = 0.5 - 0.5 + sum(float(x.sum()) for x, _, _ in pts)
    ys = sum(float(y.sum()) for _, y, _ in pts)
    assert abs(p["xsum"] - xs) <= 1e-14 and abs(p["ysum"] - ys) <= 1e-14
    # geometry with the actuator points already in it (a restart directory)
    lines = [" 0.5 0.0 0", " -0.5 0.0 0"]
    for x, y, b in pts:
        lines += [f" {float(xv)!r} {float(yv)!r} {int(bv)}" for xv, yv, bv in zip(x, y, b)]
    (tmp_path / "input" / "geom.inp").write_text(f"{len(lines)}\n" + "\n".join(lines) + "\n")
    for i, n in enumerate(npt):
        (tmp_path / "input" / f"slot.{i + 1:03d}.inp").write_text(f"{n:12d}\n")
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    p = json.loads(out)
    assert (p["n_act"], p["n_act_pt"], p["nb"]) == (2, sum(npt), 2 + sum(npt))
    (tmp_path / "input" / "slot.002.inp").unlink()
    rc, out, err = run(tmp_path)
    assert rc != 0 and "slot.002.inp" in err


def test_actuator_slots_after_spec_primitives(tmp_path):
    """Primitives from input/geom.spec, then the actuators' slot points after
    them (grid.f90:382-401: the primitives, then each actuator_slot)."""
    import oracle as O
    m = 64
    ds = 4.0 / m
    write_inp(tmp_path, f"&READ_PARAMETERS M = {m}, N = {m}, LEN = 4.0, OFFSETX = 2, OFFSETY = 2 /\n")
    (tmp_path / "input" / "geom.spec").write_text("circle 1.0 0.0 0.0 0\n")
    (tmp_path / "input" / "actuator.001.inp").write_text(
        " &READ_ACT_PARAMETERS X_J = 0.6, Y_J = 0.0, H_J = 0.25, U_J = 1.0, U_J_OSC = 0.0, "
        "THETA_J = 0.0, OMG_J = 0.0 /\n")
    rc, out, err = run(tmp_path)
    assert rc == 0, err
    p = json.loads(out)
    ncirc = int(np.pi * 1.0 / ds)
    ax, ay, _ = O.actuator_slot(0.6, 0.0, 0.25, ds, 0.0, -1)
    assert (p["n_act"], p["n_act_pt"], p["nb"]) == (1, len(ax), ncirc + len(ax))
    xc, yc = O.circle(ds, 1.0, 0.0, 0.0)
    assert abs(p["xsum"] - (xc.sum() + ax.sum())) <= 1e-13 and abs(p["ysum"] - (yc.sum() + ay.sum())) <= 1e-13
