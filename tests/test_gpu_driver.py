"""The host driver (ibfs_gpu) run end to end in a reference-style run
directory: its force.dat / restart records against the oracle, a restart from
a .var record continuing the run exactly, and input/ibfs.chd reused."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import oracle as O
import workloads as W
from conftest import PKG

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(PKG, "ibfs_gpu")
M, LEV, DT, RE, STEPS = 32, 3, 0.01, 100.0, 6


def setup_dir(d, istart=0):
    os.makedirs(d / "input", exist_ok=True)
    (d / "input" / "ibfs.inp").write_text(
        f" &READ_PARAMETERS ISTART = {istart}, ISTOP = {STEPS}, ISAVE = 3, M = {M},\n N = {M}, DT = {DT}, "
        f"RE = {RE}, CGTOL = 1.E-7, CG_MAX_ITER = 3000,\n UNIF_FLOW = T, LEN = 4.0, OFFSETX = 2, OFFSETY = 2, "
        f"MGRIDLEV = {LEV},\n MAKE_VORTEX = F, STATIONARY = T,\n /\n")
    xb, yb = W.circle(4.0 / M)
    lines = [f"{len(xb)}"] + [f" {float(x)!r} {float(y)!r} 0" for x, y in zip(xb, yb)]
    (d / "input" / "geom.inp").write_text("\n".join(lines) + "\n")
    return xb, yb


def run(d):
    r = subprocess.run([DRIVER, "-C", str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout[-2000:]
    return r


def table(path):
    return np.array([[float(v) for v in line.split()] for line in open(path) if line.strip()])


def read_record(path):
    raw = open(path, "rb").read()
    n = struct.unpack("<i", raw[:4])[0]
    assert struct.unpack("<i", raw[4 + n:8 + n])[0] == n
    return np.frombuffer(raw[4:4 + n], dtype="<f8")


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")
def test_driver_run_restart_and_cholesky_file(tmp_path):
    a = tmp_path / "a"
    xb, yb = setup_dir(a)
    run(a)
    f = table(a / "output" / "force.dat")
    assert f.shape == (STEPS, 3) and list(f[:, 0]) == list(range(1, STEPS + 1))
    assert table(a / "output" / "circ.dat").shape == (STEPS, 1 + LEV)
    assert table(a / "output" / "slip.dat").shape == (STEPS, 2)
    assert (a / "input" / "ibfs.chd").exists()
    # against the oracle, step by step
    oc = O.Case(O.make_params(M, M, DT, RE, LEV), xb, yb)
    ref = []
    for _ in range(STEPS):
        rc, o = oc.advance()
        assert rc == 0
        ref.append((o["fx"][0], o["fy"][0]))
    ref = np.array(ref)
    cd = np.abs(ref[:, 0]).max()
    assert np.abs(f[:, 1:] - ref).max() / cd < 1e-10
    rec = read_record(a / "output" / "ibfs0000006.var")
    so = oc.get_state()
    ns = (M - 1) ** 2
    om = rec[:ns * LEV]
    assert np.abs(om - so["omega"]).max() / np.abs(so["omega"]).max() < 1e-10
    # restart from the step-3 record continues the run exactly
    b = tmp_path / "b"
    setup_dir(b, istart=3)
    os.makedirs(b / "output")
    shutil.copy(a / "output" / "ibfs0000003.var", b / "output")
    shutil.copy(a / "input" / "ibfs.chd", b / "input")
    run(b)
    fb_ = open(b / "output" / "force.dat").read().splitlines()
    fa_ = open(a / "output" / "force.dat").read().splitlines()
    assert fb_ == fa_[3:]
    assert np.array_equal(read_record(b / "output" / "ibfs0000006.var"), rec)
    # a fresh run that finds input/ibfs.chd reads it instead of recomputing
    c = tmp_path / "c"
    setup_dir(c)
    shutil.copy(a / "input" / "ibfs.chd", c / "input")
    r = run(c)
    assert "Reading Cholesky premade decomposition" in r.stdout
    assert open(c / "output" / "force.dat").read() == open(a / "output" / "force.dat").read()
    # post-processing (post.f90): Tecplot files of the saved steps, every level
    r = subprocess.run([DRIVER, "-C", str(a), "--post"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    from test_gpu_parity import vertex_reference
    for it in (0, 3, 6):
        for k in range(1, LEV + 1):
            path = a / "post" / f"ibfs_g{k}t{it:07d}_vel.dat"
            lines = open(path).read().splitlines()
            assert lines[0].split("=")[-1].strip(' "') == str(it) and len(lines) == 12 + (M - 1) ** 2
            data = np.array([[float(line[14 * c:14 * c + 14]) for c in range(7)] for line in lines[12:]])
            fac, de = 2.0 ** (k - 1), 4.0 / M
            ii, jj = np.meshgrid(np.arange(2, M + 1), np.arange(2, M + 1))
            x = fac * de * (ii.ravel() - 1) - (fac - 1) / 2 * 4.0 - 2.0
            y = fac * de * (jj.ravel() - 1) - (fac - 1) / 2 * de * M - 2.0
            assert np.allclose(data[:, 0], x, rtol=1e-5, atol=1e-5) and np.allclose(data[:, 1], y, rtol=1e-5, atol=1e-5)
            if it == 6:
                ref = vertex_reference(oc, so, k, de, DT)
                for c, f in enumerate(("u", "v", "etfx", "etfy", "vort")):
                    # E14.5 keeps five significant digits: half a unit of the fifth,
                    # plus the FP64 parity bar (1e-10 of the field) for values at roundoff level
                    bar = 5.01e-5 * np.abs(ref[f]) + 1e-10 * np.abs(ref[f]).max() + 1e-300
                    assert np.all(np.abs(data[:, 2 + c] - ref[f]) <= bar), (k, f)


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")
def test_driver_actuator_jets(tmp_path):
    """input/actuator.001.inp: the driver appends the slot points to the
    geometry (bodyno -1), writes slot.001.inp and rewrites geom.inp, and runs
    the jets on the device; force.dat carries bodies -1 and 0 (write_force
    loops minval..maxval of bdyno) and matches the oracle advanced with the
    jet velocities computed on the host."""
    import math
    d = tmp_path / "act"
    xb, yb = setup_dir(d)
    a = dict(x_j=0.0, y_j=0.75, h_j=0.3, u_j=0.5, u_j_osc=0.2, theta_j=90.0, omg_j=2.0 * math.pi)
    body = ", ".join(f"{k.upper()} = {v!r}" for k, v in a.items())
    (d / "input" / "actuator.001.inp").write_text(f" &READ_ACT_PARAMETERS {body} /\n")
    run(d)
    ax, ay, ab = O.actuator_slot(a["x_j"], a["y_j"], a["h_j"], 4.0 / M, a["theta_j"], -1)
    assert int(open(d / "input" / "slot.001.inp").read().split()[0]) == len(ax)
    geo = open(d / "input" / "geom.inp").read().split()
    assert int(geo[0]) == len(xb) + len(ax)
    x, y = np.concatenate([xb, ax]), np.concatenate([yb, ay])
    bd = np.concatenate([np.zeros(len(xb), dtype=np.int32), ab])
    oc = O.Case(O.make_params(M, M, DT, RE, LEV), x, y, bd)
    acts = [dict(npt=len(ax), u_j=a["u_j"], u_j_osc=a["u_j_osc"], omg_j=a["omg_j"], theta_j=a["theta_j"])]
    ref = []
    for s in range(1, STEPS + 1):
        rc, o = oc.advance(body_vel=O.jet_velocities(np.zeros(2 * len(x)), acts, s, DT))
        assert rc == 0
        ref.append(list(o["fx"]) + list(o["fy"]))
    ref = np.array(ref)
    f = table(d / "output" / "force.dat")
    assert f.shape == (STEPS, 5)
    assert np.abs(f[:, 1:] - ref).max() <= 1e-10 * np.abs(ref).max()
