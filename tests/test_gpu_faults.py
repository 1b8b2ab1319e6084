"""Failure statuses made on the host or with bad inputs, none of which faults,
traps or hangs the GPU:

* a force system that is not positive definite stops preprocess with
  IBFS_ERR_CHOL, the reference's 'choldc failed' (operators.f90:784): a body
  point outside the grid has no faces within the support of its delta kernel,
  so its row and column of A are zero and choldc meets a zero pivot; the oracle
  fails on the same input;
* a bounded wait of the tensor-core GEMM (the single-CTA kernel, or the
  CTA-pair kernel) runs out: ibfs_set_wait_limit's probe
  makes every thread block wait on a barrier that nothing completes (2 ms
  limit) before it issues any copy or product; the advance returns
  IBFS_ERR_TIMEOUT naming that wait, each block frees its tensor memory, and a
  new handle then advances normally (its GEMM allocates the same tensor memory
  on every SM);
* the host driver stops with IBFS_ERR_IO on a truncated restart record or
  Cholesky record in a real (non dry-run) run.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import ibfs_capi as C
import oracle as O
import workloads as W
from conftest import PKG

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def test_singular_force_system_is_chol_error():
    m = 48
    xb, yb = W.circle(4.0 / m)
    xb, yb = np.append(xb, 50.0), np.append(yb, 50.0)  # far outside [-2, 2]^2
    oc = O.Case(O.make_params(m, m, 0.01, 100.0, 3), xb, yb)
    assert oc.preprocess() == 2  # ERR_CHOL in the oracle too
    g = C.Solver(C.make_params(m, m, 0.01, 100.0, 3), (xb, yb))
    with pytest.raises(C.IbfsError) as e:
        g.precompute()
    assert e.value.code == C.ERR_CHOL and "choldc failed" in str(e.value)
    with pytest.raises(C.IbfsError) as e:
        g.advance()  # advance runs preprocess at the first step and stops the same way
    assert e.value.code == C.ERR_CHOL
    g.close()
    # the same body without the stray point factors and advances
    ok = C.Solver(C.make_params(m, m, 0.01, 100.0, 3), (xb[:-1], yb[:-1]))
    ok.precompute()
    assert np.isfinite(ok.advance()["fx"]).all()


@pytest.mark.parametrize("entry,tile", [("advance", 0), ("advance_n", 0), ("advance", 4)])
def test_tensor_core_wait_limit_gives_timeout(entry, tile):
    """tile 4: every GEMM on the CTA-pair kernel, whose two CTAs meet at a
    cluster barrier before freeing their tensor memory."""
    m, lev = 128, 3
    xb, yb = W.circle(4.0 / m)
    p = C.make_params(m, m, 0.004, 100.0, lev)
    g = C.Solver(p, (xb, yb), C.make_options(precision=1, tc_tile=tile))
    g.precompute()  # the factor is FP64 (no tensor-core GEMM); made before the probe is set
    g.set_wait_limit(0.002, probe=True)  # every GEMM block waits on a barrier nothing completes
    with pytest.raises(C.IbfsError) as e:
        if entry == "advance":
            g.advance()
        else:
            g.advance_n(2, want_hist=False)
    assert e.value.code == C.ERR_TIMEOUT, str(e.value)
    assert "bounded device wait gave up" in str(e.value) and "probe" in str(e.value)
    assert "drain" not in str(e.value)  # nothing was in flight when the blocks returned
    g.close()
    # a fresh handle: its GEMM allocates tensor memory on every SM again and
    # its results follow the oracle at the split-precision bar
    g2 = C.Solver(p, (xb, yb), C.make_options(precision=1))
    oc = O.Case(O.make_params(m, m, 0.004, 100.0, lev), xb, yb)
    for _ in range(3):
        og = g2.advance()
        rc, o = oc.advance()
        assert rc == 0
    assert abs(og["fx"][0] - o["fx"][0]) / abs(o["fx"][0]) < 1e-8
    assert rel(g2.get_state()["omega"], oc.get_state()["omega"]) < 1e-8
    # a short real limit on a healthy handle does not fire; a bad one is refused
    g2.set_wait_limit(0.5)
    g2.advance_n(2, want_hist=False)
    with pytest.raises(C.IbfsError) as e:
        g2.set_wait_limit(-1.0)
    assert e.value.code == C.ERR_ARG


DRIVER = os.path.join(PKG, "ibfs_gpu")
IBFS_ERR_IO = 5


def _run_dir(d, istart, istop):
    os.makedirs(d / "input", exist_ok=True)
    (d / "input" / "ibfs.inp").write_text(
        f" &READ_PARAMETERS ISTART = {istart}, ISTOP = {istop}, ISAVE = 2, M = 32,\n N = 32, DT = 0.01, "
        "RE = 100., CGTOL = 1.E-7, CG_MAX_ITER = 3000,\n UNIF_FLOW = T, LEN = 4.0, OFFSETX = 2, OFFSETY = 2, "
        "MGRIDLEV = 3,\n MAKE_VORTEX = F, STATIONARY = T,\n /\n")


def _drive(d):
    return subprocess.run([DRIVER, "-C", str(d)], capture_output=True, text=True, timeout=300)


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")
def test_driver_truncated_records_are_io_errors(tmp_path):
    _run_dir(tmp_path, 0, 2)
    r = _drive(tmp_path)
    assert r.returncode == 0, r.stderr
    var = tmp_path / "output" / "ibfs0000002.var"
    chd = tmp_path / "input" / "ibfs.chd"
    good_var, good_chd = var.read_bytes(), chd.read_bytes()
    # restart from a truncated .var
    _run_dir(tmp_path, 2, 4)
    var.write_bytes(good_var[:len(good_var) // 3])
    r = _drive(tmp_path)
    assert r.returncode == IBFS_ERR_IO and "ibfs0000002.var" in r.stderr, (r.returncode, r.stderr)
    # restart with a good .var but a truncated .chd
    var.write_bytes(good_var)
    chd.write_bytes(good_chd[:len(good_chd) - 100])
    r = _drive(tmp_path)
    assert r.returncode == IBFS_ERR_IO and "ibfs.chd" in r.stderr, (r.returncode, r.stderr)
    # a fresh run (istart 0) that finds a truncated .chd stops the same way
    shutil.rmtree(tmp_path / "output")
    _run_dir(tmp_path, 0, 2)
    r = _drive(tmp_path)
    assert r.returncode == IBFS_ERR_IO and "ibfs.chd" in r.stderr, (r.returncode, r.stderr)
    # with the good files both runs go through
    chd.write_bytes(good_chd)
    r = _drive(tmp_path)
    assert r.returncode == 0, r.stderr
