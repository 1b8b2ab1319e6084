"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point declared in include/ibfs_capi.h (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def so_path():
    subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(ROOT, "ibfs-if2d_b200")])
    return os.path.join(ROOT, "ibfs-if2d_b200", "libibfs_b200.so")


def declared():
    text = open(os.path.join(ROOT, "include", "ibfs_capi.h")).read()
    return sorted(set(re.findall(r"\b(ibfs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "ibfs_advance" in names and "ibfs_create" in names and len(names) >= 15


def test_library_exports_all(so_path):
    lib = ctypes.CDLL(so_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_matches_header(so_path):
    import ibfs_capi
    assert sorted(ibfs_capi.EXPORTS) == declared()


def test_kernels_are_sm100a(so_path):
    out = subprocess.run(["cuobjdump", "--list-elf", so_path], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_error_statuses_without_gpu(so_path):
    """Argument and grid checks run before any CUDA call: the statuses and
    messages of the reference's STOPs (grid.f90:67-69) come back on a host
    without a GPU."""
    import ibfs_capi as C
    L = C.lib()
    h = ctypes.c_void_p()
    xb = np.zeros(4)
    yb = np.linspace(-0.2, 0.2, 4)
    p = C.make_params(30, 32, 0.01, 100.0, 3)  # m not divisible by 4
    rc = L.ibfs_create(ctypes.byref(p), None, 4, C._p(xb), C._p(yb), None, ctypes.byref(h))
    assert rc == 1 and h.value is None
    assert b"divisible by 4" in L.ibfs_last_error(None)
    rc = L.ibfs_create(None, None, 4, C._p(xb), C._p(yb), None, ctypes.byref(h))
    assert rc == 7
    rc = L.ibfs_case_sizes(None, 0, *([None] * 6))
    assert rc == 7
    assert L.ibfs_advance_n(None, 1, None) == 7
    assert L.ibfs_batch_advance(None, None, None) == 7


def test_adjoint_weight_lengths_checked():
    """The adjoint wrappers refuse objective weights that do not cover
    nsteps x nbody per case (the C side would read past them); the check
    runs before any library call, so a handle-less Solver shows it."""
    import ibfs_capi as C
    s = C.Solver.__new__(C.Solver)
    s.h, s.ncases = None, 2
    s.sizes = [dict(nbody=1, nf=10), dict(nbody=2, nf=10)]
    with pytest.raises(ValueError):
        s.adjoint_pitch_run(4, 2, np.zeros(4), np.zeros(4))  # tiled 1-D: 8 weights, 12 needed
    with pytest.raises(ValueError):
        s.adjoint_pitch_run(4, 2, np.zeros(11), np.zeros(11))
    s.ncases, s.sizes = 1, [dict(nbody=3, nf=10)]
    with pytest.raises(ValueError):
        s.adjoint_run(4, 2, None, np.zeros(4), np.zeros(4))


def test_pitching_workload_options():
    """workloads.solver_args turns pitching cases into moving-body CG options
    (relative stop, device pitching, preconditioned unless asked otherwise)
    and stationary cases into Cholesky ones."""
    import ibfs_capi as C
    import workloads as W
    cases = [W.pitching(m=64, levels=3, amp_deg=12.5), W.pitching(m=64, levels=3, amp_deg=7.0, precond=False),
             W.case(64, 3, 100.0, 0.01, "cylinder")]
    params, bodies, opts = W.solver_args(cases, C)
    assert [p.stationary for p in params] == [0, 0, 1]
    assert [o.motion_kind for o in opts] == [1, 1, 0]
    assert [o.cg_precond for o in opts] == [1, 0, 0]
    assert opts[0].cg_relative == 1 and opts[0].pitch_amp_deg == 12.5 and opts[0].pitch_freq == 0.25
    assert params[0].cgtol == 1e-12 and len(bodies[0][0]) == int(1.0 / (4.0 / 64)) + 1
