"""Failure statuses on the GPU paths, made on the host (no GPU fault): the CG
iteration cap is the reference's warning (operators.f90:435-438) -- the step
completes, its outputs match the oracle capped the same way, and later steps
run -- and calls on a finished handle report argument errors."""
import ctypes

import numpy as np
import pytest

import ibfs_capi as C
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def test_cg_iteration_cap_is_a_warning():
    m = 32
    xb, yb = W.circle(4.0 / m)
    po = O.make_params(m, m, 0.01, 100.0, 3, stationary=False, cgtol=1e-14, cg_max_iter=2)
    oc = O.Case(po, xb, yb)
    g = C.Solver(C.make_params(m, m, 0.01, 100.0, 3, stationary=False, cgtol=1e-14, cg_max_iter=2), (xb, yb))
    fo, fg = [], []
    for _ in range(3):
        rc, o = oc.advance()
        assert rc == 3
        with pytest.warns(RuntimeWarning, match="max iterations"):
            og = g.advance()
        assert g.last_cg_iterations() == 2
        fo.append(o["fx"][0])
        fg.append(og["fx"][0])
    assert g.itime.value == 3
    assert np.abs(np.array(fg) - fo).max() / np.abs(fo).max() < 1e-9
    with pytest.warns(RuntimeWarning):
        h = g.advance_n(2)
    assert g.itime.value == 5 and np.isfinite(h).all()


def test_bad_case_index_and_sizes():
    m = 32
    xb, yb = W.circle(4.0 / m)
    g = C.Solver(C.make_params(m, m, 0.01, 100.0, 3), (xb, yb))
    L = C.lib()
    assert L.ibfs_case_sizes(g.h, 1, *([None] * 6)) == 7
    assert L.ibfs_get_state(g.h, 5, None, None, None, None, None) == 7
    with pytest.raises(AssertionError):
        g.batch_advance(np.zeros(3))  # wrong body-velocity length is refused before the call
    g.close()
