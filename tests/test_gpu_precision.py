"""Split-precision form (3xBF16 tcgen05 sine transforms + one FP64 refinement
sweep per solve) against the FP64 oracle.

Bars: each refined solve (ctci, ainv) within 1e-9 of FP64 (max-abs relative;
measured ~2e-10); over an advance, forces (Cd, Cl normalised by max |Cd|)
within 1e-8 and fields within 1e-8.
"""
import numpy as np
import pytest

import ibfs_capi as C
import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("m,n,tile", [(64, 64, 0), (128, 96, 0), (200, 200, 0), (128, 96, 4), (192, 384, 4)])
def test_refined_solves(m, n, tile):
    """ctci and ainv of the split form against the oracle, square and
    rectangular grids; tile 4 puts every GEMM on the CTA-pair tile."""
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    oc = O.Case(O.make_params(m, n, 0.004, 100.0, 3), xb, yb)
    g = C.Solver(C.make_params(m, n, 0.004, 100.0, 3), (xb, yb), C.make_options(precision=1, tc_tile=tile))
    x = np.random.default_rng(5).standard_normal(oc.ns)
    assert rel(g.apply_op(1, x), oc.ctci(x)) < 1e-9
    assert rel(g.apply_op(2, x), oc.ainv(x)) < 1e-9


@pytest.mark.parametrize("body,m,lev,steps", [("cyl", 64, 3, 20), ("plate", 128, 3, 10)])
def test_precision_advance(body, m, lev, steps):
    ds = 4.0 / m
    xb, yb = O.circle(ds, 1.0, 0.0, 0.0) if body == "cyl" else O.line(ds, 1.0, 30.0)
    oc = O.Case(O.make_params(m, m, 0.004, 100.0, lev), xb, yb)
    g = C.Solver(C.make_params(m, m, 0.004, 100.0, lev), (xb, yb), C.make_options(precision=1))
    fo, fg = [], []
    for _ in range(steps):
        rc, o = oc.advance()
        og = g.advance()
        fo.append((o["fx"][0], o["fy"][0]))
        fg.append((og["fx"][0], og["fy"][0]))
    fo, fg = np.array(fo), np.array(fg)
    cd = np.abs(fo[:, 0]).max()
    assert np.abs(fg - fo).max() / cd < 1e-8
    so, sg = oc.get_state(), g.get_state()
    assert rel(sg["omega"], so["omega"]) < 1e-8
    assert rel(sg["q"], so["q"]) < 1e-8


@pytest.mark.parametrize("m,lev", [(128, 3), (256, 2), (192, 2), (384, 2)])
def test_tensor_core_tile_shapes_and_autotuner(m, lev):
    """The tensor-core GEMM's four tile configurations (128 x 128 with K
    blocks of 64 and two stages; 128 x 256, K 32, two stages; 128 x 128, K 32,
    four stages; 256 x 256 on a CTA pair, K 64, two stages) and the measured
    autotuner's per-launch-group choice all follow the FP64 oracle at the
    split-precision bar, including grids whose m - 1 is not a multiple of the
    tile (191, 383); the tuner reports a configuration for every GEMM launch
    group of the step."""
    xb, yb = O.line(4.0 / m, 1.0, 30.0)
    oc = O.Case(O.make_params(m, m, 0.004, 300.0, lev), xb, yb)
    for _ in range(4):
        oc.advance()
    ref = oc.get_state()["omega"]
    widths = {}
    for tile in (1, 2, 3, 4, 0):
        g = C.Solver(C.make_params(m, m, 0.004, 300.0, lev), (xb, yb), C.make_options(precision=1, tc_tile=tile))
        widths[tile] = g.gemm_tiles()
        g.advance_n(4, want_hist=False)
        assert rel(g.get_state()["omega"], ref) < 1e-8, tile
        x = np.random.default_rng(3).standard_normal(g.sizes[0]["ns"])
        assert rel(g.apply_op(1, x), oc.ctci(x)) < 1e-9, tile
        g.close()
    for tile in (1, 2, 3, 4):
        assert widths[tile] and set(widths[tile]) == {tile}
    assert len(widths[0]) == len(widths[1]) and set(widths[0]) <= {1, 2, 3, 4}
