"""Batched form: several independent cases of uneven size and level count in
one handle (one launch per kernel for all of them) against the oracle run
case by case, and against single-case handles."""
import numpy as np
import pytest

import ibfs_capi as C
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

SMALL = [W.case(32, 3, 100.0, 0.01, "cylinder"), W.case(48, 2, 250.0, 0.008, "plate", aoa=20.0),
         W.case(64, 3, 60.0, 0.006, "plate", aoa=35.0), W.case(32, 2, 400.0, 0.01, "plate", aoa=5.0, n=24)]


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("precision,tol,tile", [(0, 1e-10, 0), (1, 1e-8, 0), (1, 1e-8, 4)])
def test_batch_vs_oracle(precision, tol, tile):
    """tile 4: every tensor-core GEMM of the split form on the CTA-pair tile,
    the 32 x 24 case included."""
    params, bodies, opts = W.solver_args(SMALL, C, precision)
    for o in opts:
        o.tc_tile = tile
    g = C.Solver(params, bodies, opts)
    steps = 6
    hist = g.advance_n(steps)
    for ic, c in enumerate(SMALL):
        oc = O.Case(O.make_params(c["m"], c["n"], c["dt"], c["re"], c["levels"]), c["xb"], c["yb"])
        fx = []
        for _ in range(steps):
            rc, o = oc.advance()
            assert rc == 0
            fx.append((o["fx"][0], o["fy"][0]))
        fx = np.array(fx)
        fg = np.array([[g.outputs_of(hist[s], ic)["fx"][0], g.outputs_of(hist[s], ic)["fy"][0]]
                       for s in range(steps)])
        cd = np.abs(fx[:, 0]).max()
        assert np.abs(fg - fx).max() / cd < tol, ic
        so, sg = oc.get_state(), g.get_state(ic)
        assert rel(sg["omega"], so["omega"]) < tol, ic


def test_batch_equals_single_handles():
    params, bodies, opts = W.solver_args(SMALL, C, 0)
    g = C.Solver(params, bodies, opts)
    g.advance_n(4, want_hist=False)
    for ic in range(len(SMALL)):
        s = C.Solver(params[ic], bodies[ic], opts[ic])
        s.advance_n(4, want_hist=False)
        assert np.array_equal(s.get_state()["omega"], g.get_state(ic)["omega"]), ic


def test_batch_advance_per_step_call():
    """ibfs_batch_advance (host body velocities in, one step's outputs out)
    reproduces advance_n's history bit for bit, and body velocities given to
    it equal those given to single-case ibfs_advance calls."""
    params, bodies, opts = W.solver_args(SMALL, C, 0)
    a = C.Solver(params, bodies, opts)
    b = C.Solver(params, bodies, opts)
    hist = a.advance_n(3)
    rows = [b.batch_advance() for _ in range(3)]
    assert np.array_equal(np.array(rows), hist)
    rng = np.random.default_rng(5)
    vels = [0.05 * rng.standard_normal(s["nf"]) for s in b.sizes]
    row = b.batch_advance(np.concatenate(vels))
    for ic in range(len(SMALL)):
        s = C.Solver(params[ic], bodies[ic], opts[ic])
        s.advance_n(3, want_hist=False)
        o = s.advance(body_vel=vels[ic])
        assert np.array_equal(b.outputs_of(row, ic)["fx"], o["fx"]), ic
        assert np.array_equal(b.get_state(ic)["omega"], s.get_state()["omega"]), ic
