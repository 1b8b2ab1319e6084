"""Moving-body path: the CG force solve (cjgr, operators.f90:393-441) on a
fixed body, and a rigidly pitching plate whose regularisation is rebuilt on
the GPU every step (setup_reg, grid.f90:142-230), both against the oracle
driven with the same body positions and velocities."""
import math

import numpy as np
import pytest

import ibfs_capi as C
import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def test_cg_fixed_body():
    m = 48
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    po = O.make_params(m, m, 0.01, 100.0, 3, stationary=False, cgtol=1e-12)
    oc = O.Case(po, xb, yb)
    oc.set_cg_relative(True)
    g = C.Solver(C.make_params(m, m, 0.01, 100.0, 3, stationary=False, cgtol=1e-12), (xb, yb),
                 C.make_options(cg_relative=1))
    fo, fg = [], []
    for _ in range(5):
        rc, o = oc.advance()
        og = g.advance()
        fo.append(o["fx"][0])
        fg.append(og["fx"][0])
        assert g.last_cg_iterations() > 0
    ef, eo = rel(fg, fo), rel(g.get_state()["omega"], oc.get_state()["omega"])
    print(f"CG fixed body: force {ef:.2e}, omega {eo:.2e}")
    assert ef < 1e-10
    assert eo < 1e-10


def pitch_state(xb0, yb0, t, amp_deg, freq, px=0.0, py=0.0):
    amp = amp_deg * math.pi / 180.0
    al = amp * math.sin(2 * math.pi * freq * t)
    ald = amp * 2 * math.pi * freq * math.cos(2 * math.pi * freq * t)
    th, thd = -al, -ald
    c, s = math.cos(th), math.sin(th)
    x = px + c * (xb0 - px) - s * (yb0 - py)
    y = py + s * (xb0 - px) + c * (yb0 - py)
    return x, y, np.concatenate([-thd * (y - py), thd * (x - px)])


@pytest.mark.parametrize("precision", [0, 1])
def test_pitching_plate(precision):
    m, dt, amp, freq = 64, 0.01, 20.0, 0.25
    xb0, yb0 = O.line(4.0 / m, 1.0, 0.0)
    oc = O.Case(O.make_params(m, m, dt, 500.0, 3, stationary=False, cgtol=1e-12), xb0, yb0, np.ones(len(xb0)))
    oc.set_cg_relative(True)
    g = C.Solver(C.make_params(m, m, dt, 500.0, 3, stationary=False, cgtol=1e-12), (xb0, yb0),
                 C.make_options(precision=precision, cg_relative=1, motion_kind=1, pitch_amp_deg=amp,
                                pitch_freq=freq))
    fo, fg = [], []
    for s in range(1, 9):
        x, y, v = pitch_state(xb0, yb0, s * dt, amp, freq)
        oc.set_body(x, y)
        rc, o = oc.advance(body_vel=v)
        assert rc == 0
        og = g.advance()
        fo.append((o["fx"][0], o["fy"][0]))
        fg.append((og["fx"][0], og["fy"][0]))
    fo, fg = np.array(fo), np.array(fg)
    tol = 1e-10 if precision == 0 else 1e-8
    ef = np.abs(fg - fo).max() / np.abs(fo).max()
    eo = rel(g.get_state()["omega"], oc.get_state()["omega"])
    print(f"pitching plate precision={precision}: force {ef:.2e}, omega {eo:.2e}")
    assert ef < tol
    assert eo < tol


def test_pitching_batch_equals_single_handles():
    """Several pitching amplitudes advanced together (one launch per kernel,
    CG iterations until every case has converged, converged cases idle) give
    each case's single-handle result, and the first case follows the oracle."""
    import workloads as W
    cases = [W.pitching(m=48, levels=3, re=500.0, dt=0.01, amp_deg=a) for a in (5.0, 17.0, 30.0)]
    params, bodies, opts = W.solver_args(cases, C)
    g = C.Solver(params, bodies, opts)
    hist = g.advance_n(5)
    for ic in range(len(cases)):
        s = C.Solver(params[ic], bodies[ic], opts[ic])
        hs = s.advance_n(5)
        assert rel(g.get_state(ic)["omega"], s.get_state()["omega"]) < 1e-13, ic
        fb = np.array([g.outputs_of(hist[k], ic)["fx"][0] for k in range(5)])
        fs = np.array([s.outputs_of(hs[k], 0)["fx"][0] for k in range(5)])
        assert rel(fb, fs) < 1e-13, ic
        s.close()
    c = cases[0]
    oc = O.Case(O.make_params(c["m"], c["n"], c["dt"], c["re"], c["levels"], stationary=False, cgtol=1e-12),
                c["xb"], c["yb"], np.ones(len(c["xb"])))
    oc.set_cg_relative(True)
    fo = []
    for k in range(1, 6):
        x, y, v = pitch_state(c["xb"], c["yb"], k * c["dt"], c["pitch_amp_deg"], c["pitch_freq"])
        oc.set_body(x, y)
        rc, o = oc.advance(body_vel=v)
        assert rc == 0
        fo.append(o["fx"][0])
    fb = np.array([g.outputs_of(hist[k], 0)["fx"][0] for k in range(5)])
    assert rel(fb, fo) < 1e-9


def test_amplitude_derivative_by_central_differences():
    """d(mean drag)/d(pitch amplitude) from one batch of A -+ h cases: the
    central differences at two step sizes agree (O(h^2) truncation), J (the
    mean of the two neighbours, O(h^2) from J(A)) is the mean drag of a
    single-handle run at A within that, and the discrete adjoint agrees with
    the extrapolated difference."""
    import sensitivity as S
    kw = dict(m=48, levels=2, re=500.0, dt=0.01, freq=0.25)
    amps = [10.0, 25.0]
    J1, g1 = S.mean_drag_amplitude_derivative(amps, h_deg=0.05, steps=12, tail=6, **kw)
    J2, g2 = S.mean_drag_amplitude_derivative(amps, h_deg=0.025, steps=12, tail=6, **kw)
    assert np.all(np.abs(g1 - g2) <= 1e-3 * np.abs(g2) + 1e-9)
    assert np.all(np.abs(J1 - J2) <= 1e-5 * np.abs(J2))
    import workloads as W
    c = W.pitching(amp_deg=amps[0], **kw)
    p, b, o = W.solver_args([c], C)
    s = C.Solver(p[0], b[0], o[0])
    h = s.advance_n(12)
    J = np.mean([s.outputs_of(h[k], 0)["fx"][0] for k in range(6, 12)])
    assert abs(J2[0] - J) <= 1e-5 * abs(J)
    # the discrete adjoint against the Richardson extrapolation of the two
    # central differences (O(h^4))
    Ja, ga = S.mean_drag_amplitude_adjoint(amps, steps=12, tail=6, checkpoint_every=4, **kw)
    assert abs(Ja[0] - J) <= 1e-12 * abs(J)
    gr = (4.0 * g2 - g1) / 3.0
    assert np.all(np.abs(ga - gr) <= 1e-5 * np.abs(gr)), (ga, gr)


def test_preconditioned_cg_matches_plain_cg():
    """cg_precond = 1: CG preconditioned by factors at a grid of pitch angles turned with
    the plate reaches the same relative 1e-12 solution as the reference's
    unpreconditioned cjgr (forces within 1e-10) in fewer iterations; on a
    body that does not move it is the inverse of A's symmetric part (A is
    symmetric to ~1e-6, so a handful of iterations reach 1e-12)."""
    m, dt, amp, freq = 64, 0.02, 25.0, 0.25
    xb0, yb0 = O.line(4.0 / m, 1.0, 0.0)
    runs = {}
    for pre in (0, 1):
        g = C.Solver(C.make_params(m, m, dt, 500.0, 3, stationary=False, cgtol=1e-12), (xb0, yb0),
                     C.make_options(cg_relative=1, motion_kind=1, pitch_amp_deg=amp, pitch_freq=freq, cg_precond=pre))
        f, its = [], []
        for s in range(30):
            o = g.advance()
            f.append((o["fx"][0], o["fy"][0]))
            its.append(g.last_cg_iterations())
        runs[pre] = (np.array(f), np.array(its), g.get_state()["omega"])
        g.close()
    (f0, i0, w0), (f1, i1, w1) = runs[0], runs[1]
    assert np.abs(f1 - f0).max() <= 1e-10 * np.abs(f0).max()
    assert rel(w1, w0) < 1e-10
    assert i1[5:].sum() < 0.7 * i0[5:].sum(), (i0, i1)
    # fixed body: the preconditioner is the inverse of A's symmetric part
    # (compared with plain CG: the Cholesky path factors the upper triangle,
    # i.e. solves with the symmetric part, which differs from A at ~1e-6)
    xb, yb = O.circle(4.0 / 48, 1.0, 0.0, 0.0)
    pp = C.make_params(48, 48, 0.01, 100.0, 3, stationary=False, cgtol=1e-12)
    ref = C.Solver(pp, (xb, yb), C.make_options(cg_relative=1))
    g = C.Solver(pp, (xb, yb), C.make_options(cg_relative=1, cg_precond=1))
    for _ in range(5):
        a, b = g.advance(), ref.advance()
        assert g.last_cg_iterations() <= 5 and ref.last_cg_iterations() > 20
        assert abs(a["fx"][0] - b["fx"][0]) <= 1e-10 * abs(b["fx"][0])
    g.close()
    ref.close()
