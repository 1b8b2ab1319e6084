"""Discrete adjoint of the moving-body advance (ibfs_adjoint_pitch_run): a
plate pitching about mid-chord, CG force solve to a relative 1e-12, objective
the mean drag over the last steps, derivative with respect to the pitch
amplitude. Checked against central finite differences of the forward advance
and against the FP64 tangent-linear reference (complex step in the amplitude
through the independent numpy restatement, exact force solve)."""
import numpy as np
import pytest

import ibfs_capi as C
import tangent_linear as TL
import workloads as W

pytestmark = pytest.mark.gpu

KW = dict(m=48, levels=3, re=500.0, dt=0.02, freq=0.25)
STEPS, TAIL = 16, 8


def solver(amp, kw=KW):
    c = W.pitching(amp_deg=amp, **kw)
    p, b, o = W.solver_args([c], C)
    return c, C.Solver(p[0], b[0], o[0])


def forward_J(amp, steps=STEPS, tail=TAIL, kw=KW):
    _, s = solver(amp, kw)
    h = s.advance_n(steps)
    fx = [s.outputs_of(h[k], 0)["fx"][0] for k in range(steps)]
    s.close()
    return float(np.mean(fx[steps - tail:]))


def adjoint(amp, K, steps=STEPS, tail=TAIL, kw=KW):
    _, s = solver(amp, kw)
    wx = np.zeros(steps)
    wx[steps - tail:] = 1.0 / tail
    J, g, ms_f, ms_t = s.adjoint_pitch_run(steps, K, wx, np.zeros(steps))
    st = s.get_state()
    s.close()
    return J, g, ms_t / ms_f, st


@pytest.mark.parametrize("K", [5, 16])
def test_pitch_adjoint_vs_finite_differences(K):
    for amp in (10.0, 25.0):
        J, g, cost, st = adjoint(amp, K)
        assert abs(J - forward_J(amp)) <= 1e-12 * abs(J)
        h = 0.02  # degrees; fourth-order central difference
        Jp1, Jm1, Jp2, Jm2 = (forward_J(amp + d) for d in (h, -h, 2 * h, -2 * h))
        fd = (8.0 * (Jp1 - Jm1) - (Jp2 - Jm2)) / (12.0 * h)
        assert abs(g - fd) <= 1e-6 * abs(fd), (amp, K, g, fd)


def test_pitch_adjoint_vs_tangent_linear_and_state():
    amp = 17.0
    J, g, cost, st = adjoint(amp, 4)
    c, _ = solver(amp)
    Jr, tl = TL.mean_drag_amplitude_derivative(KW["m"], KW["levels"], KW["dt"], KW["re"], c["xb"], c["yb"], amp,
                                               KW["freq"], STEPS, TAIL)
    # the GPU's CG stops at a relative residual of 1e-12; the reference solves exactly
    assert abs(J - Jr) <= 1e-9 * abs(Jr)
    assert abs(g - tl) <= 1e-8 * abs(tl), (g, tl)
    # on return the state is the state after the advances
    _, s = solver(amp)
    s.advance_n(STEPS)
    ref = s.get_state()
    s.close()
    assert np.array_equal(st["omega"], ref["omega"]) and np.array_equal(st["fb"], ref["fb"])


def test_pitch_adjoint_batched_equals_single():
    """Several amplitudes (and grids) differentiated together, one slot each,
    give each case's single-handle J and dJ/dA."""
    kw2 = dict(KW, m=32, levels=2)
    cases = [W.pitching(amp_deg=a, **KW) for a in (8.0, 21.0)] + [W.pitching(amp_deg=14.0, **kw2)]
    p, b, o = W.solver_args(cases, C)
    g = C.Solver(p, b, o)
    wx = np.zeros(STEPS)
    wx[STEPS - TAIL:] = 1.0 / TAIL
    Jb, gb, ms_f, ms_t = g.adjoint_pitch_run(STEPS, 5, wx, np.zeros(STEPS))
    assert Jb.shape == (3,) and gb.shape == (3,)
    for i in range(3):
        s = C.Solver(p[i], b[i], o[i])
        Js, gs, _, _ = s.adjoint_pitch_run(STEPS, 5, wx, np.zeros(STEPS))
        s.close()
        assert abs(Jb[i] - Js) <= 1e-13 * abs(Js), i
        assert abs(gb[i] - gs) <= 1e-11 * abs(gs), (i, gb[i], gs)
    g.close()
