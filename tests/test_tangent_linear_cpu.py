"""The complex-step tangent-linear reference agrees with central finite
differences of the numpy restatement itself (CPU)."""
import numpy as np

import oracle as O
import tangent_linear as TL


def test_complex_step_matches_fd():
    m, lev, dt, re, steps, tail = 32, 3, 0.01, 150.0, 6, 3
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    th = np.arctan2(yb, xb)
    rng = np.random.default_rng(3)
    u = rng.normal(0.0, 0.1, len(xb))
    du = rng.standard_normal(len(xb))
    vel = np.concatenate([-u * np.sin(th), u * np.cos(th)])
    dvel = np.concatenate([-du * np.sin(th), du * np.cos(th)])
    J0, tl = TL.mean_lift_derivative(m, lev, dt, re, xb, yb, vel, dvel, steps, tail)
    h = 1e-4
    Jp, _ = TL.mean_lift_derivative(m, lev, dt, re, xb, yb, vel + h * dvel, dvel, steps, tail)
    Jm, _ = TL.mean_lift_derivative(m, lev, dt, re, xb, yb, vel - h * dvel, dvel, steps, tail)
    fd = (Jp - Jm) / (2 * h)
    assert abs(fd - tl) <= 1e-7 * max(abs(tl), 1.0)


def test_pitch_complex_step_matches_fd_and_oracle():
    """The pitching-plate reference (complex step in the amplitude, exact
    force solve): its J is the C oracle's (CG to a relative 1e-12, the same
    body positions and velocities) and its derivative is the central
    difference of its own J."""
    import workloads as W
    m, lev, dt, re, amp, freq, steps, tail = 32, 3, 0.02, 500.0, 12.0, 0.25, 8, 4
    c = W.pitching(m=m, levels=lev, re=re, dt=dt, amp_deg=amp, freq=freq)
    xb0, yb0 = c["xb"], c["yb"]
    J, g = TL.mean_drag_amplitude_derivative(m, lev, dt, re, xb0, yb0, amp, freq, steps, tail)
    h = 1e-3
    Jp, _ = TL.mean_drag_amplitude_derivative(m, lev, dt, re, xb0, yb0, amp + h, freq, steps, tail)
    Jm, _ = TL.mean_drag_amplitude_derivative(m, lev, dt, re, xb0, yb0, amp - h, freq, steps, tail)
    assert abs((Jp - Jm) / (2 * h) - g) <= 1e-6 * abs(g)
    oc = O.Case(O.make_params(m, m, dt, re, lev, stationary=False, cgtol=1e-12), xb0, yb0, np.ones(len(xb0)))
    oc.set_cg_relative(True)
    A, om = amp * np.pi / 180.0, 2.0 * np.pi * freq
    Jo = 0.0
    for s in range(1, steps + 1):
        th, thd = -A * np.sin(om * s * dt), -A * om * np.cos(om * s * dt)
        x = np.cos(th) * xb0 - np.sin(th) * yb0
        y = np.sin(th) * xb0 + np.cos(th) * yb0
        oc.set_body(x, y)
        rc, o = oc.advance(body_vel=np.concatenate([-thd * y, thd * x]))
        assert rc == 0
        if s > steps - tail:
            Jo += o["fx"][0] / tail
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
