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
