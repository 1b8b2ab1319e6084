"""The discrete adjoints at the differentiation benchmarks' grid sizes.

* Rotating cylinder (D=1, Re 150, 256x256 cells, 4 levels, 126 points, dt
  0.004): gradient of the mean lift over the last third of 100 steps with
  respect to the 126 tangential surface velocities (seeded N(0, 0.1^2)), with a
  checkpoint every 50 steps, against central finite differences (h = 1e-6) on 8
  seeded random unit directions.
* Pitching plate on the moving-body grid (chord 1 about mid-chord, Re 500,
  512x512 cells, 5 levels, dt 0.001, CG to a relative 1e-12, preconditioned),
  started at the phase of maximum pitch: derivative of the mean drag over the
  last 3 of 6 steps with respect to the pitch amplitude against fourth-order
  central differences.
"""
import numpy as np
import pytest

import ibfs_capi as C
import workloads as W

pytestmark = pytest.mark.gpu

M, LEV, DT, RE, NPT = 256, 4, 0.004, 150.0, 126
STEPS, TAIL, K = 100, 33, 50


def _cylinder():
    xb, yb = W.circle(4.0 / M, 1.0, 0.0, 0.0, npt=NPT)
    th = np.arctan2(yb, xb)
    return xb, yb, -np.sin(th), np.cos(th)


def _forward_J(xb, yb, vel, chol):
    g = C.Solver(C.make_params(M, M, DT, RE, LEV), (xb, yb))
    g.set_cholesky(*chol)
    first = g.advance(body_vel=vel)  # the velocities stay in force for advance_n
    hist = g.advance_n(STEPS - 1)
    fy = np.array([first["fy"][0]] + [g.outputs_of(hist[s], 0)["fy"][0] for s in range(STEPS - 1)])
    g.close()
    return float(fy[STEPS - TAIL:].mean())


def test_rotating_cylinder_gradient_vs_finite_differences():
    xb, yb, tx, ty = _cylinder()
    g0 = C.Solver(C.make_params(M, M, DT, RE, LEV), (xb, yb))
    g0.precompute()
    chol = g0.get_cholesky()
    g0.close()
    rng = np.random.default_rng(20261203)
    u0 = rng.normal(0.0, 0.1, NPT)
    vel = np.concatenate([u0 * tx, u0 * ty])
    g = C.Solver(C.make_params(M, M, DT, RE, LEV), (xb, yb))
    g.set_cholesky(*chol)
    wy = np.zeros(STEPS)
    wy[STEPS - TAIL:] = 1.0 / TAIL
    J, gv, ms_f, ms_t = g.adjoint_run(STEPS, K, vel, np.zeros(STEPS), wy)
    g.close()
    grad = gv[:NPT] * tx + gv[NPT:] * ty
    assert abs(J - _forward_J(xb, yb, vel, chol)) <= 1e-12 * max(1.0, abs(J))
    h = 1e-6
    errs = []
    for d in range(8):
        dirn = rng.standard_normal(NPT)
        dirn /= np.linalg.norm(dirn)
        up, um = u0 + h * dirn, u0 - h * dirn
        fd = (_forward_J(xb, yb, np.concatenate([up * tx, up * ty]), chol) -
              _forward_J(xb, yb, np.concatenate([um * tx, um * ty]), chol)) / (2 * h)
        ad = grad @ dirn
        errs.append(abs(fd - ad) / np.linalg.norm(grad))
        assert abs(fd - ad) <= 1e-6 * np.linalg.norm(grad), (d, fd, ad)
    print(f"rotating cylinder 256x256x4, {STEPS} steps, K={K}: |grad| {np.linalg.norm(grad):.4e}, "
          f"max |fd - ad| / |grad| {max(errs):.2e}, adjoint cost {ms_t / ms_f:.2f}x its forward pass")


MAX_PITCH_STEP = 1000  # t = 1 s at dt 0.001, f 0.25: alpha = amplitude
PSTEPS, PTAIL = 6, 3


def _pitch(amp):
    c = W.pitching(amp_deg=amp)
    p, b, o = W.solver_args([c], C)
    p[0].istart = MAX_PITCH_STEP
    return C.Solver(p[0], b[0], o[0])


def _pitch_J(amp):
    s = _pitch(amp)
    h = s.advance_n(PSTEPS)
    fx = [s.outputs_of(h[k], 0)["fx"][0] for k in range(PSTEPS)]
    s.close()
    return float(np.mean(fx[PSTEPS - PTAIL:]))


def test_pitch_adjoint_on_the_moving_body_grid():
    amp = 20.0
    s = _pitch(amp)
    wx = np.zeros(PSTEPS)
    wx[PSTEPS - PTAIL:] = 1.0 / PTAIL
    J, g, ms_f, ms_t = s.adjoint_pitch_run(PSTEPS, 3, wx, np.zeros(PSTEPS))
    s.close()
    assert abs(J - _pitch_J(amp)) <= 1e-12 * abs(J)
    # The body points' regularisation weights are C1 in the point positions
    # (Roma-Peskin-Berger kernel, grid.f90:233-249), so J(A) bends sharply
    # wherever a point's support crosses a face; on this grid (dx = 0.0078) a
    # 0.02 degree step moves the points by ~0.02 dx and the fourth-order
    # difference is off by ~6e-4. Steps of 0.002 and 0.001 degrees (J is
    # repeatable to 1e-15 at CG's relative 1e-12) resolve the derivative.
    fds = {}
    for h in (0.002, 0.001):
        Jp1, Jm1, Jp2, Jm2 = (_pitch_J(amp + d) for d in (h, -h, 2 * h, -2 * h))
        fds[h] = (8.0 * (Jp1 - Jm1) - (Jp2 - Jm2)) / (12.0 * h)
    print(f"pitching plate 512x512x5: dJ/dA adjoint {g:.10e}, fourth-order FD {fds}")
    for h, fd in fds.items():
        assert abs(g - fd) <= 1e-6 * abs(fd), (h, g, fd)
