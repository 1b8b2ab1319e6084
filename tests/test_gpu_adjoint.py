"""Discrete adjoint (ibfs_adjoint_run) of the advance, checked against central
finite differences of the forward advance on random directions.

Objective as in the differentiation benchmark: J = mean lift over the last
steps; parameters: the per-point tangential surface velocities u_t of a
cylinder, body velocity v_i = u_t,i * (-sin th_i, cos th_i). The C-ABI is
wrapped as a torch.autograd.Function here, in the test harness only.
"""
import numpy as np
import pytest
import torch

import ibfs_capi as C
import oracle as O

pytestmark = pytest.mark.gpu


def make_case(m=32, lev=3, dt=0.01, re=150.0, npt=None):
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0, npt=npt)
    th = np.arctan2(yb, xb)
    return dict(m=m, lev=lev, dt=dt, re=re, xb=xb, yb=yb, tx=-np.sin(th), ty=np.cos(th))


class MeanLift(torch.autograd.Function):
    """u_t -> J (mean lift over the last `tail` of `steps` advances)."""

    @staticmethod
    def forward(ctx, ut, case, steps, tail, K, chol):
        g = C.Solver(C.make_params(case["m"], case["m"], case["dt"], case["re"], case["lev"]),
                     (case["xb"], case["yb"]))
        g.set_cholesky(*chol)
        u = ut.detach().cpu().numpy()
        vel = np.concatenate([u * case["tx"], u * case["ty"]])
        wx = np.zeros(steps)
        wy = np.zeros(steps)
        wy[steps - tail:] = 1.0 / tail
        J, gv, ms_f, ms_t = g.adjoint_run(steps, K, vel, wx, wy)
        nb = len(u)
        gu = gv[:nb] * case["tx"] + gv[nb:] * case["ty"]
        ctx.save_for_backward(torch.from_numpy(gu))
        ctx.cost = ms_t / ms_f
        g.close()
        return ut.new_tensor(J)

    @staticmethod
    def backward(ctx, gout):
        (gu,) = ctx.saved_tensors
        return gout * gu, None, None, None, None, None


def forward_J(case, u, steps, tail, chol):
    g = C.Solver(C.make_params(case["m"], case["m"], case["dt"], case["re"], case["lev"]),
                 (case["xb"], case["yb"]))
    g.set_cholesky(*chol)
    vel = np.concatenate([u * case["tx"], u * case["ty"]])
    J = 0.0
    for s in range(steps):
        o = g.advance(body_vel=vel)
        if s >= steps - tail:
            J += o["fy"][0] / tail
    g.close()
    return J


@pytest.mark.parametrize("steps,tail,K", [(12, 6, 4), (20, 8, 20)])
def test_adjoint_vs_finite_differences(steps, tail, K):
    case = make_case()
    g0 = C.Solver(C.make_params(case["m"], case["m"], case["dt"], case["re"], case["lev"]),
                  (case["xb"], case["yb"]))
    g0.precompute()
    chol = g0.get_cholesky()
    g0.close()
    nb = len(case["xb"])
    rng = np.random.default_rng(20261203)
    u0 = rng.normal(0.0, 0.1, nb)
    ut = torch.tensor(u0, dtype=torch.float64, requires_grad=True)
    J = MeanLift.apply(ut, case, steps, tail, K, chol)
    J.backward()
    grad = ut.grad.numpy()
    assert abs(J.item() - forward_J(case, u0, steps, tail, chol)) <= 1e-12 * max(1.0, abs(J.item()))
    h = 1e-6
    for d in range(8):
        dirn = rng.standard_normal(nb)
        dirn /= np.linalg.norm(dirn)
        fd = (forward_J(case, u0 + h * dirn, steps, tail, chol) - forward_J(case, u0 - h * dirn, steps, tail, chol)) / (2 * h)
        ad = grad @ dirn
        # unit direction: the derivative's scale is |grad|; FD round-off is
        # ~1e-8 |grad| at h = 1e-6
        assert abs(fd - ad) <= 1e-6 * np.linalg.norm(grad), (d, fd, ad)


def test_adjoint_vs_tangent_linear():
    """Against the FP64 tangent-linear reference (complex step through the
    independent numpy restatement)."""
    import tangent_linear as TL
    case = make_case()
    steps, tail = 10, 5
    g0 = C.Solver(C.make_params(case["m"], case["m"], case["dt"], case["re"], case["lev"]),
                  (case["xb"], case["yb"]))
    g0.precompute()
    chol = g0.get_cholesky()
    g0.close()
    nb = len(case["xb"])
    rng = np.random.default_rng(5)
    u0 = rng.normal(0.0, 0.1, nb)
    ut = torch.tensor(u0, dtype=torch.float64, requires_grad=True)
    J = MeanLift.apply(ut, case, steps, tail, steps, chol)
    J.backward()
    grad = ut.grad.numpy()
    vel = np.concatenate([u0 * case["tx"], u0 * case["ty"]])
    for d in range(3):
        du = rng.standard_normal(nb)
        du /= np.linalg.norm(du)
        dvel = np.concatenate([du * case["tx"], du * case["ty"]])
        Jr, tl = TL.mean_lift_derivative(case["m"], case["lev"], case["dt"], case["re"], case["xb"], case["yb"],
                                         vel, dvel, steps, tail)
        assert abs(Jr - J.item()) <= 1e-10 * abs(J.item())
        assert abs(tl - grad @ du) <= 1e-9 * np.linalg.norm(grad), (d, tl, grad @ du)
