"""FP64 tangent-linear reference of the IBFS advance by complex-step
differentiation of the independent numpy restatement (make_golden.NpCase).

J(p + i h d) with h = 1e-30 gives dJ/dp . d = Im(J)/h to machine precision:
every operation on the path from the body velocities to the forces is
analytic (sums, products, the DST, the triangular solves of a Cholesky factor
that depends on the geometry only), so no subtraction error arises.

TEST INFRASTRUCTURE ONLY (checker of the GPU discrete adjoint).
"""
import numpy as np

import make_golden as G


class CplxCase(G.NpCase):
    """NpCase whose state may be complex (allocations follow the input dtype)."""

    def curl(self, x, bc):
        m, n = self.m, self.n
        dt = np.result_type(x, bc)
        left, right, bot, top = self.ring(bc)
        U = np.zeros((m + 1, n), dt)
        V = np.zeros((m, n + 1), dt)
        xe = np.zeros((m - 1, n + 1), dt)
        xe[:, 0] = bot[1:m]
        xe[:, 1:n] = x
        xe[:, n] = top[1:m]
        U[1:m, :] = xe[:, 1:] - xe[:, :-1]
        U[0, :] = left[1:] - left[:-1]
        U[m, :] = right[1:] - right[:-1]
        xe2 = np.zeros((m + 1, n - 1), dt)
        xe2[0, :] = left[1:n]
        xe2[1:m, :] = x
        xe2[m, :] = right[1:n]
        V[:, 1:n] = xe2[:-1, :] - xe2[1:, :]
        V[:, 0] = bot[:-1] - bot[1:]
        V[:, n] = top[:-1] - top[1:]
        return self.join(U, V)

    def nonlinear(self, om, qv, q0v, bc):
        m, n = self.m, self.n
        dt = np.result_type(om, qv, bc)
        left, right, bot, top = self.ring(bc)
        U, V = self.split(qv)
        U0, V0 = self.split(q0v)
        uavg = 0.5 * (U[:, 1:] + U[:, :-1] + U0[:, 1:] + U0[:, :-1])
        vavg = 0.5 * (V[1:, :] + V[:-1, :] + V0[1:, :] + V0[:-1, :])
        FU = np.zeros((m + 1, n), dt)
        FV = np.zeros((m, n + 1), dt)
        oe = np.zeros((m - 1, n + 1), dt)
        oe[:, 0] = bot[1:m]
        oe[:, 1:n] = om
        oe[:, n] = top[1:m]
        FU[1:m, :] = 0.5 * (vavg[:, 1:] * oe[:, 1:] + vavg[:, :-1] * oe[:, :-1])
        oe2 = np.zeros((m + 1, n - 1), dt)
        oe2[0, :] = left[1:n]
        oe2[1:m, :] = om
        oe2[m, :] = right[1:n]
        FV[:, 1:n] = -0.5 * (uavg[1:, :] * oe2[1:, :] + uavg[:-1, :] * oe2[:-1, :])
        return self.join(FU, FV)

    def get_bc(self, r, fac):
        m, n = self.m, self.n
        R = lambda a, b: r[a - 1, b - 1]
        dt = r.dtype
        bot, top = np.zeros(m + 1, dt), np.zeros(m + 1, dt)
        left, right = np.zeros(n + 1, dt), np.zeros(n + 1, dt)
        ie = np.arange(0, m + 1, 2)
        bot[ie] = R(m // 4 + ie // 2, n // 4)
        top[ie] = R(m // 4 + ie // 2, 3 * n // 4)
        io = np.arange(1, m, 2)
        bot[io] = 0.5 * (R(m // 4 + (io + 1) // 2, n // 4) + R(m // 4 - 1 + (io + 1) // 2, n // 4))
        top[io] = 0.5 * (R(m // 4 + (io + 1) // 2, 3 * n // 4) + R(m // 4 - 1 + (io + 1) // 2, 3 * n // 4))
        je = np.arange(0, n + 1, 2)
        left[je] = R(m // 4, n // 4 + je // 2)
        right[je] = R(3 * m // 4, n // 4 + je // 2)
        jo = np.arange(1, n, 2)
        left[jo] = 0.5 * (R(m // 4, n // 4 + (jo + 1) // 2) + R(m // 4, n // 4 - 1 + (jo + 1) // 2))
        right[jo] = 0.5 * (R(3 * m // 4, n // 4 + (jo + 1) // 2) + R(3 * m // 4, n // 4 - 1 + (jo + 1) // 2))
        return np.concatenate([left, right, bot, top]) * fac

    def vort2flux(self, omega, nlev):
        L = self.L
        vel = np.zeros((nlev, self.nq), omega.dtype)
        for k in range(1, L):
            omega[k] = self.coarsify(omega[k], omega[k - 1])
        sbc = np.zeros(2 * (self.m + 1) + 2 * (self.n + 1), omega.dtype)
        s = self.ctci(omega[L - 1])
        if nlev >= L:
            vel[L - 1] = self.curl(s, sbc)
        for k in range(L - 2, -1, -1):
            sbc = self.get_bc(s, 1.0)
            s = self.ctci(self.apply_bc(omega[k], sbc, 1.0))
            if nlev >= k + 1:
                vel[k] = self.curl(s, sbc)
        return vel

    def make_complex(self):
        self.omega = self.omega.astype(complex)
        self.rhs_old = self.rhs_old.astype(complex)
        self.q = self.q.astype(complex)
        self.fb = self.fb.astype(complex)

    def cholsl(self, b):
        import scipy.linalg as sl
        y = sl.solve_triangular(self.chol, b, lower=True)
        return sl.solve_triangular(self.chol.T, y, lower=False)

    def advance(self, body_vel=None, new_xb=None, new_yb=None):
        if self.itime == 0 and self.chol is None:
            self.preprocess()
            self.make_complex()
        self.itime += 1
        L = self.L
        cz = np.zeros(2 * (self.m + 1) + 2 * (self.n + 1), complex)
        lastbc = [self.get_bc(self.omega[k + 1], 0.25) for k in range(L - 1)] + [cz]
        for k in range(L - 1, -1, -1):
            obc = self.get_bc(self.omega[k + 1], 0.25) if k < L - 1 else cz
            rhs = self.rot(self.nonlinear(self.omega[k], self.q[k], self.q0[k], lastbc[k]))
            if self.itime == 1:
                self.rhs_old[k] = rhs
            rb = self.apply_bc(np.zeros_like(rhs), lastbc[k], self.vfac[k])
            rb = self.apply_bc(rb, obc, self.vfac[k])
            t1 = self.dst(self.con1[k] * rhs + self.con2[k] * self.rhs_old[k] + rb)
            self.omega[k] = self.dst(self.lam1i[k] * (t1 + self.lam1[k] * self.dst(self.omega[k])))
            self.rhs_old[k] = rhs
        motion = np.asarray(body_vel) * self.delta - self.regT(self.q0[0])
        vel1 = self.vort2flux(self.omega, 1)
        rhsf = self.regT(vel1[0]) - motion
        self.fb = self.cholsl(rhsf)
        self.omega[0] = self.omega[0] - self.ainv(self.rot(self.reg(self.fb)))
        self.q = self.vort2flux(self.omega, L)
        h = self.reg(self.fb / self.dt)
        return dict(fx=h[:self.nu].sum() * 2.0 * self.delta, fy=h[self.nu:].sum() * 2.0 * self.delta)


def mean_lift_derivative(m, lev, dt, re, xb, yb, vel, dvel, steps, tail, h=1e-30):
    """d/de J(vel + e dvel) at e=0, J = mean lift over the last `tail` steps."""
    c = CplxCase(m, m, dt, re, lev, xb, yb)
    v = np.asarray(vel, complex) + 1j * h * np.asarray(dvel)
    J = 0.0
    for s in range(steps):
        o = c.advance(body_vel=v)
        if s >= steps - tail:
            J = J + o["fy"] / tail
    return J.real, J.imag / h


def deltafnc_c(r, r0, dr):
    """grid.f90:233-249 continued analytically to complex positions: the branch
    is chosen by the real part and |t| becomes sgn(Re t) t, so the complex
    step carries the derivative of the kernel (C1 at both joins)."""
    t = (r - r0) / dr
    d = np.abs(t.real)
    a = np.where(t.real >= 0.0, t, -t)
    out = np.zeros(np.shape(t), complex)
    m1 = d <= 0.5
    m2 = (~m1) & (d <= 1.5)
    out[m1] = (1.0 + np.sqrt(-3.0 * t[m1] ** 2 + 1.0)) / (3.0 * dr)
    out[m2] = (5.0 - 3.0 * a[m2] - np.sqrt(-3.0 * (1.0 - a[m2]) ** 2 + 1.0)) / (6.0 * dr)
    return out


class PitchCplxCase(CplxCase):
    """Moving body with complex positions: the regularisation is rebuilt from
    them every step (setup_reg, grid.f90:142-230, box test on the real part)
    and the force system is solved exactly (dense A from a_times columns),
    the limit of the CG solve (cjgr) the GPU runs to a relative 1e-12."""

    def set_body(self, xb, yb):
        m, n, d = self.m, self.n, self.delta
        xb = np.asarray(xb, complex)
        yb = np.asarray(yb, complex)
        self.xb, self.yb = xb.copy(), yb.copy()
        sup = 1.5 * d
        E = np.zeros((self.nf, self.nq), complex)
        iu, ju = np.meshgrid(np.arange(1, m + 2), np.arange(1, n + 1), indexing="ij")
        xu = d * (iu - 1) - self.offx
        yu = d * (ju - 1) - self.offy + 0.5 * d
        idx_u = (iu + (ju - 1) * (m + 1) - 1)
        iv, jv = np.meshgrid(np.arange(1, m + 1), np.arange(1, n + 2), indexing="ij")
        xv = d * (iv - 1) - self.offx + 0.5 * d
        yv = d * (jv - 1) - self.offy
        idx_v = ((m + 1) * n + iv + (jv - 1) * m - 1)
        for k in range(self.nb):
            mk = (np.abs(xu - xb[k].real) < sup) & (np.abs(yu - yb[k].real) < sup)
            E[k, idx_u[mk]] = d * d * deltafnc_c(xu[mk], xb[k], d) * deltafnc_c(yu[mk], yb[k], d)
            mk = (np.abs(xv - xb[k].real) < sup) & (np.abs(yv - yb[k].real) < sup)
            E[self.nb + k, idx_v[mk]] = d * d * deltafnc_c(xv[mk], xb[k], d) * deltafnc_c(yv[mk], yb[k], d)
        self.E = E

    def step(self, xb, yb, vel):
        """One advance with the body at (xb, yb) moving at vel (operators.f90:62-188)."""
        if self.itime == 0:
            self.make_complex()
        self.itime += 1
        L = self.L
        cz = np.zeros(2 * (self.m + 1) + 2 * (self.n + 1), complex)
        lastbc = [self.get_bc(self.omega[k + 1], 0.25) for k in range(L - 1)] + [cz]
        for k in range(L - 1, -1, -1):
            obc = self.get_bc(self.omega[k + 1], 0.25) if k < L - 1 else cz
            rhs = self.rot(self.nonlinear(self.omega[k], self.q[k], self.q0[k], lastbc[k]))
            if self.itime == 1:
                self.rhs_old[k] = rhs
            rb = self.apply_bc(np.zeros_like(rhs), lastbc[k], self.vfac[k])
            rb = self.apply_bc(rb, obc, self.vfac[k])
            t1 = self.dst(self.con1[k] * rhs + self.con2[k] * self.rhs_old[k] + rb)
            self.omega[k] = self.dst(self.lam1i[k] * (t1 + self.lam1[k] * self.dst(self.omega[k])))
            self.rhs_old[k] = rhs
        self.set_body(xb, yb)
        motion = np.asarray(vel) * self.delta - self.regT(self.q0[0])
        vel1 = self.vort2flux(self.omega, 1)
        rhsf = self.regT(vel1[0]) - motion
        A = np.stack([self.a_times(e) for e in np.eye(self.nf)], axis=1)
        self.fb = np.linalg.solve(A, rhsf)
        self.omega[0] = self.omega[0] - self.ainv(self.rot(self.reg(self.fb)))
        self.q = self.vort2flux(self.omega, L)
        h = self.reg(self.fb / self.dt)
        return dict(fx=h[:self.nu].sum() * 2.0 * self.delta, fy=h[self.nu:].sum() * 2.0 * self.delta)


def mean_drag_amplitude_derivative(m, lev, dt, re, xb0, yb0, amp_deg, freq, steps, tail, h=1e-30,
                                   px=0.0, py=0.0):
    """J = mean drag over the last `tail` of `steps` advances of a plate pitching
    as alpha(t) = A sin(2 pi freq t) about (px, py) (the body turned by -alpha),
    and dJ/dA per degree, by complex step in A."""
    c = PitchCplxCase(m, m, dt, re, lev, xb0, yb0, stationary=False)
    A = (amp_deg + 1j * h) * np.pi / 180.0
    om = 2.0 * np.pi * freq
    J = 0.0
    for s in range(1, steps + 1):
        t = s * dt
        th = -A * np.sin(om * t)
        thd = -A * om * np.cos(om * t)
        cs, sn = np.cos(th), np.sin(th)
        rx, ry = np.asarray(xb0) - px, np.asarray(yb0) - py
        x = px + cs * rx - sn * ry
        y = py + sn * rx + cs * ry
        vel = np.concatenate([-thd * (y - py), thd * (x - px)])
        o = c.step(x, y, vel)
        if s > steps - tail:
            J = J + o["fx"] / tail
    return J.real, J.imag / h
