"""Independent numpy restatement of the IBFS advance + golden-fixture writer.

This is a second, vectorised restatement of the reference's hot path
(src/operators.f90, src/myfft.f90, src/grid.f90, src/variables.f90 of
atchieu/ibfs-if2d), written separately from the C oracle so that the two can
check each other. The DST is scipy.fft.dstn(type=1), which has the same
definition as the FFTW RODFT00 transform the reference plans
(myfft.f90:115). The Cholesky factor uses numpy.linalg.cholesky.

Running this file writes small .npz fixtures into tests/golden/:
    python tests/golden/make_golden.py
They pin the C oracle (oracle/) and, through it, the CUDA path.
"""
import math
import os
import sys

import numpy as np
import scipy.fft as sfft

PI = 3.1415926535897932384


def nlevmax(m, n):
    """grid.f90:79 with its single-precision LOG."""
    return int(math.floor(float(np.log(np.float32(min(m, n) // 2))) / math.log(2.0))) - 1


def deltafnc(r, r0, dr):
    """grid.f90:233-249, vectorised."""
    d = np.abs(r - r0)
    t = (r - r0) / dr
    a = np.abs(t)
    out = np.zeros_like(d)
    m1 = d <= 0.5 * dr
    m2 = (~m1) & (d <= 1.5 * dr)
    out[m1] = (1.0 + np.sqrt(-3.0 * t[m1] ** 2 + 1.0)) / (3.0 * dr)
    out[m2] = (5.0 - 3.0 * a[m2] - np.sqrt(-3.0 * (1.0 - a[m2]) ** 2 + 1.0)) / (6.0 * dr)
    return out


class NpCase:
    def __init__(self, m, n, dt, re, mgridlev, xb, yb, len_=4.0, offx=2.0, offy=2.0,
                 stationary=True, cgtol=1e-7, cg_max_iter=3000, cg_rel=False):
        assert m % 4 == 0 and n % 4 == 0
        self.m, self.n, self.dt, self.re = m, n, dt, re
        self.L = min(mgridlev, nlevmax(m, n))
        self.delta = len_ / m
        self.offx, self.offy = offx, offy
        self.stationary = stationary
        self.cgtol, self.cg_max_iter, self.cg_rel = cgtol, cg_max_iter, cg_rel
        self.nb = len(xb)
        self.nf = 2 * self.nb
        self.nq = (m + 1) * n + (n + 1) * m
        self.nu = (m + 1) * n
        self.set_body(np.asarray(xb, float), np.asarray(yb, float))
        # myfft.f90:46-69
        norm = 4.0 * float(np.float32(m * n))
        self.norm = norm
        i = np.arange(1, m)[:, None]
        j = np.arange(1, n)[None, :]
        lam = -2.0 * (np.cos(PI * i / m) + np.cos(PI * j / n) - 2.0)
        self.lam = lam
        self.laminv = 1.0 / lam / norm
        del2 = self.delta ** 2
        self.lam1, self.lam1i, self.con1, self.con2, self.vfac = [], [], [], [], []
        for k in range(1, self.L + 1):
            d22 = del2 * 4.0 ** (k - 1)
            self.lam1.append((1.0 - 0.5 * dt * lam / d22 / re) / norm)
            self.lam1i.append(1.0 / (1.0 + 0.5 * dt * lam / d22 / re))
            self.vfac.append(0.5 * dt / re / d22 / norm)
            self.con1.append(1.5 * dt / d22 / norm)
            self.con2.append(-0.5 * dt / d22 / norm)
        # variables.f90:55-64
        self.omega = np.zeros((self.L, m - 1, n - 1))
        self.rhs_old = np.zeros((self.L, m - 1, n - 1))
        self.q = np.zeros((self.L, self.nq))
        self.q0 = np.zeros((self.L, self.nq))
        for k in range(self.L):
            self.q0[k, :self.nu] = self.delta * 2.0 ** k
        self.fb = np.zeros(self.nf)
        self.itime = 0
        self.chol = None

    # --- regularisation: dense Nf x Nq operator (grid.f90:142-230) ----------
    def set_body(self, xb, yb):
        m, n, d = self.m, self.n, self.delta
        self.xb, self.yb = xb.copy(), yb.copy()
        sup = 1.5 * d
        E = np.zeros((self.nf, self.nq))
        iu, ju = np.meshgrid(np.arange(1, m + 2), np.arange(1, n + 1), indexing="ij")
        xu = d * (iu - 1) - self.offx
        yu = d * (ju - 1) - self.offy + 0.5 * d
        idx_u = (iu + (ju - 1) * (m + 1) - 1)
        iv, jv = np.meshgrid(np.arange(1, m + 1), np.arange(1, n + 2), indexing="ij")
        xv = d * (iv - 1) - self.offx + 0.5 * d
        yv = d * (jv - 1) - self.offy
        idx_v = ((m + 1) * n + iv + (jv - 1) * m - 1)
        for k in range(self.nb):
            mk = (np.abs(xu - xb[k]) < sup) & (np.abs(yu - yb[k]) < sup)
            w = d * d * deltafnc(xu[mk], xb[k], d) * deltafnc(yu[mk], yb[k], d)
            E[k, idx_u[mk]] = w
            mk = (np.abs(xv - xb[k]) < sup) & (np.abs(yv - yb[k]) < sup)
            w = d * d * deltafnc(xv[mk], xb[k], d) * deltafnc(yv[mk], yb[k], d)
            E[self.nb + k, idx_v[mk]] = w
        self.E = E

    def reg(self, f):
        return self.E.T @ f

    def regT(self, h):
        return self.E @ h

    # --- spectral (myfft.f90:83-124) ----------------------------------------
    @staticmethod
    def dst(x):
        return sfft.dstn(x, type=1)

    def ctci(self, x):
        return self.dst(self.laminv * self.dst(x))

    def ainv(self, x):
        return self.dst(self.lam1i[0] * self.dst(x) / self.norm)

    # --- faces as blocks ------------------------------------------------------
    def split(self, qv):
        m, n = self.m, self.n
        U = qv[:self.nu].reshape((m + 1, n), order="F")
        V = qv[self.nu:].reshape((m, n + 1), order="F")
        return U, V

    def join(self, U, V):
        return np.concatenate([U.ravel(order="F"), V.ravel(order="F")])

    # ring: left(n+1) right(n+1) bottom(m+1) top(m+1)
    def ring(self, bc):
        m, n = self.m, self.n
        return bc[0:n + 1], bc[n + 1:2 * n + 2], bc[2 * n + 2:2 * n + m + 3], bc[2 * n + m + 3:]

    def curl(self, x, bc):
        """operators.f90:243-288."""
        m, n = self.m, self.n
        left, right, bot, top = self.ring(bc)
        U = np.zeros((m + 1, n))
        V = np.zeros((m, n + 1))
        xe = np.zeros((m - 1, n + 1))
        xe[:, 0] = bot[1:m]
        xe[:, 1:n] = x
        xe[:, n] = top[1:m]
        U[1:m, :] = xe[:, 1:] - xe[:, :-1]
        U[0, :] = left[1:] - left[:-1]
        U[m, :] = right[1:] - right[:-1]
        xe2 = np.zeros((m + 1, n - 1))
        xe2[0, :] = left[1:n]
        xe2[1:m, :] = x
        xe2[m, :] = right[1:n]
        V[:, 1:n] = xe2[:-1, :] - xe2[1:, :]
        V[:, 0] = bot[:-1] - bot[1:]
        V[:, n] = top[:-1] - top[1:]
        return self.join(U, V)

    def rot(self, qv):
        """operators.f90:291-304."""
        U, V = self.split(qv)
        n = self.n
        return V[1:, 1:n] - V[:-1, 1:n] - U[1:-1, 1:] + U[1:-1, :-1]

    def nonlinear(self, om, qv, q0v, bc):
        """operators.f90:465-510."""
        m, n = self.m, self.n
        left, right, bot, top = self.ring(bc)
        U, V = self.split(qv)
        U0, V0 = self.split(q0v)
        uavg = 0.5 * (U[:, 1:] + U[:, :-1] + U0[:, 1:] + U0[:, :-1])      # (m+1, n-1), j=2..n
        vavg = 0.5 * (V[1:, :] + V[:-1, :] + V0[1:, :] + V0[:-1, :])      # (m-1, n+1), i=2..m
        FU = np.zeros((m + 1, n))
        FV = np.zeros((m, n + 1))
        oe = np.zeros((m - 1, n + 1))
        oe[:, 0] = bot[1:m]
        oe[:, 1:n] = om
        oe[:, n] = top[1:m]
        FU[1:m, :] = 0.5 * (vavg[:, 1:] * oe[:, 1:] + vavg[:, :-1] * oe[:, :-1])
        oe2 = np.zeros((m + 1, n - 1))
        oe2[0, :] = left[1:n]
        oe2[1:m, :] = om
        oe2[m, :] = right[1:n]
        FV[:, 1:n] = -0.5 * (uavg[1:, :] * oe2[1:, :] + uavg[:-1, :] * oe2[:-1, :])
        return self.join(FU, FV)

    def coarsify(self, crhs, rhs):
        """operators.f90:307-333 (numpy 0-based: node i -> i-2)."""
        m, n = self.m, self.n
        out = crhs.copy()
        I = np.arange(m // 4 + 2, 3 * m // 4 + 1)
        J = np.arange(n // 4 + 2, 3 * n // 4 + 1)
        ii = 2 * I - m // 2 - 1 - 2
        jj = 2 * J - n // 2 - 1 - 2
        a = lambda di, dj: rhs[np.ix_(ii + di, jj + dj)]
        out[np.ix_(I - 2, J - 2)] = (a(0, 0) + 0.5 * (a(-1, 0) + a(1, 0) + a(0, -1) + a(0, 1))
                                     + 0.25 * (a(-1, -1) + a(-1, 1) + a(1, -1) + a(1, 1)))
        return out

    def get_bc(self, r, fac):
        """operators.f90:336-367; r(a,b) 1-based -> r[a-1, b-1]."""
        m, n = self.m, self.n
        R = lambda a, b: r[a - 1, b - 1]
        bot = np.zeros(m + 1)
        top = np.zeros(m + 1)
        left = np.zeros(n + 1)
        right = np.zeros(n + 1)
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

    def apply_bc(self, r, bc, fac):
        """operators.f90:370-390."""
        m, n = self.m, self.n
        left, right, bot, top = self.ring(bc)
        r = r.copy()
        r[:, 0] += fac * bot[1:m]
        r[:, n - 2] += fac * top[1:m]
        r[0, :] += fac * left[1:n]
        r[m - 2, :] += fac * right[1:n]
        return r

    def vort2flux(self, omega, nlev):
        """operators.f90:191-240 (omega modified in place)."""
        L = self.L
        vel = np.zeros((nlev, self.nq))
        for k in range(1, L):
            omega[k] = self.coarsify(omega[k], omega[k - 1])
        sbc = np.zeros(2 * (self.m + 1) + 2 * (self.n + 1))
        s = self.ctci(omega[L - 1])
        if nlev >= L:
            vel[L - 1] = self.curl(s, sbc)
        for k in range(L - 2, -1, -1):
            sbc = self.get_bc(s, 1.0)
            s = self.ctci(self.apply_bc(omega[k], sbc, 1.0))
            if nlev >= k + 1:
                vel[k] = self.curl(s, sbc)
        return vel

    def a_times(self, x):
        """operators.f90:444-462."""
        vort = np.zeros_like(self.omega)
        vort[0] = self.ainv(self.rot(self.reg(x)))
        vel = self.vort2flux(vort, 1)
        return self.regT(vel[0])

    def preprocess(self):
        A = np.stack([self.a_times(e) for e in np.eye(self.nf)], axis=1)
        self.A = A
        # choldc reads only the upper triangle cholmat(i,j), j >= i
        # (operators.f90:778-779); A itself is not exactly symmetric.
        U = np.triu(A)
        self.chol = np.linalg.cholesky(U + np.triu(A, 1).T)

    def cholsl(self, b):
        import scipy.linalg as sl
        y = sl.solve_triangular(self.chol, b, lower=True)
        return sl.solve_triangular(self.chol.T, y, lower=False)

    def cjgr(self, x, b):
        """operators.f90:393-441 (with optional relative stop)."""
        r = b - self.a_times(x)
        d = r.copy()
        dn = r @ d
        eps = self.cgtol ** 2 * ((b @ b) if self.cg_rel else 1.0)
        it = 0
        while it < self.cg_max_iter and dn > eps:
            it += 1
            qv = self.a_times(d)
            alpha = dn / (d @ qv)
            x = x + alpha * d
            r = b - self.a_times(x) if it % 50 == 0 else r - alpha * qv
            do, dn = dn, r @ r
            d = r + (dn / do) * d
        return x, it

    def advance(self, body_vel=None, new_xb=None, new_yb=None):
        """operators.f90:62-188; returns fx, fy (single body), circ, slip."""
        self.itime += 1
        L = self.L
        if self.itime == 1 and self.stationary:
            self.preprocess()
        lastbc = [self.get_bc(self.omega[k + 1], 0.25) for k in range(L - 1)]
        lastbc.append(np.zeros(2 * (self.m + 1) + 2 * (self.n + 1)))
        for k in range(L - 1, -1, -1):
            obc = self.get_bc(self.omega[k + 1], 0.25) if k < L - 1 else np.zeros_like(lastbc[-1])
            rhs = self.rot(self.nonlinear(self.omega[k], self.q[k], self.q0[k], lastbc[k]))
            if self.itime == 1:
                self.rhs_old[k] = rhs
            rb = self.apply_bc(np.zeros_like(rhs), lastbc[k], self.vfac[k])
            rb = self.apply_bc(rb, obc, self.vfac[k])
            t1 = self.dst(self.con1[k] * rhs + self.con2[k] * self.rhs_old[k] + rb)
            self.omega[k] = self.dst(self.lam1i[k] * (t1 + self.lam1[k] * self.dst(self.omega[k])))
            self.rhs_old[k] = rhs
        if new_xb is not None:
            self.set_body(new_xb, new_yb)
        motion = np.zeros(self.nf) if body_vel is None else np.asarray(body_vel) * self.delta
        motion = motion - self.regT(self.q0[0])
        vel1 = self.vort2flux(self.omega, 1)
        rhsf = self.regT(vel1[0]) - motion
        iters = 0
        if self.stationary:
            self.fb = self.cholsl(rhsf)
        else:
            self.fb, iters = self.cjgr(self.fb, rhsf)
        self.omega[0] = self.omega[0] - self.ainv(self.rot(self.reg(self.fb)))
        self.q = self.vort2flux(self.omega, L)
        h = self.reg(self.fb / self.dt)
        fx = h[:self.nu].sum() * 2.0 * self.delta
        fy = h[self.nu:].sum() * 2.0 * self.delta
        circ = self.omega.sum(axis=(1, 2))
        slip = np.abs(self.regT(self.q[0]) - motion).max()
        return dict(fx=fx, fy=fy, circ=circ, slip=slip, cg_iters=iters)

    def state_flat(self):
        """Fortran-order state vectors, as in the .var record (variables.f90:152)."""
        om = np.concatenate([w.ravel(order="F") for w in self.omega])
        ro = np.concatenate([w.ravel(order="F") for w in self.rhs_old])
        return dict(omega=om, rhs_old=ro, q=self.q.ravel(), q0=self.q0.ravel(), fb=self.fb.copy())


# ----------------------------------------------------------------------------
CASES = {
    # name: (m, n, dt, re, mgridlev, body, stationary, steps)
    "cyl_m32_L3": dict(m=32, n=32, dt=0.01, re=100.0, lev=3, body="cyl", stationary=True, steps=6),
    "plate_m32x24_L2": dict(m=32, n=24, dt=0.01, re=300.0, lev=3, body="plate", stationary=True, steps=6),
    "cyl_m32_L3_cg": dict(m=32, n=32, dt=0.01, re=100.0, lev=3, body="cyl", stationary=False, steps=4),
}


def body_points(kind, m, len_=4.0):
    ds = len_ / m
    if kind == "cyl":
        npt = int(PI * 1.0 / ds)
        i = np.arange(npt, dtype=float)
        return 0.5 * np.cos(2.0 * PI * i / npt), 0.5 * np.sin(2.0 * PI * i / npt)
    angle = -30.0 * PI / 180.0
    npt = int(1.0 / ds)
    seg = np.arange(npt + 1, dtype=float) * 1.0 / npt
    return -0.5 * math.cos(angle) + seg * math.cos(angle), -0.5 * math.sin(angle) + seg * math.sin(angle)


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    rng = np.random.default_rng(20261203)
    # DST-I known answers (scipy dst type 1 == FFTW RODFT00)
    dst_fix = {}
    for (m, n) in [(16, 16), (32, 24), (200, 200)]:
        x = rng.standard_normal((m - 1, n - 1))
        dst_fix[f"x_{m}_{n}"] = x.ravel(order="F")
        dst_fix[f"y_{m}_{n}"] = sfft.dstn(x, type=1).ravel(order="F")
    np.savez_compressed(os.path.join(here, "dst_rodft00.npz"), **dst_fix)
    for name, cfg in CASES.items():
        xb, yb = body_points(cfg["body"], cfg["m"])
        c = NpCase(cfg["m"], cfg["n"], cfg["dt"], cfg["re"], cfg["lev"], xb, yb,
                   stationary=cfg["stationary"], cg_rel=True, cgtol=1e-13)
        out = {"xb": xb, "yb": yb, "params": np.array([cfg["m"], cfg["n"], cfg["dt"], cfg["re"],
                                                        cfg["lev"], float(cfg["stationary"])])}
        for s in range(cfg["steps"]):
            r = c.advance()
            for key in ("fx", "fy", "slip"):
                out.setdefault(key, []).append(r[key])
            out.setdefault("circ", []).append(r["circ"])
        st = c.state_flat()
        for key, v in st.items():
            out["final_" + key] = v
        np.savez_compressed(os.path.join(here, f"{name}.npz"), **{k: np.asarray(v) for k, v in out.items()})
        print(name, "fx", out["fx"][-1], "nlev", c.L)


if __name__ == "__main__":
    sys.exit(main())
