"""ctypes wrapper of the CPU FP64 oracle (oracle/ibfs_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline legs, where it is the checker / the timed CPU
restatement -- never by the product path. Parity of this oracle with the
reference Fortran+FFTW binary is unpinned (that binary cannot be built here);
its DST is pinned to scipy.fft.dst(type=1) and its advance is cross-checked
against an independent numpy restatement (tests/golden/make_golden.py).

Also holds the body-geometry primitives of the reference (grid.f90:431-520)
used to make test inputs.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libibfs_oracle.so")
_lib = None


class Params(ctypes.Structure):
    """Namelist READ_PARAMETERS (parameters.f90:48-50)."""
    _fields_ = [
        ("istart", ctypes.c_int), ("istop", ctypes.c_int), ("isave", ctypes.c_int),
        ("m", ctypes.c_int), ("n", ctypes.c_int),
        ("dt", ctypes.c_double), ("re", ctypes.c_double), ("cgtol", ctypes.c_double),
        ("cg_max_iter", ctypes.c_int), ("unif_flow", ctypes.c_int),
        ("len", ctypes.c_double), ("offsetx", ctypes.c_double), ("offsety", ctypes.c_double),
        ("mgridlev", ctypes.c_int), ("make_vortex", ctypes.c_int), ("stationary", ctypes.c_int),
    ]


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        P = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.or_create.argtypes = [ctypes.POINTER(Params), ctypes.c_int, P, P,
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(vp)]
        L.or_destroy.argtypes = [vp]
        L.or_sizes.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 6 + [P]
        L.or_get_state.argtypes = [vp, P, P, P, P, P]
        L.or_set_state.argtypes = [vp, P, P, P, P, P]
        L.or_get_cholesky.argtypes = [vp, P, P]
        L.or_set_cholesky.argtypes = [vp, P, P]
        L.or_set_body.argtypes = [vp, P, P]
        L.or_preprocess.argtypes = [vp]
        L.or_advance.argtypes = [vp, ctypes.POINTER(ctypes.c_int), P, P, P, P, P,
                                 ctypes.POINTER(ctypes.c_int)]
        L.or_set_cg_relative.argtypes = [vp, ctypes.c_int]
        for name in ("or_dst", "or_ctci", "or_ainv", "or_rot", "or_regT", "or_reg",
                     "or_a_times", "or_cholsl"):
            getattr(L, name).argtypes = [vp, P, P]
        L.or_curl.argtypes = [vp, P, P, P]
        L.or_nonlinear.argtypes = [vp, P, P, P, P, P]
        L.or_coarsify.argtypes = [vp, P, P, P]
        L.or_get_bc.argtypes = [vp, P, P, ctypes.c_double]
        L.or_apply_bc.argtypes = [vp, P, P, ctypes.c_double]
        L.or_vort2flux.argtypes = [vp, P, P, ctypes.c_int]
        L.or_tables.argtypes = [vp, P, P, P, P, P, P, P]
        L.or_deltafnc.argtypes = [ctypes.c_double] * 3
        L.or_deltafnc.restype = ctypes.c_double
        L.or_nlevmax.argtypes = [ctypes.c_int, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(m, n, dt, re, mgridlev, len_=4.0, offsetx=2.0, offsety=2.0,
                stationary=True, unif_flow=True, cgtol=1e-7, cg_max_iter=3000,
                istart=0, istop=400, isave=25):
    return Params(istart, istop, isave, m, n, dt, re, cgtol, cg_max_iter,
                  int(unif_flow), len_, offsetx, offsety, mgridlev, 0, int(stationary))


# --- body geometry primitives (grid.f90:431-520) -----------------------------
PI = 3.1415926535897932384


def circle(ds, dia, x, y, npt=None):
    """grid.f90:496-520; npt defaults to INT(pi*dia/ds)."""
    if npt is None:
        npt = int(PI * dia / ds)
    i = np.arange(npt, dtype=np.float64)
    xb = x + 0.5 * dia * np.cos(2.0 * PI * i / float(npt))
    yb = y + 0.5 * dia * np.sin(2.0 * PI * i / float(npt))
    return xb, yb


def line(ds, length, aoa, x=0.0, y=0.0, npt=None):
    """grid.f90:431-462 (end points included; aoa in degrees, nose-up for
    positive aoa since angle = -aoa)."""
    angle = -aoa * PI / 180.0
    x_le = -0.5 * length * math.cos(angle)
    y_le = -0.5 * length * math.sin(angle)
    if npt is None:
        npt = int(length / ds)
    seg = np.arange(npt + 1, dtype=np.float64) * length / float(npt)
    xb = x_le + seg * math.cos(angle) + 0.0 * x
    yb = y_le + seg * math.sin(angle) + 0.0 * y
    return xb, yb


def actuator_slot(x, y, hs, ds, angle, num):
    """grid.f90:636-680: the points of one actuator slot of width hs centred at
    (x, y) across the jet direction angle (degrees): INT(hs/ds)+1 points at
    spacing hs/INT(hs/ds), or the single point (x, y) when INT(hs/ds) = 0;
    body number num (negative). Returns xb, yb, bodyno."""
    npt = int(hs / ds)
    if npt == 0:
        return np.array([x]), np.array([y]), np.array([num], dtype=np.int32)
    a = PI * (angle + 90.0) / 180.0
    seg = np.arange(npt + 1, dtype=np.float64) * hs / float(npt)
    xb = x - hs / 2.0 * math.cos(a) + seg * math.cos(a)
    yb = y - hs / 2.0 * math.sin(a) + seg * math.sin(a)
    return xb, yb, np.full(npt + 1, num, dtype=np.int32)


def jet_velocities(vel, actuators, itime, dt):
    """actuation (grid.f90:579-605) with u_jet (:608-633): the last points of the
    body-velocity vector vel (x components, then y), npt per actuator in
    order, get (u_j + u_j_osc sin(omg_j dt itime)) (cos, sin)(pi/180 theta_j).
    actuators: list of dicts npt, u_j, u_j_osc, omg_j, theta_j. Returns a copy."""
    v = np.array(vel, dtype=np.float64)
    nb = v.size // 2
    k = nb - sum(a["npt"] for a in actuators)
    for a in actuators:
        u = a["u_j"] + a["u_j_osc"] * math.sin(a["omg_j"] * dt * float(itime))
        cx, sy = math.cos(PI / 180.0 * a["theta_j"]), math.sin(PI / 180.0 * a["theta_j"])
        for _ in range(a["npt"]):
            v[k] = u * cx
            v[nb + k] = u * sy
            k += 1
    return v


class Case:
    """One oracle case (grid + state), mirroring the reference's globals."""

    def __init__(self, params, xb, yb, bdyno=None):
        L = lib()
        xb = np.ascontiguousarray(xb, dtype=np.float64)
        yb = np.ascontiguousarray(yb, dtype=np.float64)
        nb = xb.size
        if bdyno is None:
            bdyno = np.zeros(nb, dtype=np.int32)
        self.bdyno = np.ascontiguousarray(bdyno, dtype=np.int32)
        h = ctypes.c_void_p()
        rc = L.or_create(ctypes.byref(params), nb, _p(xb), _p(yb),
                         self.bdyno.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                         ctypes.byref(h))
        if rc != 0:
            raise ValueError("HEY! Grid nodes must be divisible by 4!!")
        self.h = h
        self.params = params
        vals = [ctypes.c_int() for _ in range(6)]
        d = ctypes.c_double()
        L.or_sizes(h, *[ctypes.byref(v) for v in vals], ctypes.byref(d))
        self.m, self.n, self.nlev, self.nq, self.nb, self.nsmear = [v.value for v in vals]
        self.delta = d.value
        self.ns = (self.m - 1) * (self.n - 1)
        self.nf = 2 * self.nb
        self.nring = 2 * (self.m + 1) + 2 * (self.n + 1)
        self.itime = ctypes.c_int(params.istart)
        self.nbody = int(self.bdyno.max() - self.bdyno.min() + 1) if nb else 0

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.or_destroy(self.h)
            self.h = None

    # state -----------------------------------------------------------------
    def get_state(self):
        L = lib()
        om = np.zeros(self.ns * self.nlev)
        fb = np.zeros(self.nf)
        ro = np.zeros(self.ns * self.nlev)
        q = np.zeros(self.nq * self.nlev)
        q0 = np.zeros(self.nq * self.nlev)
        L.or_get_state(self.h, _p(om), _p(fb), _p(ro), _p(q), _p(q0))
        return dict(omega=om, fb=fb, rhs_old=ro, q=q, q0=q0)

    def set_state(self, omega=None, fb=None, rhs_old=None, q=None, q0=None):
        lib().or_set_state(self.h, _p(omega), _p(fb), _p(rhs_old), _p(q), _p(q0))

    def get_cholesky(self):
        cm = np.zeros(self.nf * self.nf)
        cv = np.zeros(self.nf)
        lib().or_get_cholesky(self.h, _p(cm), _p(cv))
        return cm, cv

    def set_cholesky(self, cm, cv):
        lib().or_set_cholesky(self.h, _p(cm), _p(cv))

    def set_body(self, xb, yb):
        xb = np.ascontiguousarray(xb, dtype=np.float64)
        yb = np.ascontiguousarray(yb, dtype=np.float64)
        lib().or_set_body(self.h, _p(xb), _p(yb))

    def preprocess(self):
        return lib().or_preprocess(self.h)

    def set_cg_relative(self, flag=True):
        lib().or_set_cg_relative(self.h, int(flag))

    def advance(self, body_vel=None):
        L = lib()
        fx = np.zeros(max(self.nbody, 1))
        fy = np.zeros(max(self.nbody, 1))
        circ = np.zeros(self.nlev)
        slip = np.zeros(1)
        it = ctypes.c_int()
        if body_vel is not None:
            body_vel = np.ascontiguousarray(body_vel, dtype=np.float64)
        rc = L.or_advance(self.h, ctypes.byref(self.itime), _p(body_vel), _p(fx), _p(fy),
                          _p(circ), _p(slip), ctypes.byref(it))
        return rc, dict(fx=fx, fy=fy, circ=circ, slip=float(slip[0]), cg_iters=it.value)

    # operators ---------------------------------------------------------------
    def _unary(self, name, x, nout):
        out = np.zeros(nout)
        x = np.ascontiguousarray(x, dtype=np.float64)
        getattr(lib(), name)(self.h, _p(x), _p(out))
        return out

    def dst(self, x):
        return self._unary("or_dst", x, self.ns)

    def ctci(self, x):
        return self._unary("or_ctci", x, self.ns)

    def ainv(self, x):
        return self._unary("or_ainv", x, self.ns)

    def rot(self, x):
        return self._unary("or_rot", x, self.ns)

    def reg(self, x):
        return self._unary("or_reg", x, self.nq)

    def regT(self, x):
        return self._unary("or_regT", x, self.nf)

    def a_times(self, x):
        return self._unary("or_a_times", x, self.nf)

    def cholsl(self, x):
        return self._unary("or_cholsl", x, self.nf)

    def curl(self, x, xbc):
        out = np.zeros(self.nq)
        lib().or_curl(self.h, _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(xbc)), _p(out))
        return out

    def nonlinear(self, omega, q, q0, bc):
        out = np.zeros(self.nq)
        lib().or_nonlinear(self.h, _p(omega), _p(q), _p(q0), _p(bc), _p(out))
        return out

    def coarsify(self, crhs, rhs):
        out = np.zeros(self.ns)
        lib().or_coarsify(self.h, _p(crhs), _p(rhs), _p(out))
        return out

    def get_bc(self, r, fac):
        out = np.zeros(self.nring)
        lib().or_get_bc(self.h, _p(np.ascontiguousarray(r)), _p(out), fac)
        return out

    def apply_bc(self, r, rbc, fac):
        r = np.array(r, dtype=np.float64)
        lib().or_apply_bc(self.h, _p(r), _p(np.ascontiguousarray(rbc)), fac)
        return r

    def vort2flux(self, omega, nlev):
        omega = np.array(omega, dtype=np.float64)
        vel = np.zeros(self.nq * nlev)
        lib().or_vort2flux(self.h, _p(vel), _p(omega), nlev)
        return vel, omega

    def tables(self):
        ns, L = self.ns, self.nlev
        out = dict(lam=np.zeros(ns), laminv=np.zeros(ns), lam1=np.zeros(ns * L),
                   lam1i=np.zeros(ns * L), con1=np.zeros(L), con2=np.zeros(L), vfac=np.zeros(L))
        lib().or_tables(self.h, *[_p(out[k]) for k in
                                  ("lam", "laminv", "lam1", "lam1i", "con1", "con2", "vfac")])
        return out
