"""ctypes binding of include/ibfs_capi.h (the B200 IBFS advance).

This is the Python-side caller of the C-ABI, the same seam a Fortran driver
binds through iso_c_binding. It loads the in-tree libibfs_b200.so and raises
if it is missing -- there is no CPU fallback.

Mirrors the reference's driver flow (src/main.f90:42-54): create (setup +
setup_variables), optional restart/Cholesky load, then advance per step.
"""
import ctypes
import warnings
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libibfs_b200.so")

OK, ERR_GRID, ERR_CHOL, ERR_CG_MAXITER, ERR_CUDA, ERR_IO, ERR_TIMEOUT, ERR_ARG, ERR_NOMEM = range(9)
_ERRNAMES = {1: "IBFS_ERR_GRID", 2: "IBFS_ERR_CHOL", 3: "IBFS_ERR_CG_MAXITER", 4: "IBFS_ERR_CUDA",
             5: "IBFS_ERR_IO", 6: "IBFS_ERR_TIMEOUT", 7: "IBFS_ERR_ARG", 8: "IBFS_ERR_NOMEM"}

EXPORTS = [
    "ibfs_create", "ibfs_batch_create", "ibfs_destroy", "ibfs_case_sizes", "ibfs_num_cases",
    "ibfs_set_state", "ibfs_get_state", "ibfs_set_cholesky", "ibfs_get_cholesky", "ibfs_precompute",
    "ibfs_advance", "ibfs_advance_n", "ibfs_batch_advance", "ibfs_output_offset", "ibfs_output_stride", "ibfs_apply_op",
    "ibfs_last_timing", "ibfs_kernels_per_step", "ibfs_profile_step", "ibfs_dst2d_noalloc",
    "ibfs_last_cg_iterations", "ibfs_adjoint_run", "ibfs_adjoint_pitch_run", "ibfs_vertex_fields",
    "ibfs_set_actuators", "ibfs_set_wait_limit", "ibfs_gemm_tiles",
    "ibfs_last_error",
]


class Params(ctypes.Structure):
    """ibfs_params_c == namelist READ_PARAMETERS (parameters.f90:48-50)."""
    _fields_ = [
        ("istart", ctypes.c_int), ("istop", ctypes.c_int), ("isave", ctypes.c_int),
        ("m", ctypes.c_int), ("n", ctypes.c_int),
        ("dt", ctypes.c_double), ("re", ctypes.c_double), ("cgtol", ctypes.c_double),
        ("cg_max_iter", ctypes.c_int), ("unif_flow", ctypes.c_int),
        ("len", ctypes.c_double), ("offsetx", ctypes.c_double), ("offsety", ctypes.c_double),
        ("mgridlev", ctypes.c_int), ("make_vortex", ctypes.c_int), ("stationary", ctypes.c_int),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int), ("cg_relative", ctypes.c_int), ("motion_kind", ctypes.c_int),
        ("pitch_amp_deg", ctypes.c_double), ("pitch_freq", ctypes.c_double),
        ("pivot_x", ctypes.c_double), ("pivot_y", ctypes.c_double), ("tile_cfg", ctypes.c_int),
        ("cg_precond", ctypes.c_int), ("tc_tile", ctypes.c_int), ("refine_slices", ctypes.c_int),
        ("poisson_sweeps", ctypes.c_int),
    ]


class IbfsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def lib():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise FileNotFoundError(f"{SO} not built (run __graft_entry__.build() or make -C ibfs-if2d_b200)")
        L = ctypes.CDLL(SO)
        vp = ctypes.c_void_p
        L.ibfs_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(Options), ctypes.c_int, _DP, _DP, _IP,
                                  ctypes.POINTER(vp)]
        L.ibfs_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(Params), ctypes.POINTER(Options), _IP,
                                        _DP, _DP, _IP, ctypes.POINTER(vp)]
        L.ibfs_destroy.argtypes = [vp]
        L.ibfs_case_sizes.argtypes = [vp, ctypes.c_int] + [_IP] * 6
        L.ibfs_num_cases.argtypes = [vp]
        L.ibfs_set_state.argtypes = [vp, ctypes.c_int, _DP, _DP, _DP, _DP, _DP]
        L.ibfs_get_state.argtypes = [vp, ctypes.c_int, _DP, _DP, _DP, _DP, _DP]
        L.ibfs_set_cholesky.argtypes = [vp, ctypes.c_int, _DP, _DP]
        L.ibfs_get_cholesky.argtypes = [vp, ctypes.c_int, _DP, _DP]
        L.ibfs_precompute.argtypes = [vp]
        L.ibfs_advance.argtypes = [vp, _IP, _DP, _DP, _DP, _DP, _DP]
        L.ibfs_advance_n.argtypes = [vp, ctypes.c_int, _DP]
        L.ibfs_batch_advance.argtypes = [vp, _DP, _DP]
        L.ibfs_vertex_fields.argtypes = [vp, ctypes.c_int, ctypes.c_int, _DP]
        L.ibfs_output_offset.argtypes = [vp, ctypes.c_int]
        L.ibfs_output_stride.argtypes = [vp]
        L.ibfs_apply_op.argtypes = [vp, ctypes.c_int, _DP, _DP]
        L.ibfs_last_timing.argtypes = [vp, _DP]
        L.ibfs_kernels_per_step.argtypes = [vp]
        L.ibfs_last_cg_iterations.argtypes = [vp]
        L.ibfs_adjoint_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _DP, _DP]
        L.ibfs_adjoint_pitch_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, _DP, _DP, _DP, _DP, _DP, _DP]
        L.ibfs_set_actuators.argtypes = [vp, ctypes.c_int, ctypes.c_int, _IP, _DP, _DP, _DP, _DP]
        L.ibfs_profile_step.argtypes = [vp, _DP, _IP, _DP]
        L.ibfs_set_wait_limit.argtypes = [vp, ctypes.c_double, ctypes.c_int]
        L.ibfs_gemm_tiles.argtypes = [vp, _IP, ctypes.c_int]
        L.ibfs_dst2d_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_void_p]
        L.ibfs_last_error.argtypes = [vp]
        L.ibfs_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 contiguous arrays only"
    return a.ctypes.data_as(_DP)


def make_params(m, n, dt, re, mgridlev, len_=4.0, offsetx=2.0, offsety=2.0, stationary=True,
                unif_flow=True, cgtol=1e-7, cg_max_iter=3000, istart=0, istop=400, isave=25):
    return Params(istart, istop, isave, m, n, dt, re, cgtol, cg_max_iter, int(unif_flow), len_,
                  offsetx, offsety, mgridlev, 0, int(stationary))


def make_options(precision=0, cg_relative=0, motion_kind=0, pitch_amp_deg=0.0, pitch_freq=0.0,
                 pivot_x=0.0, pivot_y=0.0, tile_cfg=-1, cg_precond=0, tc_tile=0, refine_slices=0,
                 poisson_sweeps=0):
    return Options(precision, cg_relative, motion_kind, pitch_amp_deg, pitch_freq, pivot_x, pivot_y,
                   tile_cfg, cg_precond, tc_tile, refine_slices, poisson_sweeps)


class Solver:
    """One handle: a single case (plain drop-in) or a batch of cases."""

    def __init__(self, params, bodies, options=None):
        """params: Params or list of Params; bodies: (xb, yb[, bdyno]) or list of those."""
        L = lib()
        if isinstance(params, Params):
            params, bodies = [params], [bodies]
            options = [options] if options is not None else None
        n = len(params)
        parr = (Params * n)(*params)
        oarr = (Options * n)(*options) if options is not None else None
        nb = np.array([len(b[0]) for b in bodies], dtype=np.int32)
        xb = np.ascontiguousarray(np.concatenate([np.asarray(b[0], float) for b in bodies]))
        yb = np.ascontiguousarray(np.concatenate([np.asarray(b[1], float) for b in bodies]))
        bd = np.ascontiguousarray(np.concatenate(
            [np.asarray(b[2] if len(b) > 2 else np.zeros(len(b[0])), dtype=np.int32) for b in bodies]))
        h = ctypes.c_void_p()
        rc = L.ibfs_batch_create(n, parr, oarr, nb.ctypes.data_as(_IP), _p(xb), _p(yb),
                                 bd.ctypes.data_as(_IP), ctypes.byref(h))
        if rc != 0:
            raise IbfsError(rc, L.ibfs_last_error(None).decode())
        self.h = h
        self.ncases = n
        self.sizes = []
        for i in range(n):
            v = [ctypes.c_int() for _ in range(6)]
            L.ibfs_case_sizes(h, i, *[ctypes.byref(x) for x in v])
            m_, n_, nlev, nq, nbp, nbody = [x.value for x in v]
            self.sizes.append(dict(m=m_, n=n_, nlev=nlev, nq=nq, nb=nbp, nf=2 * nbp, nbody=nbody,
                                   ns=(m_ - 1) * (n_ - 1)))
        self.itime = ctypes.c_int(params[0].istart)
        self.stride = L.ibfs_output_stride(h)

    def close(self):
        if getattr(self, "h", None) is not None:
            lib().ibfs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, step=False):
        if rc == 3 and step:  # IBFS_ERR_CG_MAXITER: the reference's warning; the step completed
            warnings.warn("IBFS: " + lib().ibfs_last_error(self.h).decode(), RuntimeWarning, stacklevel=3)
            return
        if rc != 0:
            raise IbfsError(rc, lib().ibfs_last_error(self.h).decode())

    def get_state(self, icase=0):
        s = self.sizes[icase]
        out = dict(omega=np.zeros(s["ns"] * s["nlev"]), fb=np.zeros(max(s["nf"], 1)),
                   rhs_old=np.zeros(s["ns"] * s["nlev"]), q=np.zeros(s["nq"] * s["nlev"]),
                   q0=np.zeros(s["nq"] * s["nlev"]))
        self._check(lib().ibfs_get_state(self.h, icase, *[_p(out[k]) for k in
                                                          ("omega", "fb", "rhs_old", "q", "q0")]))
        return out

    def set_state(self, icase=0, omega=None, fb=None, rhs_old=None, q=None, q0=None):
        self._check(lib().ibfs_set_state(self.h, icase, _p(omega), _p(fb), _p(rhs_old), _p(q), _p(q0)))

    def get_cholesky(self, icase=0):
        nf = self.sizes[icase]["nf"]
        cm, cv = np.zeros(nf * nf), np.zeros(nf)
        self._check(lib().ibfs_get_cholesky(self.h, icase, _p(cm), _p(cv)))
        return cm, cv

    def set_cholesky(self, cm, cv, icase=0):
        self._check(lib().ibfs_set_cholesky(self.h, icase, _p(np.ascontiguousarray(cm)),
                                            _p(np.ascontiguousarray(cv))))

    def precompute(self):
        self._check(lib().ibfs_precompute(self.h))

    def advance(self, body_vel=None):
        s = self.sizes[0]
        fx, fy = np.zeros(max(s["nbody"], 1)), np.zeros(max(s["nbody"], 1))
        circ, slip = np.zeros(s["nlev"]), np.zeros(1)
        bv = None if body_vel is None else np.ascontiguousarray(body_vel, dtype=np.float64)
        self._check(lib().ibfs_advance(self.h, ctypes.byref(self.itime), _p(bv), _p(fx), _p(fy),
                                       _p(circ), _p(slip)), step=True)
        return dict(fx=fx, fy=fy, circ=circ, slip=float(slip[0]))

    def advance_n(self, nsteps, want_hist=True):
        hist = np.zeros(nsteps * self.stride) if want_hist else None
        self._check(lib().ibfs_advance_n(self.h, nsteps, _p(hist)), step=True)
        self.itime.value += nsteps
        return hist.reshape(nsteps, self.stride) if want_hist else None

    def batch_advance(self, body_vel=None, out=None):
        """One advance of every case (ibfs_batch_advance): body_vel = all cases'
        body-point velocities concatenated (or None); returns the step's
        output row (layout of one advance_n history row)."""
        if out is None:
            out = np.zeros(self.stride)
        bv = None if body_vel is None else np.ascontiguousarray(body_vel, dtype=np.float64)
        if bv is not None:
            assert bv.size == sum(s["nf"] for s in self.sizes), "body_vel must hold every case's Nf values"
        self._check(lib().ibfs_batch_advance(self.h, _p(bv), _p(out)), step=True)
        self.itime.value += 1
        return out

    def vertex_fields(self, level, icase=0):
        """write_tecplot's vertex fields of one level (1-based): dict of u, v,
        etfx, etfy, vort, each (m-1)*(n-1) with i fastest."""
        s = self.sizes[icase]
        out = np.zeros(5 * s["ns"])
        self._check(lib().ibfs_vertex_fields(self.h, icase, level, _p(out)))
        f = out.reshape(5, s["ns"])
        return dict(u=f[0], v=f[1], etfx=f[2], etfy=f[3], vort=f[4])

    def outputs_of(self, hist_row, icase=0):
        s = self.sizes[icase]
        o = lib().ibfs_output_offset(self.h, icase)
        nb = s["nbody"]
        blk = hist_row[o:o + 2 * nb + s["nlev"] + 1]
        return dict(fx=blk[:nb], fy=blk[nb:2 * nb], circ=blk[2 * nb:2 * nb + s["nlev"]],
                    slip=blk[2 * nb + s["nlev"]])

    def last_ms(self):
        v = ctypes.c_double()
        lib().ibfs_last_timing(self.h, ctypes.byref(v))
        return v.value

    def adjoint_run(self, nsteps, checkpoint_every, body_vel, wx, wy):
        """J and dJ/d body_vel over nsteps advances (see ibfs_adjoint_run)."""
        nf = self.sizes[0]["nf"]
        bv = None if body_vel is None else np.ascontiguousarray(body_vel, dtype=np.float64)
        wx = np.ascontiguousarray(wx, dtype=np.float64)
        wy = np.ascontiguousarray(wy, dtype=np.float64)
        need = nsteps * self.sizes[0]["nbody"]
        if wx.size != need or wy.size != need:
            raise ValueError(f"wx and wy need {need} weights (nsteps x nbody), got {wx.size} and {wy.size}")
        J, ms_f, ms_t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        grad = np.zeros(nf)
        self._check(lib().ibfs_adjoint_run(self.h, nsteps, checkpoint_every, _p(bv), _p(wx), _p(wy),
                                           ctypes.byref(J), _p(grad), ctypes.byref(ms_f), ctypes.byref(ms_t)))
        self.itime.value += nsteps
        return J.value, grad, ms_f.value, ms_t.value

    def set_actuators(self, actuators, icase=0):
        """Actuator jets on the last body points of case icase (see
        ibfs_set_actuators): a list of dicts with npt, u_j, u_j_osc, omg_j,
        theta_j, in actuator order; [] removes them."""
        n = len(actuators)
        npt = np.array([a["npt"] for a in actuators] or [0], dtype=np.int32)
        col = {k: np.array([float(a[k]) for a in actuators] or [0.0]) for k in ("u_j", "u_j_osc", "omg_j", "theta_j")}
        self._check(lib().ibfs_set_actuators(self.h, icase, n, npt.ctypes.data_as(_IP), _p(col["u_j"]),
                                             _p(col["u_j_osc"]), _p(col["omg_j"]), _p(col["theta_j"])))

    def adjoint_pitch_run(self, nsteps, checkpoint_every, wx, wy):
        """J and dJ/d(pitch amplitude, per degree) over nsteps advances of the
        handle's pitching cases (see ibfs_adjoint_pitch_run). wx, wy: per case
        nsteps x nbody weights, case-major; a 1-D array of nsteps applies to
        every case (one body each). Scalars for a single case, arrays for a
        batch."""
        nc = self.ncases
        wx = np.asarray(wx, dtype=np.float64)
        wy = np.asarray(wy, dtype=np.float64)
        if wx.ndim == 1 and nc > 1:
            wx, wy = np.tile(wx, nc), np.tile(wy, nc)
        wx, wy = np.ascontiguousarray(wx.ravel()), np.ascontiguousarray(wy.ravel())
        need = nsteps * sum(sz["nbody"] for sz in self.sizes)
        if wx.size != need or wy.size != need:
            raise ValueError(f"wx and wy need {need} weights (nsteps x nbody per case, case-major), "
                             f"got {wx.size} and {wy.size}")
        J, dJ = np.zeros(nc), np.zeros(nc)
        ms_f, ms_t = ctypes.c_double(), ctypes.c_double()
        self._check(lib().ibfs_adjoint_pitch_run(self.h, nsteps, checkpoint_every, _p(wx), _p(wy), _p(J), _p(dJ),
                                                 ctypes.byref(ms_f), ctypes.byref(ms_t)), step=True)
        self.itime.value += nsteps
        if nc == 1:
            return float(J[0]), float(dJ[0]), ms_f.value, ms_t.value
        return J, dJ, ms_f.value, ms_t.value

    def set_wait_limit(self, seconds, probe=False):
        """Limit of the bounded device waits; probe=True makes every GEMM block
        wait first on a barrier nothing completes (ibfs_set_wait_limit)."""
        self._check(lib().ibfs_set_wait_limit(self.h, float(seconds), int(bool(probe))))

    def last_cg_iterations(self):
        return lib().ibfs_last_cg_iterations(self.h)

    def kernels_per_step(self):
        return lib().ibfs_kernels_per_step(self.h)

    def gemm_tiles(self):
        """Tile configurations (1..3) of the tensor-core GEMM launch groups of the step."""
        n = lib().ibfs_gemm_tiles(self.h, None, 0)
        out = np.zeros(max(n, 1), dtype=np.int32)
        lib().ibfs_gemm_tiles(self.h, out.ctypes.data_as(_IP), n)
        return [int(x) for x in out[:n]]

    TAGS = ("stencil", "gemm_f64", "gemm_tc", "chol", "split")

    def profile_step(self):
        ms, fl = np.zeros(5), np.zeros(5)
        la = np.zeros(5, dtype=np.int32)
        self._check(lib().ibfs_profile_step(self.h, _p(ms), la.ctypes.data_as(_IP), _p(fl)))
        self.itime.value += 1
        return {t: dict(ms=float(ms[i]), launches=int(la[i]), flops=float(fl[i])) for i, t in enumerate(self.TAGS)}

    def apply_op(self, op, x):
        s = self.sizes[0]
        nout = {0: s["ns"], 1: s["ns"], 2: s["ns"], 3: s["nf"], 4: s["nf"], 5: s["ns"]}[op]
        out = np.zeros(nout)
        self._check(lib().ibfs_apply_op(self.h, op, _p(np.ascontiguousarray(x, dtype=np.float64)), _p(out)))
        return out
