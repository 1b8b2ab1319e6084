"""Case definitions for the IBFS advance: the reference's body-geometry
primitives and seeded generators of the benchmark configurations.

Geometry follows grid.f90: circle() (:496-520) and line() (:431-462). All
configurations use the reference's domain convention len=4, offsetx =
offsety = 2, i.e. [-2,2]^2 on the finest level, each coarser level doubling
the extent. Inputs are synthetic and seeded: the reference runs no dataset.
"""
import math

import numpy as np

PI = 3.1415926535897932384
LEN = 4.0


def circle(ds, dia=1.0, x=0.0, y=0.0, npt=None):
    """grid.f90:496-520; npt defaults to INT(pi*dia/ds)."""
    if npt is None:
        npt = int(PI * dia / ds)
    i = np.arange(npt, dtype=np.float64)
    return x + 0.5 * dia * np.cos(2.0 * PI * i / float(npt)), y + 0.5 * dia * np.sin(2.0 * PI * i / float(npt))


def line(ds, length=1.0, aoa=0.0, npt=None):
    """grid.f90:431-462: end points included, npt = INT(len/ds) segments,
    angle = -aoa (degrees), centred on the origin."""
    angle = -aoa * PI / 180.0
    x_le = -0.5 * length * math.cos(angle)
    y_le = -0.5 * length * math.sin(angle)
    if npt is None:
        npt = int(length / ds)
    seg = np.arange(npt + 1, dtype=np.float64) * length / float(npt)
    return x_le + seg * math.cos(angle), y_le + seg * math.sin(angle)


def case(m, levels, re, dt, body, aoa=0.0, npt=None, n=None):
    """One case as a dict: grid, flow parameters and body points."""
    n = m if n is None else n
    ds = LEN / m
    if body == "cylinder":
        xb, yb = circle(ds, 1.0, npt=npt)
    else:
        xb, yb = line(ds, 1.0, aoa, npt=npt)
    return dict(m=m, n=n, levels=levels, re=float(re), dt=float(dt), body=body, aoa=float(aoa), xb=xb, yb=yb)


def cylinder_re100():
    """Stationary cylinder D=1, Re 100, 200x200 cells, 3 levels, 126 points, dt .004."""
    return case(200, 3, 100.0, 0.004, "cylinder", npt=126)


def plate_re300():
    """Flat plate chord 1 at 30 deg, Re 300, 400x400 cells, 5 levels, dt .002."""
    return case(400, 5, 300.0, 0.002, "plate", aoa=30.0)


def batch(ncases=256, seed=20261203):
    """Independent stationary cases: m in {128,192,256,384,512}, 2-5 levels,
    Re log-uniform in [50,500], cylinder or plate with angle of attack uniform
    in [0,40] deg, body-point spacing ~dx, dt at CFL 0.4 for U=1 (dt = 0.4 dx)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(ncases):
        m = int(rng.choice([128, 192, 256, 384, 512]))
        levels = int(rng.integers(2, 6))
        re = float(np.exp(rng.uniform(math.log(50.0), math.log(500.0))))
        body = "cylinder" if rng.random() < 0.5 else "plate"
        aoa = float(rng.uniform(0.0, 40.0))
        dx = LEN / m
        out.append(case(m, levels, re, 0.4 * dx, body, aoa=aoa))
    return out


def strata(cases):
    """The batch grouped by (grid size m, level count L): {(m, L): [case
    indices]}, in batch order within each group."""
    out = {}
    for i, c in enumerate(cases):
        out.setdefault((c["m"], c["levels"]), []).append(i)
    return dict(sorted(out.items()))


def stratified_sample(cases, body=None):
    """One case per (m, L) stratum of the batch: the first case of the body
    type `body` ("plate", "cylinder") in each stratum, or, with body None,
    alternately the first plate and the first cylinder (strata in (m, L)
    order), falling back to the stratum's first case. Returns (indices,
    weights), the weight being the stratum's share of the batch's cases."""
    ids, wts = [], []
    for s, (key, members) in enumerate(strata(cases).items()):
        want = body if body is not None else ("plate" if s % 2 == 0 else "cylinder")
        pick = next((i for i in members if cases[i]["body"] == want), members[0])
        ids.append(pick)
        wts.append(len(members))
    return ids, wts


def cells_per_step(cases, nlev):
    """Cell-updates per step: sum of L*m*n over cases (levels after the clamp)."""
    return int(sum(L * c["m"] * c["n"] for c, L in zip(cases, nlev)))


def case_cost(c):
    """Relative cost of one step of a case: (3L+1) sine-transform solves of
    (m-1)^2 (m-1)-long contractions dominate, so ~ (3L+1) m^3."""
    return (3 * c["levels"] + 1) * float(c["m"]) ** 3


def shard(cases, rank, world):
    """Indices of the cases one of `world` GPUs advances when a batch is split
    across GPUs (independent cases: no exchange step between shards). Greedy
    longest-first assignment to the least-loaded rank, deterministic, so that
    every rank computes the same partition without communicating."""
    order = sorted(range(len(cases)), key=lambda i: (-case_cost(cases[i]), i))
    load = [0.0] * world
    owner = [0] * len(cases)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += case_cost(cases[i])
    return [i for i in range(len(cases)) if owner[i] == rank]


def pitching(m=512, levels=5, re=500.0, dt=0.001, amp_deg=20.0, freq=0.25, cgtol=1e-12, precond=True):
    """Flat plate of chord 1 pitching sinusoidally about mid-chord,
    alpha(t) = amp sin(2 pi freq t), body points at spacing dx along the chord;
    the force system is solved by CG to a relative residual of cgtol every step
    (preconditioned by factors at a grid of pitch angles, turned with the plate, unless
    precond is False)."""
    c = case(m, levels, re, dt, "plate", aoa=0.0)
    c.update(pitch_amp_deg=float(amp_deg), pitch_freq=float(freq), cgtol=float(cgtol), cg_precond=int(bool(precond)))
    return c


def pitching_batch(ncases=32, seed=20261203, **kw):
    """Pitching plates whose amplitudes are drawn uniformly from [5, 30] degrees."""
    rng = np.random.default_rng(seed)
    return [pitching(amp_deg=float(a), **kw) for a in rng.uniform(5.0, 30.0, ncases)]


def solver_args(cases, capi, precision=0):
    """Params / bodies / options lists for ibfs_capi.Solver (pitching cases:
    moving body, CG with a relative stop, motion on the device)."""
    params, opts = [], []
    for c in cases:
        if "pitch_amp_deg" in c:
            params.append(capi.make_params(c["m"], c["n"], c["dt"], c["re"], c["levels"], stationary=False,
                                           cgtol=c["cgtol"]))
            opts.append(capi.make_options(precision=precision, cg_relative=1, motion_kind=1,
                                          pitch_amp_deg=c["pitch_amp_deg"], pitch_freq=c["pitch_freq"],
                                          cg_precond=c.get("cg_precond", 0)))
        else:
            params.append(capi.make_params(c["m"], c["n"], c["dt"], c["re"], c["levels"]))
            opts.append(capi.make_options(precision=precision))
    bodies = [(c["xb"], c["yb"]) for c in cases]
    return params, bodies, opts
