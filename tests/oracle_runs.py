"""Oracle runs of whole configurations for the GPU parity tests.

TEST INFRASTRUCTURE ONLY. The CPU oracle (oracle/ibfs_oracle.c) advances a
case for a number of steps and returns its final state and its per-step
outputs (write_force / write_circ / write_slip, operators.f90:549-699). The
large configurations take tens of seconds each on one host core, so the tests
run them in a process pool started with the `spawn` method (the GPU parity
tests hold a CUDA context; a forked child of such a process can hang), all
submitted at once so that they overlap with each other and with the GPU work.
"""
import concurrent.futures as cf
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _paths():
    for sub in ("oracle", "ibfs-if2d_b200"):
        p = os.path.join(ROOT, sub)
        if p not in sys.path:
            sys.path.insert(0, p)


def run_case(spec, steps):
    """Advance one case `steps` times with the oracle from the initial state
    (the first advance runs preprocess, operators.f90:90-92).

    spec: dict with m, n, levels, re, dt, xb, yb (as workloads.case makes).
    Returns dict(state=.var payload, fx, fy (steps x nbody), circ (steps x L),
    slip (steps), slip_scale = max |regT(q0 on level 1)|, the magnitude of the
    body-point velocities whose residual slip measures, nlev)."""
    _paths()
    import oracle as O
    oc = O.Case(O.make_params(spec["m"], spec["n"], spec["dt"], spec["re"], spec["levels"]),
                spec["xb"], spec["yb"])
    fx, fy, circ, slip = [], [], [], []
    for _ in range(steps):
        rc, o = oc.advance()
        if rc != 0:
            raise RuntimeError(f"oracle advance returned {rc}")
        fx.append(o["fx"].copy())
        fy.append(o["fy"].copy())
        circ.append(o["circ"].copy())
        slip.append(o["slip"])
    st = oc.get_state()
    slip_scale = float(np.abs(oc.regT(np.ascontiguousarray(st["q0"][:oc.nq]))).max())
    return dict(state=st, fx=np.array(fx), fy=np.array(fy), circ=np.array(circ), slip=np.array(slip),
                slip_scale=slip_scale, nlev=oc.nlev)


def run_dst(m, n, seed):
    """The oracle's dst (myfft.f90:83-94) of a seeded N(0,1) field."""
    _paths()
    import oracle as O
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    oc = O.Case(O.make_params(m, n, 0.01, 100.0, 2), xb, yb)
    x = np.random.default_rng(seed).standard_normal(oc.ns)
    return x, oc.dst(x)


class Pool:
    """A spawn-started pool whose jobs are named; submit everything first,
    then collect each result where a test needs it."""

    def __init__(self, workers=None):
        workers = workers or max(1, min(16, os.cpu_count() or 1))
        self.ex = cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"))
        self.jobs = {}

    def submit(self, name, fn, *args):
        self.jobs[name] = self.ex.submit(fn, *args)

    def get(self, name, timeout=900):
        return self.jobs[name].result(timeout=timeout)

    def close(self):
        self.ex.shutdown(wait=False, cancel_futures=True)
