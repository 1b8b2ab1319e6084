"""Derivative of the mean drag of pitching plates with respect to the pitch
amplitude.

mean_drag_amplitude_adjoint: the discrete adjoint (ibfs_adjoint_pitch_run),
all amplitudes differentiated together as the cases of one handle; the cost
is about three forward solves of the batch.

mean_drag_amplitude_derivative: central differences inside one batched run
(every amplitude A becomes the two cases A - h and A + h, advanced together),
J(A) = mean of Fx over the last `tail` steps and dJ/dA = (J(A + h) -
J(A - h)) / 2h; kept as an independent cross-check of the adjoint.
"""
import numpy as np

import ibfs_capi as C
import workloads as W


def mean_drag_amplitude_adjoint(amps_deg, steps=100, tail=None, checkpoint_every=50, batched=True, workers=1,
                                **case_kw):
    """J(A) and dJ/dA (per degree) for each amplitude in amps_deg by the
    discrete adjoint; case_kw as for workloads.pitching. batched: every
    amplitude is a case of one handle and all are differentiated together
    (one launch per stage). Otherwise one handle per amplitude; with
    workers > 1 those single-case adjoints run from that many host threads at
    once, each handle on its own stream (handles share no mutable state;
    results are bit-identical to a sequential run)."""
    tail = steps if tail is None else int(tail)
    wx = np.zeros(steps)
    wx[steps - tail:] = 1.0 / tail
    wy = np.zeros(steps)
    cases = [W.pitching(amp_deg=float(a), **case_kw) for a in np.asarray(amps_deg, dtype=np.float64)]
    if batched:
        params, bodies, opts = W.solver_args(cases, C)
        g = C.Solver(params, bodies, opts)
        try:
            J, d, _, _ = g.adjoint_pitch_run(steps, checkpoint_every, wx, wy)
        finally:
            g.close()
        return np.atleast_1d(J), np.atleast_1d(d)
    solvers = []
    for c in cases:
        params, bodies, opts = W.solver_args([c], C)
        solvers.append(C.Solver(params[0], bodies[0], opts[0]))

    def run(s):
        return s.adjoint_pitch_run(steps, checkpoint_every, wx, wy)

    try:
        if workers > 1:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(workers) as ex:
                res = list(ex.map(run, solvers))
        else:
            res = [run(s) for s in solvers]
    finally:
        for s in solvers:
            s.close()
    return np.array([r[0] for r in res]), np.array([r[1] for r in res])


def mean_drag_amplitude_derivative(amps_deg, h_deg=1e-3, steps=100, tail=None, **case_kw):
    """J(A) and dJ/dA (per degree) for each amplitude in amps_deg; case_kw as
    for workloads.pitching (m, levels, re, dt, freq, cgtol)."""
    amps = np.asarray(amps_deg, dtype=np.float64)
    tail = steps if tail is None else int(tail)
    cases = []
    for a in amps:
        cases.append(W.pitching(amp_deg=float(a - h_deg), **case_kw))
        cases.append(W.pitching(amp_deg=float(a + h_deg), **case_kw))
    params, bodies, opts = W.solver_args(cases, C)
    g = C.Solver(params, bodies, opts)
    hist = g.advance_n(steps)
    fx = np.array([[g.outputs_of(hist[s], i)["fx"][0] for s in range(steps)] for i in range(len(cases))])
    g.close()
    Jc = fx[:, steps - tail:].mean(axis=1)
    jm, jp = Jc[0::2], Jc[1::2]
    return 0.5 * (jm + jp), (jp - jm) / (2.0 * h_deg)
