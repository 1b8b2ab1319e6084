"""Derivative of the mean drag of pitching plates with respect to the pitch
amplitude, by central differences inside one batched run.

Every amplitude A becomes two cases of one batch, A - h and A + h (degrees),
advanced together on the GPU; J(A) = mean of Fx over the last `tail` steps and
dJ/dA = (J(A + h) - J(A - h)) / 2h. The cost is that of one batched forward
run with twice the cases (2x a forward solve of the amplitudes). This is a
finite-difference derivative, not a discrete adjoint: the adjoint of the
moving-body path (through the regularisation's dependence on the body
positions) is not built.
"""
import numpy as np

import ibfs_capi as C
import workloads as W


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
