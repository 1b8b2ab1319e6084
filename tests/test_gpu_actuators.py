"""Actuator jets (the reference's actuation / u_jet, grid.f90:579-633, with the
slot geometry of actuator_slot, :636-718): the device-side jet velocities of
ibfs_set_actuators against the oracle advanced with the same velocities
computed on the host, per body (the actuators are bodies -1, -2 of
write_force) and per field; the batched form equals single handles."""
import math

import numpy as np
import pytest

import ibfs_capi as C
import oracle as O

pytestmark = pytest.mark.gpu

M, LEV, DT, RE, STEPS = 48, 3, 0.01, 100.0, 10


def geometry(m=M):
    ds = 4.0 / m
    xb, yb = O.circle(ds, 1.0, 0.0, 0.0)
    bd = [np.zeros(len(xb), dtype=np.int32)]
    xs, ys = [xb], [yb]
    acts = [dict(x=0.0, y=0.75, h=0.3, u_j=0.5, u_j_osc=0.2, omg_j=2.0 * math.pi, theta_j=90.0),
            dict(x=0.1, y=-0.8, h=0.05, u_j=-0.3, u_j_osc=0.1, omg_j=3.0, theta_j=-60.0)]
    for i, a in enumerate(acts):
        ax, ay, ab = O.actuator_slot(a["x"], a["y"], a["h"], ds, a["theta_j"], -(i + 1))
        a["npt"] = len(ax)
        xs.append(ax)
        ys.append(ay)
        bd.append(ab)
    return np.concatenate(xs), np.concatenate(ys), np.concatenate(bd), acts


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def test_actuator_jets_match_oracle():
    x, y, bd, acts = geometry()
    assert [a["npt"] for a in acts] == [int(0.3 / (4.0 / M)) + 1, 1]
    g = C.Solver(C.make_params(M, M, DT, RE, LEV), (x, y, bd))
    g.set_actuators(acts)
    oc = O.Case(O.make_params(M, M, DT, RE, LEV), x, y, bd)
    nf = 2 * len(x)
    for s in range(1, STEPS + 1):
        og = g.advance()
        rc, o = oc.advance(body_vel=O.jet_velocities(np.zeros(nf), acts, s, DT))
        assert rc == 0
        assert len(og["fx"]) == 3  # bodies -2, -1, 0
        scale = np.abs(o["fx"]).max()
        assert np.abs(og["fx"] - o["fx"]).max() <= 1e-10 * scale, s
        assert np.abs(og["fy"] - o["fy"]).max() <= 1e-10 * scale, s
    assert rel(g.get_state()["omega"], oc.get_state()["omega"]) < 1e-10
    # the jets are what moves the flow: without them the forces differ
    h = C.Solver(C.make_params(M, M, DT, RE, LEV), (x, y, bd))
    h.advance_n(STEPS, want_hist=False)
    assert rel(h.get_state()["omega"], g.get_state()["omega"]) > 1e-3
    h.close()
    # removing the jets rebuilds the step without them
    g.set_actuators([])
    oc2 = O.Case(O.make_params(M, M, DT, RE, LEV), x, y, bd)
    g2 = C.Solver(C.make_params(M, M, DT, RE, LEV), (x, y, bd))
    g2.set_actuators(acts)
    g2.set_actuators([])
    for s in range(3):
        a, (rc, b) = g2.advance(), oc2.advance()
        assert np.abs(a["fx"] - b["fx"]).max() <= 1e-10 * np.abs(b["fx"]).max()
    g.close()
    g2.close()


def test_actuator_jets_batched_equal_single():
    x, y, bd, acts = geometry()
    xb, yb = O.circle(4.0 / 32, 1.0, 0.0, 0.0)
    params = [C.make_params(M, M, DT, RE, LEV), C.make_params(32, 32, DT, RE, 2)]
    g = C.Solver(params, [(x, y, bd), (xb, yb)])
    g.set_actuators(acts, icase=0)
    hist = g.advance_n(STEPS)
    s = C.Solver(params[0], (x, y, bd))
    s.set_actuators(acts)
    hs = s.advance_n(STEPS)
    assert np.array_equal(g.get_state(0)["omega"], s.get_state()["omega"])
    for k in range(STEPS):
        assert np.array_equal(g.outputs_of(hist[k], 0)["fx"], s.outputs_of(hs[k], 0)["fx"])
    t = C.Solver(params[1], (xb, yb))
    t.advance_n(STEPS, want_hist=False)
    assert np.array_equal(g.get_state(1)["omega"], t.get_state()["omega"])
    for h in (g, s, t):
        h.close()
