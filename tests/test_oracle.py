"""CPU tests of the oracle (the checker): pinned against the golden fixtures
(scipy DST-I == FFTW RODFT00; the independent numpy restatement of the
advance) and against identities that follow from the reference's math."""
import numpy as np
import pytest

import make_golden as G

import oracle as O


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.fixture(scope="module")
def case32(oracle_mod):
    xb, yb = O.circle(4.0 / 32, 1.0, 0.0, 0.0)
    return O.Case(O.make_params(32, 32, 0.01, 100.0, 3), xb, yb)


def test_dst_golden(oracle_mod):
    g = np.load(G.__file__.replace("make_golden.py", "dst_rodft00.npz"))
    for (m, n) in [(16, 16), (32, 24), (200, 200)]:
        xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
        c = O.Case(O.make_params(m, n, 0.01, 100.0, 2), xb, yb)
        assert rel(c.dst(g[f"x_{m}_{n}"]), g[f"y_{m}_{n}"]) < 1e-14


@pytest.mark.parametrize("name", list(G.CASES))
def test_advance_golden(oracle_mod, name):
    cfg = G.CASES[name]
    g = np.load(G.__file__.replace("make_golden.py", f"{name}.npz"))
    p = O.make_params(cfg["m"], cfg["n"], cfg["dt"], cfg["re"], cfg["lev"], stationary=cfg["stationary"],
                      cgtol=1e-13)
    c = O.Case(p, g["xb"], g["yb"])
    c.set_cg_relative(True)
    fx = []
    for _ in range(cfg["steps"]):
        rc, o = c.advance()
        assert rc == 0
        fx.append(o["fx"][0])
    st = c.get_state()
    for k in ("omega", "q", "rhs_old"):
        assert rel(st[k], g["final_" + k]) < 1e-12, k
    assert rel(st["fb"], g["final_fb"]) < 1e-10
    assert rel(fx, g["fx"]) < 1e-12


def test_dst_involution(case32):
    c = case32
    x = np.random.default_rng(0).standard_normal(c.ns)
    assert rel(c.dst(c.dst(x)) / (4.0 * c.m * c.n), x) < 1e-14  # myfft.f90:116


def laplacian(c, s):
    """C^T C with zero Dirichlet BCs (5-point, index units)."""
    S = s.reshape(c.n - 1, c.m - 1)  # [j][i]
    P = np.pad(S, 1)
    return (4 * S - P[1:-1, :-2] - P[1:-1, 2:] - P[:-2, 1:-1] - P[2:, 1:-1]).ravel()


def test_ctci_inverts_laplacian(case32):
    c = case32
    x = np.random.default_rng(1).standard_normal(c.ns)
    assert rel(laplacian(c, c.ctci(x)), x) < 1e-12
    zero = np.zeros(c.nring)
    assert rel(c.rot(c.curl(x, zero)), laplacian(c, x)) < 1e-13  # rot(curl) = C^T C


def test_ainv_inverts(case32):
    c = case32
    x = np.random.default_rng(2).standard_normal(c.ns)
    nu = 0.5 * c.params.dt / (c.params.re * c.delta ** 2)
    y = c.ainv(x)
    assert rel(y + nu * laplacian(c, y), x) < 1e-12


def test_rot_is_curl_transpose(case32):
    c = case32
    rng = np.random.default_rng(3)
    s, f = rng.standard_normal(c.ns), rng.standard_normal(c.nq)
    zero = np.zeros(c.nring)
    assert abs(c.curl(s, zero) @ f - s @ c.rot(f)) < 1e-10 * np.abs(f).sum()


def test_regT_is_reg_transpose(case32):
    c = case32
    rng = np.random.default_rng(4)
    f, h = rng.standard_normal(c.nf), rng.standard_normal(c.nq)
    assert abs(c.reg(f) @ h - f @ c.regT(h)) < 1e-12 * np.abs(h).sum()


def test_divergence_free(case32):
    """div(curl s) = 0 on every cell (README: divergence removed to round-off)."""
    c = case32
    m, n = c.m, c.n
    s = np.random.default_rng(5).standard_normal(c.ns)
    # a ring from get_bc of a coarser field has consistent corner values
    bc = c.get_bc(np.random.default_rng(6).standard_normal(c.ns), 1.0)
    q = c.curl(s, bc)
    U = q[:(m + 1) * n].reshape(n, m + 1)
    V = q[(m + 1) * n:].reshape(n + 1, m)
    div = (U[:, 1:] - U[:, :-1]) + (V[1:, :] - V[:-1, :])
    assert np.abs(div).max() < 1e-13


def test_delta_partition_of_unity(oracle_mod):
    d = 0.1
    for x0 in (0.0, 0.013, 0.05, 0.0731):
        r = np.arange(-5, 6) * d
        s = sum(O.lib().or_deltafnc(ri, x0, d) for ri in r) * d
        assert abs(s - 1.0) < 1e-12


def test_nlevmax(oracle_mod):
    assert O.lib().or_nlevmax(200, 200) == 5 and O.lib().or_nlevmax(400, 400) == 6
    assert O.lib().or_nlevmax(512, 512) == 7 and O.lib().or_nlevmax(128, 128) == 5


def test_grid_check(oracle_mod):
    with pytest.raises(ValueError):
        O.Case(O.make_params(30, 32, 0.01, 100.0, 2), np.zeros(1), np.zeros(1))


def test_cholesky_reproduces_A(case32):
    c = case32
    assert c.preprocess() == 0
    cm, cv = c.get_cholesky()
    nf = c.nf
    A = cm.reshape(nf, nf, order="F")
    Lf = np.tril(A, -1) + np.diag(cv)
    Au = np.triu(A) + np.triu(A, 1).T  # choldc reads the upper triangle
    assert rel(Lf @ Lf.T, Au) < 1e-12
    b = np.random.default_rng(7).standard_normal(nf)
    assert rel(Au @ c.cholsl(b), b) < 1e-10


def test_cg_matches_cholesky(oracle_mod):
    m = 32
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    a = O.Case(O.make_params(m, m, 0.01, 100.0, 3, stationary=True), xb, yb)
    b = O.Case(O.make_params(m, m, 0.01, 100.0, 3, stationary=False, cgtol=1e-14), xb, yb)
    b.set_cg_relative(True)
    for _ in range(3):
        a.advance()
        rc, o = b.advance()
        assert rc == 0 and o["cg_iters"] > 0
    # A is slightly non-symmetric (vort2flux), choldc uses its upper half:
    # the two solves agree to the size of that asymmetry
    assert rel(b.get_state()["omega"], a.get_state()["omega"]) < 1e-4


def test_cg_maxiter_reports(oracle_mod):
    m = 32
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    b = O.Case(O.make_params(m, m, 0.01, 100.0, 3, stationary=False, cgtol=1e-30, cg_max_iter=2), xb, yb)
    rc, o = b.advance()
    assert rc == 3 and o["cg_iters"] == 2


def test_cn_update_identity(case32):
    """The Crank-Nicolson/AB2 level update as the reference evaluates it with
    its spectral tables (operators.f90:126-130, tables myfft.f90:46-69),
    w = dst(lam1i (dst(con1 rhs + con2 rold) + lam1 dst(omega))), solves
    (I + nu C^T C) w = (I - nu C^T C) omega + 1.5 dt/d^2 rhs - 0.5 dt/d^2 rold
    on every level (d = delta 2^(k-1), nu = dt / (2 Re d^2); no boundary terms)."""
    c = case32
    t = c.tables()
    rng = np.random.default_rng(7)
    dt, re = c.params.dt, c.params.re
    for k in range(c.nlev):
        lam1 = t["lam1"][k * c.ns:(k + 1) * c.ns]
        lam1i = t["lam1i"][k * c.ns:(k + 1) * c.ns]
        om, rhs, rold = (rng.standard_normal(c.ns) for _ in range(3))
        w = c.dst(lam1i * (c.dst(t["con1"][k] * rhs + t["con2"][k] * rold) + lam1 * c.dst(om)))
        d2 = (c.delta * 2.0 ** k) ** 2
        nu = 0.5 * dt / (re * d2)
        lhs = w + nu * laplacian(c, w)
        rhs_ = om - nu * laplacian(c, om) + 1.5 * dt / d2 * rhs - 0.5 * dt / d2 * rold
        assert rel(lhs, rhs_) < 1e-12, k
