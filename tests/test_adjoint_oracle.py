"""CPU checks of the discrete-adjoint restatement (oracle/adjoint_ref.py) and of
the host-side ascent helpers; no GPU.

The restatement is pinned three ways: its forward RHS against the oracle (itself
bit-exact with the reference's NonlinearRHSBatch), its transposes by dot-product
identities, and its gradients against the tangent-linear fixture built on the
reference's own compiled RHS (tests/golden/make_golden.py, adjoint32_tl)."""
import os

import numpy as np
import pytest

import adjoint_ref as ar
from _util import GOLDEN
from ns2d import abi, initial
from ns2d import adjoint as nadj
from pyoracle import Oracle


def _herm(n, seed, kmax=None):
    return ar.random_field(n, seed, kmax=kmax)


def test_c2r_is_transpose_of_r2c():
    n = 32
    rng = np.random.default_rng(0)
    f = rng.standard_normal((n, n))
    for X in (_herm(n, 1), rng.standard_normal((n, n // 2 + 1)) + 1j * rng.standard_normal((n, n // 2 + 1))):
        a = ar.wdot(ar.r2c(f), X)
        b = float(np.sum(f * ar.c2r(X)))
        assert abs(a - b) <= 1e-12 * max(abs(a), 1.0)


@pytest.mark.parametrize("case", ["23", "houli", "kolm"])
def test_numpy_rhs_matches_oracle(case):
    n = 32
    kw = dict(nx=n, ny=n, nu=1e-3, quirks=0)
    if case == "houli":
        kw.update(dealias=abi.DEALIAS_HOU_LI, quirks=abi.QUIRK_HOU_LI_INT)
    if case == "kolm":
        kw.update(forcing=abi.FORCING_KOLM, force_k=4)
    p = abi.default_params(**kw)
    o = Oracle(p)
    o.compute_forcing(p.dt)
    X = _herm(n, 3, kmax=12)
    f = o.nonlinear_rhs(np.zeros_like(X))
    m = ar.Model(n, ar.bracket_for(p), dealias=p.dealias, kolm=(case == "kolm"),
                 houli_int=(case == "houli"), forcing=f)
    r = o.nonlinear_rhs(X)
    assert np.abs(r - m.rhs(X)).max() <= 1e-13 * np.abs(r).max()


def test_numpy_step_matches_oracle():
    n = 32
    p = abi.default_params(nx=n, ny=n, nu=1e-3, quirks=0)
    o = Oracle(p)
    X = _herm(n, 4, kmax=10)
    o.set_w_hat(X)
    o.rk4_step(1e-3)
    m = ar.Model(n, ar.bracket_for(p))
    w1, _ = m.step(X, 1e-3)
    assert np.abs(o.get_w_hat() - w1).max() <= 1e-14 * np.abs(w1).max()


@pytest.mark.parametrize("dealias", [0, 1])
def test_rhs_adjoint_dot_product(dealias):
    n = 32
    m = ar.Model(n, lambda k2: 1e-3 * k2, dealias=dealias)
    X, kappa = _herm(n, 5, kmax=12), _herm(n, 6)
    rng = np.random.default_rng(7)
    for dX in (_herm(n, 8), rng.standard_normal(X.shape) + 1j * rng.standard_normal(X.shape)):
        a = ar.wdot(kappa, m.rhs_tl(X, dX))
        b = ar.wdot(m.rhs_adj(X, kappa), dX)
        assert abs(a - b) <= 1e-12 * abs(a)
    # the tangent-linear equals polarisation of the nonlinear RHS
    dX = _herm(n, 9)
    t1 = m.rhs_tl(X, dX)
    t2 = ar.tl_rhs_polar(m.rhs)(X, dX)
    assert np.abs(t1 - t2).max() <= 1e-13 * np.abs(t1).max()


def test_step_adjoint_dot_product():
    n = 32
    m = ar.Model(n, lambda k2: 1e-3 * k2 + 1e-12 * k2 ** 4)
    w = _herm(n, 10, kmax=10)
    _, X = m.step(w, 2e-3)
    lam, dw = _herm(n, 11), _herm(n, 12)
    a = ar.wdot(lam, m.step_tl(X, dw, 2e-3))
    b = ar.wdot(m.step_adj(X, lam, 2e-3), dw)
    assert abs(a - b) <= 1e-12 * abs(a)


@pytest.mark.parametrize("kind", ["enstrophy", "palinstrophy"])
def test_gradient_against_central_differences(kind):
    n, dt, steps = 32, 2e-3, 8
    m = ar.Model(n, lambda k2: 1e-3 * k2)
    w0 = _herm(n, 13, kmax=8) * 50.0
    J, g = m.gradient(w0, steps, dt, kind, checkpoint_every=3)

    def J_of(w):
        for _ in range(steps):
            w, _ = m.step(w, dt)
        return m.objective(w, kind)[0]

    for s in range(3):
        d = _herm(n, 20 + s, kmax=10) * 50.0
        eps = 1e-6
        fd = (J_of(w0 + eps * d) - J_of(w0 - eps * d)) / (2 * eps)
        assert abs(fd - ar.wdot(g, d)) <= 1e-6 * abs(fd)


def test_checkpoint_interval_does_not_change_gradient():
    n, dt, steps = 32, 2e-3, 7
    m = ar.Model(n, lambda k2: 1e-3 * k2)
    w0 = _herm(n, 14, kmax=8) * 50.0
    _, g1 = m.gradient(w0, steps, dt, checkpoint_every=1)
    _, g7 = m.gradient(w0, steps, dt, checkpoint_every=7)
    _, g3 = m.gradient(w0, steps, dt, checkpoint_every=3)
    assert np.array_equal(g1, g7) and np.array_equal(g1, g3)


def test_restatement_matches_reference_tangent_linear_fixture():
    z = np.load(os.path.join(GOLDEN, "adjoint32_tl.npz"))
    p = abi.params_from_arrays(z["param_names"], z["params"])
    m = ar.Model(p.nx, ar.bracket_for(p))
    nsteps = int(z["nsteps"])
    Z, gZ = m.gradient(z["w0"], nsteps, p.dt, "enstrophy", checkpoint_every=10)
    P, gP = m.gradient(z["w0"], nsteps, p.dt, "palinstrophy", checkpoint_every=10)
    assert abs(Z - float(z["Z"])) <= 1e-12 * abs(Z)
    assert abs(P - float(z["P"])) <= 1e-12 * abs(P)
    for i, d in enumerate(z["dirs"]):
        assert abs(ar.wdot(gZ, d) - z["dZ"][i]) <= 1e-10 * np.abs(z["dZ"]).max()
        assert abs(ar.wdot(gP, d) - z["dP"][i]) <= 1e-10 * np.abs(z["dP"]).max()


def test_projection_onto_energy_and_enstrophy():
    w = initial.decaying(128, 5, k0=4.0)
    p = nadj.project(w, 0.5, 10.0)
    assert abs(initial.energy(p) - 0.5) <= 1e-12 and abs(initial.enstrophy(p) - 10.0) <= 1e-11
    ge, gz = nadj.constraint_gradients(p)
    g = initial.hermitian(np.random.default_rng(1).standard_normal(p.shape) + 0j)
    d = nadj.tangent(g, p, ge, gz)
    c = initial.weights(128, 128)
    wd = lambda a, b: float(np.sum(c * (a.real * b.real + a.imag * b.imag)))  # noqa: E731
    assert abs(wd(d, ge)) <= 1e-12 * np.sqrt(wd(g, g) * wd(ge, ge))
    assert abs(wd(d, gz)) <= 1e-12 * np.sqrt(wd(g, g) * wd(gz, gz))
    # E and Z gradients are those of the measurables' formulas
    d = g * np.sqrt(wd(p, p) / wd(g, g))
    eps = 1e-6
    for f, gr in ((initial.energy, ge), (initial.enstrophy, gz)):
        fd = (f(p + eps * d) - f(p - eps * d)) / (2 * eps)
        assert abs(fd - wd(gr, d)) <= 1e-6 * abs(fd)
