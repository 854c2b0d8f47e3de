"""Forcing of listed modes (ns2d_set_forcing_modes): the values the reference's
stochastic forcings draw on the host (force.c:104-433) are added to every RHS
at their modes and nowhere else; measurables report the forcing input."""
import numpy as np
import pytest

from _util import rel_err
from ns2d import Solver, abi, initial

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,tol", [(abi.FP64, 1e-13), (abi.FP32, 1e-5)])
def test_listed_forcing_adds_to_rhs(prec, tol):
    n = 64
    p = abi.default_params(nx=n, ny=n, nu=1e-3, quirks=0, precision=prec)
    w0 = initial.decaying(n, 3, k0=4.0, dealias="2/3")
    s = Solver(p)
    s.set_w_hat(w0)
    r0 = s.nonlinear_rhs(None)
    rng = np.random.default_rng(5)
    idx = np.array([1 * 33 + 4, 5 * 33 + 2, 60 * 33 + 7, 3], np.int32)
    val = (rng.standard_normal(4) + 1j * rng.standard_normal(4)) * np.abs(r0).max()
    s.set_forcing_modes(idx, val)
    r1 = s.nonlinear_rhs(None)
    d = (r1 - r0).ravel()
    want = np.zeros_like(d)
    want[idx] = val
    assert np.abs(d - want).max() <= tol * np.abs(r0).max() * 10
    m, _ = s.system_measurables()
    assert m[3] > 0.0  # forcing input
    s.set_forcing_modes([], [])
    assert rel_err(s.nonlinear_rhs(None), r0) <= tol


def test_listed_forcing_in_graph_loop_matches_eager():
    n = 64
    p = abi.default_params(nx=n, ny=n, nu=1e-3)
    w0 = initial.decaying(n, 4, k0=4.0, dealias="2/3")
    idx = np.array([2 * 33 + 3, 40 * 33 + 5], np.int32)
    a, b = Solver(p), Solver(p)
    for s in (a, b):
        s.set_w_hat(w0)
    b.step_n(3, 1e-3)                     # graph captured without forcing
    for k in range(3):
        a.rk4_step(1e-3)
    for k in range(4):
        val = np.array([1.0 + 0.5j * k, -0.3 + 0.1j], np.complex128) * 1e3
        a.set_forcing_modes(idx, val)
        b.set_forcing_modes(idx, val)
        a.rk4_step(1e-3)
        b.step_n(2, 1e-3) if k == 3 else b.step_n(1, 1e-3)
        if k == 3:
            a.rk4_step(1e-3)
    assert np.array_equal(a.get_w_hat(), b.get_w_hat())
