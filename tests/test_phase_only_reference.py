"""The phase-only model of the reference (Solver/Makefile:58, -D__PHASE_ONLY;
RK4Step's amplitude reset, Solver/src/solver.c:634-647, 822-824, 855-857)
built from its own sources (oracle/_ref/libns2d_ref_{rk4cn,houli}_po.so)
against the oracle restatement, one step from a seeded state.

The reference's reset `w *= |w_before| / |w_after|` divides 0 by 0 wherever
the update is exactly 0, which leaves NaN in every mode the 2/3 rule zeroes
and, with Hou-Li dealiasing, at the corner kx = ky = N/2 where the filter
underflows; the next transform spreads it to every mode.  The restatement
(and the CUDA path) keep those modes at 0 and agree with the reference on all
others.  Multi-step parity, with the reference's NaN modes set to 0 between
steps, is pinned by the po32_* golden fixtures."""
import os

import numpy as np
import pytest

from _util import make_golden
from ns2d import abi, initial
from pyoracle import Oracle, RefSolver

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libns2d_ref_{}.so")


@pytest.mark.parametrize("variant,kw,dealias", [
    ("rk4cn_po", dict(), "2/3"),
    ("houli_po", dict(dealias=abi.DEALIAS_HOU_LI, nu=5e-4), None),
])
def test_reference_phase_only_step(variant, kw, dealias):
    if not os.path.exists(REF_SO.format(variant)):
        pytest.skip("phase-only reference build absent (oracle/Makefile ref)")
    n, dt = 32, 1e-3
    kw = dict(kw)
    p = abi.default_params(nx=n, ny=n, nu=kw.pop("nu", 1e-3), model=abi.MODEL_PHASE_ONLY, dt=dt, **kw)
    w0 = initial.decaying(n, seed=31, k0=4.0, dealias=dealias)
    if dealias is None:
        w0 = w0 * make_golden.houli_filter_int(n)  # the Hou-Li build's initial filter
    ref = RefSolver(p, variant)
    ref.set_w_hat(w0)
    ref.rk4_step(dt)
    got_ref = ref.get_w_hat()
    o = Oracle(p)
    o.set_w_hat(w0)
    o.rk4_step(dt)
    got = o.get_w_hat()

    nan = np.isnan(got_ref)
    assert nan.any()                       # the reference's 0/0 is exercised
    assert np.all(got[nan] == 0)           # kept at 0 here
    fin = ~nan
    scale = np.abs(got_ref[fin]).max()
    assert np.abs(got[fin] - got_ref[fin]).max() <= 1e-15 * scale
    # amplitudes are those of the state before the step (mode (0,0) is zeroed).
    # Not on ky = 0, kx < 0: there the state was overwritten during the step by
    # ForceConjugacy of the last stage's input (solver.c:1031, 2096-2103) and
    # the reset keeps that value's amplitude.
    a0, a1 = np.abs(w0), np.abs(got)
    a0[0, 0] = 0.0
    keep = a1 > 0
    keep[n // 2 + 1:, 0] = False
    assert np.allclose(a1[keep], a0[keep], rtol=1e-14, atol=0)
    if dealias == "2/3":
        kx = np.fft.fftfreq(n, 1.0 / n).astype(int)
        ky = np.arange(n // 2 + 1)
        k2 = kx[:, None] ** 2 + ky[None, :] ** 2
        assert np.array_equal(nan, k2 >= (n // 3) ** 2)
    else:
        assert np.argwhere(nan).tolist() == [[n // 2, n // 2]]
