"""The column passes' two ways of moving tiles give the same numbers.

For the common step the first, stage and final column passes bring their
tiles in and out with TMA copies; with NS2D_DISABLE_TMA set when a handle or
ensemble is created they copy per thread instead (the fallback when the
driver offers no tensor-map encoder).  The arithmetic is the same source in
both forms, but the two kernels are compiled separately and may contract
multiply-adds differently, so the states after several steps agree to
rounding: 1e-13 of max|w_hat| in FP64, 1e-5 in FP32, for a single field
(including the 1024^2 Kolmogorov workload of the benchmark) and for a batched
ensemble."""
import os

import pytest

from _util import rel_err
from ns2d import Ensemble, Solver, abi, initial

TOL = {abi.FP64: 1e-13, abi.FP32: 1e-5}

pytestmark = pytest.mark.gpu


def _with_tma(enabled, make):
    if enabled:
        return make()
    os.environ["NS2D_DISABLE_TMA"] = "1"
    try:
        return make()
    finally:
        del os.environ["NS2D_DISABLE_TMA"]


def _steps(params, w0, nsteps, dt, tma):
    s = _with_tma(tma, lambda: Solver(params))
    try:
        s.set_w_hat(w0)
        s.step_n(nsteps, dt)
        return s.get_w_hat()
    finally:
        s.close()


@pytest.mark.parametrize("n,precision", [(16, abi.FP64), (32, abi.FP32), (256, abi.FP64), (512, abi.FP32),
                                         (1024, abi.FP32), (2048, abi.FP64)])
def test_single_field_tma_equals_per_thread_copies(n, precision):
    p = abi.default_params(nx=n, ny=n, nu=1e-3, dt=1e-3, precision=precision)
    w0 = initial.decaying(n, seed=11, k0=max(2.0, 4.0 * n / 128.0), dealias="2/3")
    a = _steps(p, w0, 6, 1e-3, True)
    b = _steps(p, w0, 6, 1e-3, False)
    err = rel_err(a, b)
    assert err <= TOL[precision], err


def test_kolmogorov_1024_fp64_tma_equals_per_thread_copies():
    """The benchmark's workload: KOLM forcing n = 4, hyperviscosity through the
    drag branch, dt = 2.5e-4."""
    n = 1024
    p = abi.default_params(nx=n, ny=n, nu=1e-4, ekmn_drag_flag=1, ekmn_alpha=2e-40, ekmn_drag_pow=8.0,
                           forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0, dt=2.5e-4)
    w0 = initial.noise(n, seed=7, amplitude=1e-3, kolm=True)
    a = _steps(p, w0, 5, 2.5e-4, True)
    b = _steps(p, w0, 5, 2.5e-4, False)
    err = rel_err(a, b)
    assert err <= TOL[abi.FP64], err


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32])
def test_ensemble_tma_equals_per_thread_copies(precision):
    sizes = [64, 128, 256, 512, 128]
    p = abi.default_params(nu=1e-3, dt=1e-3, precision=precision)
    ics = [initial.decaying(n, seed=30 + m, k0=4.0 * n / 128.0, dealias="2/3") for m, n in enumerate(sizes)]
    out = []
    for tma in (True, False):
        e = _with_tma(tma, lambda: Ensemble(p, sizes))
        try:
            for m, w in enumerate(ics):
                e.set_w_hat(m, w)
            e.step_n(6, 1e-3)
            out.append([e.get_w_hat(m) for m in range(len(sizes))])
        finally:
            e.close()
    for m in range(len(sizes)):
        err = rel_err(out[0][m], out[1][m])
        assert err <= TOL[precision], (m, err)
