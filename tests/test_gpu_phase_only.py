"""The phase-only model on the GPU (ns2d_params.model = NS2D_MODEL_PHASE_ONLY;
RK4Step's amplitude reset, Solver/src/solver.c:634-647, 822-824, 855-857)
against the oracle restatement, which the po32_* golden fixtures pin to the
reference's -D__PHASE_ONLY build; the small fixtures themselves run in
test_gpu_parity.py.  FP64 tolerance 1e-12 of max|w_hat|, FP32 1e-4.
At 1024^2 the size-independent property: every mode keeps its amplitude."""
import numpy as np
import pytest

from _util import rel_err
from ns2d import Solver, abi, initial
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kw", [
    dict(),
    dict(integrator=abi.RK4, ekmn_drag_flag=1),
    dict(dealias=abi.DEALIAS_HOU_LI, nu=5e-4),
    dict(forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0),
    dict(quirks=0, hyper_visc_flag=1, ekmn_drag_flag=1, ekmn_alpha=0.1),
])
def test_phase_only_steps_match_oracle(kw):
    n, dt, steps = 128, 1e-3, 20
    kw = dict(kw)
    p = abi.default_params(nx=n, ny=n, nu=kw.pop("nu", 1e-3), dt=dt, model=abi.MODEL_PHASE_ONLY, **kw)
    w0 = initial.decaying(n, seed=41, k0=6.0, dealias="2/3")
    o = Oracle(p)
    o.set_w_hat(w0)
    for _ in range(steps):
        o.rk4_step(dt)
    want = o.get_w_hat()
    a, b = Solver(p), Solver(p)
    a.set_w_hat(w0)
    b.set_w_hat(w0)
    for _ in range(steps):
        a.rk4_step(dt)            # per-call steps (graph replay after the first)
    b.step_n(steps, dt)           # batched steps (one captured graph)
    assert rel_err(a.get_w_hat(), want) <= 1e-12
    assert np.array_equal(a.get_w_hat(), b.get_w_hat())
    a.close()
    b.close()


def test_phase_only_changes_the_step():
    """The reset is applied: the full model's step differs, the amplitudes
    of the phase-only one do not."""
    n, dt = 64, 1e-3
    w0 = initial.decaying(n, seed=42, k0=5.0, dealias="2/3")
    out = {}
    for model in (abi.MODEL_FULL, abi.MODEL_PHASE_ONLY):
        s = Solver(abi.default_params(nx=n, ny=n, nu=1e-2, dt=dt, quirks=0, model=model))
        s.set_w_hat(w0)
        s.step_n(5, dt)
        out[model] = s.get_w_hat()
        s.close()
    a0 = np.abs(w0)
    a0[0, 0] = 0
    assert np.abs(np.abs(out[abi.MODEL_FULL]) - a0).max() > 1e-6 * a0.max()
    assert np.abs(np.abs(out[abi.MODEL_PHASE_ONLY]) - a0).max() <= 1e-13 * a0.max()


def test_phase_only_1024_amplitudes_conserved():
    """1024^2, 200 steps: with the corrected conjugacy (the quirk rewrites the
    state's ky = 0, kx < 0 modes from the stage input) every mode's amplitude
    is that of the start, the 2/3-zeroed modes stay exactly 0 and the state
    stays finite."""
    n, dt = 1024, 1e-4
    p = abi.default_params(nx=n, ny=n, nu=1e-4, dt=dt, quirks=0, model=abi.MODEL_PHASE_ONLY)
    w0 = initial.decaying(n, seed=43, k0=20.0, dealias="2/3")
    s = Solver(p)
    s.set_w_hat(w0)
    s.step_n(200, dt)
    w = s.get_w_hat()
    s.close()
    assert np.isfinite(w).all()
    a0 = np.abs(w0)
    a0[0, 0] = 0
    assert np.abs(np.abs(w) - a0).max() <= 1e-12 * a0.max()
    assert np.all(w[a0 == 0] == 0)
    assert np.abs(np.angle(w[a0 > 0]) - np.angle(w0[a0 > 0])).max() > 1e-3  # phases evolved


def test_phase_only_fp32():
    n, dt = 256, 1e-3
    w0 = initial.decaying(n, seed=44, k0=8.0, dealias="2/3")
    out = []
    for prec in (abi.FP64, abi.FP32):
        s = Solver(abi.default_params(nx=n, ny=n, nu=1e-3, dt=dt, precision=prec, model=abi.MODEL_PHASE_ONLY))
        s.set_w_hat(w0)
        s.step_n(50, dt)
        out.append(s.get_w_hat())
        s.close()
    assert rel_err(out[1], out[0]) <= 1e-4


def test_phase_only_rejects_other_steps():
    n = 64
    s = Solver(abi.default_params(nx=n, ny=n, model=abi.MODEL_PHASE_ONLY))
    s.set_w_hat(initial.decaying(n, seed=45, k0=5.0, dealias="2/3"))
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        s.ab4_step(1e-3, 1)
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        s.dp5_step(1e-3)
    s.close()
    a = Solver(abi.default_params(nx=n, ny=n, quirks=0, model=abi.MODEL_PHASE_ONLY))
    with pytest.raises(RuntimeError, match="UNSUPPORTED"):
        a.adjoint_record(4, 1e-3)
    a.close()
