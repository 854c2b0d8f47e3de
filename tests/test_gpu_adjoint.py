"""Discrete adjoint on the GPU (ns2d_adjoint_*): gradients against the CPU
restatement (oracle/adjoint_ref.py), against the tangent-linear fixture built on
the reference's own RHS, against central differences of the GPU forward, and
through the torch.autograd.Function."""
import os

import numpy as np
import pytest

import adjoint_ref as ar
from _util import GOLDEN, rel_err
from ns2d import NS2DError, Solver, abi, initial
from ns2d import adjoint as nadj

pytestmark = pytest.mark.gpu


def _params(n, **kw):
    base = dict(nx=n, ny=n, nu=1e-3, quirks=0)
    base.update(kw)
    return abi.default_params(**base)


def _cpu_model(p):
    from pyoracle import Oracle
    kolm = p.forcing == abi.FORCING_KOLM
    forcing = None
    if kolm:
        o = Oracle(p)
        o.compute_forcing(p.dt)
        forcing = o.nonlinear_rhs(np.zeros((p.nx, p.nx // 2 + 1), np.complex128))
    return ar.Model(p.nx, ar.bracket_for(p, latch=bool(p.quirks & abi.QUIRK_HYPER_LATCH)), dealias=p.dealias,
                    kolm=kolm, houli_int=bool(p.quirks & abi.QUIRK_HOU_LI_INT), forcing=forcing)


@pytest.mark.parametrize("n,steps,every", [(16, 6, 4), (32, 9, 4), (64, 30, 7), (128, 8, 3), (256, 5, 2),
                                           (512, 3, 2), (1024, 2, 1)])
def test_gradient_matches_cpu_restatement(n, steps, every):
    p = _params(n)
    dt = 2e-3 if n <= 128 else 5e-4
    w0 = initial.decaying(n, 31, k0=4.0, dealias="2/3")
    s = Solver(p)
    s.set_w_hat(w0)
    J, g = s.adjoint_gradient(steps, dt, every)
    Jc, gc = _cpu_model(p).gradient(w0, steps, dt, checkpoint_every=every)
    assert abs(J - Jc) <= 1e-12 * abs(Jc)
    assert rel_err(g, gc) <= 1e-11
    # the state is left at w(T)
    wT = w0
    m = _cpu_model(p)
    for _ in range(steps):
        wT, _ = m.step(wT, dt)
    assert rel_err(s.get_w_hat(), wT) <= 1e-12


def test_hou_li_kolmogorov_palinstrophy():
    p = _params(64, dealias=abi.DEALIAS_HOU_LI, quirks=abi.QUIRK_HOU_LI_INT | abi.QUIRK_HYPER_LATCH,
                forcing=abi.FORCING_KOLM, force_k=4)
    w0 = initial.noise(64, 9, amplitude=1.0, kolm=False)
    s = Solver(p)
    s.set_w_hat(w0)
    J, g = s.adjoint_gradient(12, 2e-3, 5, abi.OBJ_PALINSTROPHY)
    Jc, gc = _cpu_model(p).gradient(w0, 12, 2e-3, "palinstrophy", checkpoint_every=5)
    assert abs(J - Jc) <= 1e-12 * abs(Jc)
    assert rel_err(g, gc) <= 1e-11


def test_reference_tangent_linear_fixture():
    z = np.load(os.path.join(GOLDEN, "adjoint32_tl.npz"))
    p = abi.params_from_arrays(z["param_names"], z["params"])
    nsteps = int(z["nsteps"])
    for kind, key, dkey in ((abi.OBJ_ENSTROPHY, "Z", "dZ"), (abi.OBJ_PALINSTROPHY, "P", "dP")):
        s = Solver(p)
        s.set_w_hat(z["w0"])
        J, g = s.adjoint_gradient(nsteps, p.dt, 10, kind)
        assert abs(J - float(z[key])) <= 1e-12 * abs(J)
        ref = z[dkey]
        for i, d in enumerate(z["dirs"]):
            assert abs(ar.wdot(g, d) - ref[i]) <= 1e-10 * np.abs(ref).max()
        s.close()


def test_central_differences():
    """Central differences (eps = 1e-6) of the GPU forward along 16 seeded
    directions agree with <g, d>_W to 1e-6."""
    n, steps, dt = 128, 40, 2e-3
    p = _params(n)
    w0 = nadj.project(initial.decaying(n, 41, k0=4.0, dealias="2/3"), 0.5, 10.0)
    s = Solver(p)
    s.set_w_hat(w0)
    J, g = s.adjoint_gradient(steps, dt, 10)
    rng_dirs = [ar.random_field(n, 500 + i, kmax=n / 3.0) for i in range(16)]
    wn = np.sqrt(ar.wdot(w0, w0))
    eps = 1e-6
    for d in rng_dirs:
        d = d * (wn / np.sqrt(ar.wdot(d, d)))
        vals = []
        for sgn in (1.0, -1.0):
            s.set_w_hat(w0 + sgn * eps * d)
            s.step_n(steps, dt)
            vals.append(s.objective(abi.OBJ_ENSTROPHY))
        fd = (vals[0] - vals[1]) / (2 * eps)
        assert abs(fd - ar.wdot(g, d)) <= 1e-6 * abs(fd)


def test_central_differences_512():
    """The gradient workload's grid and step (512^2, nu = 1e-3, dt = 5e-4,
    checkpoints every 50 steps, w0 with E = 0.5 and Z = 10) over a 200-step
    horizon, 16 seeded directions, central differences with eps = 1e-5 and
    1e-6 (|d|_W = |w0|_W), the better of the two kept.  Enforced:
    |FD - <g, d>_W| <= 1e-9 |g|_W |d|_W on every direction (a difference of two
    objective values carries about 1e-16 J / eps of rounding, which swamps the
    relative error of a direction nearly orthogonal to g), and the relative
    error <= 1e-6 on directions with |<g, d>_W| >= 1e-2 |g|_W |d|_W."""
    n, steps, dt = 512, 200, 5e-4
    p = _params(n)
    w0 = nadj.project(initial.decaying(n, 50, k0=4.0, dealias="2/3"), 0.5, 10.0)
    s = Solver(p)
    s.set_w_hat(w0)
    J, g = s.adjoint_gradient(steps, dt, 50)
    gn = np.sqrt(ar.wdot(g, g))
    wn = np.sqrt(ar.wdot(w0, w0))
    rng = np.random.default_rng(900)
    for _ in range(16):
        d = initial.dealias_23(initial.hermitian(rng.standard_normal(w0.shape) + 1j * rng.standard_normal(w0.shape)))
        d *= wn / np.sqrt(ar.wdot(d, d))
        ad = ar.wdot(g, d)
        errs = []
        for eps in (1e-5, 1e-6):
            vals = []
            for sgn in (1.0, -1.0):
                s.set_w_hat(w0 + sgn * eps * d)
                s.step_n(steps, dt)
                vals.append(s.objective(abi.OBJ_ENSTROPHY))
            errs.append(abs((vals[0] - vals[1]) / (2 * eps) - ad))
        err = min(errs)
        assert err <= 1e-9 * gn * wn, (err / (gn * wn), ad / (gn * wn))
        if abs(ad) >= 1e-2 * gn * wn:
            assert err <= 1e-6 * abs(ad), (err / abs(ad), ad / (gn * wn))
    s.close()


def test_checkpoint_interval_is_bitwise_neutral():
    n, steps, dt = 64, 12, 2e-3
    p = _params(n)
    w0 = initial.decaying(n, 7, k0=4.0, dealias="2/3")
    grads = []
    for every in (1, 5, 12, 50):
        s = Solver(p)
        s.set_w_hat(w0)
        grads.append(s.adjoint_gradient(steps, dt, every)[1])
        s.close()
    for g in grads[1:]:
        assert np.array_equal(g, grads[0])


def test_record_then_backward_matches_gradient():
    n, steps, dt = 64, 10, 2e-3
    p = _params(n)
    w0 = initial.decaying(n, 8, k0=4.0, dealias="2/3")
    s = Solver(p)
    s.set_w_hat(w0)
    J, g = s.adjoint_gradient(steps, dt, 4)
    s.set_w_hat(w0)
    s.adjoint_record(steps, dt, 4)
    wT = s.get_w_hat()
    lam_T = 2.0 * 4.0 * np.pi ** 2 * 0.5 / float(n * n) ** 2 * wT
    lam_T[0, 0] = 0.0
    g2 = s.adjoint_backward(lam_T)
    assert rel_err(g2, g) <= 1e-14
    # a second backward over the same record gives the same result
    assert np.array_equal(s.adjoint_backward(lam_T), g2)


def test_fp32_adjoint():
    n, steps, dt = 128, 20, 2e-3
    w0 = initial.decaying(n, 12, k0=4.0, dealias="2/3")
    out = {}
    for prec in (abi.FP64, abi.FP32):
        s = Solver(_params(n, precision=prec))
        s.set_w_hat(w0)
        out[prec] = s.adjoint_gradient(steps, dt, 5)
    J64, g64 = out[abi.FP64]
    J32, g32 = out[abi.FP32]
    assert abs(J32 - J64) <= 1e-5 * abs(J64)
    assert rel_err(g32, g64) <= 1e-4


def test_torch_function():
    torch = pytest.importorskip("torch")
    n, steps, dt = 64, 10, 2e-3
    p = _params(n)
    w0 = initial.decaying(n, 13, k0=4.0, dealias="2/3")
    s = Solver(p)
    s.set_w_hat(w0)
    J, g = s.adjoint_gradient(steps, dt, 4)
    s2 = Solver(p)
    w = torch.tensor(w0, dtype=torch.complex128, device="cuda", requires_grad=True)
    wT = nadj.flow(w, s2, steps, dt, 4)
    Z = nadj.enstrophy_t(wT)
    Z.backward()
    assert abs(Z.item() - J) <= 1e-12 * abs(J)
    c = initial.weights(n, n)
    assert rel_err(w.grad.cpu().numpy(), c * g) <= 1e-13
    # a stale record is refused
    w2 = torch.tensor(w0, dtype=torch.complex128, device="cuda", requires_grad=True)
    wa = nadj.flow(w2, s2, steps, dt, 4)
    nadj.flow(w2.detach().clone().requires_grad_(True), s2, steps, dt, 4)
    with pytest.raises(RuntimeError):
        nadj.enstrophy_t(wa).backward()


def test_ascent_increases_final_enstrophy():
    n, steps, dt = 64, 20, 5e-3
    s = Solver(_params(n))
    w0 = initial.decaying(n, 17, k0=4.0)
    wbest, hist = nadj.projected_ascent(s, w0, steps, dt, iters=6, e0=0.5, z0=10.0, checkpoint_every=10)
    assert hist[-1] > hist[0]
    assert abs(initial.energy(wbest) - 0.5) <= 1e-12 and abs(initial.enstrophy(wbest) - 10.0) <= 1e-10


def test_unsupported_configurations():
    n = 32
    w0 = initial.decaying(n, 1, k0=4.0, dealias="2/3")
    for kw in (dict(quirks=abi.QUIRKS_REFERENCE), dict(integrator=abi.AB4), dict(integrator=abi.RK4)):
        s = Solver(_params(n, **kw))
        s.set_w_hat(w0)
        with pytest.raises(NS2DError) as e:
            s.adjoint_gradient(2, 1e-3, 1)
        assert e.value.status == abi.ERR_UNSUPPORTED
    s = Solver(_params(n))
    with pytest.raises(NS2DError) as e:
        s.adjoint_backward(np.zeros((n, n // 2 + 1), np.complex128))
    assert e.value.status == abi.ERR_STATE
