"""Discrete-adjoint drivers over libns2d.so: a torch.autograd.Function for the
RK4CN flow map and a projected gradient-ascent search for extreme-enstrophy
initial conditions.

The C ABI returns W-gradients (dJ = sum_j c_j Re(conj(g_j) dw_j), c_j = 1 on
ky = 0 and ky = ny/2, 2 elsewhere).  torch's gradient of a real loss with
respect to a complex tensor is dL/dRe + i dL/dIm per entry, i.e. c * g; the
Function converts between the two.

The reference's own searches (Solver/src/solver.c:1775-1853, MAX_PALIN) read
their initial conditions from files; here the ascent computes them.
"""
import numpy as np

from . import abi
from .initial import wavenumbers, weights, energy, enstrophy

_torch = None


def _t():
    global _torch
    if _torch is None:
        import torch
        _torch = torch
    return _torch


def _weights_tensor(nx, nyf, device):
    torch = _t()
    c = torch.full((1, nyf), 2.0, dtype=torch.float64, device=device)
    c[0, 0] = 1.0
    c[0, nyf - 1] = 1.0
    return c


def _make_function():
    torch = _t()

    class FlowMap(torch.autograd.Function):
        """w(T) = flow map of nsteps RK4CN steps applied to w(0), on the GPU.

        Inputs and outputs: complex128 CUDA tensors [nx][ny/2+1] in the
        reference layout.  Backward runs the checkpointed reverse sweep."""

        @staticmethod
        def forward(ctx, w0, solver, nsteps, dt, checkpoint_every):
            if w0.dtype != torch.complex128 or not w0.is_cuda:
                raise TypeError("w0 must be a complex128 CUDA tensor")
            w0c = w0.detach().contiguous()
            solver.set_stream(torch.cuda.current_stream(w0c.device).cuda_stream)
            solver.set_w_hat_device(w0c.data_ptr())
            solver.adjoint_record(nsteps, dt, checkpoint_every)
            wT = torch.empty_like(w0c)
            solver.get_w_hat_device(wT.data_ptr())
            solver._record_id = getattr(solver, "_record_id", 0) + 1
            ctx.solver = solver
            ctx.record_id = solver._record_id
            return wT

        @staticmethod
        def backward(ctx, grad_out):
            solver = ctx.solver
            if getattr(solver, "_record_id", None) != ctx.record_id:
                raise RuntimeError("the solver recorded another run since this forward; "
                                   "one backward per forward on a solver")
            c = _weights_tensor(solver.nx, solver.nyf, grad_out.device)
            lam_T = (grad_out / c).contiguous()
            lam_0 = torch.empty_like(lam_T)
            solver.set_stream(torch.cuda.current_stream(lam_T.device).cuda_stream)
            solver.adjoint_backward_device(lam_T.data_ptr(), lam_0.data_ptr())
            return lam_0 * c, None, None, None, None

    return FlowMap


_FlowMap = None


def flow(w0, solver, nsteps, dt, checkpoint_every=50):
    """Differentiable w(T) for the torch tensor w0 (see FlowMap)."""
    global _FlowMap
    if _FlowMap is None:
        _FlowMap = _make_function()
    return _FlowMap.apply(w0, solver, nsteps, dt, checkpoint_every)


def enstrophy_t(w):
    """Enstrophy of a torch half spectrum (sys_msr.c:190-227, 356-363)."""
    torch = _t()
    nx, nyf = w.shape
    c = _weights_tensor(nx, nyf, w.device)
    ny = 2 * (nyf - 1)
    s = torch.sum(c * (w.real ** 2 + w.imag ** 2)) - (w[0, 0].real ** 2 + w[0, 0].imag ** 2)
    return 4.0 * np.pi ** 2 * 0.5 / float(nx * ny) ** 2 * s


# ---------------------------------------------------------------------------
# Projected gradient ascent on {E = E0, Z = Z0}


def _band_split(n):
    kx, ky = wavenumbers(n, n)
    return np.sqrt((kx * kx + ky * ky).astype(float))


def project(w, e0, z0):
    """Rescale two wavenumber bands of w so that E(w) = e0 and Z(w) = z0.  A
    mode's enstrophy-to-energy ratio is |k|^2, so splitting at |k|^2 = z0/e0
    puts the low band's ratio below the target and the high band's above it,
    and the two amplitudes solving the two quadratic constraints are real
    whenever both bands carry energy."""
    n = w.shape[0]
    k = _band_split(n)
    low = np.where(k * k < z0 / e0, w, 0.0)
    high = w - low
    eL, eH, zL, zH = energy(low), energy(high), enstrophy(low), enstrophy(high)
    det = eL * zH - eH * zL
    if det == 0.0:
        raise ValueError("degenerate spectrum: one band is empty")
    a2 = (e0 * zH - eH * z0) / det
    b2 = (eL * z0 - e0 * zL) / det
    if a2 <= 0.0 or b2 <= 0.0:
        raise ValueError("no positive rescaling reaches (E0, Z0)")
    return np.sqrt(a2) * low + np.sqrt(b2) * high


def tangent(g, w, e0_grad, z0_grad):
    """Component of g W-orthogonal to the gradients of E and Z at w."""
    def wdot(a, b):
        n = a.shape[0]
        return float(np.sum(weights(n, n) * (a.real * b.real + a.imag * b.imag)))
    basis = []
    for v in (e0_grad, z0_grad):
        for b in basis:
            v = v - wdot(b, v) * b
        nv = np.sqrt(wdot(v, v))
        if nv > 0:
            basis.append(v / nv)
    for b in basis:
        g = g - wdot(b, g) * b
    return g


def constraint_gradients(w):
    """W-gradients of E and Z at w."""
    n = w.shape[0]
    kx, ky = wavenumbers(n, n)
    k2 = (kx * kx + ky * ky).astype(float)
    cz = 4.0 * np.pi ** 2 * 0.5 / float(n * n) ** 2
    inv = np.where(k2 > 0, 1.0 / np.where(k2 > 0, k2, 1.0), 0.0)
    gz = 2.0 * cz * w
    gz[0, 0] = 0.0
    return 2.0 * cz * inv * w, gz


def projected_ascent(solver, w0, nsteps, dt, iters=20, step=None, e0=0.5, z0=10.0, checkpoint_every=50,
                     kind=abi.OBJ_ENSTROPHY, callback=None):
    """Maximise J(w(T)) over initial conditions with E = e0, Z = z0: gradient
    from the adjoint, projected on the constraint tangent, a step of length
    `step` (default 5% of |w| in the W norm, halved whenever J falls), then the
    rescaling of `project`.  Returns (w_best, [J per iteration])."""
    w = project(np.asarray(w0, np.complex128), e0, z0)
    hist = []
    J_prev = None
    def wnorm(a):
        n = a.shape[0]
        return float(np.sqrt(np.sum(weights(n, n) * np.abs(a) ** 2)))
    h = step
    best = (None, -np.inf)
    for it in range(iters):
        solver.set_w_hat(w)
        J, g = solver.adjoint_gradient(nsteps, dt, checkpoint_every, kind)
        hist.append(J)
        if callback:
            callback(it, J)
        if J > best[1]:
            best = (w.copy(), J)
        if J_prev is not None and J < J_prev and h is not None:
            h *= 0.5
        J_prev = J
        ge, gz = constraint_gradients(w)
        d = tangent(g, w, ge, gz)
        nd = wnorm(d)
        if nd == 0.0:
            break
        if h is None:
            h = 0.05 * wnorm(w)
        w = project(w + (h / nd) * d, e0, z0)
    return best[0], hist
