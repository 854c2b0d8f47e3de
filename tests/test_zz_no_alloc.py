"""ns2d_nonlinear_rhs_noalloc: the nonlinear term for callers that cannot
allocate device memory (inside someone else's stream capture, in loops that
cannot take cudaMalloc's device-wide synchronisation, or under an application
memory pool).  The entry point keeps its intermediates in a static device array
and allocates nothing; the caller passes device input and output arrays.

Checked through the C ABI against the handle-based ns2d_nonlinear_rhs on two
calls in a row (different inputs, so stale scratch contents from the first call
would show up in the second), with the single-RHS tolerance of the parity tests
(1e-13 of max|RHS|).  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from ns2d import Solver, abi, initial, load

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-13


def _noalloc(L, p, d_in, d_out, stream):
    f = L.ns2d_nonlinear_rhs_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Params), C.c_void_p, C.c_void_p, C.c_void_p]
    return f(C.byref(p), C.c_void_p(d_in), C.c_void_p(d_out), C.c_void_p(stream))


@pytest.mark.parametrize("n,kw", [(128, {}), (256, dict(forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0))])
def test_noalloc_rhs_matches_handle_rhs_twice(n, kw):
    import torch

    L = load()
    p = abi.default_params(nx=n, ny=n, nu=1e-3, **kw)
    s = Solver(p)
    s.compute_forcing(p.dt)
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (31, 32):
        w = initial.decaying(n, seed=seed, k0=6.0, dealias="2/3")
        expect = s.nonlinear_rhs(w)
        d_in = torch.from_numpy(w.view(np.float64).copy()).cuda()
        d_out = torch.full_like(d_in, float("nan"))
        assert _noalloc(L, p, d_in.data_ptr(), d_out.data_ptr(), stream) == abi.OK
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.complex128).reshape(n, n // 2 + 1)
        err = np.max(np.abs(got - expect)) / np.max(np.abs(expect))
        assert err <= RHS_TOL, (n, seed, err)
        # the input array is read only
        assert np.array_equal(d_in.cpu().numpy(), w.view(np.float64))
    s.close()


def test_noalloc_rejects_sizes_above_limit():
    import torch

    L = load()
    for n in (512, 1024, 96):
        p = abi.default_params(nx=n, ny=n)
        d = torch.zeros(2 * n * (n // 2 + 1), dtype=torch.float64, device="cuda")
        assert _noalloc(L, p, d.data_ptr(), d.data_ptr(), 0) == abi.ERR_UNSUPPORTED
    p = abi.default_params(nx=128, ny=64)
    assert _noalloc(L, p, 0, 0, 0) in (abi.ERR_INVALID, abi.ERR_UNSUPPORTED)
