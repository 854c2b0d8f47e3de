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


@pytest.mark.parametrize("n", [16, 32, 64])
def test_noalloc_rhs_recorded_in_a_captured_graph_houli(n):
    """The use the entry point exists for: a caller that records the call into
    its own CUDA graph.  One call outside the capture does the per-device
    set-up; the call recorded inside torch.cuda.graph is then replayed on new
    input placed in the captured buffer, and equals the handle's RHS (Hou-Li
    dealiasing, the small grids with their own tile shapes)."""
    import torch

    L = load()
    p = abi.default_params(nx=n, ny=n, nu=1e-3, dealias=abi.DEALIAS_HOU_LI)
    s = Solver(p)
    nyf = n // 2 + 1
    d_in = torch.zeros(2 * n * nyf, dtype=torch.float64, device="cuda")
    d_out = torch.zeros_like(d_in)
    assert _noalloc(L, p, d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream) == abi.OK
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        rc = _noalloc(L, p, d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == abi.OK
    for seed in (41, 42):
        w = initial.decaying(n, seed=seed, k0=min(6.0, n / 8), dealias="2/3")
        expect = s.nonlinear_rhs(w)
        d_in.copy_(torch.from_numpy(w.view(np.float64).reshape(-1).copy()))
        d_out.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy().view(np.complex128).reshape(n, nyf)
        err = np.max(np.abs(got - expect)) / np.max(np.abs(expect))
        assert err <= RHS_TOL, (n, seed, err)
    del g
    s.close()


def test_noalloc_rejects_misaligned_arrays():
    """A float64 view that starts 8 bytes into an allocation is refused
    before anything is launched; the context stays usable."""
    import torch

    L = load()
    n = 64
    p = abi.default_params(nx=n, ny=n)
    elems = 2 * n * (n // 2 + 1)
    # one spare double each, so that the offset views stay inside their buffers
    a = torch.zeros(elems + 2, dtype=torch.float64, device="cuda")
    b = torch.zeros(elems + 2, dtype=torch.float64, device="cuda")
    assert a.data_ptr() % 16 == 0 and b.data_ptr() % 16 == 0
    assert _noalloc(L, p, a.data_ptr() + 8, b.data_ptr(), 0) == abi.ERR_INVALID
    assert _noalloc(L, p, a.data_ptr(), b.data_ptr() + 8, 0) == abi.ERR_INVALID
    torch.cuda.synchronize()
    # the same arrays on the 16-byte boundary are taken
    assert _noalloc(L, p, a.data_ptr(), b.data_ptr(), 0) == abi.OK
    torch.cuda.synchronize()


def test_noalloc_rejects_sizes_above_limit():
    import torch

    L = load()
    for n in (512, 1024, 96):
        p = abi.default_params(nx=n, ny=n)
        d = torch.zeros(2 * n * (n // 2 + 1), dtype=torch.float64, device="cuda")
        assert _noalloc(L, p, d.data_ptr(), d.data_ptr(), 0) == abi.ERR_UNSUPPORTED
    p = abi.default_params(nx=128, ny=64)
    assert _noalloc(L, p, 0, 0, 0) in (abi.ERR_INVALID, abi.ERR_UNSUPPORTED)
