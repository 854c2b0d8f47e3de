"""GPU set-up transforms and the mean-flow sums (ns2d_fft_r2c / ns2d_fft_c2r /
ns2d_mean_flow) against numpy: the r2c/c2r pair follows FFTW's 2-D
conventions (unnormalised, c2r reads only the real parts of the ky = 0 and
ky = ny/2 columns) and the mean flows the sums of ComputeSystemMeasurables
(Solver/src/sys_msr.c:199, 227)."""
import numpy as np
import pytest

from ns2d import Solver, abi

pytestmark = pytest.mark.gpu


def _solver(n, fp32=False):
    p = abi.default_params(nx=n, ny=n, device=0)
    if fp32:
        p.precision = abi.FP32
    return Solver(p)


@pytest.mark.parametrize("n", [16, 64, 256, 1024])
def test_r2c_matches_numpy(n):
    s = _solver(n)
    rng = np.random.default_rng(n)
    f = rng.standard_normal((n, n))
    got = s.fft_r2c(f)
    want = np.fft.rfft2(f)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    s.close()


@pytest.mark.parametrize("n", [16, 128, 512])
def test_c2r_matches_numpy(n):
    """Including imaginary parts on the ky = 0 / ny/2 columns, which the c2r
    ignores as FFTW's does."""
    s = _solver(n)
    rng = np.random.default_rng(n + 1)
    spec = rng.standard_normal((n, n // 2 + 1)) + 1j * rng.standard_normal((n, n // 2 + 1))
    got = s.fft_c2r(spec)
    x = np.fft.ifft(spec, axis=0)
    x[:, 0] = x[:, 0].real
    x[:, -1] = x[:, -1].real
    want = np.fft.irfft(x, n=n, axis=1) * n * n
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    back = s.fft_r2c(got) / (n * n)
    assert np.abs(s.fft_c2r(back) - got).max() <= 1e-12 * np.abs(got).max()
    s.close()


def test_transforms_leave_the_state_alone():
    n = 64
    s = _solver(n)
    rng = np.random.default_rng(5)
    w = np.fft.rfft2(rng.standard_normal((n, n)))
    s.set_w_hat(w)
    s.fft_r2c(rng.standard_normal((n, n)))
    s.fft_c2r(w)
    assert np.array_equal(s.get_w_hat(), w)
    s.close()


def _mean_flow_numpy(w):
    nx, nyf = w.shape
    kx = np.fft.fftfreq(nx, 1.0 / nx)
    kx[nx // 2] = nx // 2
    kx = kx[:, None]
    ky = np.arange(nyf)[None, :]
    k2 = kx * kx + ky * ky
    k2[0, 0] = 1.0
    c = np.full((1, nyf), 2.0)
    c[0, 0] = c[0, -1] = 1.0
    v = c * np.abs(kx * w / k2)
    u = c * np.abs(ky * w / k2)
    v[0, 0] = u[0, 0] = 0.0
    return u.sum(axis=0), v.sum(axis=1)


@pytest.mark.parametrize("n,fp32", [(64, False), (512, False), (128, True)])
def test_mean_flow(n, fp32):
    s = _solver(n, fp32)
    rng = np.random.default_rng(7)
    w = np.fft.rfft2(rng.standard_normal((n, n)))
    s.set_w_hat(w)
    mx, my = s.mean_flow()
    wx, wy = _mean_flow_numpy(s.get_w_hat())
    tol = 1e-5 if fp32 else 1e-12
    assert np.abs(mx - wx).max() <= tol * np.abs(wx).max()
    assert np.abs(my - wy).max() <= tol * np.abs(wy).max()
    s.close()
