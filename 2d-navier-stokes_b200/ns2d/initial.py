"""Seeded initial vorticity spectra in the reference layout [nx][ny/2+1].

These are the user-set initial conditions of the benchmark workloads (set with
ns2d_set_w_hat), not the reference's glibc-rand() generators.  Conventions
follow the reference: w_hat is the unnormalised forward DFT of w, and the
energy is E = 4 pi^2 * 0.5/(Nx Ny)^2 * sum_j c_j |w_hat|^2/|k|^2 with
c_j = 1 on the ky = 0 and ky = Ny/2 columns and 2 elsewhere
(Solver/src/sys_msr.c:190-227, 356-363).
"""
import numpy as np


def wavenumbers(nx, ny):
    kx = np.fft.fftfreq(nx, 1.0 / nx).astype(np.int64)
    kx[nx // 2] = nx // 2  # row nx/2 is +nx/2 in the reference (solver.c:2048-2056)
    ky = np.arange(ny // 2 + 1, dtype=np.int64)
    return kx[:, None], ky[None, :]


def weights(nx, ny):
    nyf = ny // 2 + 1
    c = np.full((1, nyf), 2.0)
    c[0, 0] = 1.0
    c[0, -1] = 1.0
    return c


def energy(w_hat):
    nx = w_hat.shape[0]
    ny = 2 * (w_hat.shape[1] - 1)
    kx, ky = wavenumbers(nx, ny)
    k2 = (kx * kx + ky * ky).astype(float)
    k2[0, 0] = np.inf
    s = np.sum(weights(nx, ny) * np.abs(w_hat) ** 2 / k2)
    return 4.0 * np.pi ** 2 * 0.5 / float(nx * ny) ** 2 * s


def enstrophy(w_hat):
    nx = w_hat.shape[0]
    ny = 2 * (w_hat.shape[1] - 1)
    s = np.sum(weights(nx, ny) * np.abs(w_hat) ** 2) - np.abs(w_hat[0, 0]) ** 2
    return 4.0 * np.pi ** 2 * 0.5 / float(nx * ny) ** 2 * s


def hermitian(w_hat):
    """Make the ky = 0 and ky = Ny/2 columns Hermitian in kx; zero the mean."""
    w = w_hat.copy()
    nx = w.shape[0]
    for j in (0, w.shape[1] - 1):
        col = w[:, j]
        col[nx // 2 + 1:] = np.conj(col[1:nx // 2][::-1])
        col[0] = col[0].real
        col[nx // 2] = col[nx // 2].real
        w[:, j] = col
    w[0, 0] = 0.0
    return w


def dealias_23(w_hat, kolm=False):
    """2/3 rule of the reference: zero |k|^2 >= ((int)(N/3))^2 (solver.c:1049-1068)."""
    nx = w_hat.shape[0]
    ny = 2 * (w_hat.shape[1] - 1)
    kx, ky = wavenumbers(nx, ny)
    m = int(nx / 3.0)
    mask = (kx * kx + ky * ky) >= m * m
    if kolm:
        mask = mask | (kx == 0)
    w = w_hat.copy()
    w[np.broadcast_to(mask, w.shape)] = 0.0
    return w


def taylor_green(n):
    """w = 2 sin(x) sin(y) on [0, 2pi)^2: w_hat(1,1) = -N^2/2, w_hat(-1,1) = +N^2/2."""
    w = np.zeros((n, n // 2 + 1), np.complex128)
    w[1, 1] = -0.5 * n * n
    w[n - 1, 1] = 0.5 * n * n
    return w


def decaying(n, seed, k0=6.0, e0=0.5, dealias=None):
    """Random uniform phases in [0, 2 pi), energy spectrum E(k) ~ k^4 exp(-(k/k0)^2),
    normalised to total energy e0, Hermitian ky = 0 / Ny/2 columns."""
    rng = np.random.default_rng(seed)
    kx, ky = wavenumbers(n, n)
    k = np.sqrt((kx * kx + ky * ky).astype(float))
    ek = np.where(k > 0, k ** 4 * np.exp(-(k / k0) ** 2), 0.0)
    amp = np.sqrt(np.where(k > 0, k * ek / (2.0 * np.pi), 0.0))
    phase = np.exp(2j * np.pi * rng.random((n, n // 2 + 1)))
    w = hermitian(amp * phase * (n * n))
    if dealias == "2/3":
        w = dealias_23(w)
    return w * np.sqrt(e0 / energy(w))


def noise(n, seed, amplitude=1e-3, kmax=8.0, kolm=False):
    """Low-amplitude random-phase vorticity noise: modes 1 <= |k| <= kmax with
    equal amplitudes, scaled to an RMS vorticity of `amplitude`."""
    rng = np.random.default_rng(seed)
    kx, ky = wavenumbers(n, n)
    k = np.sqrt((kx * kx + ky * ky).astype(float))
    amp = np.where((k >= 1.0) & (k <= kmax), 1.0, 0.0)
    w = hermitian(amp * np.exp(2j * np.pi * rng.random((n, n // 2 + 1))))
    w = dealias_23(w, kolm=kolm)
    c = weights(n, n)
    rms = np.sqrt(np.sum(c * np.abs(w) ** 2)) / (n * n)
    return w * (amplitude / rms)
