"""CPU restatement of the discrete adjoint of the pseudospectral RK4CN step
(TEST INFRASTRUCTURE ONLY: the checker for the CUDA adjoint, never part of it).

Only tests/ and bench.py's CPU legs import this.  numpy FP64.

The reference has no adjoint; what is restated here is the exact transpose of
the reference's own discrete step, derived from

* NonlinearRHSBatch (Solver/src/solver.c:884-1032): derived spectra
  u = i ky/k^2 w, v = -i kx/k^2 w, w_x = i kx w, w_y = i ky w; batched c2r;
  n = u w_x + v w_y; r2c; times (1/(Nx Ny))^2; zero mean; ApplyDealiasing
  (solver.c:1039-1099); plus the forcing term (solver.c:1022-1027);
* RK4Step with __RK4CN (solver.c:625-873): X1 = w, X2 = w + dt/2 r1,
  X3 = w + dt/2 r2, X4 = w + dt r3, w' = ((2-D) w + 2 dt sum b_s r_s)/(2+D),
  D = dt (bracket of solver.c:839-856), b = (1/6, 1/3, 1/3, 1/6);
* the enstrophy and palinstrophy sums of ComputeSystemMeasurables
  (Solver/src/sys_msr.c:190-227, 356-363).

Inner product on the half spectrum [Nx][Ny/2+1]:
    <a, b>_W = sum_j c_j Re(conj(a_j) b_j),  c_j = 1 on ky = 0 and ky = Ny/2, 2 else,
under which the unnormalised c2r (``c2r``) and r2c (``r2c``) are exact
transposes.  Gradients here are W-gradients: dJ = <g, dw>_W.  The tangent-linear
model ``tl_rhs`` is built on any RHS callable (the reference's own compiled
NonlinearRHS through oracle.pyoracle.RefSolver, or the restatement) by
polarisation, exact for the quadratic nonlinear term.
"""
import numpy as np

B_RK4 = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
A_RK4 = (0.5, 0.5, 1.0)


def wavenumbers(n):
    kx = np.fft.fftfreq(n, 1.0 / n).astype(np.int64)
    kx[n // 2] = n // 2  # row n/2 is +n/2 (solver.c:2048-2056)
    ky = np.arange(n // 2 + 1, dtype=np.int64)
    return kx[:, None], ky[None, :]


def weights(n):
    c = np.full((1, n // 2 + 1), 2.0)
    c[0, 0] = 1.0
    c[0, -1] = 1.0
    return c


def wdot(a, b):
    n = a.shape[0]
    return float(np.sum(weights(n) * (a.real * b.real + a.imag * b.imag)))


def c2r(X):
    """Unnormalised 2-D c2r as FFTW does it (x c2c, then y c2r with the real
    parts of ky = 0 and ky = N/2)."""
    n = X.shape[0]
    return np.fft.irfft2(X, s=(n, n), axes=(0, 1)) * float(n * n)


def r2c(f):
    return np.fft.rfft2(f, axes=(0, 1))


def dealias_factor(n, dealias=0, kolm=False, houli_int=False):
    """ApplyDealiasing as a factor per mode, zero at the mean mode
    (solver.c:1013, 1039-1099)."""
    kx, ky = wavenumbers(n)
    if dealias == 0:
        m = int(n / 3.0)
        k2 = (kx * kx + ky * ky).astype(float)
        d = np.where(k2 >= float(m * m), 0.0, 1.0)
        if kolm:
            d = np.where(kx == 0, 0.0, d)
    else:
        if houli_int:
            # C integer division (truncation toward zero), solver.c:1088
            fx = np.trunc(kx / (n // 2)).astype(float)
            fy = np.trunc(ky / (n // 2)).astype(float)
        else:
            fx = kx / (n / 2.0)
            fy = ky / (n / 2.0)
        r2 = fx * fx + fy * fy
        e = 36.0 * r2 ** 18
        d = np.where(e < 1e-17, 1.0, np.exp(-e))
    d = np.broadcast_to(d, (n, n // 2 + 1)).copy()
    d[0, 0] = 0.0
    return d


def multipliers(n):
    """m_u, m_v, m_x, m_y of the derived spectra (solver.c:904-957)."""
    kx, ky = wavenumbers(n)
    k2 = (kx * kx + ky * ky).astype(float)
    k2[0, 0] = np.inf
    mu = 1j * ky / k2
    mv = -1j * kx / k2
    mx = 1j * kx + 0 * ky
    my = 1j * ky + 0 * kx
    return [np.broadcast_to(m, (n, n // 2 + 1)).astype(np.complex128) for m in (mu, mv, mx, my)]


class Model:
    """The RK4CN step and its adjoint on an n x n grid."""

    def __init__(self, n, bracket, dealias=0, kolm=False, houli_int=False, forcing=None):
        self.n = n
        self.s2 = (1.0 / float(n * n)) ** 2
        self.D = dealias_factor(n, dealias, kolm, houli_int)
        self.m = multipliers(n)
        kx, ky = wavenumbers(n)
        k2 = (kx * kx + ky * ky).astype(float)
        self.k2 = np.broadcast_to(k2, (n, n // 2 + 1)).copy()
        self.bracket = bracket  # callable k^2 -> linear operator bracket
        self.forcing = np.zeros((n, n // 2 + 1), np.complex128) if forcing is None else forcing

    # -- nonlinear term -------------------------------------------------
    def fields(self, X):
        return [c2r(m * X) for m in self.m]  # u, v, w_x, w_y

    def rhs(self, X):
        u, v, wx, wy = self.fields(X)
        return self.s2 * self.D * r2c(u * wx + v * wy) + self.forcing

    def rhs_tl(self, X, dX):
        u, v, wx, wy = self.fields(X)
        du, dv, dwx, dwy = self.fields(dX)
        return self.s2 * self.D * r2c(du * wx + u * dwx + dv * wy + v * dwy)

    def rhs_adj(self, X, kappa, fields=None):
        u, v, wx, wy = self.fields(X) if fields is None else fields
        mu = c2r(self.s2 * self.D * kappa)
        mu_u, mu_v, mu_x, mu_y = self.m
        return (np.conj(mu_u) * r2c(wx * mu) + np.conj(mu_v) * r2c(wy * mu) + np.conj(mu_x) * r2c(u * mu)
                + np.conj(mu_y) * r2c(v * mu))

    # -- RK4CN step -----------------------------------------------------
    def cn(self, dt):
        k2 = self.k2.copy()
        k2[0, 0] = 1.0
        D = dt * self.bracket(k2)
        A = (2.0 - D) / (2.0 + D)
        B = 2.0 * dt / (2.0 + D)
        A[0, 0] = 0.0
        B[0, 0] = 0.0
        return A, B

    def step(self, w, dt, rhs=None):
        """One RK4CN step; returns (w', [X1..X4])."""
        rhs = self.rhs if rhs is None else rhs
        A, B = self.cn(dt)
        X = [w]
        tot = np.zeros_like(w)
        for s in range(4):
            r = rhs(X[s])
            tot = tot + B_RK4[s] * r
            if s < 3:
                X.append(w + A_RK4[s] * dt * r)
        return A * w + B * tot, X

    def step_tl(self, X, dw, dt, rhs_tl=None):
        rhs_tl = self.rhs_tl if rhs_tl is None else rhs_tl
        A, B = self.cn(dt)
        dX = dw
        tot = np.zeros_like(dw)
        for s in range(4):
            dr = rhs_tl(X[s], dX)
            tot = tot + B_RK4[s] * dr
            if s < 3:
                dX = dw + A_RK4[s] * dt * dr
        return A * dw + B * tot

    def step_adj(self, X, lam, dt):
        """lambda_w = A lambda' + sum_s F'(X_s)^T kappa_s with
        kappa_4 = b_4 B lambda', kappa_s = b_s B lambda' + a_{s+1} dt L_{s+1}."""
        A, B = self.cn(dt)
        lam_w = A * lam
        L = None
        for s in range(3, -1, -1):
            kappa = B_RK4[s] * B * lam
            if L is not None:
                kappa = kappa + A_RK4[s] * dt * L
            L = self.rhs_adj(X[s], kappa)
            lam_w = lam_w + L
        return lam_w

    # -- objectives ------------------------------------------------------
    def objective(self, w, kind="enstrophy"):
        """Z or P of ComputeSystemMeasurables and its W-gradient."""
        n = self.n
        cz = 4.0 * np.pi ** 2 * 0.5 / float(n * n) ** 2
        f = np.ones_like(self.k2) if kind == "enstrophy" else self.k2.copy()
        f[0, 0] = 0.0
        J = cz * float(np.sum(weights(n) * f * np.abs(w) ** 2))
        return J, 2.0 * cz * f * w

    def gradient(self, w0, nsteps, dt, kind="enstrophy", checkpoint_every=None):
        """J(w(T)) and dJ/dw0 (W-gradient) by a reverse sweep; checkpoints
        every `checkpoint_every` steps with the stages recomputed per segment."""
        C = nsteps if checkpoint_every is None else checkpoint_every
        ckpt = {}
        w = w0
        for k in range(nsteps):
            if k % C == 0:
                ckpt[k] = w
            w, _ = self.step(w, dt)
        J, lam = self.objective(w, kind)
        for seg0 in sorted(ckpt, reverse=True):
            seg1 = min(seg0 + C, nsteps)
            w = ckpt[seg0]
            stages = []
            for k in range(seg0, seg1):
                w, X = self.step(w, dt)
                stages.append(X)
            for X in reversed(stages):
                lam = self.step_adj(X, lam, dt)
        return J, lam


def bracket_for(params, hyper_flag=None, latch=False):
    """Bracket of the linear operator (solver.c:839-856) for the branch the
    step settles on (the `=` typo latches hyperviscosity on when `latch`)."""
    p = params
    hf = p.hyper_visc_flag if hyper_flag is None else hyper_flag
    if hf == 1 and p.ekmn_drag_flag == 1:
        return lambda k2: p.nu * k2 ** p.hyper_visc_pow + p.ekmn_alpha * k2 ** p.ekmn_drag_pow
    if hf != 1 and p.ekmn_drag_flag == 1:
        return lambda k2: p.nu * k2 + p.ekmn_alpha * k2 ** p.ekmn_drag_pow
    if latch:
        hf = 1
    if hf == 1:
        return lambda k2: p.nu * k2 ** p.hyper_visc_pow
    return lambda k2: p.nu * k2


def tl_rhs_polar(rhs):
    """Tangent-linear of an RHS callable by polarisation: for F(X) = Q(X, X) + f
    with Q bilinear, F'(X) dX = (F(X + dX) - F(X - dX)) / 2 exactly."""
    return lambda X, dX: 0.5 * (rhs(X + dX) - rhs(X - dX))


def hermitian(w):
    w = w.copy()
    n = w.shape[0]
    for j in (0, w.shape[1] - 1):
        col = w[:, j]
        col[n // 2 + 1:] = np.conj(col[1:n // 2][::-1])
        col[0] = col[0].real
        col[n // 2] = col[n // 2].real
        w[:, j] = col
    w[0, 0] = 0.0
    return w


def random_field(n, seed, kmax=None, scale=1.0):
    """Seeded Hermitian half spectrum (PCG64), band-limited to |k| < kmax."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal((n, n // 2 + 1)) + 1j * rng.standard_normal((n, n // 2 + 1))
    kx, ky = wavenumbers(n)
    k = np.sqrt((kx * kx + ky * ky).astype(float))
    if kmax is not None:
        w = np.where(k < kmax, w, 0.0)
    return hermitian(w * scale)
