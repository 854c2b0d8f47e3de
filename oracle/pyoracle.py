"""Python loaders for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.

* ``Oracle``    -- oracle/build/libns2d_oracle.so, our C restatement
                   (oracle/ns2d_oracle.c), same layouts as include/ns2d.h.
* ``RefSolver`` -- oracle/_ref/libns2d_ref_<variant>.so, the reference's own
                   Solver/src/{solver,force,sys_msr}.c built by oracle/Makefile
                   against the single-rank stand-ins in oracle/shim/.  Variant
                   "dropin" is the same program with its per-step entry points
                   resolved to the GPU (2d-navier-stokes_b200/compat).
* ``solve``     -- the reference's own time loop (SpectralSolve) in one of
                   those libraries; once per process.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, "build", "libns2d_oracle.so")
_REF_SO = os.path.join(HERE, "_ref", "libns2d_ref_{}.so")

_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def build(ref=True):
    """Build the restatement (always) and, with ref, the reference builds
    (when the reference sources are present: oracle/Makefile target
    `checkers`, which reads their location from NS2D_REFERENCE)."""
    subprocess.run(["make", "-s", "-C", HERE, "checkers" if ref else "restatement"], check=True)


def ref_available(variant="rk4cn"):
    return os.path.exists(_REF_SO.format(variant))


class Oracle:
    """Our CPU restatement; one instance = one simulation state."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(_ORACLE_SO):
                build(ref=False)
            L = C.CDLL(_ORACLE_SO)
            L.oracle_create.restype = C.c_void_p
            L.oracle_create.argtypes = [C.c_void_p, C.c_int]
            L.oracle_destroy.argtypes = [C.c_void_p]
            L.oracle_n_spect.argtypes = [C.c_void_p]
            for f in ("oracle_set_w_hat", "oracle_get_w_hat", "oracle_get_w_real", "oracle_force_conjugacy"):
                getattr(L, f).argtypes = [C.c_void_p, _dp]
            L.oracle_compute_forcing.argtypes = [C.c_void_p, C.c_double]
            L.oracle_nonlinear_rhs.argtypes = [C.c_void_p, _dp, _dp]
            L.oracle_rk4_step.argtypes = [C.c_void_p, C.c_double]
            L.oracle_ab4_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
            L.oracle_dp5_step.argtypes = [C.c_void_p, C.c_double, _dp]
            L.oracle_rk5dp_step.argtypes = [C.c_void_p, C.c_double, C.c_int]
            L.oracle_rk5dp_step.restype = C.c_double
            L.oracle_apply_dealiasing.argtypes = [C.c_void_p, _dp, C.c_int]
            L.oracle_get_max_data.argtypes = [C.c_void_p, C.c_int]
            L.oracle_get_max_data.restype = C.c_double
            L.oracle_get_timestep.argtypes = [C.c_void_p, C.c_double]
            L.oracle_get_timestep.restype = C.c_double
            L.oracle_set_w_max_init.argtypes = [C.c_void_p, C.c_double]
            L.oracle_hyper_visc_flag.argtypes = [C.c_void_p]
            L.oracle_system_measurables.argtypes = [C.c_void_p, _dp, _dp]
            L.oracle_ic_taylor_green.argtypes = [C.c_int, C.c_int, _dp]
            cls._lib = L
        return cls._lib

    def __init__(self, params, threads=1):
        self.L = self.lib()
        self.p = params.copy()
        self.nx, self.ny = params.nx, params.ny
        self.nyf = params.ny // 2 + 1
        self.h = self.L.oracle_create(C.byref(self.p), threads)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def _spec(self):
        return np.zeros((self.nx, self.nyf), np.complex128)

    @property
    def n_spect(self):
        return self.L.oracle_n_spect(self.h)

    def set_w_hat(self, w):
        w = np.ascontiguousarray(w, np.complex128)
        self.L.oracle_set_w_hat(self.h, _ptr(w.view(np.float64)))

    def get_w_hat(self):
        w = self._spec()
        self.L.oracle_get_w_hat(self.h, _ptr(w.view(np.float64)))
        return w

    def get_w_real(self):
        w = np.zeros((self.nx, self.ny))
        self.L.oracle_get_w_real(self.h, _ptr(w))
        return w

    def compute_forcing(self, dt):
        self.L.oracle_compute_forcing(self.h, dt)

    def nonlinear_rhs(self, w_in=None):
        out = self._spec()
        if w_in is None:
            self.L.oracle_nonlinear_rhs(self.h, None, _ptr(out.view(np.float64)))
        else:
            w_in = np.ascontiguousarray(w_in, np.complex128)
            self.L.oracle_nonlinear_rhs(self.h, _ptr(w_in.view(np.float64)), _ptr(out.view(np.float64)))
        return out

    def rk4_step(self, dt):
        self.L.oracle_rk4_step(self.h, dt)

    def ab4_step(self, dt, iters):
        self.L.oracle_ab4_step(self.h, dt, iters)

    def dp5_step(self, dt):
        e = np.zeros(1)
        self.L.oracle_dp5_step(self.h, dt, _ptr(e))
        return float(e[0])

    def set_threads(self, threads):
        """Host threads of the stand-in FFT from now on."""
        self.L.ref_set_threads(int(threads))

    def rk5dp_step(self, dt, iters):
        """RK5DPStep as the reference writes it, at iteration `iters`; DP_err."""
        return self.L.oracle_rk5dp_step(self.h, dt, iters)

    def apply_dealiasing(self, arr, dim=1):
        a = np.ascontiguousarray(arr, np.complex128).copy()
        self.L.oracle_apply_dealiasing(self.h, _ptr(a.view(np.float64)), dim)
        return a

    def force_conjugacy(self, arr=None):
        if arr is None:
            self.L.oracle_force_conjugacy(self.h, None)
        else:
            a = np.ascontiguousarray(arr, np.complex128)
            self.L.oracle_force_conjugacy(self.h, _ptr(a.view(np.float64)))

    def get_max_data(self, kind=0):
        return self.L.oracle_get_max_data(self.h, kind)

    def get_timestep(self, dt):
        return self.L.oracle_get_timestep(self.h, dt)

    def set_w_max_init(self, w):
        self.L.oracle_set_w_max_init(self.h, w)

    @property
    def hyper_visc_flag(self):
        return self.L.oracle_hyper_visc_flag(self.h)

    def system_measurables(self):
        s = np.zeros(13)
        sp = np.zeros(8 * self.n_spect)
        self.L.oracle_system_measurables(self.h, _ptr(s), _ptr(sp))
        return s, sp.reshape(8, self.n_spect)

    @classmethod
    def taylor_green(cls, nx, ny):
        w = np.zeros((nx, ny // 2 + 1), np.complex128)
        cls.lib().oracle_ic_taylor_green(nx, ny, _ptr(w.view(np.float64)))
        return w


class _RefParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nu", C.c_double), ("hyper_visc_flag", C.c_int),
        ("hyper_visc_pow", C.c_double), ("ekmn_alpha", C.c_double), ("ekmn_drag_flag", C.c_int),
        ("ekmn_drag_pow", C.c_double), ("force_k", C.c_int), ("force_scale", C.c_double),
        ("dt", C.c_double), ("t0", C.c_double), ("T", C.c_double), ("adapt_step_flag", C.c_int),
        ("cfl_cond_flag", C.c_int), ("cfl_const", C.c_double), ("save_every", C.c_int),
        ("num_print_steps", C.c_int), ("forcing", C.c_char * 64), ("u0", C.c_char * 64),
    ]


class RefSolver:
    """The reference's own compiled solver (one process-wide instance per
    variant library, because the reference keeps its state in globals)."""

    _libs = {}

    def __init__(self, params, variant="rk4cn", u0="NONE", threads=1):
        path = _REF_SO.format(variant)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        if variant in RefSolver._libs:
            raise RuntimeError("one RefSolver per variant and process (reference state is global)")
        L = C.CDLL(path)
        RefSolver._libs[variant] = L
        self.L = L
        for f in ("ref_set_w_hat", "ref_get_w_hat", "ref_nonlinear_rhs_state", "ref_get_w_real"):
            getattr(L, f).argtypes = [_dp]
        L.ref_nonlinear_rhs_input.argtypes = [_dp, _dp]
        if hasattr(L, "ref_rk4_step"):  # absent from the Dormand-Prince build
            L.ref_rk4_step.argtypes = [C.c_double]
        if variant == "dp5":
            L.ref_dp5_step.argtypes = [C.c_double, C.c_int]
            L.ref_dp5_step.restype = C.c_double
        if variant == "ab4":
            L.ref_ab4_step.argtypes = [C.c_double, C.c_int]
        L.ref_compute_forcing.argtypes = [C.c_double]
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_apply_dealiasing.argtypes = [_dp, C.c_int]
        L.ref_force_conjugacy.argtypes = [_dp]
        for f in ("ref_get_max_vort", "ref_get_max_vel", "ref_w_max_init"):
            getattr(L, f).restype = C.c_double
        L.ref_get_timestep.argtypes = [C.c_double]
        L.ref_get_timestep.restype = C.c_double
        L.ref_set_w_max_init.argtypes = [C.c_double]
        L.ref_set_dt.argtypes = [C.c_double]
        L.ref_system_measurables.argtypes = [C.c_double, C.c_int, _dp, _dp]
        forcing = {0: b"NONE", 1: b"KOLM", 2: b"ZERO"}[params.forcing]
        rp = _RefParams(nx=params.nx, ny=params.ny, nu=params.nu, hyper_visc_flag=params.hyper_visc_flag,
                        hyper_visc_pow=params.hyper_visc_pow, ekmn_alpha=params.ekmn_alpha,
                        ekmn_drag_flag=params.ekmn_drag_flag, ekmn_drag_pow=params.ekmn_drag_pow,
                        force_k=params.force_k, force_scale=params.force_scale, dt=params.dt, t0=0.0,
                        T=1.0, adapt_step_flag=params.adapt_step_flag, cfl_cond_flag=params.cfl_cond_flag,
                        cfl_const=params.cfl_const, save_every=100, num_print_steps=4,
                        forcing=forcing, u0=u0.encode())
        self.nx, self.ny, self.nyf = params.nx, params.ny, params.ny // 2 + 1
        rc = L.ref_init(C.byref(rp), 1 if u0 != "NONE" else 0, threads)
        if rc != 0:
            raise RuntimeError("ref_init failed")
        self.n_spect = L.ref_n_spect()

    def _spec(self):
        return np.zeros((self.nx, self.nyf), np.complex128)

    def set_w_hat(self, w):
        w = np.ascontiguousarray(w, np.complex128)
        self.L.ref_set_w_hat(_ptr(w.view(np.float64)))

    def get_w_hat(self):
        w = self._spec()
        self.L.ref_get_w_hat(_ptr(w.view(np.float64)))
        return w

    def compute_forcing(self, dt):
        self.L.ref_compute_forcing(dt)

    def nonlinear_rhs(self, w_in=None):
        out = self._spec()
        if w_in is None:
            self.L.ref_nonlinear_rhs_state(_ptr(out.view(np.float64)))
        else:
            w_in = np.ascontiguousarray(w_in, np.complex128)
            self.L.ref_nonlinear_rhs_input(_ptr(w_in.view(np.float64)), _ptr(out.view(np.float64)))
        return out

    def rk4_step(self, dt):
        self.L.ref_rk4_step(dt)

    def ab4_step(self, dt, iters):
        self.L.ref_ab4_step(dt, iters)

    def set_threads(self, threads):
        """Host threads of the stand-in FFT from now on."""
        self.L.ref_set_threads(int(threads))

    def rk5dp_step(self, dt, iters):
        """RK5DPStep at iteration `iters` (variant "dp5"); returns DP_err."""
        return self.L.ref_dp5_step(dt, iters)

    def apply_dealiasing(self, arr, dim=1):
        a = np.ascontiguousarray(arr, np.complex128).copy()
        self.L.ref_apply_dealiasing(_ptr(a.view(np.float64)), dim)
        return a

    def force_conjugacy(self, arr):
        a = np.ascontiguousarray(arr, np.complex128)
        self.L.ref_force_conjugacy(_ptr(a.view(np.float64)))

    def get_max_data(self, kind=0):
        return self.L.ref_get_max_vort() if kind == 0 else self.L.ref_get_max_vel()

    def get_timestep(self, dt):
        return self.L.ref_get_timestep(dt)

    def set_w_max_init(self, w):
        self.L.ref_set_w_max_init(w)

    @property
    def hyper_visc_flag(self):
        return self.L.ref_hyper_visc_flag()

    def system_measurables(self, t=0.0, it=1):
        s = np.zeros(13)
        sp = np.zeros(8 * self.n_spect)
        self.L.ref_system_measurables(t, it, _ptr(s), _ptr(sp))
        return s, sp.reshape(8, self.n_spect)


def solve(params, variant="rk4cn", u0="TG_VORT", T=0.05, save_every=10, threads=1, forcing=None):
    """Run SpectralSolve (Solver/src/solver.c:54-251) of a reference library
    from the initial condition u0 over [0, T]; returns (w_hat at the last save,
    its time, number of saves).  The library keeps global state: call once per
    process (the tests use spawned processes)."""
    path = _REF_SO.format(variant)
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    L = C.CDLL(path)
    L.ref_solve.argtypes = [C.c_void_p, C.c_int]
    L.ref_saved_w_hat.argtypes = [_dp, _dp]
    L.ref_saved_w_hat.restype = C.c_long
    forcing = forcing.encode() if forcing else {0: b"NONE", 1: b"KOLM", 2: b"ZERO"}[params.forcing]
    rp = _RefParams(nx=params.nx, ny=params.ny, nu=params.nu, hyper_visc_flag=params.hyper_visc_flag,
                    hyper_visc_pow=params.hyper_visc_pow, ekmn_alpha=params.ekmn_alpha,
                    ekmn_drag_flag=params.ekmn_drag_flag, ekmn_drag_pow=params.ekmn_drag_pow,
                    force_k=params.force_k, force_scale=params.force_scale, dt=params.dt, t0=0.0,
                    T=T, adapt_step_flag=params.adapt_step_flag, cfl_cond_flag=params.cfl_cond_flag,
                    cfl_const=params.cfl_const, save_every=save_every, num_print_steps=4,
                    forcing=forcing, u0=u0.encode())
    if L.ref_solve(C.byref(rp), threads) != 0:
        raise RuntimeError("ref_solve failed")
    w = np.zeros((params.nx, params.ny // 2 + 1), np.complex128)
    t = C.c_double()
    n = L.ref_saved_w_hat(_ptr(w.view(np.float64)), C.byref(t))
    return w, t.value, int(n)
