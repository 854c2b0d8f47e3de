"""Python mirror of the reference solver's per-step C API, over libns2d.so.

Method names follow Solver/src/solver.h and sys_msr.h (NonlinearRHSBatch ->
nonlinear_rhs, RK4Step -> rk4_step, AB4Step -> ab4_step, GetMaxData ->
get_max_data, GetTimestep -> get_timestep, SystemCheck -> system_check,
ComputeSystemMeasurables -> system_measurables).  Spectral arrays are numpy
complex128 [nx][ny/2+1] in the reference layout.
"""
import ctypes as C

import numpy as np

from . import abi
from ._lib import NS2DError, load

_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


class Solver:
    def __init__(self, params=None, **kw):
        self.L = load()
        self.p = (params.copy() if params is not None else abi.default_params())
        for k, v in kw.items():
            setattr(self.p, k, v)
        h = C.c_void_p()
        st = self.L.ns2d_create(C.byref(self.p), C.byref(h))
        if st != abi.OK:
            raise NS2DError(st, "ns2d_create failed")
        self.h = h
        nx, ny, nyf, ns = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        self.L.ns2d_dims(self.h, C.byref(nx), C.byref(ny), C.byref(nyf), C.byref(ns))
        self.nx, self.ny, self.nyf, self.n_spect = nx.value, ny.value, nyf.value, ns.value

    def close(self):
        if getattr(self, "h", None):
            self.L.ns2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st):
        if st != abi.OK:
            raise NS2DError(st, (self.L.ns2d_last_error(self.h) or b"").decode())

    def _spec(self):
        return np.zeros((self.nx, self.nyf), np.complex128)

    # state
    def set_w_hat(self, w):
        w = np.ascontiguousarray(w, np.complex128)
        assert w.shape == (self.nx, self.nyf)
        self._ck(self.L.ns2d_set_w_hat(self.h, _ptr(w.view(np.float64))))

    def get_w_hat(self):
        w = self._spec()
        self._ck(self.L.ns2d_get_w_hat(self.h, _ptr(w.view(np.float64))))
        return w

    def set_w_hat_device(self, ptr):
        self._ck(self.L.ns2d_set_w_hat_device(self.h, C.c_void_p(ptr)))

    def get_w_hat_device(self, ptr):
        self._ck(self.L.ns2d_get_w_hat_device(self.h, C.c_void_p(ptr)))

    def get_w_real(self):
        w = np.zeros((self.nx, self.ny))
        self._ck(self.L.ns2d_get_w_real(self.h, _ptr(w)))
        return w

    def fft_r2c(self, real):
        """Unnormalised r2c of a real [nx][ny] field (FFTW conventions)."""
        real = np.ascontiguousarray(real, dtype=np.float64)
        assert real.shape == (self.nx, self.ny)
        out = np.zeros((self.nx, self.ny // 2 + 1), dtype=np.complex128)
        self._ck(self.L.ns2d_fft_r2c(self.h, _ptr(real), _ptr(out)))
        return out

    def fft_c2r(self, spec):
        """Unnormalised c2r of a half spectrum [nx][ny/2+1] (FFTW conventions)."""
        spec = np.ascontiguousarray(spec, dtype=np.complex128)
        assert spec.shape == (self.nx, self.ny // 2 + 1)
        out = np.zeros((self.nx, self.ny))
        self._ck(self.L.ns2d_fft_c2r(self.h, _ptr(spec), _ptr(out)))
        return out

    def mean_flow(self):
        """(mean_x [ny/2+1], mean_y [nx]) sums of one measurables call."""
        mx = np.zeros(self.ny // 2 + 1)
        my = np.zeros(self.nx)
        self._ck(self.L.ns2d_mean_flow(self.h, _ptr(mx), _ptr(my)))
        return mx, my

    # reference entry points
    def compute_forcing(self, dt):
        self._ck(self.L.ns2d_compute_forcing(self.h, dt))

    def nonlinear_rhs(self, w_in=None):
        out = self._spec()
        if w_in is None:
            self._ck(self.L.ns2d_nonlinear_rhs(self.h, None, _ptr(out.view(np.float64))))
        else:
            w_in = np.ascontiguousarray(w_in, np.complex128)
            self._ck(self.L.ns2d_nonlinear_rhs(self.h, _ptr(w_in.view(np.float64)), _ptr(out.view(np.float64))))
        return out

    def rk4_step(self, dt):
        self._ck(self.L.ns2d_rk4_step(self.h, dt))

    def ab4_step(self, dt, iters):
        self._ck(self.L.ns2d_ab4_step(self.h, dt, iters))

    def set_forcing_modes(self, idx, values):
        """Forcing of listed modes (flat indices into [nx][ny/2+1], complex
        values), added to every RHS until changed; empty removes it."""
        idx = np.ascontiguousarray(idx, np.int32)
        values = np.ascontiguousarray(values, np.complex128)
        assert idx.shape == values.shape
        self._ck(self.L.ns2d_set_forcing_modes(self.h, len(idx), idx.ctypes.data_as(C.POINTER(C.c_int32)),
                                               _ptr(values.view(np.float64)) if len(idx) else None))

    def dp5_step(self, dt):
        """One Dormand-Prince 5(4) trial step (RK5DPStep, corrected); returns
        the scaled error estimate."""
        e = C.c_double()
        self._ck(self.L.ns2d_dp5_step(self.h, dt, C.byref(e)))
        return e.value

    def rk5dp_step(self, dt, iters):
        """RK5DPStep as the reference writes it, at SpectralSolve iteration
        `iters`; returns DP_err (unchanged when iters == 1)."""
        e = C.c_double()
        self._ck(self.L.ns2d_rk5dp_step(self.h, dt, int(iters), C.byref(e)))
        return e.value

    def step_n(self, n, dt):
        self._ck(self.L.ns2d_step_n(self.h, n, dt))

    def apply_dealiasing(self, arr, dim=1):
        a = np.ascontiguousarray(arr, np.complex128).copy()
        self._ck(self.L.ns2d_apply_dealiasing(self.h, _ptr(a.view(np.float64)), dim))
        return a

    def force_conjugacy(self, arr=None):
        if arr is None:
            self._ck(self.L.ns2d_force_conjugacy(self.h, None))
        else:
            a = np.ascontiguousarray(arr, np.complex128)
            self._ck(self.L.ns2d_force_conjugacy(self.h, _ptr(a.view(np.float64))))

    def get_max_data(self, kind=abi.MAX_VORT):
        v = C.c_double()
        self._ck(self.L.ns2d_get_max_data(self.h, kind, C.byref(v)))
        return v.value

    def get_timestep(self, dt):
        v = C.c_double(dt)
        self._ck(self.L.ns2d_get_timestep(self.h, C.byref(v)))
        return v.value

    def set_w_max_init(self, w):
        self._ck(self.L.ns2d_set_w_max_init(self.h, w))

    def system_check(self, dt, iters):
        return self.L.ns2d_system_check(self.h, dt, iters)

    def system_measurables(self):
        m = abi.Measures()
        sp = np.zeros(8 * self.n_spect)
        self._ck(self.L.ns2d_system_measurables(self.h, C.byref(m), _ptr(sp)))
        return np.array(m.as_list()), sp.reshape(8, self.n_spect)

    def rk4_step_host(self, w_hat, dt):
        """RK4Step on a host array (complex128, reference layout), in place."""
        assert w_hat.dtype == np.complex128 and w_hat.flags.c_contiguous
        self._ck(self.L.ns2d_rk4_step_host(self.h, _ptr(w_hat.view(np.float64)), dt))

    def step_async(self, n, dt):
        self._ck(self.L.ns2d_step_async(self.h, n, dt))

    def check(self):
        self._ck(self.L.ns2d_check(self.h))

    @property
    def stream(self):
        s = C.c_void_p()
        self._ck(self.L.ns2d_get_stream(self.h, C.byref(s)))
        return s.value

    def set_stream(self, ptr):
        self._ck(self.L.ns2d_set_stream(self.h, C.c_void_p(ptr)))

    def set_kernel_timing(self, on=True):
        self._ck(self.L.ns2d_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        ms = np.zeros(5)
        n = np.zeros(5, np.int64)
        self._ck(self.L.ns2d_kernel_times(self.h, _ptr(ms), n.ctypes.data_as(C.POINTER(C.c_int64)), 5))
        return ms, n

    def synchronize(self):
        self._ck(self.L.ns2d_synchronize(self.h))

    # discrete adjoint (W-gradients: dJ = sum_j c_j Re(conj(g_j) dw_j))
    def adjoint_record(self, nsteps, dt, checkpoint_every=50):
        """Advance nsteps RK4CN steps keeping checkpoints for adjoint_backward."""
        self._ck(self.L.ns2d_adjoint_record(self.h, nsteps, dt, checkpoint_every))

    def adjoint_backward(self, lam_T):
        """(dw(T)/dw(0))^T lam_T over the recorded run (host arrays)."""
        lam_T = np.ascontiguousarray(lam_T, np.complex128)
        out = self._spec()
        self._ck(self.L.ns2d_adjoint_backward(self.h, _ptr(lam_T.view(np.float64)), _ptr(out.view(np.float64))))
        return out

    def adjoint_backward_device(self, d_lam_T, d_lam_0):
        self._ck(self.L.ns2d_adjoint_backward_device(self.h, C.c_void_p(d_lam_T), C.c_void_p(d_lam_0)))

    def objective(self, kind=abi.OBJ_ENSTROPHY, d_grad=None):
        v = C.c_double()
        self._ck(self.L.ns2d_objective(self.h, kind, C.byref(v), C.c_void_p(d_grad) if d_grad else None))
        return v.value

    def adjoint_gradient(self, nsteps, dt, checkpoint_every=50, kind=abi.OBJ_ENSTROPHY):
        """J(w(T)) and dJ/dw(0) from the current state (the state ends at w(T))."""
        g = self._spec()
        v = C.c_double()
        self._ck(self.L.ns2d_adjoint_gradient(self.h, nsteps, dt, checkpoint_every, kind, C.byref(v),
                                              _ptr(g.view(np.float64))))
        return v.value, g

    def adjoint_times(self):
        """Device ms of the last adjoint_record and of the last reverse sweep."""
        a, b = C.c_double(), C.c_double()
        self._ck(self.L.ns2d_adjoint_times(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def wdot_device(self, d_a, d_b):
        v = C.c_double()
        self._ck(self.L.ns2d_wdot_device(self.h, C.c_void_p(d_a), C.c_void_p(d_b), C.byref(v)))
        return v.value

    @property
    def launch_count(self):
        return self.L.ns2d_launch_count(self.h)
