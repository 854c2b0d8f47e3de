"""Loader for lib/libns2d.so (the CUDA product).  There is no CPU fallback: if
the library or a CUDA device is missing, calls raise."""
import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "lib", "libns2d.so"))

_dp = C.POINTER(C.c_double)
_lib = None


class NS2DError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {msg}")


def load():
    """Load libns2d.so once and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} not built (run `make -C 2d-navier-stokes_b200` or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    sig = {
        "ns2d_abi_version": (C.c_int, []),
        "ns2d_status_string": (C.c_char_p, [C.c_int]),
        "ns2d_last_error": (C.c_char_p, [H]),
        "ns2d_params_default": (C.c_int, [C.POINTER(abi.Params)]),
        "ns2d_create": (C.c_int, [C.POINTER(abi.Params), C.POINTER(H)]),
        "ns2d_destroy": (C.c_int, [H]),
        "ns2d_dims": (C.c_int, [H, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "ns2d_set_w_hat": (C.c_int, [H, _dp]),
        "ns2d_get_w_hat": (C.c_int, [H, _dp]),
        "ns2d_set_w_hat_device": (C.c_int, [H, C.c_void_p]),
        "ns2d_get_w_hat_device": (C.c_int, [H, C.c_void_p]),
        "ns2d_compute_forcing": (C.c_int, [H, C.c_double]),
        "ns2d_nonlinear_rhs": (C.c_int, [H, _dp, _dp]),
        "ns2d_rk4_step": (C.c_int, [H, C.c_double]),
        "ns2d_ab4_step": (C.c_int, [H, C.c_double, C.c_int32]),
        "ns2d_step_n": (C.c_int, [H, C.c_int32, C.c_double]),
        "ns2d_apply_dealiasing": (C.c_int, [H, _dp, C.c_int32]),
        "ns2d_force_conjugacy": (C.c_int, [H, _dp]),
        "ns2d_get_max_data": (C.c_int, [H, C.c_int32, _dp]),
        "ns2d_get_timestep": (C.c_int, [H, _dp]),
        "ns2d_dt_range": (C.c_int, [H, _dp, _dp]),
        "ns2d_set_w_max_init": (C.c_int, [H, C.c_double]),
        "ns2d_system_check": (C.c_int, [H, C.c_double, C.c_int64]),
        "ns2d_system_measurables": (C.c_int, [H, C.POINTER(abi.Measures), _dp]),
        "ns2d_get_w_real": (C.c_int, [H, _dp]),
        "ns2d_fft_r2c": (C.c_int, [H, _dp, _dp]),
        "ns2d_fft_c2r": (C.c_int, [H, _dp, _dp]),
        "ns2d_mean_flow": (C.c_int, [H, _dp, _dp]),
        "ns2d_set_stream": (C.c_int, [H, C.c_void_p]),
        "ns2d_synchronize": (C.c_int, [H]),
        "ns2d_launch_count": (C.c_int64, [H]),
        "ns2d_rk4_step_host": (C.c_int, [H, _dp, C.c_double]),
        "ns2d_step_async": (C.c_int, [H, C.c_int32, C.c_double]),
        "ns2d_check": (C.c_int, [H]),
        "ns2d_get_stream": (C.c_int, [H, C.POINTER(C.c_void_p)]),
        "ns2d_set_kernel_timing": (C.c_int, [H, C.c_int32]),
        "ns2d_kernel_times": (C.c_int, [H, _dp, C.POINTER(C.c_int64), C.c_int32]),
        "ns2d_dp5_step": (C.c_int, [H, C.c_double, _dp]),
        "ns2d_rk5dp_step": (C.c_int, [H, C.c_double, C.c_int32, _dp]),
        "ns2d_set_forcing_modes": (C.c_int, [H, C.c_int32, C.POINTER(C.c_int32), _dp]),
        "ns2d_adjoint_record": (C.c_int, [H, C.c_int32, C.c_double, C.c_int32]),
        "ns2d_adjoint_backward": (C.c_int, [H, _dp, _dp]),
        "ns2d_adjoint_backward_device": (C.c_int, [H, C.c_void_p, C.c_void_p]),
        "ns2d_objective": (C.c_int, [H, C.c_int32, _dp, C.c_void_p]),
        "ns2d_adjoint_gradient": (C.c_int, [H, C.c_int32, C.c_double, C.c_int32, C.c_int32, _dp, _dp]),
        "ns2d_adjoint_times": (C.c_int, [H, _dp, _dp]),
        "ns2d_wdot_device": (C.c_int, [H, C.c_void_p, C.c_void_p, _dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.ns2d_abi_version() != abi.NS2D_ABI_VERSION:
        raise RuntimeError("libns2d.so ABI version mismatch")
    _lib = L
    return L


def exported_symbols():
    """Names the header declares (used by the CPU export test)."""
    hdr = os.path.normpath(os.path.join(_HERE, "..", "..", "include", "ns2d.h"))
    import re
    names = re.findall(r"^\s*(?:ns2d_status|int|int64_t|const char\*)\s+(ns2d_\w+)\s*\(", open(hdr).read(), re.M)
    return sorted(set(names))
