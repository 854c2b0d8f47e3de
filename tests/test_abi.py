"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/ns2d.h declares, and agrees with the ctypes mirror."""
import ctypes as C
import os
import re
import subprocess

import pytest

from ns2d import abi
from ns2d._lib import LIB_PATH, exported_symbols, load

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    assert os.path.exists(LIB_PATH), "libns2d.so not built"
    names = exported_symbols()
    assert len(names) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    defined = set(re.findall(r"\sT\s(\w+)", out))
    missing = [n for n in names if n not in defined]
    assert not missing, missing


def test_library_loads_and_defaults_match_reference_cli():
    L = load()
    p = abi.Params()
    assert L.ns2d_params_default(C.byref(p)) == abi.OK
    q = abi.default_params()
    for name, _ in abi.Params._fields_:
        assert getattr(p, name) == getattr(q, name), name
    # Solver/src/utils.c:57-83
    assert (p.nx, p.ny, p.nu, p.dt, p.cfl_const) == (64, 64, 1e-4, 1e-4, 0.9)
    assert L.ns2d_status_string(abi.ERR_BLOWUP) == b"NS2D_ERR_BLOWUP"


def test_struct_layout_matches_header(tmp_path):
    """Compile a probe against include/ns2d.h and compare every field offset."""
    fields = [n for n, _ in abi.Params._fields_]
    mfields = [n for n, _ in abi.Measures._fields_]
    body = "\n".join(f'printf("P {n} %zu\\n", offsetof(ns2d_params, {n}));' for n in fields)
    body += "\n" + "\n".join(f'printf("M {n} %zu\\n", offsetof(ns2d_measures, {n}));' for n in mfields)
    prog = tmp_path / "probe.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ns2d.h"\nint main(void){\n'
                    + body + '\nprintf("S %zu %zu\\n", sizeof(ns2d_params), sizeof(ns2d_measures));return 0;}\n')
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in out:
        parts = line.split()
        if not parts:
            continue
        if parts[0] == "P":
            assert getattr(abi.Params, parts[1]).offset == int(parts[2]), parts[1]
        elif parts[0] == "M":
            assert getattr(abi.Measures, parts[1]).offset == int(parts[2]), parts[1]
        else:
            assert (C.sizeof(abi.Params), C.sizeof(abi.Measures)) == (int(parts[1]), int(parts[2]))


def test_create_without_device_reports_no_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("device present")
    except Exception:
        pass
    L = load()
    p = abi.default_params()
    h = C.c_void_p()
    assert L.ns2d_create(C.byref(p), C.byref(h)) == abi.ERR_NO_DEVICE


def test_invalid_sizes_rejected_before_device_use():
    L = load()
    for nx, ny in ((96, 96), (64, 32), (8, 8), (4096, 4096)):
        p = abi.default_params(nx=nx, ny=ny)
        h = C.c_void_p()
        assert L.ns2d_create(C.byref(p), C.byref(h)) == abi.ERR_UNSUPPORTED


def test_phase_only_combinations_rejected_before_device_use():
    """The phase-only model is RK4Step's (solver.c:822-857): AB4 and DP5 with
    it are unsupported; model values other than 0 and 1 are invalid."""
    L = load()
    h = C.c_void_p()
    for integ in (abi.AB4, abi.DP5):
        p = abi.default_params(integrator=integ, model=abi.MODEL_PHASE_ONLY)
        assert L.ns2d_create(C.byref(p), C.byref(h)) == abi.ERR_UNSUPPORTED
    for model in (-1, 2):
        p = abi.default_params(model=model)
        assert L.ns2d_create(C.byref(p), C.byref(h)) == abi.ERR_INVALID
    p = abi.default_params(model=2)
    e = C.c_void_p()
    assert L.ns2d_ensemble_create(C.byref(p), 1, (C.c_int32 * 1)(64), C.byref(e)) == abi.ERR_INVALID


def test_triad_sector_sums_rejects_bad_arguments_before_device_use():
    """ns2d_triad_sector_sums validates its geometry before touching a device:
    missing tables or a kmax_sqr that would let k2 leave the tables are
    invalid."""
    L = load()

    class Geo(C.Structure):
        _fields_ = [("kmax", C.c_int32), ("n_k3", C.c_int32), ("n_k1", C.c_int32), ("reserved", C.c_int32),
                    ("kmax_sqr", C.c_double), ("kmax_c_sqr", C.c_double)] + [
                       (n, C.POINTER(C.c_double)) for n in ("k3_lwr", "k3_upr", "k1_lwr", "k1_upr", "angle", "angle_neg")]

    buf = (C.c_double * 1024)()
    p = C.cast(buf, C.POINTER(C.c_double))
    g = Geo(kmax=5, n_k3=2, n_k1=2, kmax_sqr=25.0, kmax_c_sqr=4.0, k3_lwr=p, k3_upr=p, k1_lwr=p, k1_upr=p,
            angle=p, angle_neg=p)
    L.ns2d_triad_sector_sums.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    bad = Geo.from_buffer_copy(g)
    bad.kmax_sqr = 26.0
    assert L.ns2d_triad_sector_sums(0, C.byref(bad), buf, buf, buf) == abi.ERR_INVALID
    bad = Geo.from_buffer_copy(g)
    bad.angle = None
    assert L.ns2d_triad_sector_sums(0, C.byref(bad), buf, buf, buf) == abi.ERR_INVALID
    assert L.ns2d_triad_sector_sums(0, C.byref(g), None, buf, buf) == abi.ERR_INVALID


def test_noalloc_rhs_argument_checks_before_device_use():
    """ns2d_nonlinear_rhs_noalloc refuses misaligned arrays and parameter sets
    that ns2d_create refuses before it touches a device (the pointers here are
    never dereferenced)."""
    L = load()
    f = L.ns2d_nonlinear_rhs_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(abi.Params), C.c_void_p, C.c_void_p, C.c_void_p]
    p = abi.default_params(nx=64, ny=64)
    # an array starting 8 bytes past a 16-byte boundary
    assert f(C.byref(p), C.c_void_p(0x10008), C.c_void_p(0x20000), None) == abi.ERR_INVALID
    assert f(C.byref(p), C.c_void_p(0x10000), C.c_void_p(0x20008), None) == abi.ERR_INVALID
    # KOLM forcing whose mode lies outside the array
    q = abi.default_params(nx=64, ny=64, forcing=abi.FORCING_KOLM, force_k=64 * 33, force_scale=1.0)
    assert f(C.byref(q), C.c_void_p(0x10000), C.c_void_p(0x20000), None) == abi.ERR_INVALID
    # model and integrator out of range
    q = abi.default_params(nx=64, ny=64)
    q.model = 2
    assert f(C.byref(q), C.c_void_p(0x10000), C.c_void_p(0x20000), None) == abi.ERR_INVALID
    q = abi.default_params(nx=64, ny=64, integrator=7)
    assert f(C.byref(q), C.c_void_p(0x10000), C.c_void_p(0x20000), None) == abi.ERR_INVALID
