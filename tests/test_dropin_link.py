"""The drop-in build (oracle/_ref/libns2d_ref_dropin.so) links the reference's
own objects with 2d-navier-stokes_b200/compat/ns2d_compat.c: the six per-step
entry points it exports are the compat ones, which call into libns2d.so, and
the reference code reaches them through the dynamic symbol table (no CPU path
left behind them).  Link-level checks only; tests/test_gpu_dropin.py runs it."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
DROPIN = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libns2d_ref_dropin.so")
SYMS = ["RK4Step", "NonlinearRHSBatch", "ApplyDealiasing", "ForceConjugacy", "GetMaxData", "GetTimestep"]

pytestmark = pytest.mark.skipif(not os.path.exists(DROPIN) or not shutil.which("nm"),
                                reason="drop-in library not built")


def test_entry_points_are_the_gpu_ones():
    out = subprocess.run(["nm", "-D", "--defined-only", DROPIN], capture_output=True, text=True, check=True).stdout
    defined = {line.split()[-1]: line.split()[1] for line in out.splitlines() if len(line.split()) == 3}
    for s in SYMS:
        assert defined.get(s) == "T", s  # one strong definition each
    und = subprocess.run(["nm", "-D", "--undefined-only", DROPIN], capture_output=True, text=True, check=True).stdout
    for s in ("ns2d_rk4_step_host", "ns2d_nonlinear_rhs", "ns2d_apply_dealiasing", "ns2d_get_max_data",
              "ns2d_get_timestep", "ns2d_create"):
        assert s in und
    needed = subprocess.run(["readelf", "-d", DROPIN], capture_output=True, text=True, check=True).stdout
    assert "libns2d.so" in needed
