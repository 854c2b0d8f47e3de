"""Drop-in proof: the reference program with its per-step entry points
(RK4Step, NonlinearRHSBatch, ApplyDealiasing, ForceConjugacy, GetMaxData,
GetTimestep) resolved to 2d-navier-stokes_b200/compat/ns2d_compat.c over the
GPU, and nothing else changed (oracle/_ref/libns2d_ref_dropin.so, built by
oracle/Makefile target `dropin`), reproduces the reference's own CPU outputs:
the golden programs through the harness, and a whole SpectralSolve run.

Each run is a spawned process: the reference keeps its state in globals."""
import multiprocessing as mp
import os

import numpy as np
import pytest

from _util import GOLDEN, load_case, rel_err

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DROPIN = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libns2d_ref_dropin.so")
REF_CPU = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libns2d_ref_rk4cn.so")

needs_dropin = pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in library not built (oracle/Makefile dropin)")


def _program_worker(name, q):
    import make_golden
    from pyoracle import RefSolver
    p, w0, _ = load_case(name)
    ref = RefSolver(p, "dropin")
    _, _, ic, program = make_golden.cases()[name]
    q.put(make_golden.run_program(ref, w0, program, True))


def _solve_worker(variant, kw, u0, T, every, forcing, q):
    import pyoracle
    from ns2d import abi
    q.put(pyoracle.solve(abi.default_params(**kw), variant, u0, T=T, save_every=every, forcing=forcing))


def _spawn(target, *args):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=target, args=args + (q,))
    proc.start()
    out = q.get(timeout=600)
    proc.join(60)
    assert proc.exitcode == 0
    return out


@needs_dropin
@pytest.mark.parametrize("name", ["tg64_rk4cn", "dec64_rk4cn", "kolm64_rk4cn", "nonherm32_rhs", "cfl32"])
def test_reference_harness_on_gpu_entry_points(name):
    """The golden programs (steps, RHS calls, GetMaxData, GetTimestep,
    ComputeSystemMeasurables) run by the reference's harness with the GPU
    entry points match the reference's CPU outputs."""
    p, w0, golden = load_case(name)
    outs = _spawn(_program_worker, name)
    assert len(outs) == len(golden)
    for got, want in zip(outs, golden):
        got, want = np.asarray(got), np.asarray(want)
        if want.size == 1:
            assert abs(float(got) - float(want)) <= 1e-11 * max(abs(float(want)), 1e-300)
        else:
            scale = np.abs(want).max()
            floor = 1e-14 * scale if scale else 1e-14
            assert np.abs(got - want).max() <= max(1e-11 * scale, floor)


@needs_dropin
@pytest.mark.parametrize("u0,kw,T,every,forcing", [
    ("TG_VORT", dict(nx=64, ny=64, nu=1e-3, dt=1e-3, ekmn_drag_flag=1), 0.05, 10, None),
    ("DECAY_TURB_BB", dict(nx=64, ny=64, nu=1e-3, dt=1e-3), 0.05, 10, None),
    ("DECAY_TURB_BB", dict(nx=64, ny=64, nu=1e-3, dt=1e-3, adapt_step_flag=1, cfl_cond_flag=1, cfl_const=0.9),
     0.5, 1, None),
    # the reference's stochastic forcings draw their values with rand() on the
    # host; the drop-in passes them to the GPU every step
    ("DECAY_TURB_BB", dict(nx=64, ny=64, nu=1e-3, dt=1e-3, force_k=4, force_scale=1.0), 0.03, 10, "STOC"),
    ("DECAY_TURB_BB", dict(nx=64, ny=64, nu=1e-3, dt=1e-3, force_k=4, force_scale=1.0), 0.03, 10, "STOC_GAUSS"),
    ("DECAY_TURB_BB", dict(nx=64, ny=64, nu=1e-3, dt=1e-3, force_k=2), 0.03, 10, "ZERO"),
])
def test_spectral_solve_on_gpu_entry_points(u0, kw, T, every, forcing):
    """The reference's own SpectralSolve loop (initial condition, forcing,
    steps, saves, measurables, adaptive dt, SystemCheck): the state it saves
    last agrees between the CPU build and the drop-in build to 1e-12."""
    w_cpu, t_cpu, n_cpu = _spawn(_solve_worker, "rk4cn", kw, u0, T, every, forcing)
    w_gpu, t_gpu, n_gpu = _spawn(_solve_worker, "dropin", kw, u0, T, every, forcing)
    assert n_gpu == n_cpu and n_cpu >= 2
    assert abs(t_gpu - t_cpu) <= 1e-12 * max(t_cpu, 1.0)
    assert rel_err(w_gpu, w_cpu) <= 1e-12
