"""The plain FP64 form against the reference's own compiled solver on the two
long FP64 workloads, at their full sizes:

* Kolmogorov flow at 1024^2 (n = 4, F = 1, nu = 1e-4, hyperviscosity
  nu_h |k|^16 through the RK4CN drag branch of solver.c:839-841, dt = 2.5e-4,
  seeded 1e-3 random-phase noise): 100 RK4CN steps through the graph-replayed
  step loop; w_hat within 1e-12 of max|w_hat| (the target stated for the
  plain form) and the energy, enstrophy and palinstrophy within 1e-11.
* Decaying turbulence at 256^2 (nu = 5e-4, the reference's integer Hou-Li
  filter, CFL 0.9 adaptive step with its row-index quirk, solver.c:2376-2490):
  all 2000 steps, every dt equal to the reference's within 1e-12 and w_hat
  within 1e-12 after 200 and after 2000 steps.

The checker is oracle/_ref/libns2d_ref_{rk4cn,houli}.so: the reference's
Solver/src/{solver,force,sys_msr}.c compiled by oracle/Makefile.  It runs in a
spawned process (the reference keeps its state in globals) on the host cores.
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

from _util import rel_err
from ns2d import Solver, abi, initial

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libns2d_ref_{}.so")


def _needs(variant):
    return pytest.mark.skipif(not os.path.exists(REF.format(variant)),
                              reason=f"reference build {variant} missing (oracle/Makefile ref)")


def kolmogorov_params():
    return abi.default_params(nx=1024, ny=1024, nu=1e-4, ekmn_drag_flag=1, ekmn_alpha=2e-40, ekmn_drag_pow=8.0,
                              forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0, dt=2.5e-4)


def decaying_houli_params():
    return abi.default_params(nx=256, ny=256, nu=5e-4, dealias=abi.DEALIAS_HOU_LI, adapt_step_flag=1,
                              cfl_cond_flag=1, cfl_const=0.9, dt=1e-3)


def _threads():
    return max(1, min(16, os.cpu_count() or 1))


def _kolmogorov_worker(q):
    from pyoracle import RefSolver
    p = kolmogorov_params()
    ref = RefSolver(p, "rk4cn", threads=_threads())
    ref.set_w_hat(initial.noise(1024, seed=7, amplitude=1e-3, kolm=True))
    out = {}
    for it in range(1, 101):
        ref.rk4_step(p.dt)
        if it in (50, 100):
            out[it] = (ref.get_w_hat(), ref.system_measurables()[0])
    q.put(out)


def _decaying_worker(steps, keep, q):
    from pyoracle import RefSolver
    p = decaying_houli_params()
    ref = RefSolver(p, "houli", threads=_threads())
    ref.set_w_hat(initial.decaying(256, seed=2, k0=6.0))
    dts, kept = [], {}
    dt = ref.get_timestep(p.dt)
    for it in range(1, steps + 1):
        dts.append(dt)
        ref.rk4_step(dt)
        dt = ref.get_timestep(dt)
        if it in keep:
            kept[it] = ref.get_w_hat()
    q.put((np.array(dts), kept))


def _spawn(target, *args):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=target, args=args + (q,))
    proc.start()
    out = q.get(timeout=900)
    proc.join(60)
    assert proc.exitcode == 0
    return out


@_needs("rk4cn")
def test_kolmogorov_1024_fp64_100_steps_against_reference():
    ref = _spawn(_kolmogorov_worker)
    p = kolmogorov_params()
    s = Solver(p)
    s.set_w_hat(initial.noise(1024, seed=7, amplitude=1e-3, kolm=True))
    for it in (50, 100):
        s.step_n(50, p.dt)
        w_ref, m_ref = ref[it]
        err = rel_err(s.get_w_hat(), w_ref)
        assert err <= 1e-12, (it, err)
        m, _ = s.system_measurables()
        for q in (0, 1, 2):  # energy, enstrophy, palinstrophy
            assert abs(m[q] - m_ref[q]) <= 1e-11 * abs(m_ref[q]), (it, q, m[q], m_ref[q])
    s.close()


@_needs("houli")
def test_decaying_256_houli_cfl_2000_steps_against_reference():
    steps, keep = 2000, (200, 2000)
    dts_ref, kept = _spawn(_decaying_worker, steps, keep)
    p = decaying_houli_params()
    s = Solver(p)
    s.set_w_hat(initial.decaying(256, seed=2, k0=6.0))
    dt = s.get_timestep(p.dt)
    worst_dt = 0.0
    for it in range(1, steps + 1):
        worst_dt = max(worst_dt, abs(dt - dts_ref[it - 1]) / dts_ref[it - 1])
        assert worst_dt <= 1e-12, (it, dt, dts_ref[it - 1])
        s.rk4_step(dt)
        dt = s.get_timestep(dt)
        if it in keep:
            err = rel_err(s.get_w_hat(), kept[it])
            assert err <= 1e-12, (it, err)
    s.close()
