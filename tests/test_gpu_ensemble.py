"""Batched ensembles on the GPU (the uneven 64-member ensemble workload, scaled down).

FP64 members must reproduce single-trajectory handles (same per-column and
per-row arithmetic; only the launch grouping differs), to 1e-14 of max|w_hat|.
FP32 members: enstrophy within 1e-5 (relative) of the FP64 oracle after 100
RK4CN steps, the target stated for the batched form."""
import numpy as np
import pytest

from _util import rel_err
from ns2d import Ensemble, Solver, abi, initial
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _ics(sizes, seed0=0):
    rng = np.random.default_rng(1234)
    return [initial.decaying(n, seed=seed0 + m, k0=float(rng.choice([4, 6, 8])) * n / 128.0, dealias="2/3")
            for m, n in enumerate(sizes)]


def test_fp64_ensemble_equals_single_handles():
    sizes = [64, 128, 64, 256, 512, 128]
    p = abi.default_params(nu=1e-3, dt=1e-3)
    ics = _ics(sizes)
    e = Ensemble(p, sizes)
    for m, w in enumerate(ics):
        e.set_w_hat(m, w)
    e.step_n(12, 1e-3)
    for m, n in enumerate(sizes):
        s = Solver(abi.default_params(nx=n, ny=n, nu=1e-3, dt=1e-3))
        s.set_w_hat(ics[m])
        s.step_n(12, 1e-3)
        assert rel_err(e.get_w_hat(m), s.get_w_hat()) <= 1e-14, (m, n)
        s.close()
    assert e.launch_count > 0
    e.close()


def test_phase_only_ensemble_equals_single_handles():
    """The phase-only model (RK4Step's amplitude reset) in an FP64 ensemble
    of mixed sizes equals single phase-only handles."""
    sizes = [64, 128, 256]
    p = abi.default_params(nu=1e-3, dt=1e-3, model=abi.MODEL_PHASE_ONLY)
    ics = _ics(sizes, seed0=40)
    e = Ensemble(p, sizes)
    for m, w in enumerate(ics):
        e.set_w_hat(m, w)
    e.step_n(10, 1e-3)
    for m, n in enumerate(sizes):
        s = Solver(abi.default_params(nx=n, ny=n, nu=1e-3, dt=1e-3, model=abi.MODEL_PHASE_ONLY))
        s.set_w_hat(ics[m])
        s.step_n(10, 1e-3)
        assert rel_err(e.get_w_hat(m), s.get_w_hat()) <= 1e-14, (m, n)
        s.close()
    e.close()


def test_fp32_ensemble_enstrophy_vs_fp64_oracle():
    sizes = [128, 256, 128]
    p = abi.default_params(nu=1e-3, dt=1e-3, precision=abi.FP32)
    ics = _ics(sizes, seed0=40)
    e = Ensemble(p, sizes)
    for m, w in enumerate(ics):
        e.set_w_hat(m, w)
    e.step_n(100, 1e-3)
    for m, n in enumerate(sizes):
        o = Oracle(abi.default_params(nx=n, ny=n, nu=1e-3, dt=1e-3), threads=8)
        o.set_w_hat(ics[m])
        for _ in range(100):
            o.rk4_step(1e-3)
        z_ref = initial.enstrophy(o.get_w_hat())
        z32 = e.measurables(m).enstrophy
        assert abs(z32 - z_ref) <= 1e-5 * z_ref, (m, n, z32, z_ref)
    e.close()


def test_autotuner_and_graph_replay_keep_results():
    sizes = [64, 128, 256]
    p = abi.default_params(nu=1e-3, dt=1e-3)
    ics = _ics(sizes, seed0=70)
    e = Ensemble(p, sizes)
    cg, rg = e.tune(1e-3)
    assert cg >= 1 and rg >= 1
    for m, w in enumerate(ics):
        e.set_w_hat(m, w)
    e.step_n(6, 1e-3)
    ref = Ensemble(p, sizes)
    for m, w in enumerate(ics):
        ref.set_w_hat(m, w)
    for _ in range(6):
        ref.step_n(1, 1e-3)
    for m in range(len(sizes)):
        assert rel_err(e.get_w_hat(m), ref.get_w_hat(m)) <= 1e-15
    e.close()
    ref.close()


@pytest.mark.parametrize("col_threads,row_threads", [(128, 128), (128, 256), (256, 128)])
def test_block_size_choices_keep_results(col_threads, row_threads):
    """The autotuner's tile-shape choices (block size of the column and of the
    row launches) change only how members are cut into tiles: every member
    equals the default 256-thread shape's result."""
    sizes = [64, 512, 128, 256]
    p = abi.default_params(nu=1e-3, dt=1e-3)
    ics = _ics(sizes, seed0=90)
    ref = Ensemble(p, sizes)
    e = Ensemble(p, sizes)
    sh = e.shape
    assert (sh["col_threads"], sh["row_threads"]) == (256, 256)
    e.set_shape(col_threads, 2 * 148, row_threads, 3 * 148)
    sh = e.shape
    assert (sh["col_threads"], sh["row_threads"]) == (col_threads, row_threads)
    assert sh["col_grid"] <= sh["col_items"] and sh["row_grid"] <= sh["row_items"]
    for m, w in enumerate(ics):
        ref.set_w_hat(m, w)
        e.set_w_hat(m, w)
    ref.step_n(5, 1e-3)
    e.step_n(5, 1e-3)
    for m in range(len(sizes)):
        assert rel_err(e.get_w_hat(m), ref.get_w_hat(m)) <= 1e-15, m
    e.close()
    ref.close()


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32])
def test_one_launch_per_stage_equals_nine_launches(precision):
    """One persistent launch per RK stage (tasks wait only for the same
    member's earlier tasks) runs the same bodies on the same tiles as the
    nine-launch step: every member equals it, eagerly and from the captured
    graph, over several steps -- bit for bit in FP64, within FP32 rounding
    (1e-5 of max|w_hat|; the two kernels may contract differently) in FP32."""
    sizes = [512, 64, 256, 128, 128, 512]
    p = abi.default_params(nu=1e-3, dt=1e-3, precision=precision)
    ics = _ics(sizes, seed0=120)
    ref = Ensemble(p, sizes)
    e = Ensemble(p, sizes)
    e.set_shape(256, 8 * 148, 256, 8 * 148, stage_launch=1, stage_grid=2 * 148)
    sh = e.shape
    assert sh["stage_launch"] == 1 and sh["stage_grid"] >= 1
    ref.set_shape(256, 8 * 148, 256, 8 * 148, stage_launch=0)
    for m, w in enumerate(ics):
        ref.set_w_hat(m, w)
        e.set_w_hat(m, w)
    l0 = e.launch_count
    ref.step_n(7, 1e-3)
    e.step_n(7, 1e-3)
    e.check()
    assert e.launch_count - l0 < 7 * 9  # four launches a step (plus the first steps' tables)
    tol = 1e-15 if precision == abi.FP64 else 1e-5
    for m in range(len(sizes)):
        assert rel_err(e.get_w_hat(m), ref.get_w_hat(m)) <= tol, m
    e.close()
    ref.close()
