"""The FP32 forms on their full workloads, against the FP64 form (itself pinned
to the reference's compiled solver, tests/test_gpu_reference_long.py and the
golden fixtures).

* Kolmogorov flow at 1024^2 (n = 4, F = 1, nu = 1e-4, hyperviscosity
  nu_h |k|^16, dt = 2.5e-4, seeded 1e-3 random-phase noise), 5000 RK4CN steps
  in FP32 and in FP64 with the energy, enstrophy and palinstrophy totals
  (ComputeSystemMeasurables, sys_msr.c:146-372) saved every 50 steps.  The
  FP32 series drifts from the FP64 one roughly linearly in the step count
  (measured on a B200: max relative deviation 4.6e-5 for E, 4.0e-5 for Z,
  1.1e-5 for P over the 5000 steps, 4.7e-7 after the first 50); the bound here
  is 1e-4 for each series.
* The uneven 64-member ensemble (32 x 128^2, 24 x 256^2, 8 x 512^2; decaying
  spectra with k0 drawn from {4, 6, 8}; nu = 1e-3, dt = 1e-3), 1000 steps of
  the FP32 ensemble (autotuned grids, graph-replayed steps) against the FP64
  ensemble (equal to single FP64 handles to 1e-14, tests/test_gpu_ensemble.py):
  every member's enstrophy within 1e-5 relative, the target stated for the
  batched form (measured: 3.6e-6).
"""
import numpy as np
import pytest

from ns2d import Ensemble, Solver, abi, initial

pytestmark = pytest.mark.gpu

ENS_SIZES = [128] * 32 + [256] * 24 + [512] * 8


def _kolmogorov(precision):
    return abi.default_params(nx=1024, ny=1024, nu=1e-4, ekmn_drag_flag=1, ekmn_alpha=2e-40, ekmn_drag_pow=8.0,
                              forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0, dt=2.5e-4, precision=precision)


def test_kolmogorov_1024_fp32_series_against_fp64():
    w0 = initial.noise(1024, seed=7, amplitude=1e-3, kolm=True)
    series = {}
    for prec in (abi.FP64, abi.FP32):
        s = Solver(_kolmogorov(prec))
        s.set_w_hat(w0)
        rows = []
        for _ in range(100):
            s.step_n(50, 2.5e-4)
            m, _ = s.system_measurables()
            rows.append(m[:3].copy())
        s.close()
        series[prec] = np.array(rows)
    dev = np.abs(series[abi.FP32] - series[abi.FP64]) / np.abs(series[abi.FP64])
    worst = dev.max(axis=0)
    assert np.all(worst <= 1e-4), worst
    assert np.all(np.isfinite(series[abi.FP64])) and np.all(series[abi.FP64] > 0.0)


def test_ensemble_64_members_fp32_enstrophy_1000_steps():
    rng = np.random.default_rng(100)
    ics = [initial.decaying(n, seed=m, k0=float(rng.choice([4, 6, 8])), dealias="2/3")
           for m, n in enumerate(ENS_SIZES)]
    z = {}
    for prec in (abi.FP64, abi.FP32):
        e = Ensemble(abi.default_params(nu=1e-3, dt=1e-3, precision=prec), ENS_SIZES)
        if prec == abi.FP32:
            e.tune(1e-3)
        for m, w in enumerate(ics):
            e.set_w_hat(m, w)
        e.step_n(1000, 1e-3)
        z[prec] = np.array([e.measurables(m).enstrophy for m in range(len(ENS_SIZES))])
        e.close()
    rel = np.abs(z[abi.FP32] - z[abi.FP64]) / np.abs(z[abi.FP64])
    assert rel.max() <= 1e-5, (int(rel.argmax()), rel.max())
