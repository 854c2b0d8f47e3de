"""bin/ns2d_post (GPU post-processing of a saved run) against the reference
post-processing program's own spectra code (PostProcessing/src/full_field.c:
EnergySpectrum, EnstrophySpectrum, FluxSpectra, FullFieldData), built on the
CPU behind oracle/post_harness.c and run on the same snapshots: every
per-snapshot dataset and the set-C sums agree to 1e-10 of their scale (the
scale floor of test_gpu_cli.py for quantities that vanish up to rounding).
256^2 runs put modes on the dealiasing circle |k| = N/3, where the
post-processing program's edge (|k| > N/3 zeroed) differs from the solver's.
"""
import ctypes as C
import glob
import os
import subprocess

import numpy as np
import pytest

import h5read
from test_gpu_cli import _mismatch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NS2D = os.path.join(ROOT, "2d-navier-stokes_b200", "bin", "ns2d")
POST = os.path.join(ROOT, "2d-navier-stokes_b200", "bin", "ns2d_post")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "libns2d_post_ref.so")

needs_ref = pytest.mark.skipif(not os.path.exists(HARNESS), reason="post-processing harness not built (oracle/Makefile cli)")

SPEC = ["EnergySpectrum", "EnstrophySpectrum", "EnstrophyTimeDerivativeSpectrum", "EnstrophyFluxSpectrum",
        "EnstrophyDissSpectrum", "EnergyTimeDerivativeSpectrum", "EnergyFluxSpectrum", "EnergyDissSpectrum"]
FULL = ["FullFieldPhases", "FullFieldAmplitudes", "FullFieldEnergySpectrum", "FullFieldEnstrophySpectrum"]
CSUM = ["EnstrophyFluxC", "EnstrophyDissC", "EnergyFluxC", "EnergyDissC"]


def _run(args, cwd):
    r = subprocess.run(args, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (args[0], r.stdout[-1500:], r.stderr[-1500:])


def _harness(n, nu, hyper, hpow, alpha, drag, dpow, kfrac):
    L = C.CDLL(HARNESS)
    L.post_init.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double]
    L.post_snapshot.argtypes = [C.c_void_p] * 4
    n_spec = L.post_init(n, nu, hyper, hpow, alpha, drag, dpow, kfrac)
    kmax = L.post_kmax()
    return L, n_spec, kmax


@needs_ref
@pytest.mark.parametrize("n,visc,drag,kfrac", [
    (64, (1e-3, 0, 2.0), (0.0, 0, -2.0), 0.5),
    (64, (1e-3, 1, 2.0), (0.1, 1, -1.0), 1.0),
    (256, (1e-3, 0, 2.0), (0.05, 1, -2.0), 0.3),
])
def test_post_processing_matches_reference(n, visc, drag, kfrac, tmp_path):
    _run([NS2D, "--quiet", "-n", str(n), "-n", str(n), "-e", "0.002", "-h", "0.001", "-p", "1", "-v", "0.001",
          "-i", "DECAY_TURB_BB", "-o", "run/"], tmp_path)
    run_dir = os.path.join(glob.glob(str(tmp_path / "run" / "*"))[0], "")
    args = [POST, "-i", run_dir, "-o", str(tmp_path / "post") + "/", "-v", str(visc[0]), "-v", str(visc[1]),
            "-v", str(visc[2]), "-d", str(drag[0]), "-d", str(drag[1]), "-d", str(drag[2]), "-k", str(kfrac),
            "-t", "T"]
    _run(args, tmp_path)
    out = glob.glob(str(tmp_path / "post" / "PostProcessing_HDF_Data_SECTORS[[]24,8[]]_KFRAC*_TAG[[]T[]].h5"))
    assert len(out) == 1
    got, attrs = h5read.flatten(h5read.read(out[0]))
    run, run_attrs = h5read.flatten(h5read.read(run_dir + "Main_HDF_Data.h5"))
    snaps = sorted(k.split("/")[1] for k in run if k.endswith("/w_hat"))
    assert len(snaps) == 3

    L, n_spec, kmax = _harness(n, visc[0], visc[1], visc[2], drag[0], drag[1], drag[2], kfrac)
    m = (2 * kmax + 1) ** 2
    bad, csum = [], np.zeros((4, len(snaps)))
    for s, it in enumerate(snaps):
        w = np.ascontiguousarray(run[f"/{it}/w_hat"])
        spec = np.zeros(8 * n_spec)
        full = np.zeros(4 * m)
        c = np.zeros(4)
        L.post_snapshot(w.ctypes.data, spec.ctypes.data, full.ctypes.data, c.ctypes.data)
        csum[:, s] = c
        g = f"/Snap_{s:05d}"
        assert np.array_equal(got[g + "/w_hat"], w)
        assert float(attrs[g]["TimeValue"][0]) == float(run_attrs[f"/{it}"]["TimeValue"][0])
        sfloor = 1e-6 * max(np.abs(spec[:2 * n_spec]).max(), np.abs(spec).max())
        for k, name in enumerate(SPEC):
            mm = _mismatch(got[f"{g}/{name}"], spec[k * n_spec:(k + 1) * n_spec], sfloor)
            if mm:
                bad.append(f"{g}/{name}: {mm}")
        for k, name in enumerate(FULL):
            want = full[k * m:(k + 1) * m].reshape(2 * kmax + 1, 2 * kmax + 1)
            mm = _mismatch(got[f"{g}/{name}"], want, 1e-6 * np.abs(want).max())
            if mm:
                bad.append(f"{g}/{name}: {mm}")
    for k, name in enumerate(CSUM):
        mm = _mismatch(got["/" + name], csum[k], 1e-6 * np.abs(csum).max())
        if mm:
            bad.append(f"{name}: {mm}")
    assert not bad, bad[:20]
    assert np.array_equal(got["/kx"], np.r_[np.arange(n // 2 + 1), np.arange(-n // 2 + 1, 0)])
    assert np.array_equal(got["/ky"], np.arange(n // 2 + 1))
    assert np.allclose(got["/Time"], [float(run_attrs[f"/{it}"]["TimeValue"][0]) for it in snaps])


def test_post_processing_rejects_bad_arguments(tmp_path):
    for args in (["-k", "0"], ["-k", "1.5"], ["-v", "-1"], ["-d", "0", "-d", "0", "-d", "1"], ["-i", "/nonexistent/"],
                 ["-q"]):
        r = subprocess.run([POST] + args, cwd=tmp_path, capture_output=True, text=True, timeout=60)
        assert r.returncode == 1, args
