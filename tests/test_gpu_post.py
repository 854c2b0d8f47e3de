"""bin/ns2d_post (GPU post-processing of a saved run) against the reference
post-processing program's own spectra code (PostProcessing/src/full_field.c:
EnergySpectrum, EnstrophySpectrum, FluxSpectra, FullFieldData), built on the
CPU behind oracle/post_harness.c and run on the same snapshots: every
per-snapshot dataset and the set-C sums agree to 1e-10 of their scale (the
scale floor of test_gpu_cli.py for quantities that vanish up to rounding).
256^2 runs put modes on the dealiasing circle |k| = N/3, where the
post-processing program's edge (|k| > N/3 zeroed) differs from the solver's.
--phase-sync is checked against that program's phase_sync.c (-D__SEC_PHASE_SYNC)
behind oracle/phase_sync_harness.c.
"""
import ctypes as C
import glob
import os
import subprocess
import sys

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


PS_HARNESS = os.path.join(ROOT, "oracle", "_ref", "libns2d_ps_ref.so")

# Runs the reference's phase-sync code (oracle/phase_sync_harness.c) on the
# snapshots of a saved run, in its own process (the reference keeps its state
# in globals) and in a directory where its triad search can write its
# wavevector file (phase_sync.c:1725-1730).
_PS_CHILD = r"""
import ctypes as C, sys, numpy as np
sys.path.insert(0, sys.argv[1])
import h5read
lib, run, out, n, kfrac, a3, a1, red = sys.argv[2], sys.argv[3], sys.argv[4], int(sys.argv[5]), float(sys.argv[6]), int(sys.argv[7]), int(sys.argv[8]), int(sys.argv[9])
L = C.CDLL(lib)
L.ps_init.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
kmax = L.ps_init(n, 1e-3, 0, 2.0, 0.05, 1, -2.0, kfrac, a3, a1, red)
data, _ = h5read.flatten(h5read.read(run))
snaps = sorted(k.split("/")[1] for k in data if k.endswith("/w_hat"))
nt, res = 7, {}
def arr(*shape, dt=np.float64):
    return np.zeros(shape, dt)
for s, it in enumerate(snaps):
    w = np.ascontiguousarray(data[f"/{it}/w_hat"])
    L.ps_snapshot(w.ctypes.data)
    num, num1, num2 = arr(nt, a3, dt=np.int32), arr(nt, a3, dt=np.int32), arr(nt, a3, a1, dt=np.int32)
    L.ps_get_counts(num.ctypes.data, num1.ctypes.data, num2.ctypes.data)
    r, p, r1, p1, r2, p2 = arr(nt, a3), arr(nt, a3), arr(nt, a3), arr(nt, a3), arr(nt, a3, a1), arr(nt, a3, a1)
    L.ps_get_sync(*(x.ctypes.data for x in (r, p, r1, p1, r2, p2)))
    f, f1, f2 = arr(nt, a3), arr(nt, a3), arr(nt, a3, a1)
    L.ps_get_flux(f.ctypes.data, f1.ctypes.data, f2.ctypes.data)
    cs = [arr(nt, a3, dt=np.complex128) for _ in range(4)] + [arr(nt, a3, a1, dt=np.complex128) for _ in range(2)]
    L.ps_get_collective(*(x.ctypes.data for x in cs))
    fl, di, od = arr(a3), arr(a3), arr(a3, dt=np.complex128)
    df, t3, t1 = np.zeros_like(w), arr(a3), arr(a1)
    L.ps_get_c_theta(*(x.ctypes.data for x in (fl, di, od, df, t3, t1)))
    g = f"/Snap_{s:05d}/"
    res.update({g + "TriadPhaseSync": r, g + "TriadAverageAngle": p, g + "TriadPhaseSync_1D": r1,
                g + "TriadAverageAngle_1D": p1, g + "TriadPhaseSync_2D": r2, g + "TriadAverageAngle_2D": p2,
                g + "EnstrophyFluxPerSector": f, g + "EnstrophyFluxPerSector_1D": f1, g + "EnstrophyFluxPerSector_2D": f2,
                g + "EnstrophyFlux_C_theta": fl, g + "EnstrophyDiss_C_theta": di, g + "CollectivePhaseOrder_C_theta": od,
                g + "EnstrophyDissipationField": df})
    for name, x in zip(["", "_Unidirectional", "_1D", "_1D_Unidirectional", "_2D", "_2D_Unidirectional"], cs):
        res[g + "CollectivePhaseOrder_C_theta_Triads" + name] = x
    res.update({"/NumTriadsPerSector": num, "/NumTriadsPerSector_1D": num1, "/NumTriadsPerSector_2D": num2,
                "/SectorAngles_k3": t3, "/SectorAngles_k1": t1})
np.savez(out, **{k.replace("/", "|"): v for k, v in res.items()})
"""


@pytest.mark.skipif(not os.path.exists(PS_HARNESS), reason="phase-sync harness not built (oracle/Makefile cli)")
@pytest.mark.parametrize("n,kfrac,sectors", [(32, 0.5, []), (64, 0.6, ["-a", "12"]), (32, 0.4, ["-a", "12", "-a", "8", "-a", "x"]),
                                             (32, 0.5, ["-a", "12", "-a", "1"])])
def test_phase_sync_matches_reference(n, kfrac, sectors, tmp_path):
    """bin/ns2d_post --phase-sync (triad sums on the GPU) against the reference
    post-processing program's phase_sync.c and the -D__SEC_PHASE_SYNC parts of
    full_field.c on the same snapshots: triad counts equal, per-sector fluxes
    and collective sums to 1e-10 of their scale, order parameters to 1e-10
    (average angles where the order parameter exceeds 1e-6); default sectors,
    a full 12 x 12 search, the reduced 8-sector k1 search, and one k1 sector
    (k1 anywhere, phase_sync.c:1762-1766)."""
    _run([NS2D, "--quiet", "-n", str(n), "-n", str(n), "-e", "0.002", "-h", "0.001", "-p", "1", "-v", "0.001",
          "-i", "DECAY_TURB_BB", "-o", "run/"], tmp_path)
    run_dir = os.path.join(glob.glob(str(tmp_path / "run" / "*"))[0], "")
    _run([POST, "--phase-sync", "-i", run_dir, "-o", str(tmp_path / "post") + "/", "-v", "0.001", "-v", "0", "-v", "2.0",
          "-d", "0.05", "-d", "1", "-d", "-2.0", "-k", str(kfrac), "-t", "P"] + sectors, tmp_path)
    out = glob.glob(str(tmp_path / "post" / "PostProcessing_HDF_Data_SECTORS*_TAG[[]P[]].h5"))
    assert len(out) == 1
    got, _ = h5read.flatten(h5read.read(out[0]))
    a3 = int(sectors[1]) if sectors else 24
    a1 = 8 if len(sectors) >= 6 else (int(sectors[3]) if len(sectors) >= 4 else (a3 if sectors else 8))
    red = 1 if len(sectors) >= 6 else 0
    cwd = tmp_path / "ref"
    (cwd / "Data" / "PostProcess" / "PhaseSync").mkdir(parents=True)
    npz = str(tmp_path / "ref.npz")
    r = subprocess.run([sys.executable, "-c", _PS_CHILD, os.path.dirname(__file__), PS_HARNESS, run_dir + "Main_HDF_Data.h5",
                        npz, str(n), str(kfrac), str(a3), str(a1), str(red)], cwd=cwd, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    want = {k.replace("|", "/"): v for k, v in np.load(npz).items()}
    assert want["/NumTriadsPerSector"][0].sum() > 0
    bad = []
    for k, v in want.items():
        g = np.asarray(got[k])
        if v.dtype.kind == "i":
            if not np.array_equal(g, v):
                bad.append(f"{k}: counts differ")
            continue
        if k.endswith("EnstrophyDissipationField"):
            v, g = v.copy(), g.copy()
            v[0, 0] = g[0, 0] = 0  # the reference leaves mode (0, 0) unset
        if "AverageAngle" in k:
            rk = k.replace("AverageAngle", "PhaseSync")
            sel = want[rk] > 1e-6
            d = np.abs(np.angle(np.exp(1j * (g[sel] - v[sel]))))
            if d.size and d.max() > 1e-8:
                bad.append(f"{k}: angle err {d.max():.3e}")
            continue
        # order parameters lie in [0, 1]: absolute 1e-10; the rest 1e-10 of the dataset's scale
        mm = _mismatch(g, v, 1.0 if "PhaseSync" in k else 0.0)
        if mm:
            bad.append(f"{k}: {mm}")
    assert not bad, bad[:20]
    for name in ("PhaseSync", "AverageAngle", "TriadPhaseSyncTest", "TriadAverageAngleTest", "EnstrophyFluxTest"):
        assert not np.any(got[f"/Snap_00000/{name}"])
    assert np.array_equal(got["/NumTriadsTest"], np.zeros(7, np.int32))
