"""bin/ns2d (GPU) against the reference program (oracle/_ref/solver_ref: the
reference's main.c, utils.c, hdf5_funcs.c, solver.c, force.c and sys_msr.c on
the CPU, its HDF5 writes logged by the oracle's stand-in), run with the same
argv: the same output directory, and in Main_HDF_Data.h5,
Spectra_HDF_Data.h5 and SystemMeasures_HDF_Data.h5 the same datasets and
group attributes with values equal to 1e-10 of each dataset's largest
magnitude (the FP64 state itself agrees to ~1e-13).  Our files are read with
the strict reader tests/h5read.py.

Left out of the comparison, with the reason in the reference's source:
MeanFlow_x (sys_msr.c:338-348 indexes the ky array with the row counter);
the RANDOM, GAUSS_BLOB and CONST_GAUSS set-ups (they read uninitialised or
out-of-bounds memory: solver.c:1891-1912, 1865, force.c:355-357); a start time
t0 > 0 with fixed steps (the loop's t = iters * dt restarts the clock at 0,
solver.c:230, so the run takes more saves than the measures arrays hold and
sys_msr.c:60 writes past them)."""
import ctypes as C
import glob
import os
import subprocess

import numpy as np
import pytest

import h5log
import h5read

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NS2D = os.path.join(ROOT, "2d-navier-stokes_b200", "bin", "ns2d")
REF = os.path.join(ROOT, "oracle", "_ref", "solver_ref")
H5LIB = os.path.join(ROOT, "2d-navier-stokes_b200", "lib", "libns2d_h5.so")

needs_ref = pytest.mark.skipif(not os.path.exists(REF), reason="reference program not built (oracle/Makefile cli)")

BASE = "-n 64 -n 64 -s 0.0 -v 0.001 -t T"
CASES = {
    "decay_fixed": "-e 0.02 -h 0.001 -p 5 -i DECAY_TURB_BB",
    "decay_adaptive": "-e 0.1 -h 0.001 -h 1 -c 1 -c 0.9 -p 2 -i DECAY_TURB_BB",
    "tg_drag": "-e 0.01 -h 0.001 -p 3 -i TG_VORT -d 0.0 -d 1 -d -2.0",
    "hyper": "-e 0.01 -h 0.001 -p 4 -i DECAY_TURB_NB -v 0.001 -v 1 -v 2.0",
    "kolm": "-e 0.01 -h 0.001 -p 5 -i DECAY_TURB_BB -f KOLM -f 4 -f 1.0",
    "stoc": "-e 0.01 -h 0.001 -p 5 -i DECAY_TURB_BB -f STOC -f 4 -f 1.0",
    "stoc_gauss": "-e 0.01 -h 0.001 -p 5 -i DECAY_TURB_BB -f STOC_GAUSS -f 4 -f 1.0",
    "zero": "-e 0.01 -h 0.001 -p 5 -i DECAY_TURB_BB -f ZERO -f 2",
    "transient": "-e 0.02 -h 0.001 -p 2 -T 1 -T 0.5 -i DECAY_TURB_BB",
    "decay_alt": "-e 0.004 -h 0.001 -p 2 -i DECAY_TURB_ALT",
    "decay_exp": "-e 0.004 -h 0.001 -p 2 -i DECAY_TURB_EXP",
    "gauss_decay": "-e 0.004 -h 0.001 -p 2 -i GAUSS_DECAY_TURB",
    "extrm_ens": "-e 0.004 -h 0.001 -p 2 -i EXTRM_ENS",
    "ring": "-e 0.004 -h 0.001 -p 2 -i RING",
    "unif": "-e 0.004 -h 0.001 -p 2 -i UNIF",
    "shear": "-e 0.004 -h 0.001 -p 2 -i DOUBLE_SHEAR_LAYER",
    "tg_vel": "-e 0.004 -h 0.001 -p 2 -i TG_VEL",
    "testing": "-e 0.004 -h 0.001 -p 2 -i TESTING",
    "zero_kolm": "-e 0.004 -h 0.001 -p 2 -i ZERO_KOLM",
    "unknown_ic": "-e 0.004 -h 0.001 -p 2 -i NO_SUCH_IC",
}
FILES = ("Main_HDF_Data.h5", "Spectra_HDF_Data.h5", "SystemMeasures_HDF_Data.h5")
SKIP = {"/MeanFlow_x"}


def _run(exe, args, cwd, extra=()):
    r = subprocess.run([exe] + list(extra) + args.split(), cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
    return r


def _mismatch(got, want, floor=0.0):
    """None if got equals want to 1e-10 of max(|want|, floor), else the error.
    The floor lets quantities that vanish up to rounding (the divergence of
    the velocity, the flux spectra of a state whose transfer cancels) be
    compared on the scale of their group's other datasets."""
    got, want = np.asarray(got), np.asarray(want)
    if got.shape != want.shape:
        return f"shape {got.shape} != {want.shape}"
    if want.dtype.kind in "iu":
        return None if np.array_equal(got, want) else "integers differ"
    if not want.size:
        return None
    scale = max(np.abs(want).max(), floor)
    err = np.abs(got - want).max()
    return None if err <= 1e-10 * scale + 1e-300 else f"err {err:.3e} of scale {scale:.3e}"


def _close(got, want, what):
    bad = _mismatch(got, want)
    assert bad is None, (what, bad)


def _compare_file(got, want, fname):
    """All float datasets of a group share a floor of 1e-6 x the group's
    largest magnitude."""
    group_max = {}
    for k, v in want.items():
        if k not in SKIP and np.asarray(v).dtype.kind in "fc" and np.asarray(v).size:
            g = k.rsplit("/", 1)[0]
            group_max[g] = max(group_max.get(g, 0.0), float(np.abs(v).max()))
    bad = []
    for k in want:
        if k in SKIP:
            continue
        m = _mismatch(got[k], want[k], 1e-6 * group_max.get(k.rsplit("/", 1)[0], 0.0))
        if m:
            bad.append(f"{fname}:{k}: {m}")
    return bad


@needs_ref
@pytest.mark.parametrize("case", sorted(CASES))
def test_outputs_match_reference_program(case, tmp_path):
    args = f"{BASE} {CASES[case]} -o out/"
    (tmp_path / "ref").mkdir()
    (tmp_path / "gpu").mkdir()
    _run(REF, args, tmp_path / "ref")
    _run(NS2D, args, tmp_path / "gpu", ["--quiet"])
    rdirs = sorted(os.listdir(tmp_path / "ref" / "out"))
    gdirs = sorted(os.listdir(tmp_path / "gpu" / "out"))
    assert rdirs == gdirs and len(rdirs) == 1, (rdirs, gdirs)
    rdir = tmp_path / "ref" / "out" / rdirs[0]
    gdir = tmp_path / "gpu" / "out" / gdirs[0]
    assert (gdir / "SimulationDetails.txt").exists()
    bad = []
    for fname in FILES:
        want, want_attrs, _ = h5log.read(str(rdir / fname))
        got, got_attrs = h5read.flatten(h5read.read(str(gdir / fname)))
        assert set(got) == set(want), (fname, sorted(set(got) ^ set(want)))
        bad += _compare_file(got, want, fname)
        assert set(got_attrs) == set(want_attrs), fname
        for g, av in want_attrs.items():
            for name, v in av.items():
                assert abs(float(got_attrs[g][name][0]) - v) <= 1e-12 * max(abs(v), 1e-300), (fname, g, name)
    assert not bad, bad[:20]


def test_max_palin_reads_its_input_file(tmp_path):
    """MAX_PALIN (solver.c:1775-1853) reads /psi from
    <input_dir>MaxPalinstrophy/maxdpdt_P10000_N<N>_IG0_psi_f.h5 and starts
    from w = -k^2 psi_hat, dealiased, conjugate-symmetric on ky = 0."""
    n = 64
    L = C.CDLL(H5LIB)
    L.ns2d_h5_create.restype = C.c_void_p
    L.ns2d_h5_create.argtypes = [C.c_char_p]
    L.ns2d_h5_dataset.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.c_void_p]
    L.ns2d_h5_close.argtypes = [C.c_void_p]
    d = tmp_path / "Data" / "Solver" / "InitialConditions" / "MaxPalinstrophy"
    d.mkdir(parents=True)
    x = 2 * np.pi * np.arange(n) / n
    psi = np.sin(3 * x)[:, None] * np.cos(2 * x)[None, :] + 0.1 * np.cos(x)[:, None]
    f = L.ns2d_h5_create(str(d / f"maxdpdt_P10000_N{n}_IG0_psi_f.h5").encode())
    dims = (C.c_uint64 * 2)(n, n)
    assert L.ns2d_h5_dataset(f, b"/psi", 0, 2, dims, psi.ctypes.data_as(C.c_void_p)) == 0
    assert L.ns2d_h5_close(f) == 0
    _run(NS2D, f"-n {n} -n {n} -e 0.002 -h 0.001 -p 1 -i MAX_PALIN -o out/", tmp_path, ["--quiet"])
    main = glob.glob(str(tmp_path / "out" / "*" / "Main_HDF_Data.h5"))[0]
    got, _ = h5read.flatten(h5read.read(main))
    kx = np.fft.fftfreq(n, 1.0 / n)
    kx[n // 2] = n // 2
    ky = np.arange(n // 2 + 1)
    k2 = kx[:, None] ** 2 + ky[None, :] ** 2
    want = -k2 * np.fft.rfft2(psi)
    want[k2 >= (n // 3) ** 2] = 0
    want[n // 2 + 1:, 0] = np.conj(want[1:n // 2, 0][::-1])
    w0 = got["/Iter_00000/w_hat"]
    assert np.abs(w0 - want).max() <= 1e-12 * np.abs(want).max()


@needs_ref
def test_blowup_exits_with_status_1_and_valid_files(tmp_path):
    """SystemCheck (solver.c:2301-2326): a run that blows up (dt = 20) stops
    with status 1 in both programs, after the same saves; our files written
    up to then are complete HDF5 files and hold what the reference wrote."""
    args = "-n 64 -n 64 -e 2000.0 -h 20.0 -p 10 -v 0.0 -i DECAY_TURB_BB -o out/"
    res = {}
    for name, exe, extra in (("ref", REF, []), ("gpu", NS2D, ["--quiet"])):
        (tmp_path / name).mkdir()
        res[name] = subprocess.run([exe] + extra + args.split(), cwd=tmp_path / name, capture_output=True, text=True,
                                   timeout=600)
        assert res[name].returncode == 1, (name, res[name].stdout[-500:], res[name].stderr[-500:])
    assert "SOLVER FAILURE" in res["gpu"].stderr
    want, _, _ = h5log.read(glob.glob(str(tmp_path / "ref" / "out" / "*" / "Main_HDF_Data.h5"))[0])
    got, _ = h5read.flatten(h5read.read(glob.glob(str(tmp_path / "gpu" / "out" / "*" / "Main_HDF_Data.h5"))[0]))
    assert set(got) == set(want) and "/Iter_00000/w_hat" in got
    for k in want:
        _close(got[k], want[k], k)


@pytest.mark.parametrize("variant,extra", [("rk4", "--integrator=RK4"), ("houli", "--dealias=HOU_LI")])
@pytest.mark.parametrize("case", ["decay_fixed", "decay_adaptive", "tg_drag", "stoc"])
def test_compile_time_variants_match_reference_program(variant, extra, case, tmp_path):
    """The reference program built with -D__RK4 (explicit RK4 with its
    linear-term quirk) or with Hou-Li dealiasing (its header switched to
    __DEALIAS_HOU_LI) against bin/ns2d with the matching run-time option."""
    exe = REF + "_" + variant
    if not os.path.exists(exe):
        pytest.skip("variant of the reference program not built")
    args = f"{BASE} {CASES[case]} -o out/"
    (tmp_path / "ref").mkdir()
    (tmp_path / "gpu").mkdir()
    _run(exe, args, tmp_path / "ref")
    _run(NS2D, args, tmp_path / "gpu", ["--quiet", extra])
    rdirs = sorted(os.listdir(tmp_path / "ref" / "out"))
    assert rdirs == sorted(os.listdir(tmp_path / "gpu" / "out")) and len(rdirs) == 1
    bad = []
    for fname in FILES:
        want, _, _ = h5log.read(str(tmp_path / "ref" / "out" / rdirs[0] / fname))
        got, _ = h5read.flatten(h5read.read(str(tmp_path / "gpu" / "out" / rdirs[0] / fname)))
        assert set(got) == set(want)
        bad += _compare_file(got, want, fname)
    assert not bad, bad[:20]


@pytest.mark.parametrize("extra", [["--integrator=RK4"], ["--integrator=AB4"], ["--integrator=DP5"],
                                   ["--precision=FP32"], ["--dealias=HOU_LI"]])
def test_variants_run(extra, tmp_path):
    """The compile-time variants of the reference as run-time options (in the
    corrected forms: explicit RK4 with the reference's quirk adds the linear
    term with the wrong sign and gains energy) write complete files with
    finite fields and decaying energy."""
    _run(NS2D, "-n 64 -n 64 -e 0.02 -h 0.001 -p 5 -v 0.001 -i DECAY_TURB_BB -o out/", tmp_path,
         extra + ["--quiet", "--no-quirks"])
    main = glob.glob(str(tmp_path / "out" / "*" / "Main_HDF_Data.h5"))[0]
    data, attrs = h5read.flatten(h5read.read(main))
    assert len([k for k in data if k.endswith("/w_hat")]) >= 2
    assert all(np.isfinite(v).all() for v in data.values())
    msr = glob.glob(str(tmp_path / "out" / "*" / "SystemMeasures_HDF_Data.h5"))[0]
    m, _ = h5read.flatten(h5read.read(msr))
    e = m["/TotalEnergy"]
    assert e[0] > 0 and np.all(np.diff(e[e > 0]) < 1e-6 * e[0])  # unforced decay


def test_file_only_output(tmp_path):
    """A second -o writes the files straight into the output directory, the
    run's parameters in their names (hdf5_funcs.c:446-490)."""
    _run(NS2D, "-n 64 -n 64 -e 0.004 -h 0.001 -p 2 -i TG_VORT -o out/ -o x", tmp_path, ["--quiet"])
    names = sorted(os.listdir(tmp_path / "out"))
    assert len(names) == 3 and all(n.endswith(".h5") for n in names)
    assert names[0].startswith("Main_HDF_Data_SIM[NAV-RK4CN-FULL]_N[64,64]")
    for n in names:
        h5read.read(str(tmp_path / "out" / n))


def test_phase_only_matches_reference_program(tmp_path):
    """--phase-only against the reference program built with -D__PHASE_ONLY
    (Solver/Makefile:58): the PHAEONLY directory, the a_k / phi_k datasets
    (the initial save's row-indexed form, hdf5_funcs.c:264-290), and after one
    step every mode the reference leaves finite.  The reference's reset divides
    0 by 0 in the modes the 2/3 rule zeroes (NaN there, and everywhere from the
    next transform on); bin/ns2d keeps them at 0."""
    exe = REF + "_phase_only"
    if not os.path.exists(exe):
        pytest.skip("phase-only reference program not built")
    args = f"{BASE} -e 0.001 -h 0.001 -p 1 -i DECAY_TURB_BB -o out/"
    (tmp_path / "ref").mkdir()
    (tmp_path / "gpu").mkdir()
    _run(exe, args, tmp_path / "ref")
    _run(NS2D, args, tmp_path / "gpu", ["--quiet", "--phase-only"])
    rdirs = sorted(os.listdir(tmp_path / "ref" / "out"))
    assert rdirs == sorted(os.listdir(tmp_path / "gpu" / "out")) and len(rdirs) == 1
    assert "_PHAEONLY_" in rdirs[0]
    want, _, _ = h5log.read(str(tmp_path / "ref" / "out" / rdirs[0] / "Main_HDF_Data.h5"))
    got, _ = h5read.flatten(h5read.read(str(tmp_path / "gpu" / "out" / rdirs[0] / "Main_HDF_Data.h5")))
    assert set(got) == set(want) and "/Iter_00001/a_k" in got
    bad = [k for k in want if k.startswith("/Iter_00000/") and _mismatch(got[k], want[k])]
    assert not bad, bad
    nan = np.isnan(want["/Iter_00001/w_hat"])
    assert nan.any() and not np.isnan(got["/Iter_00001/w_hat"]).any()
    for name in ("w_hat", "a_k", "phi_k"):
        g, w = got[f"/Iter_00001/{name}"], want[f"/Iter_00001/{name}"]
        assert np.all(g[nan] == 0), name
        assert _mismatch(g[~nan], w[~nan]) is None, name
    details = (tmp_path / "gpu" / "out" / rdirs[0] / "SimulationDetails.txt").read_text()
    assert "Model Type: PHAEONLY" in details


def test_phase_only_run_keeps_amplitudes(tmp_path):
    """A longer --phase-only run (corrected conjugacy): finite fields, every
    save's a_k equal to |w_hat| and to the initial amplitudes."""
    _run(NS2D, "-n 64 -n 64 -e 0.02 -h 0.001 -p 5 -v 0.001 -i DECAY_TURB_BB -o out/", tmp_path,
         ["--quiet", "--phase-only", "--no-quirks"])
    main = glob.glob(str(tmp_path / "out" / "*" / "Main_HDF_Data.h5"))[0]
    data, _ = h5read.flatten(h5read.read(main))
    a0 = np.abs(data["/Iter_00000/w_hat"])
    a0[0, 0] = 0
    iters = sorted({k.split("/")[1] for k in data})
    assert len(iters) == 5
    for it in iters:
        w = data[f"/{it}/w_hat"]
        assert np.isfinite(w).all() and np.isfinite(data[f"/{it}/w"]).all()
        assert np.abs(data[f"/{it}/a_k"] - np.abs(w)).max() <= 1e-15 * a0.max()
        dphi = data[f"/{it}/phi_k"] - np.angle(w)
        assert np.abs(dphi).max() <= 1e-14, np.abs(dphi).max()
        assert np.abs(np.abs(w) - a0).max() <= 1e-12 * a0.max()
