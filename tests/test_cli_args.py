"""bin/ns2d's command-line grammar against the reference's own parser
(GetCMLArgs, Solver/src/utils.c:34-460, built alone as oracle/_ref/args_ref):
the parsed parameters of `ns2d --dry-run` equal the reference's for the
argument vectors below, and both exit with status 1 on the same errors.
CPU only (a dry run touches no GPU)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NS2D = os.path.join(ROOT, "2d-navier-stokes_b200", "bin", "ns2d")
REF = os.path.join(ROOT, "oracle", "_ref", "args_ref")

pytestmark = pytest.mark.skipif(not (os.path.exists(NS2D) and os.path.exists(REF)),
                                reason="bin/ns2d or oracle/_ref/args_ref not built")

# run_solver.py:270's argument vector, with its formats
DRIVER = ("-o ../Data/Tmp/ -n 128 -n 128 -s 0.00000 -e 1.00000 -T 0 -c 1 -c 0.900000 -h 0.000100 -h 1 "
          "-v 0.0001000000 -v 0 -v 2.0 -d 0.000000 -d 0 -d -2.0 -i DECAY_TURB_BB -t RUN -f NONE -f 0 -f 1 -p 100")

VALID = [
    "",
    DRIVER,
    "-n 256 -n 256 -e 2.5 -h 0.001 -i TG_VORT",
    "-o a/ -o b/ -o c/",                        # later -o: file-only output
    "-h 0.01 -h 1 -h 0",                        # later -h: adaptive flag again
    "-c 0 -c 0.5 -c 0.25",                      # later -c: CFL constant
    "-v 0.01 -v 1 -v 4 -v 8",                   # later -v: hyperviscosity power
    "-d 0.1 -d 1 -d -1 -d 0",                   # later -d: drag power
    "-f FOO -f KOLM -f 4 -f 2.5 -f 3.5",        # unknown first name ignored
    "-f STOC_GAUSS -f ZERO -f 7",               # second -f is force_k even if a name
    "-T 1 -T 0.3 -T 0.7",
    "-i NOT_AN_IC",                             # unknown initial condition -> NONE
    "-i MAX_PALIN -t tag_with_chars-123",
    "-s 0.5 -e 0.5",
    "-p 7 -p 9",
    "-n 64 -i RING -f CONST_GAUSS",             # one -n sets Nx only
]

ERRORS = [
    "-n 3", "-n 2", "-n 0", "-s -1", "-e -1", "-s 2 -e 1", "-h 0", "-h -1", "-h 0.1 -h 2",
    "-c 2", "-c 1 -c 0", "-c 1 -c -3", "-v -1", "-v 1 -v 3", "-v 1 -v 1 -v 0", "-d -1", "-d 0 -d 2",
    "-d 0 -d 1 -d 1", "-T 2", "-T 1 -T 1.5", "-T 1 -T 0", "-z /nonexistent/file.h5", "-q", "-n",
]


def _run(exe, args, extra=()):
    return subprocess.run([exe] + list(extra) + args.split(), capture_output=True, text=True, timeout=60)


@pytest.mark.parametrize("args", VALID)
def test_same_parameters_as_reference(args):
    ref = _run(REF, args)
    got = _run(NS2D, args, ["--dry-run"])
    assert ref.returncode == 0 and got.returncode == 0, (ref.stderr, got.stderr)
    want, have = json.loads(ref.stdout), json.loads(got.stdout)
    for k, v in want.items():
        assert have[k] == v, (k, have[k], v)


@pytest.mark.parametrize("args", ERRORS)
def test_same_rejections_as_reference(args):
    ref = _run(REF, args)
    got = _run(NS2D, args, ["--dry-run"])
    assert ref.returncode == 1 and got.returncode == 1, (ref.stdout, got.stdout)


@pytest.mark.parametrize("args", ["-n 64 -n 64 -n 64", "-p 0", "-p -5", "--integrator=RK5", "--precision=FP16"])
def test_rejections_the_reference_lacks(args):
    """A third -n (the reference writes past N[2]) and -p 0 (the reference
    divides by it every step) stop here; unknown long-option values too."""
    assert _run(NS2D, args, ["--dry-run"]).returncode == 1


def test_extensions():
    got = json.loads(_run(NS2D, "--integrator=AB4 --dealias=HOU_LI --precision=FP32 --no-quirks --dry-run").stdout)
    assert (got["integrator"], got["dealias"], got["precision"], got["quirks"]) == ("AB4", "HOU_LI", "FP32", 0)


def test_other_mpi_ranks_exit_quietly():
    """Under `mpirun -n P` (run_solver.py) only rank 0 works."""
    env = dict(os.environ, OMPI_COMM_WORLD_RANK="3")
    r = subprocess.run([NS2D, "-n", "64", "-n", "64"], capture_output=True, text=True, timeout=60, env=env)
    assert r.returncode == 0 and r.stdout == ""
