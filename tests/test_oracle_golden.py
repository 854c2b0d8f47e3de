"""The oracle restatement (oracle/ns2d_oracle.c) against golden outputs of the
reference's own sources (tests/golden/make_golden.py).  Same FFT, same
operation order: the results must agree to the last bit or within 1e-15."""
import numpy as np
import pytest

from _util import load_case, make_golden, rel_err
from pyoracle import Oracle

CASES = sorted(make_golden.cases())


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_fixture(name):
    p, w0, ref_outs = load_case(name)
    _, _, _, program = make_golden.cases()[name]
    o = Oracle(p)
    outs = make_golden.run_program(o, w0, program, False)
    assert len(outs) == len(ref_outs)
    for k, (a, b) in enumerate(zip(outs, ref_outs)):
        assert a.shape == b.shape, (name, k)
        assert rel_err(a, b) <= 1e-15, (name, k, rel_err(a, b))


def test_taylor_green_decay_matches_analytic():
    """The 64^2 Taylor-Green workload: w0 = 2 sin x sin y, nu = 0.01, dt = 1e-3, 100 steps:
    the amplitude decays as exp(-2 nu t) (solver.c:2526-2530)."""
    p, w0, outs = load_case("tg64_rk4cn")
    w100 = outs[0]
    ratio = np.abs(w100[1, 1]) / np.abs(w0[1, 1])
    assert abs(ratio - np.exp(-2 * 0.01 * 0.1)) < 1e-12


def test_fixture_non_hermitian_column_is_exercised():
    p, w0, outs = load_case("nonherm32_rhs")
    x = outs[0]
    col = x[:, 0]
    n = len(col)
    assert np.max(np.abs(col[n // 2 + 1:] - np.conj(col[1:n // 2][::-1]))) > 1e-3 * np.abs(col).max()
