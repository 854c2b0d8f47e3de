"""Fixed-dt time loops (ns2d_step_n / ns2d_step_async) replay one captured step
as a CUDA graph; the results must equal eager steps bit for bit, across dt
changes and the hyperviscosity latch."""
import numpy as np
import pytest

from ns2d import Solver, abi, initial

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("quirks", [0, abi.QUIRKS_REFERENCE])
@pytest.mark.parametrize("n", [64, 1024])
def test_graph_replay_matches_eager_steps(n, quirks):
    p = abi.default_params(nx=n, ny=n, nu=1e-3, quirks=quirks)
    w0 = initial.decaying(n, 3, k0=4.0, dealias="2/3")
    a, b = Solver(p), Solver(p)
    a.set_w_hat(w0)
    b.set_w_hat(w0)
    dts = [1e-3] * 6 + [5e-4] * 5 + [1e-3] * 3
    for dt in dts:
        a.rk4_step(dt)                      # eager, one call per step
    i = 0
    while i < len(dts):                     # runs of equal dt through the loop form
        j = i
        while j < len(dts) and dts[j] == dts[i]:
            j += 1
        b.step_n(j - i, dts[i])
        i = j
    assert np.array_equal(a.get_w_hat(), b.get_w_hat())
    # graph replays count their kernels; the fused loop launches fewer
    assert 0 < b.launch_count <= a.launch_count


def test_step_async_then_timing_mode():
    n = 128
    p = abi.default_params(nx=n, ny=n, nu=1e-3)
    w0 = initial.decaying(n, 5, k0=4.0, dealias="2/3")
    a, b = Solver(p), Solver(p)
    a.set_w_hat(w0)
    b.set_w_hat(w0)
    a.step_async(8, 1e-3)
    a.check()
    b.step_async(3, 1e-3)
    b.set_kernel_timing(True)               # eager launches with events
    b.step_async(5, 1e-3)
    b.check()
    ms, cnt = b.kernel_times()
    # per step: 3 stage column passes, 1 final, 4 row passes; the first column
    # pass only when the previous step did not produce it (fused final pass)
    assert cnt[1] == 15 and cnt[2] == 5 and cnt[3] == 20 and cnt[0] <= 5
    assert np.array_equal(a.get_w_hat(), b.get_w_hat())


def test_fused_first_pass_is_invalidated_by_other_calls():
    """A call between loop steps that launches anything (here a state read-back
    and an RHS evaluation that overwrites the derived spectra) makes the next
    loop step recompute its first column pass; results equal eager steps."""
    n = 64
    p = abi.default_params(nx=n, ny=n, nu=1e-3)
    w0 = initial.decaying(n, 8, k0=4.0, dealias="2/3")
    a, b = Solver(p), Solver(p)
    a.set_w_hat(w0)
    b.set_w_hat(w0)
    for _ in range(3):
        a.rk4_step(1e-3)
    a.nonlinear_rhs(None)
    for _ in range(3):
        a.rk4_step(1e-3)
    b.step_n(3, 1e-3)
    b.nonlinear_rhs(None)
    b.step_n(3, 1e-3)
    assert np.array_equal(a.get_w_hat(), b.get_w_hat())
