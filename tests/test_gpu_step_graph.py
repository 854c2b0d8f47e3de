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
    assert b.launch_count >= a.launch_count  # graph replays count their kernels


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
    assert cnt[0] == 5 and cnt[1] == 15 and cnt[2] == 5 and cnt[3] == 20
    assert np.array_equal(a.get_w_hat(), b.get_w_hat())

