"""Generate tests/golden/*.npz from the reference solver's own sources.

Runs oracle/_ref/libns2d_ref_<variant>.so (Solver/src/{solver,force,sys_msr}.c
compiled unmodified by oracle/Makefile against single-rank MPI/FFTW stand-ins)
on small seeded cases and stores inputs, parameters and outputs.  Each case
runs in a fresh process because the reference keeps its state in globals.

    python tests/golden/make_golden.py          # needs the reference sources
"""
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "2d-navier-stokes_b200"), os.path.join(ROOT, "oracle")]

from ns2d import abi, initial  # noqa: E402


def cases():
    """name -> (variant, params kwargs, initial condition spec, program)."""
    return {
        # the 64^2 Taylor-Green workload: Taylor-Green, nu|k|^2 via the drag-flag recipe
        # of InitFiles/TaylorGreen/tg.ini (EKMN_DRAG_FLAG = 1, alpha = 0).
        "tg64_rk4cn": ("rk4cn", dict(nx=64, ny=64, nu=0.01, ekmn_drag_flag=1, ekmn_alpha=0.0, dt=1e-3),
                       ("tg",), [("steps", 100, 1e-3), ("w_hat",), ("max", 0), ("meas",)]),
        # stock flags: hyperviscosity latch (nu |k|^4), decaying spectrum
        "dec64_rk4cn": ("rk4cn", dict(nx=64, ny=64, nu=1e-3, dt=1e-3),
                        ("decaying", 11, 6.0), [("rhs_state",), ("steps", 20, 1e-3), ("w_hat",), ("meas",),
                                                ("max", 0), ("max", 1), ("cfl", 1e-3), ("w_hat",)]),
        # Kolmogorov forcing n = 4, F = 1, nu k^2 + hyperviscosity alpha k^16
        "kolm64_rk4cn": ("rk4cn", dict(nx=64, ny=64, nu=1e-3, ekmn_drag_flag=1, ekmn_alpha=1e-20,
                                        ekmn_drag_pow=8.0, forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0,
                                        dt=2.5e-3),
                         ("noise", 5), [("steps", 30, 2.5e-3), ("w_hat",), ("meas",), ("max", 0)]),
        # explicit RK4 with the reference's +D X stage term
        "dec32_rk4": ("rk4", dict(nx=32, ny=32, nu=1e-3, integrator=abi.RK4, ekmn_drag_flag=1, dt=1e-3),
                      ("decaying", 3, 4.0), [("steps", 10, 1e-3), ("w_hat",)]),
        # AB4 with three RK4CN start-up steps
        "dec32_ab4": ("ab4", dict(nx=32, ny=32, nu=1e-3, integrator=abi.AB4, dt=1e-3),
                      ("decaying", 4, 4.0), [("ab4", 10, 1e-3), ("w_hat",)]),
        # one RHS of an input whose ky = 0 column is not Hermitian (FFTW c2r
        # reads only the real parts there) and the conjugacy side effect
        "nonherm32_rhs": ("rk4cn", dict(nx=32, ny=32, nu=1e-3, dt=1e-3),
                          ("decaying", 5, 4.0), [("rhs_input", 77), ("w_hat",)]),
        # Hou-Li filter (integer k/(N/2) as in solver.c:1088) at 32^2 where the
        # Nyquist row/column are populated; reference built with __DEALIAS_HOU_LI
        "houli32": ("houli", dict(nx=32, ny=32, nu=5e-4, dealias=abi.DEALIAS_HOU_LI, dt=1e-3),
                    ("decaying", 8, 6.0, None), [("rhs_state",), ("steps", 10, 1e-3), ("w_hat",)]),
        # ZERO forcing: modes with |kx| <= 2 or |ky| <= 2 killed every step
        "zero32_rk4cn": ("rk4cn", dict(nx=32, ny=32, nu=1e-3, forcing=abi.FORCING_ZERO, force_k=2, dt=1e-3),
                         ("decaying", 9, 6.0), [("steps", 10, 1e-3), ("w_hat",), ("meas",)]),
        # phase-only model (-D__PHASE_ONLY): amplitudes reset after each update.
        # The reference's reset divides 0 by 0 wherever the update is exactly 0
        # (outside the 2/3 disc; the Hou-Li corner kx = ky = N/2); each step here
        # starts from the previous step's output with those NaN modes set to 0.
        "po32_rk4cn": ("rk4cn_po", dict(nx=32, ny=32, nu=1e-3, model=abi.MODEL_PHASE_ONLY, dt=1e-3),
                       ("decaying", 12, 4.0), [("po_steps", 10, 1e-3), ("w_hat",)]),
        "po32_rk4": ("rk4_po", dict(nx=32, ny=32, nu=1e-3, integrator=abi.RK4, model=abi.MODEL_PHASE_ONLY,
                                    ekmn_drag_flag=1, dt=1e-3),
                     ("decaying", 13, 4.0), [("po_steps", 10, 1e-3), ("w_hat",)]),
        "po32_kolm": ("rk4cn_po", dict(nx=32, ny=32, nu=1e-3, model=abi.MODEL_PHASE_ONLY, forcing=abi.FORCING_KOLM,
                                       force_k=4, force_scale=1.0, ekmn_drag_flag=1, ekmn_alpha=0.05, dt=1e-3),
                      ("decaying", 15, 4.0), [("po_steps", 10, 1e-3), ("w_hat",), ("meas",)]),
        "po32_houli": ("houli_po", dict(nx=32, ny=32, nu=5e-4, dealias=abi.DEALIAS_HOU_LI,
                                        model=abi.MODEL_PHASE_ONLY, dt=1e-3),
                       ("decaying", 14, 6.0, None, "houli_ic"), [("po_steps", 10, 1e-3), ("w_hat",)]),
        # RK5DPStep as written (reference built with -D__DPRK5 from a copy with
        # its three compile defects fixed, oracle/Makefile): DP_err of
        # SpectralSolve iterations 1..6 (0 at the first, which computes none),
        # then the state; stock flags (the hyperviscosity bracket with == only)
        "dp5_32": ("dp5", dict(nx=32, ny=32, nu=1e-3, dt=1e-3),
                   ("decaying", 16, 4.0), [("rk5dp", 6, 1e-3), ("w_hat",)]),
        # the same with drag + hyperviscosity on alpha |k|^16 and Kolmogorov forcing
        "dp5_32_kolm": ("dp5", dict(nx=32, ny=32, nu=1e-3, ekmn_drag_flag=1, ekmn_alpha=1e-12, ekmn_drag_pow=8.0,
                                    forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0, dt=2e-3),
                        ("decaying", 17, 4.0), [("rk5dp", 6, 2e-3), ("w_hat",), ("meas",)]),
        # adaptive CFL step with the reference's row-index quirk
        "cfl32": ("rk4cn", dict(nx=32, ny=32, nu=1e-3, adapt_step_flag=1, cfl_cond_flag=1, cfl_const=0.9, dt=1e-3),
                  ("decaying", 6, 4.0), [("cfl", 1e-3), ("steps", 5, 2e-3), ("cfl", 2e-3), ("w_hat",)]),
    }


def houli_filter_int(n):
    """The Hou-Li filter that ends InitialConditions in a Hou-Li build
    (solver.c:1088, 1994), with its integer ratios k/(N/2): 1 inside, exp(-36)
    on the Nyquist row and column, 0 (underflow) at their corner."""
    kx = np.fft.fftfreq(n, 1.0 / n).astype(int)
    kx[n // 2] = -(n // 2)
    ky = np.arange(n // 2 + 1)
    fx = np.trunc(kx / (n // 2))[:, None]
    fy = np.trunc(ky / (n // 2))[None, :]
    return np.exp(-36.0 * np.sqrt(fx ** 2 + fy ** 2) ** 36)


def make_ic(spec, n):
    if spec[0] == "tg":
        return initial.taylor_green(n)
    if spec[0] == "decaying":
        w = initial.decaying(n, seed=spec[1], k0=spec[2], dealias=spec[3] if len(spec) > 3 else "2/3")
        if len(spec) > 4 and spec[4] == "houli_ic":
            w = w * houli_filter_int(n)
        return w
    if spec[0] == "noise":
        return initial.noise(n, seed=spec[1], amplitude=1e-3, kolm=True)
    raise ValueError(spec)


def run_program(solver, w0, program, record):
    solver.set_w_hat(w0)
    outs = []
    for op in program:
        kind = op[0]
        if kind == "steps":
            for _ in range(op[1]):
                solver.rk4_step(op[2])
        elif kind == "po_steps":
            for _ in range(op[1]):
                solver.rk4_step(op[2])
                w = solver.get_w_hat()
                if np.isnan(w).any():
                    w[np.isnan(w)] = 0.0
                    solver.set_w_hat(w)
        elif kind == "ab4":
            for it in range(1, op[1] + 1):
                solver.ab4_step(op[2], it)
        elif kind == "rk5dp":
            outs.append(np.array([solver.rk5dp_step(op[2], it) for it in range(1, op[1] + 1)]))
        elif kind == "w_hat":
            outs.append(solver.get_w_hat())
        elif kind == "max":
            outs.append(np.array([solver.get_max_data(op[1])]))
        elif kind == "cfl":
            outs.append(np.array([solver.get_timestep(op[1])]))
        elif kind == "meas":
            s, sp = solver.system_measurables()
            outs.append(np.asarray(s))
            outs.append(np.asarray(sp))
        elif kind == "rhs_state":
            outs.append(solver.nonlinear_rhs(None))
        elif kind == "rhs_input":
            rng = np.random.default_rng(op[1])
            x = w0 + 1e-3 * np.abs(w0).max() * (rng.standard_normal(w0.shape) + 1j * rng.standard_normal(w0.shape))
            x[:, 0] += 0.01 * np.abs(w0).max() * rng.standard_normal(w0.shape[0])  # non-Hermitian column 0
            outs.append(x)
            outs.append(solver.nonlinear_rhs(x))
        else:
            raise ValueError(kind)
    return outs


def _ref_worker(name, q):
    from pyoracle import RefSolver
    variant, kw, ic, program = cases()[name]
    p = abi.default_params(**kw)
    w0 = make_ic(ic, p.nx)
    ref = RefSolver(p, variant)
    q.put(run_program(ref, w0, program, True))


def generate(name):
    variant, kw, ic, program = cases()[name]
    p = abi.default_params(**kw)
    w0 = make_ic(ic, p.nx)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=_ref_worker, args=(name, q))
    proc.start()
    outs = q.get(timeout=600)
    proc.join()
    params = {f: getattr(p, f) for f, _ in abi.Params._fields_}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), w0=w0, n_out=len(outs),
                        params=np.array([float(params[f]) for f, _ in abi.Params._fields_]),
                        param_names=np.array([f for f, _ in abi.Params._fields_]),
                        variant=variant, **{f"out{i}": o for i, o in enumerate(outs)})
    return len(outs)


# ---------------------------------------------------------------------------
# Tangent-linear fixture for the discrete adjoint: directional derivatives of
# the final enstrophy and palinstrophy along seeded directions, propagated by a
# tangent-linear RK4CN step whose RHS derivative is taken from the reference's
# own NonlinearRHSBatch by polarisation (exact for its quadratic term).

ADJOINT_CASE = dict(nx=32, ny=32, nu=1e-3, quirks=0, dt=2e-3)
ADJOINT_STEPS = 25
ADJOINT_DIRS = 4


def _adjoint_worker(q):
    import adjoint_ref as ar
    from pyoracle import RefSolver
    p = abi.default_params(**ADJOINT_CASE)
    n, dt = p.nx, p.dt
    ref = RefSolver(p, "rk4cn")
    rhs = ref.nonlinear_rhs
    model = ar.Model(n, ar.bracket_for(p))
    tl = ar.tl_rhs_polar(rhs)
    w0 = initial.decaying(n, seed=21, k0=4.0, dealias="2/3")
    dirs = [ar.random_field(n, 100 + i, kmax=n / 3.0, scale=np.abs(w0).max()) for i in range(ADJOINT_DIRS)]
    traj = []
    w = w0
    for _ in range(ADJOINT_STEPS):
        w, X = model.step(w, dt, rhs=rhs)
        traj.append(X)
    Z, gZ = model.objective(w, "enstrophy")
    P, gP = model.objective(w, "palinstrophy")
    dZ, dP = [], []
    for d in dirs:
        dw = d
        for X in traj:
            dw = model.step_tl(X, dw, dt, rhs_tl=tl)
        dZ.append(ar.wdot(gZ, dw))
        dP.append(ar.wdot(gP, dw))
    q.put((w0, np.array(dirs), w, Z, P, np.array(dZ), np.array(dP)))


def generate_adjoint():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=_adjoint_worker, args=(q,))
    proc.start()
    w0, dirs, wT, Z, P, dZ, dP = q.get(timeout=600)
    proc.join()
    p = abi.default_params(**ADJOINT_CASE)
    params = {f: getattr(p, f) for f, _ in abi.Params._fields_}
    np.savez_compressed(os.path.join(HERE, "adjoint32_tl.npz"), w0=w0, dirs=dirs, wT=wT, Z=Z, P=P, dZ=dZ, dP=dP,
                        nsteps=ADJOINT_STEPS,
                        params=np.array([float(params[f]) for f, _ in abi.Params._fields_]),
                        param_names=np.array([f for f, _ in abi.Params._fields_]))


if __name__ == "__main__":
    import pyoracle
    pyoracle.build(ref=True)
    only = sys.argv[1:]
    for name in cases():
        if not only or name in only:
            print(name, generate(name))
    if not only or "adjoint32_tl" in only:
        generate_adjoint()
        print("adjoint32_tl")
