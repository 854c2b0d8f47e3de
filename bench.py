#!/usr/bin/env python
"""RK4 steps/s of the pseudospectral time step at 1024^2 (FP64), B200.

Workload (the 1024^2 configuration of the headline metric): Kolmogorov-forced
flow, n = 4, F = 1, nu = 1e-4 plus hyperviscosity nu_h |k|^16 (nu_h = 2e-40)
through the RK4CN drag branch, dt = 2.5e-4, 2/3 dealiasing, FP64, from seeded
1e-3-amplitude random-phase noise (synthetic input; no dataset involved).

One "step" = one RK4CN step (4 nonlinear-term evaluations + update) of one
1024^2 trajectory.  With --gpus N (torchrun, one process per GPU) every rank
advances its own trajectory (replicas: the path has no exchange step), so
`value` is the job's total steps/s and scaling is weak.

  value   device time (CUDA events on the solver's stream) per step, state
          resident in HBM; L2 is flushed (256 MiB write) between timed steps,
          outside the events.
  e2e     ns2d_rk4_step_host: the reference-facing RK4Step contract with the
          state in pinned host memory, copied in and out every step (wall
          clock per step, L2 flushed between steps).
  roofline  the dominant kernel class against the measured HBM bandwidth
          (algorithmic bytes per launch over the scaled event time);
          roofline_by_kernel gives the same for every pass class.
  --impl reference   the reference's own CPU solver (Solver/src built by
          oracle/Makefile; FFTW replaced by the oracle's FFT) on the host cores.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "2d-navier-stokes_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

METRIC = "RK4 steps/s at 1024^2 (FP64 plain vs FP32 batched); adjoint/forward time"
N = 1024
DT = 2.5e-4
NU_H = 2e-40
WORKLOAD = "kolmogorov_1024_fp64_rk4cn"
S_BYTES = 16 * N * (N // 2 + 1)  # one FP64 half spectrum
# algorithmic bytes per launch, in units of S, per kernel class: 0 first column
# pass (read w, write 4 fields: 5), 1 column pass with stage combine (read n,
# w, acc; write acc + 4 fields: 8; stage 1 has no acc read: 7; mean 23/3),
# 2 final column pass (read n, w, acc, CN table; write w: 5), 3 row pass (read
# 4, write 1: 5).
CLASS_NAMES = ["col_p1", "col_stage", "col_final", "row", "other"]
CLASS_BYTES_PER_LAUNCH = {0: 5.0, 1: 23.0 / 3.0, 2: 5.0, 3: 5.0}
# the read part of the same (stage pass: n, w, and acc in stages 2-3; final
# pass: n, w, acc and the Crank-Nicolson table)
CLASS_READ_PER_LAUNCH = {0: 1.0, 1: 8.0 / 3.0, 2: 4.0, 3: 4.0}
# what `roofline.traffic` holds: ncu's dram__bytes_read.sum + dram__bytes_write.sum
# of one launch captured alone (caches flushed before it).  Its writes stay in
# the 126 MB L2 when the kernel ends and are written back during later kernels,
# so the figure is close to the DRAM reads of the launch; compare it with
# algorithmic_read_bytes_per_launch.
NCU_TRAFFIC_KIND = "ncu dram read+write of one launch (writes mostly still in L2 at kernel end)"
MODEL_BYTES_PER_STEP = 58  # the 2-pass minimal model (58 S per RK4 step)


def params(device=0):
    from ns2d import abi
    return abi.default_params(nx=N, ny=N, nu=1e-4, ekmn_drag_flag=1, ekmn_alpha=NU_H, ekmn_drag_pow=8.0,
                              forcing=abi.FORCING_KOLM, force_k=4, force_scale=1.0, dt=DT, device=device)


def config(parallelism):
    return {"workload": WORKLOAD, "grid": f"{N}x{N}", "nu": 1e-4, "nu_h": NU_H, "hyperviscosity": "|k|^16",
            "dt": DT, "forcing": "KOLM n=4 F=1", "integrator": "RK4CN", "dealias": "2/3",
            "l2": "flushed between timed steps (256 MiB write outside the timed events)",
            "parallelism": parallelism}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(cls):
    """DRAM bytes per launch for a kernel class from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "col_row_1024_fp64.md")
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(rf"traffic_bytes_per_launch\s+{CLASS_NAMES[cls]}\s+([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """SM clock and throttle reasons sampled while the timed steps run.

    The timed region of the default run is tens of milliseconds, shorter than
    nvidia-smi's 200 ms sampling period, so the clocks are read through NVML
    (the library nvidia-smi reports from) every 2 ms by a thread; the fields
    are nvidia-smi's clocks.sm, clocks.max.sm and clocks_event_reasons.*.
    Without NVML, `nvidia-smi -lms 200` runs instead (and may see no sample
    inside a short region)."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.sm, self.mx, self.reasons = [], None, set()
        self.source = None
        self._stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            prop = torch.cuda.get_device_properties(self.device)
            bus = f"{prop.pci_domain_id:08X}:{prop.pci_bus_id:02X}:{prop.pci_device_id:02X}.0"
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
        self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        return pynvml, h

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            self.source = "nvml, 2 ms period"
            self.t = threading.Thread(target=self._poll, daemon=True)
        except Exception:
            self.nvml = None
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.SMI_FIELDS,
                                              "--format=csv,noheader,nounits", "-lms", "200", "-i", str(self.device)],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi -lms 200"
                self.t = threading.Thread(target=self._read, daemon=True)
            except Exception:
                self.proc = None
                return self
        self.t.start()
        return self

    def _poll(self):
        pynvml, h = self.nvml
        bits = [(name, getattr(pynvml, const)) for name, const in self.REASONS]
        while not self._stop.is_set():
            try:
                self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.reasons.update(name for name, b in bits if r & b)
            except Exception:
                return
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 9:
                continue
            try:
                self.sm.append(float(parts[1]))
                self.mx = float(parts[2])
            except ValueError:
                continue
            for (name, _), v in zip(self.REASONS, parts[5:9]):
                if v.lower() == "active":
                    self.reasons.add(name)

    def __exit__(self, *exc):
        self._stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.nvml or self.proc:
            self.t.join(timeout=5)
        if self.nvml:
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.mx, "reasons": ["unavailable"], "source": self.source}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.mx, "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": self.source}


def cpu_reference(steps, warmup, threads, budget_s=None):
    """The reference's own solver (oracle/_ref) on the host: steps/s."""
    from ns2d import initial
    from pyoracle import RefSolver, build, ref_available
    if not ref_available("rk4cn"):
        build(ref=True)
    ref = RefSolver(params(), "rk4cn", threads=threads)
    ref.set_w_hat(initial.noise(N, seed=7, amplitude=1e-3, kolm=True))
    for _ in range(warmup):
        ref.rk4_step(DT)
    if budget_s is not None:
        t0 = time.perf_counter()
        ref.rk4_step(DT)
        one = time.perf_counter() - t0
        steps = max(2, min(steps, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        ref.rk4_step(DT)
    el = time.perf_counter() - t0
    return steps / el, steps, el


# The reference's CPU solver on the three FP64 workloads (host cores): the
# 64^2 Taylor-Green case (nu |k|^2 through the drag flag, dt = 1e-3), the 256^2
# decaying case (Hou-Li build, CFL 0.9 adaptive step, nu = 5e-4) and the 1024^2
# Kolmogorov case of the headline metric.
CPU_TABLE = (("taylor_green_64_fp64_rk4cn", 64), ("decaying_256_houli_cfl_fp64_rk4cn", 256),
             ("kolmogorov_1024_fp64_rk4cn", 1024))


def _cpu_case(name):
    from ns2d import abi, initial
    if name.startswith("taylor_green"):
        p = abi.default_params(nx=64, ny=64, nu=0.01, ekmn_drag_flag=1, ekmn_alpha=0.0, dt=1e-3)
        return p, "rk4cn", initial.taylor_green(64), False
    if name.startswith("decaying"):
        p = abi.default_params(nx=256, ny=256, nu=5e-4, dealias=abi.DEALIAS_HOU_LI, adapt_step_flag=1,
                               cfl_cond_flag=1, cfl_const=0.9, dt=1e-3)
        return p, "houli", initial.decaying(256, seed=2, k0=6.0), True
    return params(), "rk4cn", initial.noise(N, seed=7, amplitude=1e-3, kolm=True), False


def _cpu_table_worker(name, thread_counts, runs, budget_s, q):
    """Median steps/s of `runs` timed runs after one warm-up step, for each
    thread count, in a process of its own (the reference keeps global state)."""
    from pyoracle import RefSolver
    p, variant, w0, adaptive = _cpu_case(name)
    ref = RefSolver(p, variant, threads=thread_counts[0])
    ref.set_w_hat(w0)
    dt = ref.get_timestep(p.dt) if adaptive else p.dt
    out = []
    for th in thread_counts:
        ref.set_threads(th)
        t0 = time.perf_counter()
        ref.rk4_step(dt)
        if adaptive:
            dt = ref.get_timestep(dt)
        one = time.perf_counter() - t0
        k = max(1, min(200, int(budget_s / (runs * max(one, 1e-4)))))
        rates = []
        for _ in range(runs):
            t0 = time.perf_counter()
            for _ in range(k):
                ref.rk4_step(dt)
                if adaptive:
                    dt = ref.get_timestep(dt)
            rates.append(k / (time.perf_counter() - t0))
        out.append({"threads": th, "steps_per_run": k, "runs": runs,
                    "steps_per_s_median": statistics.median(rates), "steps_per_s_runs": rates})
    q.put(out)


def cpu_table(threads, runs=5, budget_s=4.0):
    """The reference on each workload at T = threads and T = 1; each case in a
    spawned process, about budget_s seconds of timed work per thread count."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    rows = []
    for name, n in CPU_TABLE:
        q = ctx.Queue()
        proc = ctx.Process(target=_cpu_table_worker, args=(name, (threads, 1) if threads > 1 else (1,), runs,
                                                          budget_s, q))
        proc.start()
        res = q.get(timeout=600)
        proc.join(60)
        for r in res:
            r.update({"workload": name, "grid": f"{n}x{n}"})
            rows.append(r)
    return rows


def run_reference(args, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    value, steps, el = cpu_reference(args.steps, args.warmup, threads)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config("reference CPU (1 process, OpenMP FFT)"),
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "reference",
                             "sample": f"{steps} RK4CN steps of the {N}^2 Kolmogorov workload: the reference's "
                                       "Solver/src (solver.c, force.c, sys_msr.c) built by oracle/Makefile, "
                                       "FFTW-MPI replaced by the oracle's OpenMP FFT"},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


ENS_SIZES = [128] * 32 + [256] * 24 + [512] * 8  # 4,194,304 points = 4 x 1024^2
ENS_DT = 1e-3


def ensemble_bench(stream, flush, steps, warmup, rank):
    """The uneven-ensemble workload: 64 members (32 x 128^2, 24 x 256^2, 8 x 512^2), FP32
    RK4CN, nu = 1e-3, decaying spectra with k0 drawn from {4, 6, 8}; every pass
    of a step is one launch for all members, the step replayed from a CUDA
    graph, block sizes (tile shapes) and persistent grids picked by the
    autotuner.  Returns ensemble steps/s (device time, L2 flushed between
    steps) and the tuned launch shape."""
    import torch
    from ns2d import Ensemble, abi, initial
    p = abi.default_params(nu=1e-3, dt=ENS_DT, precision=abi.FP32)
    e = Ensemble(p, ENS_SIZES)
    e.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(100 + rank)
    ics = [initial.decaying(n, seed=1000 * rank + m, k0=float(rng.choice([4, 6, 8])), dealias="2/3")
           for m, n in enumerate(ENS_SIZES)]
    e.tune(ENS_DT)
    grids = e.shape
    for m, w in enumerate(ics):
        e.set_w_hat(m, w)
    e.step_async(warmup, ENS_DT)
    e.check()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    l0 = e.launch_count
    with torch.cuda.stream(stream):
        for e0, e1 in evs:
            e0.record(stream)
            e.step_async(1, ENS_DT)
            e1.record(stream)
            flush.zero_()
    torch.cuda.synchronize()
    e.check()
    launches = e.launch_count - l0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    z = [e.measurables(m).enstrophy for m in (0, 32, 56)]
    e.close()
    return steps / (ms * 1e-3), ms / steps, grids, launches, z


def ensemble_error(stream, steps, rank):
    """Largest relative enstrophy difference over the 64 members between the
    FP32 ensemble (tuned grids, graph-replayed steps) and the FP64 ensemble
    after `steps` steps of the same workload."""
    from ns2d import Ensemble, abi, initial
    rng = np.random.default_rng(100 + rank)
    ics = [initial.decaying(n, seed=1000 * rank + m, k0=float(rng.choice([4, 6, 8])), dealias="2/3")
           for m, n in enumerate(ENS_SIZES)]
    z = {}
    for prec in (abi.FP64, abi.FP32):
        e = Ensemble(abi.default_params(nu=1e-3, dt=ENS_DT, precision=prec), ENS_SIZES)
        e.set_stream(stream.cuda_stream)
        if prec == abi.FP32:
            e.tune(ENS_DT)
        for m, w in enumerate(ics):
            e.set_w_hat(m, w)
        e.step_n(steps, ENS_DT)
        z[prec] = np.array([e.measurables(m).enstrophy for m in range(len(ENS_SIZES))])
        e.close()
    rel = np.abs(z[abi.FP32] - z[abi.FP64]) / np.abs(z[abi.FP64])
    return float(rel.max()), int(rel.argmax())


ADJ_N, ADJ_DT, ADJ_EVERY = 512, 5e-4, 50


def adjoint_bench(stream, nsteps, rank, precision, g_ref=None, n_dirs=16):
    """Discrete adjoint at 512^2 (nu = 1e-3, dt = 5e-4, RK4CN, checkpoints every
    50 steps): device time of one gradient of the final enstrophy (record +
    objective + checkpointed reverse sweep) over the time of the forward solve
    alone, from w0 = decaying spectrum (k0 = 4) projected to E = 0.5, Z = 10.
    FP64: central differences (eps in 1e-5, 1e-6, 1e-7, |d|_W = |w0|_W) of the
    forward along n_dirs seeded directions; the headline `fd` figures are those
    of the one eps whose worst direction agrees best (the same eps for every
    direction), the whole sweep is reported beside them.  FP32: the gradient
    against the FP64 one (g_ref)."""
    import torch
    from ns2d import Solver, abi, initial
    from ns2d import adjoint as nadj
    p = abi.default_params(nx=ADJ_N, ny=ADJ_N, nu=1e-3, quirks=0, dt=ADJ_DT, precision=precision)
    s = Solver(p)
    s.set_stream(stream.cuda_stream)
    w0 = nadj.project(initial.decaying(ADJ_N, seed=50 + rank, k0=4.0, dealias="2/3"), 0.5, 10.0)
    c = initial.weights(ADJ_N, ADJ_N)

    def wdot(a, b):
        return float(np.sum(c * (a.real * b.real + a.imag * b.imag)))

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    def forward():
        s.step_async(nsteps, ADJ_DT)

    def gradient():
        return s.adjoint_gradient(nsteps, ADJ_DT, ADJ_EVERY, abi.OBJ_ENSTROPHY)

    # warm-up (allocations, kernel set-up), then timed
    s.set_w_hat(w0)
    gradient()
    s.set_w_hat(w0)
    ms_fwd, _ = timed(forward)
    s.check()
    s.set_w_hat(w0)
    ms_grad, (J, g) = timed(gradient)
    ms_rec, ms_rev = s.adjoint_times()
    out = {"precision": "f64" if precision == abi.FP64 else "f32", "forward_ms": ms_fwd, "gradient_ms": ms_grad,
           "adjoint_over_forward": ms_grad / ms_fwd, "record_ms": ms_rec, "reverse_sweep_ms": ms_rev,
           "J_final_enstrophy": J}
    if precision == abi.FP64:
        rng = np.random.default_rng(900 + rank)
        eps_list = (1e-5, 1e-6, 1e-7)
        rel = {e: [] for e in eps_list}
        scaled = {e: [] for e in eps_list}
        gn = np.sqrt(wdot(g, g))
        for _ in range(n_dirs):
            d = initial.dealias_23(initial.hermitian(rng.standard_normal(w0.shape) + 1j * rng.standard_normal(w0.shape)))
            d *= np.sqrt(wdot(w0, w0) / wdot(d, d))
            ad = wdot(g, d)
            for eps in eps_list:
                vals = []
                for sgn in (1.0, -1.0):
                    s.set_w_hat(w0 + sgn * eps * d)
                    s.step_n(nsteps, ADJ_DT)
                    vals.append(s.objective(abi.OBJ_ENSTROPHY))
                fd = (vals[0] - vals[1]) / (2.0 * eps)
                rel[eps].append(abs(fd - ad) / abs(fd))
                scaled[eps].append(abs(fd - ad) / (gn * np.sqrt(wdot(d, d))))
        if n_dirs:
            best_rel = [min(rel[e][i] for e in eps_list) for i in range(n_dirs)]
            best_scaled = [min(scaled[e][i] for e in eps_list) for i in range(n_dirs)]
            eps_h = min(eps_list, key=lambda e: max(rel[e]))
            out["fd"] = {"eps": eps_h, "directions": n_dirs, "max_rel_err": max(rel[eps_h]),
                         "median_rel_err": float(np.median(rel[eps_h])),
                         "max_err_over_grad_norm": max(scaled[eps_h]),
                         "eps_sweep": list(eps_list),
                         "max_rel_err_by_eps": [max(rel[e]) for e in eps_list],
                         "max_rel_err_best_eps": max(best_rel),
                         "max_err_over_grad_norm_best_eps": max(best_scaled)}
        out["gradient"] = g
    elif g_ref is not None:
        out["grad_rel_err_vs_f64"] = float(np.abs(g - g_ref).max() / np.abs(g_ref).max())
    s.close()
    return out


def run_part(args, local_rank):
    """One part of the benchmark alone (--only): its JSON object on one line.
    Used for profiling runs, which should hold few launches."""
    import torch
    from ns2d import abi
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    if args.only == "ensemble":
        v, ms, grids, launches, z = ensemble_bench(stream, flush, args.ens_steps, args.warmup, 0)
        out = {"part": "ensemble", "ensemble_steps_per_s": v, "ms_per_step": ms, "tuned_shape": grids,
               "gpu_launches": launches, "enstrophy_sample": z}
    else:
        out = {"part": "adjoint", "run": adjoint_bench(stream, args.adj_steps, 0, abi.FP64, n_dirs=0)}
        out["run"].pop("gradient", None)
        if args.ascent:
            out["ascent"] = adjoint_ascent(stream, args.adj_steps, args.ascent)
    print(json.dumps(out), flush=True)
    return 0


def adjoint_ascent(stream, nsteps, iters):
    """Projected gradient ascent of the final enstrophy over initial conditions
    with E = 0.5 and Z = 10 fixed (the extreme-enstrophy search), at 512^2 with
    the adjoint workload's horizon: Z(T) at the first and the best iterate."""
    import torch
    from ns2d import Solver, abi, initial
    from ns2d import adjoint as nadj
    p = abi.default_params(nx=ADJ_N, ny=ADJ_N, nu=1e-3, quirks=0, dt=ADJ_DT)
    s = Solver(p)
    s.set_stream(stream.cuda_stream)
    w0 = initial.decaying(ADJ_N, seed=50, k0=4.0, dealias="2/3")
    t0 = time.perf_counter()
    wbest, hist = nadj.projected_ascent(s, w0, nsteps, ADJ_DT, iters=iters, e0=0.5, z0=10.0,
                                       checkpoint_every=ADJ_EVERY)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    out = {"iterations": iters, "J_first": hist[0], "J_best": max(hist), "J_history": hist, "wall_s": wall,
           "E_best": initial.energy(wbest), "Z0_best": initial.enstrophy(wbest)}
    s.close()
    return out


def run_gpu(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from ns2d import Solver, initial

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    s = Solver(params(local_rank))
    stream = torch.cuda.Stream(device=dev)
    s.set_stream(stream.cuda_stream)
    w0 = initial.noise(N, seed=7 + rank, amplitude=1e-3, kolm=True)
    s.set_w_hat(w0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    s.step_async(args.warmup, DT)
    s.check()
    # timed region: K steps, each bracketed by events; L2 flush between them
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize(dev)
    l0 = s.launch_count
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            for e0, e1 in evs:
                e0.record(stream)
                s.step_async(1, DT)
                e1.record(stream)
                flush.zero_()
        torch.cuda.synchronize(dev)
        s.check()
    launches = s.launch_count - l0
    barrier()
    ms_total = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    # per-kernel device times (events around every launch; eager launches, so
    # this loop is separate from the timed steps above, which replay a graph)
    s.set_kernel_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            s.step_async(1, DT)
            flush.zero_()
    torch.cuda.synchronize(dev)
    s.check()
    kms, kn = s.kernel_times()
    s.set_kernel_timing(False)
    t = torch.tensor([ms_total], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max * 1e-3)

    # end to end through the reference-facing host-buffer call
    host = torch.empty((N, N // 2 + 1, 2), dtype=torch.float64, pin_memory=True)
    hw = host.numpy().view(np.complex128).reshape(N, N // 2 + 1)
    hw[:] = w0
    ke = max(3, min(args.steps, 20))
    s.rk4_step_host(hw, DT)
    walls = []
    barrier()
    for _ in range(ke):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s.rk4_step_host(hw, DT)
        walls.append(time.perf_counter() - t0)
    te = torch.tensor([sum(walls)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * ke / float(te.item())

    full = args.only != "plain"
    if full:
        # FP32 batched ensemble (same process, same GPU)
        ens_v, ens_ms, ens_grids, ens_launches, ens_z = ensemble_bench(stream, flush, args.ens_steps, args.warmup,
                                                                       rank)
        ens_err, ens_err_member = ensemble_error(stream, 1000, rank)
        te2 = torch.tensor([ens_ms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(te2, op=dist.ReduceOp.MAX)
        ens_total = world * 1e3 / float(te2.item())

        # discrete adjoint at 512^2, FP64 and FP32 (same process, same GPU)
        from ns2d import abi as _abi
        adj64 = adjoint_bench(stream, args.adj_steps, rank, _abi.FP64)
        adj32 = adjoint_bench(stream, args.adj_steps, rank, _abi.FP32, g_ref=adj64.pop("gradient"))
        adj = [adj64, adj32]

    if rank != 0:
        s.close()
        return 0

    # roofline of the dominant kernel class.  The per-kernel times come from a
    # second run with an event pair around every launch, which adds a few
    # microseconds per launch; they are scaled by one factor so that they sum
    # to the device time of the un-instrumented steps (the gaps between
    # launches are spread over the kernels, so `achieved` is a lower bound).
    peak, peak_kind = peaks()
    scale = ms_total / max(float(kms[:4].sum()), 1e-30)
    kms_scaled = kms * scale
    dom = int(np.argmax(kms[:4]))
    per_launch_bytes = CLASS_BYTES_PER_LAUNCH[dom] * S_BYTES
    avg_ms = kms_scaled[dom] / kn[dom]
    achieved = per_launch_bytes / (avg_ms * 1e-3) / 1e9
    step_ms = ms_max / args.steps
    model_gbs = MODEL_BYTES_PER_STEP * S_BYTES / (step_ms * 1e-3) / 1e9
    # the same figures for every pass class of the step (the dominant one is `roofline`)
    by_kernel = {}
    for k in range(4):
        if kn[k]:
            kb = CLASS_BYTES_PER_LAUNCH[k] * S_BYTES
            kms_avg = kms_scaled[k] / kn[k]
            ka = kb / (kms_avg * 1e-3) / 1e9
            by_kernel[CLASS_NAMES[k]] = {"achieved": ka, "frac": ka / peak, "algorithmic_bytes_per_launch": kb,
                                         "avg_launch_ms": kms_avg, "traffic": ncu_traffic(k)}
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random-phase noise, 1e-3 amplitude)",
        "config": config("replicas" if world > 1 else "single GPU"),
        "roofline": {"bound": "hbm", "kernel": CLASS_NAMES[dom], "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": ncu_traffic(dom), "traffic_kind": NCU_TRAFFIC_KIND,
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "algorithmic_read_bytes_per_launch": CLASS_READ_PER_LAUNCH[dom] * S_BYTES,
                     "avg_launch_ms": avg_ms},
        "step_roofline": {"model_bytes_per_step": MODEL_BYTES_PER_STEP * S_BYTES, "achieved": model_gbs,
                          "frac": model_gbs / peak, "unit": "GB/s"},
        "roofline_by_kernel": by_kernel,
        "kernels": {CLASS_NAMES[k]: {"ms_total": float(kms_scaled[k]), "ms_total_instrumented": float(kms[k]),
                                     "launches": int(kn[k]),
                                     "share": float(kms[k] / max(kms.sum(), 1e-30))} for k in range(5) if kn[k]},
        "kernels_note": "ms_total: instrumented per-launch event times scaled to the un-instrumented steps' device "
                        "time (they sum to steps x ms_per_step); share: of the instrumented run",
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": S_BYTES, "d2h_bytes_per_step": S_BYTES,
                "call": "ns2d_rk4_step_host"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if full:
        line["fp32_batched"] = {
            "workload": "ensemble 32x128^2 + 24x256^2 + 8x512^2 (4 x 1024^2 points), FP32 RK4CN, nu=1e-3, dt=1e-3",
            "ensemble_steps_per_s": ens_total, "ms_per_step": float(te2.item()),
            "equiv_1024_steps_per_s": 4.0 * ens_total, "ratio_vs_fp64_plain": 4.0 * ens_total / value,
            "tuned_shape": ens_grids, "gpu_launches": int(ens_launches),
            "enstrophy_sample": ens_z, "launches_per_step": ens_launches / max(args.ens_steps, 1),
            "enstrophy_max_rel_err_vs_fp64": ens_err, "enstrophy_err_member": ens_err_member,
            "enstrophy_err_steps": 1000,
        }
        line["adjoint"] = {
            "workload": f"gradient of Z(T) w.r.t. w0, {ADJ_N}^2, nu=1e-3, RK4CN dt={ADJ_DT}, {args.adj_steps} steps, "
                        f"checkpoints every {ADJ_EVERY} steps with stage recomputation",
            "adjoint_over_forward": adj[0]["adjoint_over_forward"], "runs": adj,
        }
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        table = cpu_table(threads, runs=5, budget_s=args.cpu_seconds / 6.0)
        main_row = [r for r in table if r["grid"] == f"{N}x{N}" and r["threads"] == threads][0]
        line["cpu_baseline"] = {
            "value": main_row["steps_per_s_median"], "unit": "steps/s", "cores": threads, "kind": "reference",
            "sample": f"median of 5 timed runs of {main_row['steps_per_run']} RK4CN steps each (after one warm-up "
                      f"step) of the same {N}^2 workload on {threads} host threads: the reference's Solver/src "
                      "built by oracle/Makefile, FFTW-MPI replaced by the oracle's OpenMP FFT",
            "table": table}
    print(json.dumps(line), flush=True)
    s.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ns2d", choices=["ns2d", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ens-steps", type=int, default=20)
    ap.add_argument("--adj-steps", type=int, default=2000)
    ap.add_argument("--ascent", type=int, default=20,
                    help="--only adjoint: projected-ascent iterations of the final enstrophy (0 = none)")
    ap.add_argument("--only", choices=["plain", "ensemble", "adjoint"], default=None,
                    help="one part alone (profiling runs): plain = the 1024^2 FP64 line without the "
                         "ensemble and adjoint parts; ensemble / adjoint print that part's JSON object")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.only in ("ensemble", "adjoint"):
        return run_part(args, local_rank)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        return run_gpu(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
