#!/usr/bin/env python
"""Benchmark of the classic 2D wave-propagation step (ClawSolver2D.step ->
step2/flux2) on the B200.

Workload: 2D Euler, Roe 4-wave solver with entropy fix, gamma = 1.4, 1024 x
1024 cells on [0,1]^2, FP64, extrapolation BCs, MC limiter, unsplit step with
transverse corrections (trans_cor); four-quadrant Riemann data split at
x = y = 0.8.  A step is one pass of the hot path: device ghost-cell fill +
the fused step2 kernel + the grid-wide CFL reduction, with q resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is device-timed (CUDA events on the
stream the kernels run on, L2 flushed between steps, max over ranks); `e2e`
is the same metric through the public patch API with a pinned host -> device
upload of q and a device -> host download of the result inside every step.
`--impl reference` times the CPU restatement of the reference's Fortran
step2 (the oracle; the reference's Fortran cannot be compiled in this image)
on all host cores.
"""
import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s on 1 B200 (FP64, % HBM roofline); batched & learned-guess speedup"
UNIT = "cell-updates/s"
N = 1024
MEQN = 4
BYTES_PER_CELL = 2 * MEQN * 8  # read q^n + write q^{n+1}, FP64
WORKLOAD = "euler_quadrants_roe_1024x1024_unsplit_trans_cor_mc"
# One ncu capture of the step kernel on this workload (profiles/k_step_unsplit_euler_roe_1024.md):
# dram__bytes_read.sum + dram__bytes_write.sum per launch, and the FP64 pipe's busy fraction.
# The launch's 33.5 MB of output stays in L2 while it runs, so DRAM shows the reads only.
NCU_TRAFFIC_BYTES = {1024: 34.801e6 + 0.926e6}
NCU_FP64_PIPE_ACTIVE = {1024: 0.435}


def step_kernel_name(variant):
    """The unsplit step kernel a launch variant runs (claw2_tune_set)."""
    if variant == 8:
        return "k_step_unsplit_ws<RPEulerRoe,128>"
    if variant == 4:
        return "k_step_unsplit2<RPEulerRoe,128>"
    return "k_step_unsplit%s<RPEulerRoe,128,%d>" % ("_tma" if variant & 2 else "", 3 if variant & 1 else 2)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=N, help="grid size override (profiling runs only)")
    ap.add_argument("--secondary", type=int, default=1, help="also time the other benchmark problems")
    ap.add_argument("--learned", type=int, default=1, help="include the learned-guess exact solver")
    ap.add_argument("--shape", default=None, help="fixed launch shape 'variant,rows' (skips the autotuner)")
    ap.add_argument("--pre-t", type=float, default=0.4,
                    help="advance the problem to this time (untimed) before warm-up")
    ap.add_argument("--only", default=None, choices=["shallow_4096", "acoustics_200", "batched_512", "learned_2048"],
                    help="profiling aid: run one of the other workloads alone (with --shape: no autotuning) "
                         "and print its JSON")
    ap.add_argument("--train-problems", type=int, default=1 << 24,
                    help="training-set size of the learned guess (2^24 in the benchmark)")
    ap.add_argument("--epochs", type=int, default=16, help="training epochs of the learned guess")
    ap.add_argument("--learned-n", type=int, default=2048,
                    help="grid size of the learned-guess workload (2048 in the benchmark; smaller for profiling)")
    ap.add_argument("--learned-pre-t", type=float, default=0.4,
                    help="time the learned-guess workload's state is advanced to (0.4 in the benchmark)")
    ap.add_argument("--replicas", action="store_true",
                    help="with --gpus N > 1: N independent copies of the problem instead of the row-slab "
                         "decomposition")
    ap.add_argument("--overlap", action="store_true",
                    help="row slabs: step the interior row blocks while the halo rows move (two launches per "
                         "step; off by default: at 1024^2 the second launch's tail costs more than the "
                         "exchange it hides)")
    ap.add_argument("--slab", action="store_true",
                    help="use the row-slab code path even on one GPU (one slab: no neighbours)")
    ap.add_argument("--state", default=None,
                    help="profiling aid: .npy file of the advanced state; loaded if it exists (no "
                         "advance), else written after the advance")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def config(extra=None):
    c = {"workload": WORKLOAD, "mx": N, "my": N, "num_eqn": MEQN, "riemann": "euler_4wave_2D (Roe, efix)",
         "limiter": "MC", "transverse": "trans_cor", "dimensional_split": False, "bc": "extrap",
         "l2": "flushed between timed steps (256 MiB write, not timed)"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML reads only)
# ---------------------------------------------------------------------------
class ClockSampler(object):
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index):
        self.samples, self.reasons = [], set()
        self._stop = threading.Event()
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for b, name in self.REASONS.items():
                    if bits & b and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self._nv is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._nv is not None:
            self._t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# ---------------------------------------------------------------------------
# CPU legs (the oracle): single-thread baseline and the all-core reference arm
# ---------------------------------------------------------------------------
def cpu_rate(threads, budget_s, max_steps=None, warmup=1):
    """cell-updates/s of the oracle's step2 on the benchmark workload, after
    `warmup` untimed steps (the first also sets dt near CFL 0.9)."""
    from oracle import pyoracle
    from pyclaw_b200 import workloads
    pyoracle.set_threads(threads)
    claw = workloads.euler_quadrants_unsplit(pyoracle.make_solver_class(), n=N)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    s.dt = 2.5e-4
    s.step_hyperbolic(sol)  # warm-up (also sets dt near CFL 0.9)
    s.dt = s.dt * 0.9 / max(s.cfl.get_cached_max(), 1e-12)
    for _ in range(max(warmup, 1) - 1):
        s.step_hyperbolic(sol)
    steps, t0 = 0, time.perf_counter()
    while True:
        s.step_hyperbolic(sol)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_steps is not None and steps >= max_steps):
            break
    return N * N * steps / el, steps, el


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    ncores = len(os.sched_getaffinity(0))
    budget = max(5.0, min(120.0, 0.5 * args.steps))
    warmup = max(args.warmup, 1)
    value, steps, el = cpu_rate(ncores, budget, max_steps=args.steps, warmup=warmup)
    sample = ("%d full steps of the %dx%d workload (oracle step2 + host ghost fill), OpenMP over row "
              "colours, %.1f s" % (steps, N, N, el))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": warmup, "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config({"reference": "C++ restatement of step2.f90/flux2.f90/limiter.f90/philim.f90 "
                                           "(oracle/claw_oracle.cpp); the reference Fortran needs gfortran, "
                                           "absent from this image"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
def copy_bound(nbytes, reps):
    """Wall-clock rate of the copies alone: reps times, nbytes from pinned host
    memory to the device on one stream while nbytes go the other way on a
    second one (both PCIe directions at once, as in the e2e pipeline).
    Returns (seconds per pair, H2D GB/s alone, D2H GB/s alone)."""
    import torch
    n = nbytes // 8
    hi = torch.empty(n, dtype=torch.float64, pin_memory=True)
    hi.fill_(1.0)
    ho = torch.empty(n, dtype=torch.float64, pin_memory=True)
    d1 = torch.empty(n, dtype=torch.float64, device="cuda")
    d2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def run(h2d, d2h):
        for k in range(reps + 2):  # two untimed rounds first
            if k == 2:
                torch.cuda.synchronize()
                t0 = time.perf_counter()
            if h2d:
                with torch.cuda.stream(s1):
                    d1.copy_(hi, non_blocking=True)
            if d2h:
                with torch.cuda.stream(s2):
                    ho.copy_(d2, non_blocking=True)
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    # the host link's rate varies with the host's other traffic: the best of
    # three rounds of each (the bound is the fastest the copies went)
    up = min(run(True, False) for _ in range(3))
    down = min(run(False, True) for _ in range(3))
    both = min(run(True, True) for _ in range(3))
    return both, nbytes / up / 1e9, nbytes / down / 1e9


def time_patch(patch, dt, steps, flush, stream):
    """Mean step and step-kernel times (ms) of a device patch, L2 flushed
    between steps; the state advances (every step accepted)."""
    import torch
    patch.set_stream(stream.cuda_stream)
    patch.set_timing(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    kern = []
    for k in range(steps):
        flush.zero_()
        ev[k][0].record(stream)
        patch.step(dt, want_cfl=False)
        patch.accept(True)
        ev[k][1].record(stream)
        kern.append(patch.kernel_ms())
    torch.cuda.synchronize()
    patch.sync()
    return statistics.mean(a.elapsed_time(b) for a, b in ev), statistics.mean(kern)


def batched_workload(n_instances=512, steps=100, plain=True):
    """The batched form: n independent Euler quadrant problems of uneven size
    (side 64..512), 100 steps with per-problem dt; aggregate cell-updates/s of
    the graph-captured persistent form and (plain=True) of the plain
    per-problem loop."""
    import numpy as np
    from pyclaw_b200 import batch as pb, workloads
    claws, sides = workloads.batched_quadrants(n_instances)
    bat = pb.Batch(claws)
    dt0 = [c.solver.dt_initial for c in claws]
    rows, trials, choice = pb.autotune_rows(bat, sides)
    cells = sides.astype(np.float64) ** 2
    out = {"instances": n_instances, "cells_total": float(cells.sum()), "steps": steps,
           "rows_per_bucket": [int(c) for c in choice], "bucket_edges": [128, 256],
           "plain_loop_rows": "single-problem heuristic (0)"}
    ntiles, grid = bat.tiles()
    out["tiles"], out["persistent_grid"] = ntiles, grid
    for mode, name in ((0, "graph_persistent"), (2, "plain_per_instance_loop"))[:2 if plain else 1]:
        if mode == 2:
            # the plain loop launches each problem alone: give every launch the
            # single-problem heuristic shape (most CTAs per launch), not the
            # row heights tuned for the persistent kernel
            bat.set_rows(np.zeros(n_instances, dtype=np.intc))
        bat.upload()
        bat.set_time(dt0, 0.0, 1e99)
        bat.run(1, mode=mode)  # warm (captures the graph for 1 step)
        bat.upload()
        bat.set_time(dt0, 0.0, 1e99)
        ms = bat.run(steps, mode=mode)
        st = bat.state()
        upd = float((cells * st["nsteps"]).sum())
        out[name] = {"ms": ms, "value": upd / (ms * 1e-3), "unit": UNIT,
                     "accepted_steps": int(st["nsteps"].sum()), "rejected_steps": int(st["nreject"].sum()),
                     "failed_instances": int(st["failed"].sum()),
                     "failed_instance_ids": [int(i) for i in np.nonzero(st["failed"])[0]],
                     "failed_note": "retired when a step produced a non-finite value (Roe's linearisation "
                                    "loses positivity in their strong rarefactions); the oracle fails at the "
                                    "same attempt (tests/test_gpu_headline.py)"}
    if plain:
        out["speedup"] = out["graph_persistent"]["value"] / out["plain_per_instance_loop"]["value"]
    bat.close()
    return out


def learned_workload(stream, flush, n=2048, steps=10, n_train=1 << 24, epochs=16, pre_t=0.4, shape=None):
    """Exact Euler solver on the quadrant problem (n^2, unsplit trans_cor, MC),
    Newton started from the adaptive PVRS guess vs from the learned guess of a
    network trained here on n_train seeded problems by the library's kernels.
    shape: a fixed launch shape (variant, rows) instead of the autotuner's."""
    fixed_shape = tuple(shape) if shape is not None else None
    import numpy as np
    import torch
    from pyclaw_b200 import learned, riemann, workloads
    out = {"n": n, "train_problems": n_train, "epochs": epochs}
    t0 = time.perf_counter()
    net = learned.Network(seed=2024)
    out["valid_problems"] = net.generate(n_train, seed=7)
    torch.cuda.synchronize()
    out["generate_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    out["final_loss"] = net.train(epochs=epochs, batch=16384, lr=3e-3)
    out["train_s"] = time.perf_counter() - t0
    # advance the Roe problem to mid-run, then hand the state to the exact solver
    claw = workloads.euler_quadrants_unsplit(n=n)
    s, sol = claw.solver, claw.solution
    s.setup(sol)
    p = s._dev
    t, dt, cfl = 0.0, 1e-4, None
    while t < pre_t:
        dt = min(dt if cfl is None else dt * 0.9 / cfl, pre_t - t)
        cfl = p.step(dt)
        p.accept(cfl <= 1.0)
        if cfl <= 1.0:
            t += dt
    q_mid = sol.state.get_q_global()
    p.close()
    res = {}
    # converged guesses with a fixed relative error of the size a guess of
    # that precision carries (half an ulp of BF16, FP16, FP32), where the
    # adaptive guess needs Newton steps (the adaptive guess elsewhere)
    precision = {"bf16": 2.0 ** -9, "fp16": 2.0 ** -12, "fp32": 2.0 ** -25}
    for mode in ("pvrs", "learned", "learned_mma_sync", "converged") + tuple(precision):
        ce = workloads.euler_quadrants_unsplit(n=n)
        ce.solver.rp = riemann.euler_exact_2D
        ce.solver.num_waves = 3
        ce.solution.state.q = q_mid
        ce.solver.setup(ce.solution)
        pe = ce.solver._dev
        # the network's tensor-core path: tcgen05 (the default) or, for the
        # comparison, the warp-level mma.sync form
        net.set_engine("mma.sync" if mode == "learned_mma_sync" else "tcgen05")
        learned.attach(ce.solver, net if mode.startswith("learned") else None)
        if mode == "converged":
            # the floor for any guess: every step starts from the converged p*
            # (pre-pass outside the kernel timing)
            learned.converged_guess(ce.solver)
        elif mode in precision:
            learned.converged_guess(ce.solver, rel_error=precision[mode])
        c1 = pe.step(dt)
        pe.accept(False)
        dte = dt * 0.9 / c1
        # launch shape tuned once on the PVRS run (cached per solver and size,
        # so the learned run uses the same one)
        from pyclaw_b200 import tune
        if fixed_shape is not None:
            tune.set_shape(pe.desc.riemann, *fixed_shape)
            shape = fixed_shape
        else:
            pe.set_stream(stream.cuda_stream)
            shape, _ = tune.autotune(pe, dte, before_step=flush.zero_)
        learned.newton_counts(ce.solver)
        step_ms, kern_ms = time_patch(pe, dte, steps, flush, stream)
        it, applied, ns = learned.newton_counts(ce.solver)
        res[mode] = {"value": n * n / (step_ms * 1e-3), "unit": UNIT, "ms_per_step": step_ms,
                     "kernel_ms": kern_ms, "newton_per_interface": it / max(ns, 1),
                     "newton_applied_per_interface": applied / max(ns, 1), "solves": ns,
                     "launch_shape": list(shape)}
        # one step from the same state for the same-answer check
        ce.solution.state.q = q_mid
        pe.push(ce.solution.state)
        pe.step(dte, want_cfl=False)
        pe.accept(True)
        res[mode]["_q"] = ce.solution.state.get_q_global()
        pe.close()
    qa, qb, qc = res["pvrs"].pop("_q"), res["learned"].pop("_q"), res["converged"].pop("_q")
    qm = res["learned_mma_sync"].pop("_q")
    out["pvrs_guess"], out["learned_guess"] = res["pvrs"], res["learned"]
    out["learned_guess_mma_sync"] = res["learned_mma_sync"]
    out["converged_guess_floor"] = res["converged"]
    out["max_rel_diff_one_step"] = float(np.max(np.abs(qa - qb)) / np.max(np.abs(qa)))
    out["max_rel_diff_one_step_mma_sync"] = float(np.max(np.abs(qa - qm)) / np.max(np.abs(qa)))
    out["max_rel_diff_one_step_converged"] = float(np.max(np.abs(qa - qc)) / np.max(np.abs(qa)))
    out["speedup"] = res["learned"]["value"] / res["pvrs"]["value"]
    out["speedup_ceiling"] = res["pvrs"]["kernel_ms"] / res["converged"]["kernel_ms"]
    out["precision_ceilings"] = {}
    for mode, rel in precision.items():
        r = res[mode]
        r.pop("_q")
        out["precision_ceilings"][mode] = {
            "rel_error": rel, "newton_per_interface": r["newton_per_interface"],
            "kernel_ms": r["kernel_ms"], "speedup_ceiling": res["pvrs"]["kernel_ms"] / r["kernel_ms"]}
    out["note"] = ("kernel_ms of the learned guess includes its tensor-core guess pre-pass; that of the "
                   "converged-guess floor excludes its pre-pass (the step kernel alone with perfect "
                   "guesses): speedup_ceiling = PVRS step kernel / that, the most any guess can gain on "
                   "this workload.  newton_per_interface counts the steps needed (a final step below "
                   "tolerance is applied but not counted), newton_applied_per_interface counts it too.  "
                   "precision_ceilings: the same floor with the converged p* off by a fixed relative "
                   "error of up to half an ulp of that format where the PVRS guess needs Newton steps "
                   "(PVRS elsewhere), i.e. the most a guess of that precision can gain with PVRS as "
                   "its fallback (tolerance 1e-12)")
    net.close()
    return out


def secondary_workloads(stream, flush, peaks, only=None, shape=None):
    """The shallow-water dam break at 4096^2, 200 steps at CFL 0.9 from its
    initial state, and the walled acoustics problem at 200^2 run to t = 0.6
    at CFL 0.9 (48 B/cell each), unsplit trans_cor, MC."""
    import math
    import torch
    from pyclaw_b200 import tune, workloads
    out = {}
    for name, make, bpc in [("shallow_roe_dam_break_4096", lambda: workloads.shallow_dam_break_unsplit(n=4096), 48),
                            ("acoustics_wall_200", lambda: workloads.acoustics_wall(n=200), 48)]:
        if only is not None and name != only:
            continue
        claw = make()
        s, sol = claw.solver, claw.solution
        s.setup(sol)
        p = s._dev
        p.set_stream(stream.cuda_stream)
        dt = s.dt_initial if name.startswith("acoustics") else 1e-4
        cfl = p.step(dt)
        p.accept(False)
        dt = dt * 0.9 / cfl
        if shape is not None:
            use = tuple(shape)
            tune.set_shape(p.desc.riemann, *use)
        else:
            use, _ = tune.autotune(p, dt, before_step=flush.zero_)
        steps = 200 if name.startswith("shallow") else int(math.ceil(0.6 / dt))
        step_ms, kern_ms = time_patch(p, dt, steps, flush, stream)
        n = sol.state.grid.num_cells[0] * sol.state.grid.num_cells[1]
        gbs = n * bpc / (kern_ms * 1e-3) / 1e9
        out[name] = {"value": n / (step_ms * 1e-3), "unit": UNIT, "ms_per_step": step_ms, "kernel_ms": kern_ms,
                     "bytes_per_cell": bpc, "achieved_gbs": gbs, "hbm_frac": gbs / peaks["hbm_gbs"],
                     "launch_shape": list(use), "steps": steps}
        p.close()
        if name.startswith("acoustics"):
            # the whole run as a user runs it: Controller.run() to t = 0.6 on the
            # device time loop (one output time), wall clock including setup,
            # upload and the final download; best of three
            best = None
            for _ in range(3):
                c = workloads.acoustics_wall(n=200)
                c.keep_copy, c.output_format, c.num_output_times = False, None, 1
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                c.run()
                el = time.perf_counter() - t0
                best = el if best is None else min(best, el)
            out[name]["controller_run"] = {"ms": best * 1e3, "steps": c.solver.status['numsteps'],
                                           "value": n * c.solver.status['numsteps'] / best, "unit": UNIT,
                                           "what": "Controller.run() to t = 0.6, device time loop, wall clock "
                                                   "with setup, upload and download"}
    return out

def run_one(args):
    """One of the other workloads alone (profiling aid)."""
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream(torch.device("cuda", 0))
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    shape = tuple(int(x) for x in args.shape.split(",")) if args.shape else None
    if args.only == "shallow_4096":
        out = secondary_workloads(stream, flush, measured_peaks()[0], "shallow_roe_dam_break_4096", shape)
    elif args.only == "acoustics_200":
        out = secondary_workloads(stream, flush, measured_peaks()[0], "acoustics_wall_200", shape)
    elif args.only == "batched_512":
        out = {"batched_quadrants_512": batched_workload(plain=False)}
    else:
        out = {"learned_exact_euler_%d" % args.learned_n: learned_workload(
            stream, flush, n=args.learned_n, n_train=args.train_problems, epochs=args.epochs,
            pre_t=args.learned_pre_t, shape=shape)}
    torch.cuda.synchronize()
    print(json.dumps(out), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    from pyclaw_b200 import _lib, workloads

    if args.only:
        return run_one(args)
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)  # one non-default stream: kernels, flushes and events
    torch.cuda.set_stream(stream)
    n = args.n

    # weak scaling.  With N > 1 ranks the default is the row-slab
    # decomposition: rank r owns an n x n slab of an n x (n N) grid (the
    # quadrant data repeated along y), and every step exchanges two halo rows
    # with each neighbour (NCCL, device to device) and reduces the Courant
    # number (all-reduce MAX) before the accept decision, as petclaw does.
    # --replicas runs N independent copies instead.
    slab = (world > 1 and not args.replicas) or args.slab
    if slab:
        from pyclaw_b200 import classic, slabs
        claw = workloads.euler_quadrants_unsplit(slabs.make_slab_solver_class(classic.ClawSolver2D), n=n)
        claw.solver.slab = (rank, world, False, None)
        claw.solver.global_delta = tuple(claw.solution.state.grid.delta)
    else:
        claw = workloads.euler_quadrants_unsplit(n=n)
    solver, sol = claw.solver, claw.solution
    solver.device = local
    solver.setup(sol)
    patch = solver._dev
    patch.set_stream(stream.cuda_stream)

    side = torch.cuda.Stream(dev) if slab else None

    def slab_step(dt):
        """One decomposed step: the halo rows in, the local step, the global
        Courant number and the same accept decision on every rank (--overlap:
        the interior row blocks on the patch's stream while the halo rows move
        on a side stream, then the edge row blocks)."""
        if not args.overlap:
            planes = slabs.DevicePlanes(patch)
            slabs.exchange_rows(planes.get_rows, planes.set_rows, n, rank, world, False)
            local = patch.step(dt)
        else:
            ready = torch.cuda.Event()
            ready.record(stream)
            patch.step_part(dt, 1)
            with torch.cuda.stream(side):
                side.wait_event(ready)
                planes = slabs.DevicePlanes(patch)
                slabs.exchange_rows(planes.get_rows, planes.set_rows, n, rank, world, False)
                moved = torch.cuda.Event()
                moved.record(side)
            stream.wait_event(moved)
            local = patch.step_part(dt, 2)
        cfl = slabs.global_cfl(local, device=dev)
        patch.accept(cfl <= 1.0)
        return cfl

    # advance (untimed) to the middle of the run so the timed steps see a
    # developed flow, with the reference's dt rule (cfl_desired 0.9)
    t, dt, cfl = 0.0, 2.5e-4, None
    if args.state and os.path.exists(args.state):
        q = np.asfortranarray(np.load(args.state))
        _lib.check(_lib.load().claw2_patch_upload_q(patch.h, _lib.dptr(q)))
        patch.host_dirty, patch.device_newer = False, True
        t = args.pre_t
    while t < args.pre_t:
        dt = min(dt, args.pre_t - t) if cfl is None else min(dt * 0.9 / cfl, args.pre_t - t)
        if slab:
            cfl = slab_step(dt)
            ok = cfl <= 1.0
        else:
            cfl = patch.step(dt)
            ok = cfl <= 1.0
            patch.accept(ok)
        if ok:
            t += dt
    if args.state and not os.path.exists(args.state):
        q = np.empty((MEQN, n, n), order="F")
        _lib.check(_lib.load().claw2_patch_download_q(patch.h, _lib.dptr(q)))
        np.save(args.state, q)
    # fixed dt for CFL 0.9 from a probe step
    cfl = patch.step(dt)
    patch.accept(False)
    if slab:
        cfl = slabs.global_cfl(cfl, device=dev)
    dt = dt * 0.9 / cfl
    # launch shape from the autotuner (trial steps are rejected: state unchanged),
    # each trial after the same L2 flush as the timed steps
    from pyclaw_b200 import tune
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    if args.shape:
        shape, trials = tuple(int(x) for x in args.shape.split(",")), {}
        tune.set_shape(patch.desc.riemann, *shape)
    else:
        shape, trials = tune.autotune(patch, dt, before_step=flush.zero_)
    patch.set_timing(True)
    for _ in range(args.warmup):
        flush.zero_()
        if slab:
            slab_step(dt)
        else:
            patch.step(dt, want_cfl=False)
            patch.accept(True)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kern_ms = []
    launches0 = ctypes.c_longlong(0)
    _lib.check(_lib.load().claw2_patch_launch_count(patch.h, ctypes.byref(launches0)))
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            if slab:
                slab_step(dt)
            else:
                patch.step(dt, want_cfl=False)
                patch.accept(True)
            ev[k][1].record(stream)
            kern_ms.append(patch.kernel_ms())
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches1 = ctypes.c_longlong(0)
    _lib.check(_lib.load().claw2_patch_launch_count(patch.h, ctypes.byref(launches1)))
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    patch.sync()  # raises if any step produced a non-finite value
    last_cfl = patch.cfl()

    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    cells = n * n
    value = world * cells * args.steps / (total_ms * 1e-3)

    # roofline of the dominant kernel (the fused step)
    peaks, peak_src = measured_peaks()
    kms = statistics.mean(kern_ms)
    achieved = cells * BYTES_PER_CELL / (kms * 1e-3) / 1e9
    fp64 = ctypes.c_double(0.0)
    _lib.check(_lib.load().claw2_probe_fp64(local, ctypes.byref(fp64)))

    # end to end through the public patch API with pinned host buffers: every
    # step uploads its input state and downloads its result
    e2e = None
    if args.e2e_steps > 0:
        qh = torch.empty((n * n * MEQN,), dtype=torch.float64, pin_memory=True).numpy()
        qh[:] = sol.state.get_q_global().reshape(-1, order="F")
        qd = torch.empty_like(torch.from_numpy(qh)).pin_memory().numpy()
        L = _lib.load()
        e2e_patch = patch
        if slab:
            # host-to-host steps of independent states (each rank its own
            # pipeline; a decomposed run keeps its state on the devices)
            ec = workloads.euler_quadrants_unsplit(n=n)
            ec.solver.device = local
            ec.solver.setup(ec.solution)
            e2e_patch = ec.solver._dev
            e2e_patch.set_stream(stream.cuda_stream)
        h = e2e_patch.h
        cflv = ctypes.c_double(0.0)
        K = args.e2e_steps
        # the copies alone, before the e2e runs (and again after them below):
        # the host link's rate moves with the host's other traffic
        pair_a = copy_bound(qh.nbytes, K)
        # (1) one call per step: upload, step (waits for the CFL), accept, download
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(K):
            _lib.check(L.claw2_patch_upload_q(h, _lib.dptr(qh)))
            _lib.check(L.claw2_patch_step(h, ctypes.c_double(dt), ctypes.byref(cflv)))
            _lib.check(L.claw2_patch_accept(h, 1))
            _lib.check(L.claw2_patch_download_q(h, _lib.dptr(qd)))
        el_seq = time.perf_counter() - t0
        # (2) claw2_patch_run_host: the same K host-to-host steps with the next
        # input's copy overlapping this step's compute and result copy
        qin = [qh.reshape((MEQN, n, n), order="F")] * K
        qout = [qd.reshape((MEQN, n, n), order="F")] * K
        e2e_patch.run_host(qin[:2], qout[:2], [dt, dt])  # allocates the staging buffers
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_patch.run_host(qin, qout, [dt] * K)
        el = time.perf_counter() - t0
        e2e_val, seq_val = cells * K / el, cells * K / el_seq
        pair_b = copy_bound(qh.nbytes, K)
        pair_s = min(pair_a[0], pair_b[0])
        up_gbs, down_gbs = max(pair_a[1], pair_b[1]), max(pair_a[2], pair_b[2])
        if world > 1:
            t = torch.tensor([el, el_seq], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_val, seq_val = world * cells * K / float(t[0].item()), world * cells * K / float(t[1].item())
        e2e = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": qh.nbytes,
               "d2h_bytes_per_step": qd.nbytes + 8, "steps": K,
               "path": "claw2_patch_run_host: per step, pinned host state -> device, ghost fill + step + CFL, "
                       "result -> pinned host; uploads and downloads on their own streams overlap the "
                       "compute of the neighbouring steps; wall clock",
               "copy_bound": {"value": cells / pair_s, "unit": UNIT, "frac": e2e_val / world / (cells / pair_s),
                              "h2d_gbs": up_gbs, "d2h_gbs": down_gbs,
                              "both_gbs_each": qh.nbytes / pair_s / 1e9,
                              "what": "the step's upload and download alone (pinned, both directions at once, "
                                      "no compute; fastest of rounds before and after the e2e runs): the rate "
                                      "e2e cannot exceed on this host link"},
               "one_call_per_step": {"value": seq_val, "unit": UNIT,
                                     "path": "claw2_patch_upload_q + claw2_patch_step (returns CFL) + "
                                             "claw2_patch_accept + claw2_patch_download_q"}}

    secondary = {}
    if rank == 0 and world == 1 and args.secondary:
        secondary = secondary_workloads(stream, flush, peaks)
        secondary["batched_quadrants_512"] = batched_workload()
        if args.learned:
            secondary["learned_exact_euler_2048"] = learned_workload(stream, flush, n_train=args.train_problems,
                                                                     epochs=args.epochs)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and n == N:
        v, s, el = cpu_rate(1, args.cpu_sample_s)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "%d full %dx%d steps of the oracle step2 (single thread), %.1f s" % (s, N, N, el)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "ours",
                "config": config({"dt": dt, "cfl_last": last_cfl, "mx": n, "my": n,
                                  "parallelism": ("row slabs: %d x %d grid, one %d x %d slab per rank, halo "
                                                  "exchange (NCCL%s) + CFL all-reduce every step"
                                                  % (n, n * world, n, n,
                                                     ", overlapping the interior row blocks" if args.overlap
                                                     else "")) if slab else
                                                 ("%d independent replicas" % world),
                                  "launch_shape": {"variant": shape[0], "rows": shape[1],
                                                   "trials_ms": {"%d/%d" % k: round(v, 4)
                                                                 for k, v in sorted(trials.items())}},
                                  "state": "quadrant problem advanced to t=%g before warm-up" % args.pre_t}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                             "frac": achieved / peaks["hbm_gbs"], "traffic": NCU_TRAFFIC_BYTES.get(n),
                             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch "
                                               "(profiles/k_step_unsplit_euler_roe_1024.md)",
                             "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_src,
                             "kernel": "%s (launch variant %d, H = %d)" % (step_kernel_name(shape[0]), shape[0],
                                                                           shape[1]),
                             "kernel_ms": kms,
                             "algorithmic_bytes_per_launch": cells * BYTES_PER_CELL,
                             "fp64_probe_tflops": fp64.value,
                             "fp64_pipe_active_ncu": NCU_FP64_PIPE_ACTIVE.get(n),
                             "note": "FP64-latency-bound kernel (10.8 warps/SM at the tuned 3-CTA shape, "
                                     "dependency waits the top stall): ~870 FP64 instructions per developed "
                                     "cell-update cap it near 2.1e10 cell-updates/s (21% of HBM) on this part; "
                                     "warps whose interfaces all have equal cells on both sides (37% of this "
                                     "state's) skip the finish"},
                "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
                "secondary": secondary,
                "gpu_launches": int(launches1.value - launches0.value)}
        print(json.dumps(line), flush=True)
    solver._dev.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
