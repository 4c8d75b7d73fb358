#!/usr/bin/env python3
"""Benchmark of the 2D pseudo-spectral vorticity DNS step on B200.

Workload: plain DNS at N=4096 (6144 x 6144 dealiased physical grid), Re=1e5, K0=4, CFL=0.1,
ADAPT_VISC=0, diagnostics (NEXTDT + OM2PHYS + display sigma) every UPDATE=100 steps as in the
reference's mem_cuda loop.  A "step" is one time step (row pass + column pass); the timed K
steps include their diagnostic steps, like the reference's "Steady FPS".  Initial field: seeded
random-phase k^4 exp(-2(k/K0)^2) spectrum, E = 1/2 (synthetic).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--gpus N > 1 runs under torchrun, one independent replica per GPU (the solver does not shard;
value = all replicas' steps / max-over-ranks device time).  --impl reference runs the
reference's own cuFFT build (oracle/_ref/mem_cuda, compiled from its unmodified sources) on the
same arguments and reports its Steady FPS; when that binary is absent it times the FP64 oracle.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

# dns4096: the headline configuration.  dns29400: the large run of the reference's README
# (mem_cuda 29400 1E7 4 41 0.1 20 0: 41 steps, its Steady FPS after 20 warm-up steps).
# dns16384: the reference's recorded N=16384 run (mem_cuda 16384 1E6 5 21 0.2 10 0), with 41 steps.
WORKLOADS = {
    "dns4096": dict(N=4096, Re=1.0e5, K0=4.0, CFL=0.1, UPDATE=100, ADAPT_VISC=0, seed=0, steps=500, warmup=100),
    "dns16384": dict(N=16384, Re=1.0e6, K0=5.0, CFL=0.2, UPDATE=10, ADAPT_VISC=0, seed=0, steps=31, warmup=10),
    "dns29400": dict(N=29400, Re=1.0e7, K0=4.0, CFL=0.1, UPDATE=20, ADAPT_VISC=0, seed=0, steps=21, warmup=20),
}
WORKLOAD = dict(WORKLOADS["dns4096"])
METRIC = "steps/s (2D vorticity DNS time step, N=4096, 6144^2 padded grid)"


def select_workload(name: str, n: int | None):
    global METRIC
    WORKLOAD.clear()
    WORKLOAD.update(WORKLOADS.get(name, WORKLOADS["dns4096"]))
    if n:
        WORKLOAD["N"] = n
    N = WORKLOAD["N"]
    METRIC = f"steps/s (2D vorticity DNS time step, N={N}, {3 * N // 2}^2 padded grid)"


def workload_text(N: int) -> str:
    w = WORKLOAD
    return (f"plain DNS N={N} ({3 * N // 2}^2 padded grid), Re={w['Re']:.0e}, K0={w['K0']:g}, CFL={w['CFL']:g}, "
            f"ADAPT_VISC=0, UPDATE={w['UPDATE']}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--cpu-steps", type=int, default=24,
                    help="FP64 oracle steps for cpu_baseline (about 10 s on 16 host cores at N=4096)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--profile", choices=["step", "closure", "network", "training", "training-tc"], default=None,
                    help="short run for an ncu capture, nothing timed or printed as a bench line: 'step' = "
                         "k^4 field (seed 1), NEXTDT, 1 + 3 steps of size --n through the step graphs; "
                         "'closure' = 3 closed steps at N=256 with a 6 x 32 network; 'network' = the "
                         "persistent network launch on a 384^2 image with its per-tile trace, summarised; "
                         "'training' = Adam iterations of the 6 x 32 closure network (batch 4 at 384^2 and "
                         "batch 32 at 48^2) with FP32 and with tensor-core convolutions, timed; 'training-tc' = "
                         "3 tensor-core Adam iterations at 384^2, batch 4 (for an ncu launch list)")
    ap.add_argument("--windows", type=int, default=0,
                    help="number of timed K-step windows (0: as many as fill about 1 s of device time)")
    ap.add_argument("--workload", choices=["dns4096", "dns16384", "dns29400", "ensemble"], default="dns4096",
                    help="dns16384 / dns29400: N=16384 (24576^2 grid) / N=29400 (44100^2 grid), the "
                         "reference's recorded and README large runs; "
                         "ensemble: the 64-member batched configuration (32xN=128, 24xN=256, 8xN=512)")
    a = ap.parse_args()
    select_workload(a.workload, a.n)
    a.n = WORKLOAD["N"]
    if a.steps is None:
        a.steps = WORKLOAD["steps"]
    if a.warmup is None:
        a.warmup = WORKLOAD["warmup"]
    if a.workload in ("dns16384", "dns29400"):
        # the FP64 oracle needs tens of GB of host memory here, and a host round trip of the
        # multi-GB state per step would dominate the e2e figure: both are reported at N=4096
        a.no_cpu_baseline = True
        a.no_e2e = True
    return a


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The maximum of a per-rank value over all ranks (the slowest replica's time)."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(steps: int, ms_max: float, world: int) -> float:
    """Whole-job steps/s of `world` independent replicas that each ran `steps` steps, timed by
    the slowest one."""
    return world * steps / (ms_max / 1e3)


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------------------------------
# clock sampling during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# the run loop of the reference (cuda/mem_cuda.cu:1848-1897), through the C ABI
# ------------------------------------------------------------------------------------------
def segments(it_from, it_to, update):
    """Lengths of the dns2d_step calls advance() makes from it_from to it_to."""
    out, it = [], it_from
    while it < it_to:
        nxt = 1 if it < 1 else min(it_to, (it // update + 1) * update)
        out.append(nxt - it)
        it = nxt
    return out


def advance(s, it_to, update, steps_total, counts, history=False):
    """Advance a Solver to step it_to with the reference's diagnostic cadence."""
    hist = []
    while True:
        it = s.scalars()["it"]
        if it >= it_to:
            break
        nxt = it_to
        if it < 1:
            nxt = 1
        else:
            nxt = min(it_to, (it // update + 1) * update)
        n = nxt - it
        r = s.step(n, history=history)
        if history:
            hist.append(r)
        counts["kernels"] += 2 * n + (n + 127) // 128
        if nxt == 1 or nxt % update == 0 or nxt == steps_total:
            s.next_dt()
            s.om2phys()
            s.display_sigma(2)
            counts["kernels"] += 5
    return hist


def window_plan(W: int, K: int, update: int, ms_per_step_est: float, target_ms: float = 1000.0,
                max_windows: int = 200):
    """Start steps of the timed windows: consecutive K-step windows after the W warm-up steps,
    as many as fill about target_ms of device time (at least 3, at most max_windows)."""
    n = int(target_ms / max(1e-6, ms_per_step_est * K)) + 1
    n = max(3, min(max_windows, n))
    return [W + i * K for i in range(n)]


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import optimizec_b200 as P

    N, K, W = args.n, args.steps, args.warmup
    up = WORKLOAD["UPDATE"]
    torch.cuda.set_device(local_rank)
    tuning = P.autotune(N, local_rank)  # kernel variants with identical arithmetic; fastest kept
    s = P.Solver(N, WORKLOAD["Re"], WORKLOAD["K0"], WORKLOAD["CFL"], device=local_rank)
    s.init_k4(WORKLOAD["seed"] + rank)
    s.next_dt()
    stream = torch.cuda.ExternalStream(s.stream(), device=local_rank)
    counts = {"kernels": 0}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    advance(s, W, up, W, counts)  # warm-up, ending with a diagnostic step like every window
    e1.record(stream)
    s.sync()
    est = e0.elapsed_time(e1) / max(1, W)
    starts = window_plan(W, K, up, est) if args.windows <= 0 else [W + i * K for i in range(args.windows)]
    if world > 1:  # every rank runs the same number of windows
        starts = starts[:int(-max_over_ranks(-len(starts), world, device=f"cuda:{local_rank}"))]
    for w0 in starts:  # graph capture stays out of the timed region
        for n in set(segments(w0, w0 + K, up)):
            s.prepare(n)
    s.sync()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in starts]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    counts = {"kernels": 0}
    for (a, b), w0 in zip(evs, starts):
        a.record(stream)
        # one window: K steps with the reference's diagnostic cadence, ending on a diagnostic
        # step as the reference's run ends on it == STEPS
        advance(s, w0 + K, up, w0 + K, counts)
        b.record(stream)
    s.sync()
    torch.cuda.synchronize()
    ck = clocks.stop()
    win = [a.elapsed_time(b) for a, b in evs]
    ms = statistics.median(win)
    ms_max = max_over_ranks(ms, world, device=f"cuda:{local_rank}")
    if world > 1:
        torch.distributed.barrier()
    value = replica_throughput(K, ms_max, world)

    E_end, Z_end = s.energy_enstrophy()
    if not (np.isfinite(E_end) and np.isfinite(Z_end) and 0.0 < E_end < 1.0):
        raise RuntimeError(f"the field is not a valid state after the timed steps: E={E_end} Z={Z_end}")

    # per-kernel device time (CUDA events around each launch, on the solver's stream)
    s.phase_timing(True)
    s.step(20)
    ph_ms, ph_n = s.phase_report()
    s.phase_timing(False)
    rows_ms = ph_ms[0] / max(ph_n[0], 1)
    cols_ms = ph_ms[1] / max(ph_n[1], 1)
    s.close()
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(P, N, K, W, up, local_rank, world)
    return dict(value=value, ms=ms_max, K=K, W=W, N=N, kernels=counts["kernels"], clocks=ck,
                rows_ms=rows_ms, cols_ms=cols_ms, e2e=e2e, tuning=tuning,
                windows={"count": len(win), "median_ms": round(ms, 4), "min_ms": round(min(win), 4),
                         "max_ms": round(max(win), 4), "first_ms": round(win[0], 4)})


def run_e2e(P, N, K, W, up, local_rank, world, min_reps: int = 5, target_s: float = 1.0):
    """Same metric through the public API with host buffers, as a user runs an initial-value
    problem: the initial vorticity (pinned host memory) -> device, K steps with the per-step FP64
    energy/enstrophy returned to the host, the final vorticity -> pinned host memory.  Each
    repetition restarts from the same field; the median repetition is reported."""
    import numpy as np
    import torch

    H = N // 2
    pin_om = torch.empty((N, H, 2), dtype=torch.float32, pin_memory=True).numpy()
    pin_om[...] = P.k4_spectrum(N, WORKLOAD["K0"], WORKLOAD["seed"]).view(np.float32).reshape(N, H, 2)
    om_in = pin_om.view(np.complex64).reshape(N, H)
    out_om = torch.empty((N, H, 2), dtype=torch.float32, pin_memory=True).numpy().view(np.complex64).reshape(N, H)
    s = P.Solver(N, WORKLOAD["Re"], WORKLOAD["K0"], WORKLOAD["CFL"], device=local_rank)

    def one():
        s.init_vorticity(om_in)  # FNM1 starts at zero on the device, as in a fresh run
        s.next_dt()
        advance(s, K, up, K, {"kernels": 0}, history=True)
        s.om2(out=out_om)  # result into pinned host memory

    one()  # builds the graphs of this state's segment lengths
    for n in set(segments(0, K, up)):
        s.prepare(n)
    s.sync()
    reps = []
    while len(reps) < min_reps or (sum(reps) < target_s and len(reps) < 100):
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        one()
        reps.append(time.perf_counter() - t0)
    sec = max_over_ranks(statistics.median(reps), world, device=f"cuda:{local_rank}")
    s.close()
    state_bytes = N * H * 8
    return {"value": world * K / sec, "unit": "steps/s",
            "h2d_bytes_per_step": state_bytes / K,
            "d2h_bytes_per_step": (state_bytes + 16 * K) / K,
            "repetitions": len(reps),
            "what": "pinned host initial vorticity -> device, K steps with per-step E/Z to host, final vorticity -> "
                    "pinned host (wall clock, median repetition)"}


def cpu_baseline(args):
    from oracle import oracle as O
    N = args.n
    o = O.Oracle(N, WORKLOAD["Re"], WORKLOAD["K0"], WORKLOAD["CFL"])
    o.init_om2(O.k4_spectrum(N, WORKLOAD["K0"], WORKLOAD["seed"]))
    k = max(1, args.cpu_steps)
    t0 = time.perf_counter()
    o.run(k, 1000000, 1000000, want_diag=False)
    sec = time.perf_counter() - t0
    o.close()
    return {"value": k / sec, "unit": "steps/s", "cores": O.threads(), "kind": "port",
            "sample": f"{k} time steps of the FP64 oracle (oracle/dns2d_oracle.c, OpenMP) at N={N}, "
                      f"{sec:.1f} s"}


def ncu_traffic():
    p = os.path.join(REPO, "profiles", "ncu_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def main_ours(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device(f"cuda:{local_rank}"))
    r = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    N = r["N"]
    peak, peak_kind = measured_peaks()
    bytes_rows = 24 * N * N   # read U,W (12 N^2), write D,E (12 N^2)
    bytes_cols = 40 * N * N   # read D,E + om2,fnm1 (20 N^2), write U,W + om2,fnm1 (20 N^2)
    if r["rows_ms"] >= r["cols_ms"]:
        name, b, ms = "k_rows_step", bytes_rows, r["rows_ms"]
    else:
        name, b, ms = "k_cols_step", bytes_cols, r["cols_ms"]
    achieved = b / (ms / 1e3) / 1e9
    tr = ncu_traffic().get(f"{name}<{N}>")
    steps_s = r["value"] / max(1, int(os.environ.get("WORLD_SIZE", "1")))
    line = {
        "metric": METRIC,
        "value": round(r["value"], 3),
        "unit": "steps/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": r["K"],
        "warmup": r["W"],
        "ms_per_step": round(r["ms"] / r["K"], 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload_text(N) + ", k^4 exp(-2(k/K0)^2) IC",
                   "N": N, "padded_grid": 3 * N // 2, "parallelism": "replicas",
                   "l2": f"inputs larger than L2 (work 12N^2 + state 8N^2 bytes = {20 * N * N / 1e6:.0f} MB)",
                   "autotuned": r["tuning"],
                   "timing": "value = K / median device time of consecutive K-step windows (CUDA events on "
                             "the solver's stream), each window ending on a diagnostic step"},
        "mpts_steps_per_s": round(r["value"] * N * N / 1e6, 1),
        "step_roofline": {"bytes_per_step_model": 76 * N * N, "bytes_per_step_min": 64 * N * N,
                          "frac_model": round(76 * N * N * steps_s / (peak * 1e9), 4),
                          "frac_min": round(64 * N * N * steps_s / (peak * 1e9), 4)},
        "roofline": {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": tr, "bytes_per_launch": b, "launch_ms": round(ms, 4)},
        "kernel_ms": {"k_rows_step": round(r["rows_ms"], 4), "k_cols_step": round(r["cols_ms"], 4)},
        "windows": r["windows"],
        "gpu_launches": r["kernels"],
        "gpu_launches_note": "kernels of this library launched in all timed windows together",
        "clocks": r["clocks"],
    }
    if r["e2e"]:
        line["e2e"] = r["e2e"]
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    elif args.workload in ("dns16384", "dns29400"):
        line["cpu_baseline"] = None
        line["cpu_baseline_note"] = f"FP64 oracle needs tens of GB of host memory at N={args.n}; see the N=4096 line"
    print(json.dumps(line), flush=True)


def reference_cadence(W: int, K: int, update: int):
    """(BENCH_WARMUP_STEPS, STEPS) for the reference's mem_cuda so that its "Steady FPS" covers
    exactly the K steps after a warm-up.  Its steady timer starts only inside a diagnostic step
    (it == 1, a multiple of UPDATE, or it == STEPS) once it >= BENCH_WARMUP_STEPS
    (cuda/mem_cuda.cu:1859,1912-1920), so the warm-up is rounded down to the last diagnostic step
    at or before W: the largest multiple of UPDATE <= W, else step 1."""
    warm = (W // update) * update if W >= update else 1
    return warm, warm + K


_STEADY = re.compile(r"Steady frames per second \(FPS\)\s*=\s*([0-9.eE+-]+)\s*\((\d+) steps after warmup\)")


def parse_reference_stdout(text: str):
    """(steady steps/s, steps in the steady window) from the reference's end-of-run lines
    (cuda/mem_cuda.cu:2024-2036), or None when it printed no steady window."""
    m = _STEADY.search(text)
    if not m:
        return None
    return float(m.group(1)), int(m.group(2))


def run_reference_binary(exe: str, argv: list, warm: int, cwd: str, timeout: int = 1800):
    """One run of the reference CLI; returns (steps/s, steady steps, wall seconds) or raises
    RuntimeError with the reason and the end of its output."""
    env = dict(os.environ, BENCH_WARMUP_STEPS=str(warm))
    t0 = time.perf_counter()
    p = subprocess.run([exe, *map(str, argv)], env=env, cwd=cwd, capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    r = parse_reference_stdout(p.stdout)
    if p.returncode != 0 or r is None:
        why = f"exit code {p.returncode}" if p.returncode != 0 else "no 'Steady frames per second' line"
        tail = (p.stdout[-300:] + " | " + p.stderr[-200:]).replace("\n", " / ")
        raise RuntimeError(f"reference mem_cuda {' '.join(map(str, argv))}: {why}; output tail: {tail}")
    return r[0], r[1], wall


def reference_initial_field(N: int, path: str) -> str:
    """The seeded k^4 exp(-2(k/K0)^2) field of our arm, set up by the FP64 oracle (velocity
    recovery, C2R, NEXTDT init) and written as restart.bin v2 for the reference's loader."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    o = O.Oracle(N, WORKLOAD["Re"], WORKLOAD["K0"], WORKLOAD["CFL"])
    o.init_om2(O.k4_spectrum(N, WORKLOAD["K0"], WORKLOAD["seed"]))
    O.write_restart_v2(path, o, WORKLOAD["Re"], WORKLOAD["K0"], WORKLOAD["CFL"])
    o.close()
    return f"seeded k^4 exp(-2(k/K0)^2) field (seed {WORKLOAD['seed']}) via restart.bin v2 written by the FP64 oracle " \
           f"({time.perf_counter() - t0:.1f} s, outside the timed runs)"


def main_reference(args, runs: int = 3):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import tempfile
    N, K, W = args.n, args.steps, args.warmup
    up = WORKLOAD["UPDATE"]
    exe = os.path.join(REPO, "oracle", "_ref", "mem_cuda")
    base = {"impl": "reference", "metric": METRIC, "unit": "steps/s", "n_gpus": 1, "steps": K,
            "warmup": W, "higher_is_better": True, "scaling": "weak", "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_text(N), "N": N}}
    if not os.path.exists(exe):
        cb = cpu_baseline(args)
        line = dict(base, value=cb["value"], ms_per_step=1e3 / cb["value"], vs_baseline=None, cpu_baseline=cb,
                    e2e={"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        line["config"]["reference_note"] = "reference binary not built (oracle/_ref/mem_cuda); FP64 oracle timed instead"
        print(json.dumps(line), flush=True)
        return
    warm, steps_total = reference_cadence(W, K, up)
    with tempfile.TemporaryDirectory(prefix="dns2d_refarm_") as tmp:
        argv = [N, f"{WORKLOAD['Re']:.0E}", f"{WORKLOAD['K0']:g}", steps_total, f"{WORKLOAD['CFL']:g}", up, 0]
        try:
            if args.workload == "dns4096":
                ic = reference_initial_field(N, os.path.join(tmp, "restart.bin"))
                argv.append(os.path.join(tmp, "restart.bin"))
            else:
                ic = "PAO-k^-3 (the reference CLI's own initialiser; the FP64 oracle cannot hold this size)"
            res = [run_reference_binary(exe, argv, warm, tmp) for _ in range(runs)]
        except (RuntimeError, OSError, subprocess.TimeoutExpired, MemoryError) as e:
            print(json.dumps({"impl": "reference", "unavailable": str(e)[:600]}), flush=True)
            return
    vals = sorted(r[0] for r in res)
    v = statistics.median(vals)
    steady = res[0][1]
    line = dict(base, value=round(v, 3), ms_per_step=round(1e3 / v, 5), vs_baseline=None,
                mpts_steps_per_s=round(v * N * N / 1e6, 1),
                runs=[round(x, 3) for x in vals],
                cpu_baseline={"value": round(v, 3), "unit": "steps/s", "cores": 1, "kind": "reference",
                              "sample": f"reference cuFFT build (oracle/_ref/mem_cuda, sm_100a, unmodified source) "
                                        f"{' '.join(map(str, argv[:7]))} [restart.bin], BENCH_WARMUP_STEPS={warm}; "
                                        f"median of {runs} runs of its own 'Steady FPS' over {steady} steps on cuda:0 "
                                        f"(one host thread driving the GPU; {sum(r[2] for r in res):.1f} s wall)",
                              "device": "cuda:0"},
                e2e={"value": round(v, 3), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    line["config"]["reference_ic"] = ic
    line["config"]["steady_window"] = f"steps {warm + 1}..{steps_total} ({steady} steps), diagnostics every {up} " \
                                      f"steps and at the last step, as in our arm's window"
    print(json.dumps(line), flush=True)


def time_ensemble(ms, K, W, up, mode, tune, clocks=None):
    """Device time (ms) of K ensemble steps after W warm-up steps, NEXTDT every UPDATE steps:
    mode 0 = one graph per chunk (a branch per size group), 1 = one persistent launch per chunk."""
    import torch
    import optimizec_b200 as P
    b = P.Batch(ms)
    if tune:
        b.autotune()  # each size group's kernel variants at its own member count
    b.set_mode(mode)
    b.init_k4()
    b.next_dt()
    it = 0

    def advance(to):
        nonlocal it
        while it < to:
            nxt = 1 if it < 1 else min(to, (it // up + 1) * up)
            b.step(nxt - it)
            it = nxt
            if it == 1 or it % up == 0:
                b.next_dt()
    advance(W)
    if mode == 0:
        for n in set(segments(W, W + K, up)):  # graph capture stays out of the timed region
            b.prepare(n)
    b.sync()
    stream = torch.cuda.ExternalStream(b.stream(), device=0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if clocks:
        clocks.start()
        time.sleep(0.3)
    e0.record(stream)
    advance(W + K)
    e1.record(stream)
    b.sync()
    torch.cuda.synchronize()
    ck = clocks.stop() if clocks else None
    b.close()
    return e0.elapsed_time(e1), ck


def main_ensemble(args):
    """64 independent decaying runs (32 x N=128, 24 x N=256, 8 x N=512; Re log-uniform in
    [1e3, 1e5], K0 in [2, 8], seeds 0..63, CFL 0.1) advanced together; NEXTDT every UPDATE steps.
    The line's value is the default stepping mode (one graph per chunk, autotuned); the persistent
    launch (every member in one cooperative kernel per chunk) is timed beside it."""
    import optimizec_b200 as P
    ms = P.ensemble_members()
    K, W, up = args.steps, args.warmup, WORKLOAD["UPDATE"]
    ms_, ck = time_ensemble(ms, K, W, up, 0, True, ClockSampler(0))
    ms_p, _ = time_ensemble(ms, K, W, up, 1, False)
    member_steps = len(ms) * K / (ms_ / 1e3)
    pts = sum(m[0] ** 2 for m in ms)
    peak, peak_kind = measured_peaks()
    byts = sum(64 * m[0] ** 2 for m in ms)
    line = {"metric": "member-steps/s (64-member batched 2D DNS ensemble)", "value": round(member_steps, 1),
            "unit": "member-steps/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": round(ms_ / K, 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ensemble 32xN=128 + 24xN=256 + 8xN=512, Re log-uniform [1e3,1e5], "
                                   "K0 in [2,8], seeds 0..63, CFL 0.1, UPDATE 100, one graph per chunk",
                       "autotuned": "per size group at its member count (dns2d_batch_autotune)"},
            "ensemble_steps_per_s": round(K / (ms_ / 1e3), 2),
            "mpts_steps_per_s": round(pts * K / (ms_ / 1e3) / 1e6, 1),
            "hbm_frac_64N2": round(byts * K / (ms_ / 1e3) / (peak * 1e9), 4), "clocks": ck,
            "persistent_launch": {"ms_per_step": round(ms_p / K, 5),
                                  "member_steps_s": round(len(ms) * K / (ms_p / 1e3), 1),
                                  "what": "dns2d_batch_set_mode(1): every member in one cooperative kernel per "
                                          "chunk, default radix plans, 8 row tiles / 4 column groups per item"}}
    print(json.dumps(line), flush=True)


def network_trace_summary(tr, layers, T, S, G):
    """Medians of a persistent network launch's per-tile trace ([tiles, 10] ns; tiles in layer
    order, T tile rows x S strips per layer, CTA c took tiles c, c + G, ...)."""
    import numpy as np
    names = ["taken", "inputs", "stage", "copy", "landed", "issued", "epilogue", "tmem", "stores", "released"]
    tr = tr.astype(np.int64)
    tr = tr - tr.min()
    per = T * S
    out = {"tiles": int(len(tr)), "ctas": int(G), "span_us": round(float(tr[:, 9].max() - tr[:, 0].min()) / 1e3, 2),
           "layers": []}
    for j in range(layers - 1):
        a = tr[j * per:(j + 1) * per]
        d = np.median(np.diff(a, axis=1), axis=0) / 1e3
        out["layers"].append({"layer": j + 1, "first_taken_us": round(float(a[:, 0].min()) / 1e3, 2),
                              "last_released_us": round(float(a[:, 9].max()) / 1e3, 2),
                              "median_us": {f"{names[i]}->{names[i + 1]}": round(float(d[i]), 3) for i in range(9)}})
    gaps = [np.diff(tr[np.arange(c, len(tr), G), 0]) for c in range(G)]
    out["tile_interval_per_cta_us"] = round(float(np.median(np.concatenate(gaps))) / 1e3, 3)
    return out


def main_profile(args):
    """The short runs the ncu summaries under profiles/ were captured from."""
    import numpy as np
    import optimizec_b200 as P
    if args.profile == "training-tc":
        rng = np.random.default_rng(2)
        x = rng.standard_normal((4, 3, 384, 384)).astype(np.float32)
        t = rng.standard_normal((4, 1, 384, 384)).astype(np.float32)
        net = P.CNN(6, 32, seed=1)
        net.set_train_tc(True)
        net.set_dataset(x, t)
        net.train(3, 4, 1e-3, seed=1)
        print("profile run done", flush=True)
        net.close()
        return
    if args.profile == "training":
        import time
        rng = np.random.default_rng(2)
        out = {}
        for (n, hw, batch) in ((8, 384, 4), (64, 48, 32)):
            x = rng.standard_normal((n, 3, hw, hw)).astype(np.float32)
            t = rng.standard_normal((n, 1, hw, hw)).astype(np.float32)
            for tc in (False, True):
                net = P.CNN(6, 32, seed=1)
                net.set_train_tc(tc)
                net.set_dataset(x, t)
                net.train(3, batch, 1e-3, seed=1)  # warm-up: buffers, weights
                iters = 20 if tc else 5
                t0 = time.perf_counter()
                losses = net.train(iters, batch, 1e-3, seed=2)
                ms = (time.perf_counter() - t0) / iters * 1e3
                out[f"{hw}x{hw}_batch{batch}_{'tensor' if tc else 'fp32'}_ms_per_iter"] = round(ms, 3)
                out[f"{hw}x{hw}_batch{batch}_{'tensor' if tc else 'fp32'}_last_loss"] = round(float(losses[-1]), 5)
                net.close()
        print(json.dumps(out), flush=True)
        return
    if args.profile == "network":
        net = P.CNN(6, 32, seed=1)
        x = np.random.default_rng(1).standard_normal((1, 3, 384, 384)).astype(np.float32)
        net.set_trace(True)
        for _ in range(5):
            net.forward_tc(x)
        print(json.dumps(network_trace_summary(net.read_trace(), 6, 192, 3, net.tc_info()[1])), flush=True)
        net.close()
        return
    if args.profile == "closure":
        s = P.Solver(256, 1e5, 4.0, 0.1)
        s.init_k4(1)
        s.next_dt()
        net = P.CNN(6, 32, seed=1)
        s.attach_closure(net, np.array([5.0, 1.0, 1.0, 0.01], np.float32), energy_check=1)
        s.step(3)
        s.sync()
        print("profile run done", s.closure_stats())
        return
    s = P.Solver(args.n, 1e5, 4.0, 0.1)
    s.init_k4(1)
    s.next_dt()
    s.step(1)
    s.next_dt()
    s.step(3)
    s.sync()
    print("profile run done, it =", s.scalars()["it"])


if __name__ == "__main__":
    a = parse()
    if a.profile:
        main_profile(a)
    elif a.workload == "ensemble" and a.impl == "ours":
        main_ensemble(a)
    elif a.workload == "ensemble":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched ensemble: each "
                              "member would be its own mem_cuda process"}), flush=True)
    elif a.impl == "reference":
        main_reference(a)
    else:
        main_ours(a)
