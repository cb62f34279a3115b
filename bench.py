"""Benchmark: shots/s of the Schrodinger-VM executor on the B200.

Workload (one "step"): `sample_survivors` of the noisy 7x7 memory-grid
program (n = 49, 10 rounds, DEPOLARIZE1/2 + X_ERROR at p = 1e-3, 12 magic
gates, post-selection on all 240 detectors) for 10^6 shots per GPU, bytecode
after the reference's own bytecode passes (tests/golden/programs/cfg1.npz,
written by tests/golden/make_golden.py). Synthetic seeded data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl clifft_b200|reference]

Reported `value` = survivor-sampled shots per second, whole job (sum over
ranks, max-over-ranks device time), statevector in complex FP32 with FP64
probability sums. `e2e` = the same metric through the public Python API
(`clifft_b200.sample_survivors` on a freshly uploaded program, records read
back to host numpy). `extras` carry the plain-FP64 executor on the same
workload and the k = 10 / 16 / 24 programs side by side.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PROGRAMS = os.path.join(ROOT, "tests", "golden", "programs")
SHOTS_PER_GPU = 1_000_000
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_program(name):
    from clifft_b200.program import Program
    return Program.load(os.path.join(PROGRAMS, f"{name}.npz"))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
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
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ GPU helpers
def device_run(prog, dp, shots, seed, first_shot, precision, stream, bufs):
    """One device-resident sampling step: program resident, outputs in HBM."""
    import ctypes
    from clifft_b200 import _native as N
    a = N.SampleArgs(shots=shots, seed=seed, first_shot=first_shot,
                     precision=N.CLIFFT_GPU_FP32 if precision == "fp32" else N.CLIFFT_GPU_FP64,
                     flags=N.CLIFFT_GPU_SURVIVORS | N.CLIFFT_GPU_DEVICE_PTRS,
                     stream=stream.cuda_stream)
    o = N.Outputs()
    for field, t in bufs.items():
        setattr(o, field, t.data_ptr() if t.numel() else None)
    N.check(N.lib().clifft_gpu_sample(dp.handle, ctypes.byref(a), ctypes.byref(o)), "clifft_gpu_sample")
    return o


def output_buffers(torch, prog, shots, dev):
    mw = (prog.num_measurements + 63) // 64
    dw = (prog.num_detectors + 63) // 64
    ow = (prog.num_observables + 63) // 64
    return {
        "meas": torch.empty((shots, mw), dtype=torch.int64, device=dev),
        "det": torch.empty((shots, dw), dtype=torch.int64, device=dev),
        "obs": torch.empty((shots, ow), dtype=torch.int64, device=dev),
        "survived": torch.empty(shots, dtype=torch.uint8, device=dev),
    }


def time_device(torch, prog, shots, precision, steps, warmup, rank, flush):
    import clifft_b200 as cb
    dev = torch.device("cuda", torch.cuda.current_device())
    dp = cb.load(prog)
    stream = torch.cuda.current_stream()
    bufs = output_buffers(torch, prog, shots, dev)
    first = rank * shots
    for w in range(warmup):
        device_run(prog, dp, shots, 1000 + w, first, precision, stream, bufs)
    torch.cuda.synchronize()
    times, kernel_ms, launches, passed, alg_bytes, groups = [], [], 0, 0, 0, set()
    for s in range(steps):
        flush.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        o = device_run(prog, dp, shots, 7 + s, first, precision, stream, bufs)
        ev1.record(stream)
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
        kernel_ms.append(o.kernel_ms)
        launches += o.kernel_launches
        passed += o.passed_shots
        alg_bytes += o.algorithmic_bytes
        groups.add(o.group_threads)
    return {"ms": times, "kernel_ms": kernel_ms, "launches": launches, "passed": passed,
            "alg_bytes": alg_bytes, "group_threads": sorted(groups)}


def time_e2e(prog_path, shots, steps, rank, torch):
    """Public-API path with host buffers: fresh upload of the program image
    (H2D), sampling, packed records read back (D2H) and unpacked to numpy."""
    import numpy as np
    import clifft_b200 as cb
    from clifft_b200.program import Program
    times, h2d, d2h = [], 0, 0
    for s in range(steps + 1):
        prog = Program.load(prog_path)  # host-side program, not yet on the device
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = cb.sample_survivors(prog, shots, seed=50 + s, keep_records=True, precision="fp32")
        dt = time.perf_counter() - t0
        if s == 0:
            continue  # first call pays one-time CUDA context / kernel attribute setup
        times.append(dt)
        h2d = cb.load(prog).device_bytes
        words = ((prog.num_measurements + 63) // 64 + (prog.num_detectors + 63) // 64 +
                 (prog.num_observables + 63) // 64)
        d2h = shots * (words * 8 + 1) + 8 * (6 + prog.num_observables)
        prog._device_program.free()
    return times, h2d, d2h


def cpu_baseline(shots_hint=200_000, target_s=12.0):
    """The reference executor (oracle/_ref) on this host's cores, shot-parallel,
    on a bounded sample of the workload; falls back to the C oracle port."""
    from oracle import pyoracle as O
    prog = load_program("cfg1")
    cores = len(os.sched_getaffinity(0))
    if O.ref_available():
        probe = 20_000
        t = O.ref_time_sample(prog, probe, 3, cores, True)
        n = int(min(5_000_000, max(probe, probe * target_s / max(t, 1e-3))))
        t = O.ref_time_sample(prog, n, 4, cores, True)
        return {"value": n / t, "unit": "shots/s", "cores": cores, "kind": "reference",
                "sample": f"{n} shots of the cfg1 program, {cores} threads x clifft::sample_survivors "
                          f"(oracle/_ref, dispatch {O.ref_backend()})"}
    n = 20_000
    t0 = time.perf_counter()
    O.run(prog, n, seed=3, rng=O.RNG_XOSHIRO)
    t = time.perf_counter() - t0
    return {"value": n / t, "unit": "shots/s", "cores": 1, "kind": "port",
            "sample": f"{n} shots of the cfg1 program through the C oracle, 1 thread"}


def k_sweep(torch, flush):
    """FP32 vs FP64 shots/s on the k = 10 / 16 / 24 programs (configs 2 and 3)."""
    import numpy as np
    from clifft_b200.program import Program
    out = {}
    peaks = {}
    for name in sorted(os.listdir(PROGRAMS)):
        if name.startswith("cfg2_"):
            p = Program.load(os.path.join(PROGRAMS, name))
            peaks.setdefault(p.peak_rank, name[:-4])
    picks = [(10, peaks.get(10), 10_000), (16, peaks.get(16), 10_000), (24, "cfg3", 256)]
    for k, name, shots in picks:
        if name is None:
            continue
        prog = load_program(name)
        row = {"program": name, "shots": shots}
        for prec in ("fp32", "fp64"):
            r = time_device(torch, prog, shots, prec, steps=2, warmup=1, rank=0, flush=flush)
            ms = min(r["ms"])
            kms = min(r["kernel_ms"])
            row[f"{prec}_shots_per_s"] = shots / (ms / 1e3)
            row[f"{prec}_kernel_GBps"] = (r["alg_bytes"] / len(r["ms"])) / (kms / 1e3) / 1e9
        row["fp32_over_fp64"] = row["fp32_shots_per_s"] / row["fp64_shots_per_s"]
        out[f"k{k}"] = row
    return out


# --------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="clifft_b200", choices=["clifft_b200", "reference"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--profile", metavar="PROGRAM", default=None,
                    help="only run --warmup + --steps device steps of tests/golden/programs/PROGRAM "
                         "(for ncu captures); prints one summary line")
    ap.add_argument("--shots", type=int, default=SHOTS_PER_GPU)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    args = ap.parse_args()
    if args.profile:
        import torch
        torch.cuda.set_device(0)
        prog = load_program(args.profile)
        flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
        r = time_device(torch, prog, args.shots, args.precision, args.steps, args.warmup, 0, flush)
        print(json.dumps({"program": args.profile, "shots": args.shots, "precision": args.precision,
                          "ms": r["ms"], "kernel_ms": r["kernel_ms"], "alg_bytes": r["alg_bytes"],
                          "launches": r["launches"], "group_threads": r["group_threads"]}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": "cfg1: 7x7 noisy memory grid, n=49, 10 rounds, p=1e-3, 12 magic, "
                          "post-select all 240 detectors; sample_survivors",
              "shots_per_gpu_per_step": SHOTS_PER_GPU, "global_batch_shots": SHOTS_PER_GPU * world,
              "peak_k": None, "parallelism": f"shot-sharded x{world}",
              "l2": "256 MiB buffer zeroed between timed steps (inputs are on-chip sized)"}

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import pyoracle as O
        prog = load_program("cfg1")
        config["peak_k"] = prog.peak_rank
        cores = len(os.sched_getaffinity(0))
        if not O.ref_available():
            print(json.dumps({"impl": "reference", "unavailable":
                              "reference harness oracle/_ref not built on this machine"}))
            return
        per_step = 200_000
        for w in range(args.warmup):
            O.ref_time_sample(prog, 20_000, 900 + w, cores, True)
        ts = [O.ref_time_sample(prog, per_step, 10 + s, cores, True) for s in range(args.steps)]
        ms = 1e3 * sum(ts) / len(ts)
        val = per_step / (ms / 1e3)
        line = {"metric": "survivor-sampled shots/s (cfg1 memory grid, FP64 reference executor)",
                "value": val, "unit": "shots/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config, "impl": "reference",
                "cpu_baseline": {"value": val, "unit": "shots/s", "cores": cores, "kind": "reference",
                                 "sample": f"{per_step} shots per step, {cores} threads x "
                                           f"clifft::sample_survivors (oracle/_ref)"},
                "e2e": {"value": val, "unit": "shots/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    import clifft_b200 as cb
    if not cb.backend_name().startswith("cuda:sm_100a"):
        raise SystemExit(f"no sm_100 device: {cb.backend_name()}")
    prog = load_program("cfg1")
    config["peak_k"] = prog.peak_rank
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        barrier()
        r = time_device(torch, prog, SHOTS_PER_GPU, "fp32", args.steps, args.warmup, rank, flush)
        barrier()
    total_ms = sum(r["ms"])
    step_ms = total_ms / args.steps
    passed = r["passed"]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([step_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms = float(t.item())
        pt = torch.tensor([passed], device="cuda", dtype=torch.float64)
        dist.all_reduce(pt, op=dist.ReduceOp.SUM)
        passed = int(pt.item())
    value = SHOTS_PER_GPU * world / (step_ms / 1e3)

    # roofline of the sampling kernel (device time from events inside the call)
    peak, peak_kind = measured_peaks()
    kms = sum(r["kernel_ms"]) / len(r["kernel_ms"])
    bytes_per_launch = r["alg_bytes"] / args.steps
    achieved = bytes_per_launch / (kms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                traffic = json.load(f).get("cfg1_fp32_dram_bytes_per_launch")
        except Exception:
            traffic = None

    extras = {}
    e2e = None
    cpu = None
    if rank == 0:
        e_times, h2d, d2h = time_e2e(os.path.join(PROGRAMS, "cfg1.npz"), SHOTS_PER_GPU,
                                     max(2, min(args.steps, 3)), rank, torch)
        e2e = {"value": SHOTS_PER_GPU / (sum(e_times) / len(e_times)), "unit": "shots/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": 1e3 * sum(e_times) / len(e_times)}
        if not args.no_extras:
            r64 = time_device(torch, prog, SHOTS_PER_GPU, "fp64", 2, 1, 0, flush)
            extras["fp64_plain_executor_shots_per_s"] = SHOTS_PER_GPU / (min(r64["ms"]) / 1e3)
            extras["fp32_over_fp64"] = value / world / extras["fp64_plain_executor_shots_per_s"]
            extras["k_sweep"] = k_sweep(torch, flush)
        world_cpu = world == 1
        if world_cpu:
            cpu = cpu_baseline()
    line = {
        "metric": "survivor-sampled shots/s (cfg1 memory grid, batched FP32 statevector, FP64 sums)",
        "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 state / f64 reductions",
        "data": "synthetic (seeded generator, reference bytecode passes)",
        "config": config,
        "survivors_per_step": passed / args.steps,
        "gpu_launches": r["launches"],
        "group_threads": r["group_threads"],
        "clocks": clocks.summary(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "note": f"algorithmic statevector bytes / kernel time; peak {peak_kind}; "
                             "statevectors are shared-memory resident at this k, so frac > 1 "
                             "means on-chip, not HBM"},
        "e2e": e2e,
        "cpu_baseline": cpu,
        "extras": extras,
    }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
