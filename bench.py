"""Benchmark: shots/s of the Schrodinger-VM executor on the B200.

Headline workload (one "step"): `sample` of the k = 24 program (random
near-Clifford circuit, n = 64, 400 layers, 24 T gates, peak rank 24; bytecode
after the reference's own bytecode passes, tests/golden/programs/cfg3.npz
written by tests/golden/make_golden.py) for 296 shots per GPU, i.e. one
resident wave of two 256-thread CTAs per SM, each holding a 128 MiB
complex-FP32 statevector.
Synthetic seeded data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl clifft_b200|reference]

`value` = shots per second of the batched FP32 executor (statevector in
complex FP32, probability sums and renormalisation in FP64, fused tile sweeps,
autotuned launch shape), whole job (sum over ranks, max-over-ranks device
time). `e2e` = the same metric through the public Python API
(`clifft_b200.sample` on a freshly uploaded program, records read back and
unpacked on the host). `extras` put the plain FP64 executor (one pass per
opcode, fixed launch heuristic) beside it on the same workload, the k = 10 and
k = 16 programs, the noisy memory-grid survivor workload, the k = 24 program at
10^3 shots with 128 resident, and (a check, not a timing) the largest FP32 and
FP64 errors against the reference executor of every measurement probability
and of the amplitudes at peak rank.

`--impl reference` times the reference's own executor (oracle/_ref, built
from the reference sources) on this host's cores on the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PROGRAMS = os.path.join(ROOT, "tests", "golden", "programs")
HEADLINE = "cfg3"
SHOTS_PER_GPU = 296  # one wave of two resident CTAs on each of the 148 SMs
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
METRIC = "shots/sec at k=10/16/24, FP32-batched vs FP64 GPU (1e-5 prob tol); HBM GB/s vs peak"
WORKLOAD = ("cfg3: random near-Clifford n=64, 400 layers, 24 T, peak k=24 (2^24 amplitudes/shot); "
            "clifft.sample, 296 shots per GPU per step")


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
def device_run(dp, shots, seed, first_shot, precision, stream, bufs, survivors=False, plain=False, group=0,
               max_resident=0, extra_flags=0):
    """One device-resident sampling step: program resident, outputs in HBM.
    plain = the plain executor: one pass per opcode, fixed heuristic launch
    shape, one launch per call (no fusion, no autotuning, no survivor
    compaction). extra_flags: further CLIFFT_GPU_* flags (e.g. TENSOR_DENSE)."""
    import ctypes
    from clifft_b200 import _native as N
    flags = N.CLIFFT_GPU_DEVICE_PTRS | extra_flags
    if survivors:
        flags |= N.CLIFFT_GPU_SURVIVORS
    if plain:
        flags |= N.CLIFFT_GPU_NO_FUSION | N.CLIFFT_GPU_NO_AUTOTUNE | N.CLIFFT_GPU_NO_SEGMENTS
    a = N.SampleArgs(shots=shots, seed=seed, first_shot=first_shot,
                     precision=N.CLIFFT_GPU_FP32 if precision == "fp32" else N.CLIFFT_GPU_FP64,
                     flags=flags, group_threads=group, stream=stream.cuda_stream, max_resident=max_resident)
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
        "exp_vals": torch.empty((shots, prog.num_exp_vals), dtype=torch.float64, device=dev),
        "survived": torch.empty(shots, dtype=torch.uint8, device=dev),
    }


def time_device(torch, prog, shots, precision, steps, warmup, rank, flush, survivors=False, plain=False,
                group=0, max_resident=0, extra_flags=0):
    import clifft_b200 as cb
    dev = torch.device("cuda", torch.cuda.current_device())
    dp = cb.load(prog)
    stream = torch.cuda.current_stream()
    bufs = output_buffers(torch, prog, shots, dev)
    first = rank * shots
    for w in range(warmup):
        device_run(dp, shots, 1000 + w, first, precision, stream, bufs, survivors, plain, group, max_resident,
                   extra_flags)
    torch.cuda.synchronize()
    times, kernel_ms, launches, passed, alg_bytes, streamed, groups = [], [], 0, 0, 0, 0, set()
    for s in range(steps):
        flush.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        o = device_run(dp, shots, 7 + s, first, precision, stream, bufs, survivors, plain, group, max_resident,
                       extra_flags)
        ev1.record(stream)
        ev1.synchronize()
        times.append(ev0.elapsed_time(ev1))
        kernel_ms.append(o.kernel_ms)
        launches += o.kernel_launches
        passed += o.passed_shots
        alg_bytes += o.algorithmic_bytes
        streamed += o.streamed_bytes
        groups.add(o.group_threads)
    return {"ms": times, "kernel_ms": kernel_ms, "launches": launches, "passed": passed,
            "alg_bytes": alg_bytes, "streamed_bytes": streamed, "group_threads": sorted(groups)}


def time_e2e(name, shots, steps, torch, first_shot=0):
    """Public-API path with host buffers: fresh upload of the program image
    (H2D), sampling, packed records read back (D2H) and unpacked to numpy."""
    import clifft_b200 as cb
    from clifft_b200.program import Program
    path = os.path.join(PROGRAMS, f"{name}.npz")
    times, h2d, d2h = [], 0, 0
    for s in range(steps + 1):
        prog = Program.load(path)  # host-side program, not yet on the device
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cb.sample(prog, shots, seed=50 + s, precision="fp32", first_shot=first_shot)
        dt = time.perf_counter() - t0
        if s == 0:
            continue  # first call pays one-time CUDA context / kernel attribute setup
        times.append(dt)
        h2d = cb.load(prog).device_bytes
        words = ((prog.num_measurements + 63) // 64 + (prog.num_detectors + 63) // 64 +
                 (prog.num_observables + 63) // 64)
        d2h = shots * (words * 8 + 1 + 8 * prog.num_exp_vals) + 8 * (6 + prog.num_observables)
        prog._device_program.free()
    return times, h2d, d2h


def reference_errors(name, shots):
    """Largest error against the reference executor (oracle/_ref, FP64) of
    every measurement probability of `shots` forced trajectories (outcomes of
    an FP64 GPU run), and, for a prefix of the program that ends where k
    first reaches its peak, of the normalised amplitudes (max abs, relative
    L2, 1 - |overlap|), for the FP32 and FP64 statevectors. A check, not a
    timing: the reference replays the same bytecode on the host."""
    import numpy as np
    import clifft_b200 as cb
    from clifft_b200.program import ACTIVE_MEAS, Program
    from oracle import pyoracle as O
    if not O.ref_available():
        return None
    prog = load_program(name)
    f = cb.run(prog, shots, 5, precision="fp64")
    bits = cb.api._unpack(f["meas_words"], prog.num_measurements)
    fm = np.zeros((shots, prog.total_meas_slots), np.uint8)
    fm[:, :prog.num_measurements] = bits
    ref = O.ref_forced(prog, fm)
    out = {"program": name, "shots": shots}
    for prec in ("fp32", "fp64"):
        g = cb.run(prog, shots, 0, precision=prec, forced_meas=fm, trace=True)
        out[f"{prec}_max_abs_prob_err"] = float(np.max(np.abs(np.nan_to_num(g["meas_prob"]) -
                                                            np.nan_to_num(ref["meas_prob"])), initial=0.0))
    hist, ops = prog.active_k_history(), prog.opcodes.tolist()
    first = int(np.argmax(hist == prog.peak_rank))
    cut = next((pc for pc in range(first, len(ops)) if ops[pc] in ACTIVE_MEAS), len(ops))
    d = prog.to_npz_dict()
    d["instructions"] = prog.instructions[:cut].copy()
    pre = Program.from_npz_dict(d)
    n = 2
    f = cb.run(pre, n, 3, precision="fp64")
    fm = np.zeros((n, pre.total_meas_slots), np.uint8)
    fm[:, :pre.num_measurements] = cb.api._unpack(f["meas_words"], pre.num_measurements)
    r = O.ref_forced(pre, fm)
    k = int(r["final_k"][0])
    ra = (r["final_gamma"][:, 0] + 1j * r["final_gamma"][:, 1])[:, None] * r["final_v"][:, :1 << k]
    del r
    for prec in ("fp32", "fp64"):
        g = cb.run(pre, n, 0, precision=prec, forced_meas=fm, trace=True, dump_shots=n)
        ga = (g["final_gamma"][:, 0] + 1j * g["final_gamma"][:, 1])[:, None] * g["final_v"][:, :1 << k]
        del g
        mx = rl2 = ov = 0.0
        for s_ in range(n):
            a_, b_ = ga[s_] / np.linalg.norm(ga[s_]), ra[s_] / np.linalg.norm(ra[s_])
            mx = max(mx, float(np.abs(a_ - b_).max() / np.abs(b_).max()))
            rl2 = max(rl2, float(np.linalg.norm(ga[s_] - ra[s_]) / np.linalg.norm(ra[s_])))
            ov = max(ov, float(1.0 - abs(np.vdot(a_, b_))))
        out[f"{prec}_amplitudes_at_k{k}"] = {"max_abs_err_rel_to_largest": mx, "rel_l2_err": rl2,
                                            "one_minus_overlap": ov}
        del ga
    return out


# ------------------------------------------------------------ CPU reference
def ref_modes(prog, cores, budget_s):
    """The reference executor on this host: shot-parallel (one std::thread per
    core, OpenMP team of 1) and intra-shot (one thread, OpenMP team of all
    cores, the executor's own large-k parallelism). Returns [(mode, shots/s,
    shots, seconds)] with each sample sized to about budget_s seconds."""
    from oracle import pyoracle as O
    out = []
    surv = bool(prog.has_postselection)
    for mode, thr, omp in (("shot-parallel", cores, 1), ("intra-shot OpenMP", 1, cores)):
        n = max(thr, 2)
        t = O.ref_time_sample(prog, n, 3, thr, surv, omp)
        n = int(max(n, min(50_000_000, n * budget_s / max(t, 1e-3))))
        n = max(thr, (n // thr) * thr)
        t = O.ref_time_sample(prog, n, 4, thr, surv, omp)
        out.append((mode, n / t, n, t))
    return out


def cpu_baseline(name):
    from oracle import pyoracle as O
    prog = load_program(name)
    cores = len(os.sched_getaffinity(0))
    if O.ref_available():
        O.ref_select_native()
        modes = ref_modes(prog, cores, 6.0)
        best = max(modes, key=lambda m: m[1])
        t1 = O.ref_time_sample(prog, 2, 5, 1, bool(prog.has_postselection), 1)
        desc = "; ".join(f"{m}: {n} shots in {t:.1f} s = {v:.3g}/s" for m, v, n, t in modes)
        return {"value": best[1], "unit": "shots/s", "cores": cores, "kind": "reference",
                "sample": f"{name} program, reference clifft::sample built from its sources (oracle/_ref, "
                          f"{O.ref_build_kind()} build, dispatch {O.ref_backend()}); best of [{desc}]; "
                          f"1 core: {2 / t1:.3g}/s"}
    n = 2
    t0 = time.perf_counter()
    O.run(prog, n, seed=3, rng=O.RNG_XOSHIRO)
    t = time.perf_counter() - t0
    return {"value": n / t, "unit": "shots/s", "cores": 1, "kind": "port",
            "sample": f"{n} shots of the {name} program through the C oracle, 1 thread"}


def reference_arm(args, config):
    from oracle import pyoracle as O
    prog = load_program(HEADLINE)
    cores = len(os.sched_getaffinity(0))
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference executor (oracle/_ref) not built on this machine"}))
        return
    O.ref_select_native()
    # the faster of the reference's two parallel modes on a short probe
    modes = ref_modes(prog, cores, 2.0)
    mode = max(modes, key=lambda m: m[1])[0]
    thr, omp = (cores, 1) if mode == "shot-parallel" else (1, cores)
    per_step = 4 * cores
    for w in range(args.warmup):
        O.ref_time_sample(prog, thr, 900 + w, thr, False, omp)
    ts = [O.ref_time_sample(prog, per_step, 10 + s, thr, False, omp) for s in range(args.steps)]
    ms = 1e3 * sum(ts) / len(ts)
    val = per_step / (ms / 1e3)
    line = {"metric": METRIC, "value": val, "unit": "shots/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128 state / f64", "data": "synthetic", "config": config,
            "impl": "reference",
            "cpu_baseline": {"value": val, "unit": "shots/s", "cores": cores, "kind": "reference",
                             "sample": f"{per_step} shots per step of the {HEADLINE} program, {mode} "
                                       f"({thr} threads x OpenMP team {omp}), reference clifft::sample "
                                       f"(oracle/_ref, {O.ref_build_kind()} build)"},
            "e2e": {"value": val, "unit": "shots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def k_sweep(torch, flush, head_fp32, head_fp64):
    """Batched FP32 vs plain FP64 shots/s on the k = 10 / 16 programs of the
    multi-program set (seeds 100..163) plus the k = 24 headline numbers."""
    from clifft_b200.program import Program
    peaks = {}
    for name in sorted(os.listdir(PROGRAMS)):
        if name.startswith("cfg2_"):
            p = Program.load(os.path.join(PROGRAMS, name))
            peaks.setdefault(p.peak_rank, name[:-4])
    out = {}
    for k, name, shots in ((10, peaks.get(10), 10_000), (16, peaks.get(16), 10_000)):
        if name is None:
            continue
        prog = load_program(name)
        row = {"program": name, "shots": shots}
        for prec, plain in (("fp32", False), ("fp64", True)):
            r = time_device(torch, prog, shots, prec, steps=3, warmup=2, rank=0, flush=flush, plain=plain)
            kms = min(r["kernel_ms"])
            key = "fp32_batched" if prec == "fp32" else "fp64_plain"
            row[f"{key}_shots_per_s"] = shots / (statistics.median(r["ms"]) / 1e3)
            row[f"{key}_kernel_shots_per_s"] = shots / (kms / 1e3)
            row[f"{key}_alg_GBps"] = (r["alg_bytes"] / len(r["ms"])) / (kms / 1e3) / 1e9
            row[f"{key}_group_threads"] = r["group_threads"]
        row["fp32_over_fp64"] = row["fp32_batched_shots_per_s"] / row["fp64_plain_shots_per_s"]
        row["fp32_over_fp64_kernel"] = row["fp32_batched_kernel_shots_per_s"] / row["fp64_plain_kernel_shots_per_s"]
        out[f"k{k}"] = row
    out["k24"] = {"program": HEADLINE, "shots": SHOTS_PER_GPU, "fp32_batched_shots_per_s": head_fp32,
                  "fp64_plain_shots_per_s": head_fp64, "fp32_over_fp64": head_fp32 / head_fp64}
    return out


def multi_program(torch, flush):
    """The 64 seed programs (peak k 4..18) x 10^4 shots: one launch per
    program vs one CUDA-graph launch of the whole batch (FP32)."""
    from clifft_b200.batch import ProgramBatch
    import clifft_b200 as cb
    names = sorted(n[:-4] for n in os.listdir(PROGRAMS) if n.startswith("cfg2_"))
    progs = [load_program(n) for n in names]
    shots = 10_000
    b = ProgramBatch(progs, shots, precision="fp32")
    b.run()
    graph_ms = min(b.run(list(range(100 + 64 * i, 164 + 64 * i))) for i in range(3))
    b.free()
    stream = torch.cuda.current_stream()
    dev = torch.device("cuda", torch.cuda.current_device())
    dps = [cb.load(p) for p in progs]
    bufs = [output_buffers(torch, p, shots, dev) for p in progs]
    for dp, bf in zip(dps, bufs):
        device_run(dp, shots, 1, 0, "fp32", stream, bf)
    sep = []
    for _ in range(3):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i, (dp, bf) in enumerate(zip(dps, bufs)):
            device_run(dp, shots, 100 + i, 0, "fp32", stream, bf)
        e1.record(stream)
        e1.synchronize()
        sep.append(e0.elapsed_time(e1))
    total = len(progs) * shots
    return {"programs": len(progs), "shots_each": shots, "graph_shots_per_s": total / (graph_ms / 1e3),
            "separate_launches_shots_per_s": total / (min(sep) / 1e3), "graph_over_separate": min(sep) / graph_ms}


def literal_cfg3(torch, flush):
    """The k = 24 program as its configuration states it: 10^3 shots per call
    with at most 128 statevectors resident (16 GiB FP32), next to the default
    residency (one wave: two CTAs on every SM)."""
    prog = load_program(HEADLINE)
    out = {"program": HEADLINE, "shots": 1000}
    for key, cap in (("resident_128", 128), ("resident_one_wave", 0)):
        r = time_device(torch, prog, 1000, "fp32", steps=2, warmup=1, rank=0, flush=flush, max_resident=cap)
        out[f"{key}_shots_per_s"] = 1000 / (min(r["ms"]) / 1e3)
    return out


def dense_blocks(torch, flush):
    """The dense k = 20 program (U2 / U4 / H runs; peak 2^20 amplitudes, FP32)
    with its dense blocks on the tensor cores (3xTF32 MMAs) and on the CUDA
    cores: kernel-time shots/s of each and their ratio. The configured
    programs form no dense block, so the flag does not change them."""
    from clifft_b200 import _native as N
    prog = load_program("dense_k20")
    shots = 592  # four waves of two CTAs on every SM
    out = {"program": "dense_k20", "peak_k": prog.peak_rank, "shots": shots, "group_threads": 288}
    for key, fl in (("tensor_cores", N.CLIFFT_GPU_TENSOR_DENSE), ("cuda_cores", 0)):
        r = time_device(torch, prog, shots, "fp32", steps=3, warmup=3, rank=0, flush=flush, group=288,
                        extra_flags=fl)
        out[f"{key}_shots_per_s"] = shots / (min(r["kernel_ms"]) / 1e3)
        out[f"{key}_kernel_ms"] = min(r["kernel_ms"])
    out["tensor_over_cuda_cores"] = out["tensor_cores_shots_per_s"] / out["cuda_cores_shots_per_s"]
    return out


def gradients():
    """Adjoint d<P_j>/dphi_i on the rotation workload (n = 40, 32 rotations,
    16 probes redrawn on the active axes), 256 phase vectors."""
    import numpy as np
    from clifft_b200 import grad as GR
    from clifft_b200.workloads import active_probes
    base = load_program("cfg4")
    rng = np.random.default_rng(3)
    phases = rng.uniform(0.0, 2 * np.pi, size=(256, GR.num_rot_params(base)))
    out = {"program": "cfg4 (n=40, 120 Clifford layers, 32 RZ), 256 phase vectors"}
    for label, prog in (("config_probes", base), ("active_probes", active_probes(base))):
        for prec in ("fp64", "fp32"):
            GR.expval_grad(prog, phases, precision=prec)
            ts = []
            for _ in range(3):
                t0 = time.perf_counter()
                GR.expval_grad(prog, phases, precision=prec)
                ts.append(time.perf_counter() - t0)
            out[f"{label}_{prec}_vectors_per_s"] = 256 / min(ts)
            out[f"{label}_{prec}_ms_per_call"] = 1e3 * min(ts)
    return out


def k_fault_sampling():
    """sample_k_survivors on the memory grid, k = 2 faults per shot, 10^6 shots (FP32)."""
    import clifft_b200 as cb
    prog = load_program("cfg1")
    cb.run(prog, 100_000, 1, precision="fp32", survivors=True, want_records=False, k_faults=2)
    ts = []
    for s in range(3):
        t0 = time.perf_counter()
        r = cb.run(prog, 1_000_000, 2 + s, precision="fp32", survivors=True, want_records=False, k_faults=2)
        ts.append((time.perf_counter() - t0, r["kernel_ms"]))
    wall, kms = min(ts)
    return {"program": "cfg1", "k": 2, "shots": 1_000_000, "shots_per_s_wall": 1e6 / wall,
            "sampling_kernel_ms": kms}


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
    ap.add_argument("--plain", action="store_true", help="with --profile: the plain executor")
    ap.add_argument("--group", type=int, default=0,
                    help="with --profile: fixed group_threads (no autotuning trial launches)")
    ap.add_argument("--tensor-dense", action="store_true",
                    help="with --profile: dense blocks of fused sweeps on the tensor cores")
    args = ap.parse_args()
    if args.profile:
        import torch
        torch.cuda.set_device(0)
        prog = load_program(args.profile)
        flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
        from clifft_b200 import _native as N
        r = time_device(torch, prog, args.shots, args.precision, args.steps, args.warmup, 0, flush,
                        survivors=bool(prog.has_postselection), plain=args.plain, group=args.group,
                        extra_flags=N.CLIFFT_GPU_TENSOR_DENSE if args.tensor_dense else 0)
        print(json.dumps({"program": args.profile, "shots": args.shots, "precision": args.precision,
                          "plain": args.plain, "tensor_dense": args.tensor_dense,
                          "ms": r["ms"], "kernel_ms": r["kernel_ms"],
                          "alg_bytes": r["alg_bytes"], "streamed_bytes": r["streamed_bytes"],
                          "launches": r["launches"], "group_threads": r["group_threads"]}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": WORKLOAD, "shots_per_gpu_per_step": SHOTS_PER_GPU,
              "global_batch_shots": SHOTS_PER_GPU * world, "peak_k": 24,
              "parallelism": f"shot-sharded x{world}",
              "l2": "statevectors (128 MiB each, 296 resident) far exceed L2; a 256 MiB buffer is also "
                    "zeroed between timed steps"}

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, config)
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
    prog = load_program(HEADLINE)
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
    step_ms = sum(r["ms"]) / args.steps
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([step_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms = float(t.item())
    value = SHOTS_PER_GPU * world / (step_ms / 1e3)

    # roofline of the sampling kernel: algorithmic statevector bytes of one
    # launch / its device time (CUDA events on the launching stream, recorded
    # inside the library)
    peak, peak_kind = measured_peaks()
    kms = sum(r["kernel_ms"]) / len(r["kernel_ms"])
    bytes_per_launch = r["alg_bytes"] / args.steps
    achieved = bytes_per_launch / (kms / 1e3) / 1e9
    streamed_gbps = (r["streamed_bytes"] / args.steps) / (kms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                per_shot = json.load(f).get("cfg3_fp32_dram_bytes_per_shot")
            if per_shot:
                traffic = per_shot * SHOTS_PER_GPU
        except Exception:
            traffic = None

    extras = {}
    cpu = None
    # end to end on every rank (each samples its own shots through the public
    # API); the step time is the slowest rank's
    barrier()
    e_times, h2d, d2h = time_e2e(HEADLINE, SHOTS_PER_GPU, max(2, min(args.steps, 3)), torch,
                                 first_shot=rank * SHOTS_PER_GPU)
    e_ms = 1e3 * sum(e_times) / len(e_times)
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    e2e = {"value": SHOTS_PER_GPU * world / (e_ms / 1e3), "unit": "shots/s",
           "h2d_bytes_per_step": int(h2d) * world, "d2h_bytes_per_step": int(d2h) * world,
           "ms_per_step": e_ms}
    if rank == 0:
        if not args.no_extras and world == 1:  # single-GPU comparisons; an N-GPU run holds all N GPUs
            r64 = time_device(torch, prog, SHOTS_PER_GPU, "fp64", 2, 1, 0, flush, plain=True)
            fp64 = SHOTS_PER_GPU / (min(r64["ms"]) / 1e3)
            extras["fp64_plain_executor_shots_per_s"] = fp64
            extras["fp64_plain_alg_GBps"] = (r64["alg_bytes"] / 2) / (min(r64["kernel_ms"]) / 1e3) / 1e9
            extras["fp32_over_fp64"] = (value / world) / fp64
            extras["fp32_streamed_GBps"] = streamed_gbps
            extras["k_sweep"] = k_sweep(torch, flush, value / world, fp64)
            c1 = load_program("cfg1")
            r1 = time_device(torch, c1, 1_000_000, "fp32", 2, 2, 0, flush, survivors=True)
            r1p = time_device(torch, c1, 1_000_000, "fp64", 2, 1, 0, flush, survivors=True, plain=True)
            extras["memory_grid_survivors"] = {
                "program": "cfg1 (7x7 noisy memory grid, post-selected on all detectors)",
                "shots": 1_000_000, "fp32_batched_shots_per_s": 1e9 / min(r1["ms"]),
                "fp64_plain_shots_per_s": 1e9 / min(r1p["ms"]), "survivors_per_step": r1["passed"] / 2}
            extras["literal_cfg3"] = literal_cfg3(torch, flush)
            extras["dense_blocks"] = dense_blocks(torch, flush)
            extras["multi_program_batch"] = multi_program(torch, flush)
            extras["expval_gradients"] = gradients()
            extras["sample_k"] = k_fault_sampling()
        if world == 1:
            cpu = cpu_baseline(HEADLINE)
            if not args.no_extras:
                extras["error_vs_reference"] = {
                    "k24": reference_errors(HEADLINE, 4), "k16": reference_errors(extras["k_sweep"]["k16"]["program"], 16)}
    line = {
        "metric": METRIC,
        "value": value, "unit": "shots/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64 state / f64 reductions",
        "data": "synthetic (seeded generator, reference bytecode passes)",
        "config": config,
        "gpu_launches": r["launches"],
        "group_threads": r["group_threads"],
        "clocks": clocks.summary(),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "dram_achieved": streamed_gbps, "dram_frac": streamed_gbps / peak,
                     "note": f"achieved = algorithmic statevector bytes per launch (one pass per opcode, the "
                             f"reference's algorithm) / kernel time; fused blocks stream fewer bytes, so it can "
                             f"exceed the copy peak ({peak_kind}); dram_achieved = bytes actually streamed "
                             f"(library counter, equal to ncu DRAM traffic within 3 %) / kernel time"},
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
