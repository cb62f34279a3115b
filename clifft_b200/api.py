"""Python surface of the CUDA backend, shaped like the reference's bindings.

`sample` and `sample_survivors` take the same arguments and raise the same
exception types as `clifft.sample` / `clifft.sample_survivors`
(src/python/bindings.cc:885-918 and 1019-1038): a post-selected program passed
to `sample` raises ValueError; malformed programs raise ValueError; device
failures raise RuntimeError. Records come back as uint8 arrays (rows, count)
exactly as the reference returns them; on the device they are bit-packed.

Extra keyword arguments select the executor: `precision="fp32"` (default: the
batched FP32 statevector with FP64 reductions) or `"fp64"` (the plain FP64
executor), and `group_threads` (0 = autotuned launch shape).
"""

from __future__ import annotations

import ctypes
import os
import weakref
from typing import Dict, Optional, Sequence

import numpy as np

from . import _native as N
from ._sample_result import SampleResult
from .program import Program

_PRECISIONS = {"fp32": N.CLIFFT_GPU_FP32, "fp64": N.CLIFFT_GPU_FP64}


class DeviceProgram:
    """A program uploaded to the current CUDA device (clifft_gpu_load)."""

    def __init__(self, program: Program):
        self.program = program
        h = ctypes.c_void_p()
        N.check(N.lib().clifft_gpu_load(ctypes.byref(program.image()), ctypes.byref(h)),
                "clifft_gpu_load")
        self.handle = h
        self._fin = weakref.finalize(self, N.lib().clifft_gpu_free, h)

    def free(self) -> None:
        self._fin()

    @property
    def device_bytes(self) -> int:
        return int(N.lib().clifft_gpu_program_device_bytes(self.handle))


def load(program: Program) -> DeviceProgram:
    """Upload (and cache on the Program object) the device image of `program`."""
    dp = getattr(program, "_device_program", None)
    if dp is None or not dp._fin.alive:
        dp = DeviceProgram(program)
        program._device_program = dp
    return dp


def _seed(seed: Optional[int]) -> int:
    if seed is None:
        return int.from_bytes(os.urandom(8), "little")
    if seed < 0:
        raise ValueError("seed must be non-negative")
    return int(seed) & 0xFFFFFFFFFFFFFFFF


def _unpack(words: np.ndarray, count: int) -> np.ndarray:
    if count == 0:
        return np.zeros((words.shape[0], 0), np.uint8)
    bits = np.unpackbits(np.ascontiguousarray(words).view(np.uint8), axis=1, bitorder="little")
    return np.ascontiguousarray(bits[:, :count])


def _csr(lists, shots):
    off = np.zeros(shots + 1, np.uint32)
    flat = []
    for i in range(shots):
        l = lists[i] if lists is not None and i < len(lists) else []
        flat.extend(l)
        off[i + 1] = len(flat)
    return off, np.array(flat, np.uint32)


def run(program: Program, shots: int, seed: Optional[int] = None, *, precision: str = "fp32",
        survivors: bool = False, forced_meas: Optional[np.ndarray] = None,
        faults: Optional[Sequence[Sequence[tuple]]] = None,
        readout_faults: Optional[Sequence[Sequence[int]]] = None, trace: bool = False,
        dump_shots: int = 0, group_threads: int = 0, first_shot: int = 0,
        dust_eps: float = 0.0, want_records: bool = True, fusion: Optional[bool] = None,
        profile: bool = False, autotune: bool = True, k_faults: Optional[int] = None,
        segments: bool = True, max_resident: int = 0, raw_parity: bool = False,
        tensor_dense: bool = False) -> Dict[str, object]:
    """Low-level call of clifft_gpu_sample with host buffers; returns packed
    records plus everything the call reports. `fusion`: None / True = runs of
    consecutive opcodes share one pass over a global-memory statevector,
    False = one pass per opcode (the plain executor). `autotune`: with
    group_threads == 0, let the library time candidate launch shapes on the
    first large call and keep the fastest (False = fixed heuristic).
    `k_faults`: condition every shot on exactly that many fault events
    (clifft_gpu_sample_k). `max_resident`: at most this many statevectors
    resident at once (0 = one full wave of the launch). `raw_parity`:
    detectors / observables without their expected parities and POSTSELECT
    recorded instead of discarding (CLIFFT_GPU_RAW_PARITY). `tensor_dense`:
    FP32 dense blocks of fused sweeps on the tensor cores
    (CLIFFT_GPU_TENSOR_DENSE)."""
    if precision not in _PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
    if shots < 0:
        raise ValueError("shots must be non-negative")
    dp = load(program)
    p = program
    mw, dw, ow = (p.num_measurements + 63) // 64, (p.num_detectors + 63) // 64, (p.num_observables + 63) // 64
    res: Dict[str, object] = {}
    keep = []
    a = N.SampleArgs(shots=shots, seed=_seed(seed), first_shot=first_shot,
                     precision=_PRECISIONS[precision], group_threads=group_threads,
                     dust_eps=dust_eps, max_resident=max_resident)
    flags = 0
    if survivors:
        flags |= N.CLIFFT_GPU_SURVIVORS
    if forced_meas is not None:
        fm = np.ascontiguousarray(forced_meas, np.uint8).reshape(shots, p.total_meas_slots)
        keep.append(fm)
        a.forced_meas = fm.ctypes.data if fm.size else None  # zero slots: nothing to force
        flags |= N.CLIFFT_GPU_FORCED_MEAS
    if faults is not None or readout_faults is not None:
        fo, fs = _csr([[f[0] for f in sh] for sh in faults] if faults is not None else None, shots)
        _, fc = _csr([[f[1] for f in sh] for sh in faults] if faults is not None else None, shots)
        ro, re_ = _csr(readout_faults, shots)
        keep += [fo, fs, fc, ro, re_]
        a.fault_offsets, a.readout_offsets = fo.ctypes.data, ro.ctypes.data
        a.fault_sites = fs.ctypes.data if fs.size else None
        a.fault_channels = fc.ctypes.data if fc.size else None
        a.readout_entries = re_.ctypes.data if re_.size else None
        flags |= N.CLIFFT_GPU_FORCED_FAULTS
    if trace:
        flags |= N.CLIFFT_GPU_TRACE
    if profile:
        flags |= N.CLIFFT_GPU_PROFILE
    if not autotune:
        flags |= N.CLIFFT_GPU_NO_AUTOTUNE
    if not segments:
        flags |= N.CLIFFT_GPU_NO_SEGMENTS
    if raw_parity:
        flags |= N.CLIFFT_GPU_RAW_PARITY
    if tensor_dense:
        flags |= N.CLIFFT_GPU_TENSOR_DENSE
    if fusion is False:
        flags |= N.CLIFFT_GPU_NO_FUSION
    elif fusion is True:
        flags |= N.CLIFFT_GPU_FORCE_FUSION
    a.flags = flags
    o = N.Outputs()
    if want_records:
        res["meas_words"] = np.zeros((shots, mw), np.uint64)
        res["det_words"] = np.zeros((shots, dw), np.uint64)
        res["obs_words"] = np.zeros((shots, ow), np.uint64)
        res["exp_vals"] = np.zeros((shots, p.num_exp_vals), np.float64)
    res["survived"] = np.zeros(shots, np.uint8)
    if trace:
        res["meas_prob"] = np.zeros((shots, p.total_meas_slots), np.float64)
        res["log_prob"] = np.zeros(shots, np.float64)
        res["final_k"] = np.zeros(shots, np.uint32)
        res["final_gamma"] = np.zeros((shots, 2), np.float64)
        res["final_px"] = np.zeros((shots, p.num_words), np.uint64)
        res["final_pz"] = np.zeros((shots, p.num_words), np.uint64)
        if dump_shots:
            res["final_v"] = np.zeros((min(dump_shots, shots), 1 << p.peak_rank, 2), np.float64)
            o.dump_shots = min(dump_shots, shots)
    names = {"meas_words": "meas", "det_words": "det", "obs_words": "obs", "exp_vals": "exp_vals",
             "survived": "survived", "meas_prob": "meas_prob", "log_prob": "log_prob",
             "final_k": "final_k", "final_gamma": "final_gamma", "final_px": "final_px",
             "final_pz": "final_pz", "final_v": "final_v"}
    for key, field in names.items():
        arr = res.get(key)
        if arr is not None and arr.size:
            setattr(o, field, arr.ctypes.data)
    ones = np.zeros(max(1, p.num_observables), np.uint64)
    o.observable_ones = ones.ctypes.data
    if k_faults is None:
        N.check(N.lib().clifft_gpu_sample(dp.handle, ctypes.byref(a), ctypes.byref(o)),
                "clifft_gpu_sample")
    else:
        if k_faults < 0:
            raise ValueError("k must be non-negative")
        N.check(N.lib().clifft_gpu_sample_k(dp.handle, ctypes.byref(a), int(k_faults), ctypes.byref(o)),
                "clifft_gpu_sample_k")
    if "final_v" in res:
        fv = res["final_v"]
        res["final_v"] = fv[..., 0] + 1j * fv[..., 1]
    res.update(passed_shots=int(o.passed_shots), logical_errors=int(o.logical_errors),
               observable_ones=ones[:p.num_observables].copy(), dust_clamps=int(o.dust_clamps),
               algorithmic_bytes=int(o.algorithmic_bytes), streamed_bytes=int(o.streamed_bytes),
               fused=bool(o.fused), phase_cycles=list(o.phase_cycles),
               kernel_ms=float(o.kernel_ms), kernel_launches=int(o.kernel_launches),
               group_threads=int(o.group_threads), state_in_smem=bool(o.state_in_smem))
    return res


def _stats(r) -> dict:
    return {k: r[k] for k in ("kernel_ms", "kernel_launches", "group_threads", "state_in_smem",
                              "dust_clamps", "algorithmic_bytes", "streamed_bytes", "fused")}


def sample(program: Program, shots: int, seed: Optional[int] = None, *,
           precision: str = "fp32", group_threads: int = 0, first_shot: int = 0) -> SampleResult:
    """clifft.sample (src/clifft/svm/svm.cc:191-255) on the GPU. `first_shot`
    offsets the per-shot streams (a shard of a larger run)."""
    if program.has_postselection:
        raise ValueError(
            "sample() cannot be used with post-selected programs because it returns a fixed "
            "number of rows and cannot discard shots. Use sample_survivors(program, shots, "
            "keep_records=True) instead.")
    r = run(program, shots, seed, precision=precision, group_threads=group_threads, first_shot=first_shot)
    return SampleResult(_unpack(r["meas_words"], program.num_measurements),
                        _unpack(r["det_words"], program.num_detectors),
                        _unpack(r["obs_words"], program.num_observables),
                        exp_vals=r["exp_vals"], stats=_stats(r))


def sample_survivors(program: Program, shots: int, seed: Optional[int] = None,
                     keep_records: bool = False, *, precision: str = "fp32",
                     group_threads: int = 0) -> SampleResult:
    """clifft.sample_survivors (src/clifft/svm/svm.cc:266-345) on the GPU.

    Rows are the surviving shots in shot order."""
    r = run(program, shots, seed, precision=precision, survivors=True,
            group_threads=group_threads, want_records=keep_records)
    return _survivor_result(program, r, keep_records, shots)


def _survivor_result(p: Program, r: Dict[str, object], keep_records: bool, shots: int) -> SampleResult:
    if keep_records:
        keep = r["survived"].astype(bool)
        meas = _unpack(r["meas_words"][keep], p.num_measurements)
        det = _unpack(r["det_words"][keep], p.num_detectors)
        obs = _unpack(r["obs_words"][keep], p.num_observables)
        ev = r["exp_vals"][keep]
    else:
        meas = np.zeros((0, p.num_measurements), np.uint8)
        det = np.zeros((0, p.num_detectors), np.uint8)
        obs = np.zeros((0, p.num_observables), np.uint8)
        ev = np.zeros((0, p.num_exp_vals), np.float64)
    return SampleResult(meas, det, obs, total_shots=int(shots), passed_shots=r["passed_shots"],
                        logical_errors=r["logical_errors"], observable_ones=r["observable_ones"],
                        exp_vals=ev, stats=_stats(r))


def trim() -> None:
    """Return the statevector slabs that released programs left parked for
    the next upload (clifft_gpu_trim) to the device."""
    N.lib().clifft_gpu_trim()


def compute_reference_syndrome(program: Program, *, precision: str = "fp64") -> Dict[str, np.ndarray]:
    """Noiseless reference syndrome: the detector and observable parities of
    one noise-free shot with seed 0 (clifft::compute_reference_syndrome,
    src/clifft/api/reference_syndrome.cc:9-30), which the reference uses to
    normalise syndromes. The reference strips the noise from its HIR and
    lowers again without post-selection or expected parities; on the
    compiled program the same shot runs with every noise site and readout
    flip switched off (forced-fault mode with no faults), detectors and
    observables without their expected parities, and POSTSELECT instructions
    recorded in their detector slots instead of discarding. Returns
    {"detectors": uint8[num_detectors], "observables": uint8[num_observables]}."""
    p = program
    r = run(p, 1, 0, precision=precision, faults=[[]], readout_faults=[[]], raw_parity=True)
    return {"detectors": _unpack(r["det_words"], p.num_detectors)[0].copy(),
            "observables": _unpack(r["obs_words"], p.num_observables)[0].copy()}


def record_probabilities(program: Program, records: np.ndarray, *,
                         precision: str = "fp64") -> np.ndarray:
    """Batched forced replay: natural-log probability that `sample` emits each
    record (clifft::record_probabilities, src/clifft/api/record_probabilities.cc:122-191).

    `records` is (num_records, num_measurements) of 0/1 in execution order.
    Unreachable records return -DBL_MAX, like kUnreachableLogProb
    (src/clifft/svm/svm.h:392). Noise, detectors, observables and
    post-selection are rejected as in the reference (record_probabilities.cc:25-91)."""
    p = program
    ops = set(p.opcodes.tolist())
    from .program import OP
    banned = {OP["NOISE"], OP["NOISE_BLOCK"], OP["READOUT_NOISE"], OP["DETECTOR"],
              OP["POSTSELECT"], OP["OBSERVABLE"]}
    if ops & banned:
        raise ValueError("record_probabilities: program must not contain noise, detectors, "
                         "observables or post-selection")
    if p.num_measurements == 0:
        raise ValueError("record_probabilities: program has no measurements")
    rec = np.ascontiguousarray(records, np.uint8)
    if rec.ndim != 2 or rec.shape[1] != p.num_measurements:
        raise ValueError(f"records must have shape (n, {p.num_measurements})")
    if rec.size and rec.max() > 1:
        raise ValueError("records must hold 0/1 values")
    n = rec.shape[0]
    if p.total_meas_slots != p.num_measurements:
        raise ValueError("record_probabilities: hidden measurement slots are not supported")
    if n == 0:
        return np.zeros(0, np.float64)
    r = run(p, n, 0, precision=precision, forced_meas=rec, trace=True, want_records=False)
    out = r["log_prob"].copy()
    out[r["survived"] == 0] = np.finfo(np.float64).min
    return out


def noise_site_probabilities(program: Program) -> np.ndarray:
    """Per fault site its total probability: the noise sites (sum of their
    channel probabilities), then the readout entries
    (clifft::noise_site_probabilities, src/clifft/svm/svm.cc:356-369)."""
    p = program
    off = p.noise_site_offsets.astype(np.int64)
    sites = [float(sum(p.noise_channel_prob[off[i]:off[i + 1]].tolist())) for i in range(len(off) - 1)]
    return np.array(sites + [float(x) for x in p.readout_prob], np.float64)


def sample_k(program: Program, shots: int, k: int, seed: Optional[int] = None, *,
             precision: str = "fp32", group_threads: int = 0) -> SampleResult:
    """clifft.sample_k (src/clifft/svm/svm.cc:548-613): every shot conditioned
    on exactly k fault events."""
    r = run(program, shots, seed, precision=precision, group_threads=group_threads, k_faults=k)
    return SampleResult(_unpack(r["meas_words"], program.num_measurements),
                        _unpack(r["det_words"], program.num_detectors),
                        _unpack(r["obs_words"], program.num_observables),
                        exp_vals=r["exp_vals"], stats=_stats(r))


def sample_k_survivors(program: Program, shots: int, k: int, seed: Optional[int] = None,
                       keep_records: bool = False, *, precision: str = "fp32",
                       group_threads: int = 0) -> SampleResult:
    """clifft.sample_k_survivors (src/clifft/svm/svm.cc:615-711). Rows are the
    surviving shots in shot order."""
    r = run(program, shots, seed, precision=precision, survivors=True, group_threads=group_threads,
            want_records=keep_records, k_faults=k)
    return _survivor_result(program, r, keep_records, shots)
