"""Several programs sampled by one CUDA-graph launch (clifft_gpu_batch_*).

    b = ProgramBatch(programs, shots=10_000, precision="fp32")
    ms = b.run(seeds=[...])          # one graph launch for every program
    rows = b.results()               # per program: records (numpy) + counters

Each program keeps its own autotuned launch shape; the graph has one
independent branch per program, so programs of different peak rank run side
by side instead of one launch after another. Records stay in device buffers
(torch tensors) until `results()` copies them to the host.
"""

from __future__ import annotations

import ctypes
import weakref
from typing import Dict, List, Optional, Sequence, Union

import numpy as np

from . import _native as N
from . import api
from .program import Program


class ProgramBatch:
    def __init__(self, programs: Sequence[Program], shots: Union[int, Sequence[int]], *,
                 seeds: Optional[Sequence[int]] = None, precision: str = "fp32",
                 survivors: Union[bool, Sequence[bool]] = False, fusion: Optional[bool] = None,
                 group_threads: int = 0):
        import torch
        if precision not in api._PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(api._PRECISIONS)}")
        n = len(programs)
        if n == 0:
            raise ValueError("empty batch")
        shots = [int(shots)] * n if np.isscalar(shots) else [int(s) for s in shots]
        surv = [bool(survivors)] * n if np.isscalar(survivors) else [bool(s) for s in survivors]
        seeds = list(seeds) if seeds is not None else list(range(1, n + 1))
        if len(shots) != n or len(surv) != n or len(seeds) != n:
            raise ValueError("shots, survivors and seeds need one entry per program")
        dev = torch.device("cuda", torch.cuda.current_device())
        self.programs = list(programs)
        self.shots = shots
        self._dps = [api.load(p) for p in programs]
        self._bufs: List[Dict[str, object]] = []
        self._ones = []
        self._args = (N.SampleArgs * n)()
        self._outs = (N.Outputs * n)()
        for i, p in enumerate(programs):
            s = shots[i]
            mw, dw, ow = (p.num_measurements + 63) // 64, (p.num_detectors + 63) // 64, (p.num_observables + 63) // 64
            b = {"meas": torch.zeros((s, mw), dtype=torch.int64, device=dev),
                 "det": torch.zeros((s, dw), dtype=torch.int64, device=dev),
                 "obs": torch.zeros((s, ow), dtype=torch.int64, device=dev),
                 "exp_vals": torch.zeros((s, p.num_exp_vals), dtype=torch.float64, device=dev),
                 "survived": torch.zeros(s, dtype=torch.uint8, device=dev)}
            self._bufs.append(b)
            flags = N.CLIFFT_GPU_DEVICE_PTRS | (N.CLIFFT_GPU_SURVIVORS if surv[i] else 0)
            if fusion is False:
                flags |= N.CLIFFT_GPU_NO_FUSION
            a = self._args[i]
            a.shots, a.seed, a.first_shot = s, api._seed(seeds[i]), 0
            a.precision, a.flags, a.group_threads = api._PRECISIONS[precision], flags, group_threads
            o = self._outs[i]
            for field, t in b.items():
                setattr(o, field, t.data_ptr() if t.numel() else None)
            ones = np.zeros(max(1, p.num_observables), np.uint64)
            self._ones.append(ones)
            o.observable_ones = ones.ctypes.data
        handles = (ctypes.c_void_p * n)(*[dp.handle.value for dp in self._dps])
        h = ctypes.c_void_p()
        torch.cuda.synchronize()
        N.check(N.lib().clifft_gpu_batch_create(handles, self._args, self._outs, n, ctypes.byref(h)),
                "clifft_gpu_batch_create")
        self._handle = h
        self._fin = weakref.finalize(self, N.lib().clifft_gpu_batch_free, h)

    def run(self, seeds: Optional[Sequence[int]] = None) -> float:
        """One graph launch over every program; returns its device time in ms."""
        import torch
        n = len(self.programs)
        sp = None
        if seeds is not None:
            if len(seeds) != n:
                raise ValueError("one seed per program")
            sp = (ctypes.c_uint64 * n)(*[api._seed(s) for s in seeds])
        ms = ctypes.c_float(0.0)
        stream = torch.cuda.current_stream().cuda_stream
        N.check(N.lib().clifft_gpu_batch_run(self._handle, sp, ctypes.c_void_p(stream), ctypes.byref(ms)),
                "clifft_gpu_batch_run")
        return float(ms.value)

    def results(self) -> List[Dict[str, object]]:
        """Per program: packed records (numpy u64 words), exp-vals, survivor
        flags and the counters of the last run."""
        out = []
        for i, p in enumerate(self.programs):
            b = self._bufs[i]
            o = self._outs[i]
            out.append({
                "meas_words": b["meas"].cpu().numpy().view(np.uint64),
                "det_words": b["det"].cpu().numpy().view(np.uint64),
                "obs_words": b["obs"].cpu().numpy().view(np.uint64),
                "exp_vals": b["exp_vals"].cpu().numpy(),
                "survived": b["survived"].cpu().numpy(),
                "passed_shots": int(o.passed_shots), "logical_errors": int(o.logical_errors),
                "observable_ones": self._ones[i][:p.num_observables].copy(),
                "algorithmic_bytes": int(o.algorithmic_bytes), "group_threads": int(o.group_threads),
            })
        return out

    def free(self) -> None:
        self._fin()
