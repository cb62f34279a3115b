"""Multi-program batches (one CUDA-graph launch): every program's records and
counters equal a separate clifft_gpu_sample call with the same seed."""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.batch import ProgramBatch
from clifft_b200.program import Program

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")
NAMES = ["cfg2_00", "cfg2_12", "cfg2_36", "cfg2_05", "cfg0", "cfg1", "cfg2_01"]  # k 11,10,16,4,7,5,18


def _load(name):
    return Program.load(os.path.join(PROGRAMS, f"{name}.npz"))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_matches_separate_calls(precision):
    progs = [_load(n) for n in NAMES]
    peaks = sorted({p.peak_rank for p in progs})
    assert len(peaks) >= 4  # different peak ranks in one graph
    surv = [bool(p.has_postselection) for p in progs]
    shots = [3000, 2000, 1500, 2500, 4000, 5000, 600]
    b = ProgramBatch(progs, shots, seeds=list(range(10, 17)), precision=precision, survivors=surv)
    for seeds in (list(range(10, 17)), list(range(40, 47))):
        ms = b.run(seeds)
        assert ms > 0
        got = b.results()
        for p, s, sd, sv, r in zip(progs, shots, seeds, surv, got):
            ref = cb.run(p, s, sd, precision=precision, survivors=sv)
            assert np.array_equal(r["meas_words"], ref["meas_words"])
            assert np.array_equal(r["det_words"], ref["det_words"])
            assert np.array_equal(r["obs_words"], ref["obs_words"])
            assert np.array_equal(r["survived"], ref["survived"])
            np.testing.assert_allclose(r["exp_vals"], ref["exp_vals"], atol=1e-12)
            assert r["passed_shots"] == ref["passed_shots"]
            assert np.array_equal(r["observable_ones"], ref["observable_ones"])
    b.free()


def test_batch_rejects_host_buffers():
    import ctypes
    from clifft_b200 import _native as N
    p = _load("cfg0")
    dp = cb.load(p)
    args = (N.SampleArgs * 1)()
    args[0].shots, args[0].precision = 10, N.CLIFFT_GPU_FP32
    outs = (N.Outputs * 1)()
    h = ctypes.c_void_p()
    handles = (ctypes.c_void_p * 1)(dp.handle.value)
    with pytest.raises(ValueError, match="DEVICE_PTRS"):
        N.check(N.lib().clifft_gpu_batch_create(handles, args, outs, 1, ctypes.byref(h)), "batch")
