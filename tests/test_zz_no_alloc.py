"""clifft_gpu_sample_noalloc: the allocation-free sampling entry point.

Each case calls it twice in a row through the C ABI and compares both calls
with clifft_gpu_sample on the same arguments (same kernel, same Philox
streams, so records and counters must agree exactly and expectation values
to 1e-12). The second call checks that the static scratch is cleared between
calls. The file name sorts last so the module also runs after every other GPU
test of a session; it passes on its own as well.
"""

from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
EXP_TOL = 1e-12


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _program(name):
    from clifft_b200.program import Program
    return Program.load(os.path.join(GOLD, "programs", f"{name}.npz"))


def _fixture(name):
    from golden.make_golden import load_case
    return load_case(os.path.join(GOLD, f"{name}.npz"))


def _call(entry, prog, shots, seed, precision, flags, forced=None, stream=None, device=0):
    """One call of `entry` ("clifft_gpu_sample" or "clifft_gpu_sample_noalloc")
    with device buffers for every input and output, on `stream` (a
    torch.cuda.Stream; None = the legacy default stream) of cuda:`device`."""
    torch = _torch()
    from clifft_b200 import _native as N
    from clifft_b200 import api as cb

    torch.cuda.set_device(device)
    dp = cb.load(prog)
    dev = torch.device("cuda", device)
    mw, dw, ow = (prog.num_measurements + 63) // 64, (prog.num_detectors + 63) // 64, \
        (prog.num_observables + 63) // 64
    bufs = {
        "meas": torch.zeros((shots, max(mw, 1)), dtype=torch.int64, device=dev),
        "det": torch.zeros((shots, max(dw, 1)), dtype=torch.int64, device=dev),
        "obs": torch.zeros((shots, max(ow, 1)), dtype=torch.int64, device=dev),
        "exp": torch.zeros((shots, max(prog.num_exp_vals, 1)), dtype=torch.float64, device=dev),
        "surv": torch.zeros(shots, dtype=torch.uint8, device=dev),
    }
    a = N.SampleArgs()
    a.shots, a.seed, a.first_shot = shots, seed, 0
    a.precision = N.CLIFFT_GPU_FP64 if precision == "fp64" else N.CLIFFT_GPU_FP32
    a.flags = flags | N.CLIFFT_GPU_DEVICE_PTRS
    a.stream = stream.cuda_stream if stream is not None else None
    keep = []
    if forced is not None:
        for key, field in (("forced_meas", "forced_meas"), ("fault_offsets", "fault_offsets"),
                           ("fault_sites", "fault_sites"), ("fault_channels", "fault_channels"),
                           ("readout_offsets", "readout_offsets"), ("readout_entries", "readout_entries")):
            arr = forced[key]
            t = torch.from_numpy(np.ascontiguousarray(arr)).to(dev) if arr.size else \
                torch.zeros(1, dtype=torch.int32, device=dev)
            keep.append(t)
            setattr(a, field, t.data_ptr())
    o = N.Outputs()
    o.meas, o.det, o.obs = (bufs[k].data_ptr() for k in ("meas", "det", "obs"))
    o.exp_vals, o.survived = bufs["exp"].data_ptr(), bufs["surv"].data_ptr()
    ones = (ctypes.c_uint64 * max(prog.num_observables, 1))()
    o.observable_ones = ctypes.cast(ones, ctypes.c_void_p)
    torch.cuda.synchronize()
    N.check(getattr(N.lib(), entry)(dp.handle, ctypes.byref(a), ctypes.byref(o)), entry)
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in bufs.items()}
    res.update(passed=o.passed_shots, logical=o.logical_errors, dust=o.dust_clamps,
               alg=o.algorithmic_bytes, launches=o.kernel_launches,
               ones=list(ones)[:prog.num_observables])
    return res


def _same(a, b):
    for k in ("meas", "det", "obs", "surv"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_allclose(a["exp"], b["exp"], rtol=0, atol=EXP_TOL)
    for k in ("passed", "logical", "dust", "alg", "ones"):
        assert a[k] == b[k], k


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_sample_on_memory_grid_survivors(precision):
    from clifft_b200 import _native as N
    prog = _program("cfg1")
    shots, seed, flags = 20000, 77, N.CLIFFT_GPU_SURVIVORS
    ref = _call("clifft_gpu_sample", prog, shots, seed, precision, flags)
    first = _call("clifft_gpu_sample_noalloc", prog, shots, seed, precision, flags)
    second = _call("clifft_gpu_sample_noalloc", prog, shots, seed, precision, flags)
    assert first["launches"] == 1 and ref["passed"] > 0
    _same(first, ref)
    _same(second, ref)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_sample_on_free_sampling_with_exp_vals(precision):
    prog, _ = _fixture("fuzz_k9")
    shots, seed = 3000, 5
    ref = _call("clifft_gpu_sample", prog, shots, seed, precision, 0)
    first = _call("clifft_gpu_sample_noalloc", prog, shots, seed, precision, 0)
    second = _call("clifft_gpu_sample_noalloc", prog, shots, seed, precision, 0)
    _same(first, ref)
    _same(second, ref)


def test_noalloc_matches_sample_on_forced_replay():
    from clifft_b200 import _native as N
    prog, d = _fixture("fuzz_k9")
    forced = {"forced_meas": d["forced_meas_in"].astype(np.uint8)}
    for key in ("fault_offsets", "fault_sites", "fault_channels", "readout_offsets", "readout_entries"):
        forced[key] = d[key].astype(np.uint32)
    shots = forced["forced_meas"].shape[0]
    flags = N.CLIFFT_GPU_FORCED_MEAS | N.CLIFFT_GPU_FORCED_FAULTS
    ref = _call("clifft_gpu_sample", prog, shots, 0, "fp64", flags, forced)
    first = _call("clifft_gpu_sample_noalloc", prog, shots, 0, "fp64", flags, forced)
    second = _call("clifft_gpu_sample_noalloc", prog, shots, 0, "fp64", flags, forced)
    _same(first, ref)
    _same(second, ref)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_orders_its_work_on_the_callers_stream(precision):
    # clear, launch and read-back of the static scratch all go on args->stream
    torch = _torch()
    from clifft_b200 import _native as N
    prog = _program("cfg1")
    shots, seed, flags = 20000, 91, N.CLIFFT_GPU_SURVIVORS
    ref = _call("clifft_gpu_sample", prog, shots, seed, precision, flags)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        first = _call("clifft_gpu_sample_noalloc", prog, shots, seed, precision, flags, stream=s)
        second = _call("clifft_gpu_sample_noalloc", prog, shots, seed, precision, flags, stream=s)
    _same(first, ref)
    _same(second, ref)


def test_noalloc_on_a_second_device():
    # the scratch address is looked up per device
    torch = _torch()
    if torch.cuda.device_count() < 2:
        pytest.skip("one CUDA device visible")
    from clifft_b200 import _native as N
    prog = _program("cfg1")
    shots, seed, flags = 5000, 13, N.CLIFFT_GPU_SURVIVORS
    try:
        ref = _call("clifft_gpu_sample", prog, shots, seed, "fp32", flags, device=1)
        first = _call("clifft_gpu_sample_noalloc", prog, shots, seed, "fp32", flags, device=1)
        second = _call("clifft_gpu_sample_noalloc", prog, shots, seed, "fp32", flags, device=1)
    finally:
        torch.cuda.set_device(0)
    _same(first, ref)
    _same(second, ref)


def test_noalloc_rejects_more_observables_than_the_static_scratch_holds():
    from clifft_b200 import _native as N
    prog = _program("cfg1")
    limit = N.NOALLOC_SCRATCH_WORDS - 15
    ok = dataclasses.replace(prog, num_observables=limit,
                             expected_observables=np.zeros(limit, np.uint8))
    r = _call("clifft_gpu_sample_noalloc", ok, 64, 1, "fp32", 0)
    assert r["launches"] == 1
    big = dataclasses.replace(prog, num_observables=limit + 1,
                              expected_observables=np.zeros(limit + 1, np.uint8))
    with pytest.raises(ValueError, match="static scratch holds 512"):
        _call("clifft_gpu_sample_noalloc", big, 64, 1, "fp32", 0)


def test_noalloc_rejects_host_buffers_trace_and_global_statevectors():
    torch = _torch()
    from clifft_b200 import _native as N
    from clifft_b200 import api as cb
    prog = _program("cfg1")
    dp = cb.load(prog)
    a = N.SampleArgs()
    a.shots, a.seed, a.precision = 16, 1, N.CLIFFT_GPU_FP32
    o = N.Outputs()
    with pytest.raises(ValueError, match="CLIFFT_GPU_DEVICE_PTRS"):
        N.check(N.lib().clifft_gpu_sample_noalloc(dp.handle, ctypes.byref(a), ctypes.byref(o)), "noalloc")
    a.flags = N.CLIFFT_GPU_DEVICE_PTRS | N.CLIFFT_GPU_TRACE
    with pytest.raises(ValueError, match="CLIFFT_GPU_TRACE"):
        N.check(N.lib().clifft_gpu_sample_noalloc(dp.handle, ctypes.byref(a), ctypes.byref(o)), "noalloc")
    big, _ = _fixture("fuzz_k16")
    with pytest.raises(ValueError, match="do not fit in shared memory"):
        _call("clifft_gpu_sample_noalloc", big, 4, 1, "fp64", 0)
    torch.cuda.synchronize()
