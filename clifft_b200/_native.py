"""Loader for the in-tree CUDA library (libclifft_gpu.so) and its C ABI.

There is no CPU fallback: if the shared library is missing or no sm_100
device is visible, every sampling call raises. Build the library with
`python -m clifft_b200.build` (or `__graft_entry__.build()`).
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclifft_gpu.so")

CLIFFT_GPU_FP64 = 0
CLIFFT_GPU_FP32 = 1
CLIFFT_GPU_SURVIVORS = 0x01
CLIFFT_GPU_FORCED_MEAS = 0x02
CLIFFT_GPU_FORCED_FAULTS = 0x04
CLIFFT_GPU_DEVICE_PTRS = 0x08
CLIFFT_GPU_TRACE = 0x10
CLIFFT_GPU_NO_FUSION = 0x20
CLIFFT_GPU_FORCE_FUSION = 0x40
CLIFFT_GPU_PROFILE = 0x80
CLIFFT_GPU_NO_AUTOTUNE = 0x100
CLIFFT_GPU_NO_SEGMENTS = 0x200
CLIFFT_GPU_RAW_PARITY = 0x400
CLIFFT_GPU_TENSOR_DENSE = 0x800

STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "device error", -4: "out of memory"}

P = ctypes.c_void_p


class SampleArgs(ctypes.Structure):
    _fields_ = [
        ("shots", ctypes.c_uint64), ("seed", ctypes.c_uint64), ("first_shot", ctypes.c_uint64),
        ("precision", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("group_threads", ctypes.c_uint32), ("max_resident", ctypes.c_uint32),
        ("dust_eps", ctypes.c_double),
        ("forced_meas", P), ("fault_offsets", P), ("fault_sites", P), ("fault_channels", P),
        ("readout_offsets", P), ("readout_entries", P), ("stream", P),
    ]


class Outputs(ctypes.Structure):
    _fields_ = [
        ("meas", P), ("det", P), ("obs", P), ("exp_vals", P), ("survived", P),
        ("meas_prob", P), ("log_prob", P), ("final_k", P), ("final_gamma", P),
        ("final_px", P), ("final_pz", P), ("final_v", P), ("dump_shots", ctypes.c_uint64),
        ("passed_shots", ctypes.c_uint64), ("logical_errors", ctypes.c_uint64),
        ("observable_ones", P), ("dust_clamps", ctypes.c_uint64),
        ("algorithmic_bytes", ctypes.c_uint64), ("streamed_bytes", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint32), ("kernel_ms", ctypes.c_float),
        ("group_threads", ctypes.c_uint32), ("state_in_smem", ctypes.c_uint32),
        ("fused", ctypes.c_uint32), ("phase_cycles", ctypes.c_uint64 * 5),
    ]


class GradArgs(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_uint64), ("precision", ctypes.c_uint32), ("flags", ctypes.c_uint32),
        ("phases", P), ("stream", P),
    ]


_lib = None
_lock = threading.Lock()


class NativeError(RuntimeError):
    pass


def lib():
    """The loaded C ABI. Raises if the extension was not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise NativeError(
                    f"CUDA extension not built: {LIB_PATH} is missing "
                    "(run `python -m clifft_b200.build`); there is no CPU fallback")
            L = ctypes.CDLL(LIB_PATH)
            L.clifft_gpu_load.restype = ctypes.c_int
            L.clifft_gpu_load.argtypes = [P, ctypes.POINTER(P)]
            L.clifft_gpu_free.restype = None
            L.clifft_gpu_free.argtypes = [P]
            L.clifft_gpu_trim.restype = None
            L.clifft_gpu_trim.argtypes = []
            L.clifft_gpu_sample.restype = ctypes.c_int
            L.clifft_gpu_sample.argtypes = [P, ctypes.POINTER(SampleArgs), ctypes.POINTER(Outputs)]
            L.clifft_gpu_sample_noalloc.restype = ctypes.c_int
            L.clifft_gpu_sample_noalloc.argtypes = [P, ctypes.POINTER(SampleArgs), ctypes.POINTER(Outputs)]
            L.clifft_gpu_batch_create.restype = ctypes.c_int
            L.clifft_gpu_batch_create.argtypes = [ctypes.POINTER(P), ctypes.POINTER(SampleArgs),
                                                  ctypes.POINTER(Outputs), ctypes.c_uint32, ctypes.POINTER(P)]
            L.clifft_gpu_batch_run.restype = ctypes.c_int
            L.clifft_gpu_batch_run.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), P,
                                               ctypes.POINTER(ctypes.c_float)]
            L.clifft_gpu_batch_free.restype = None
            L.clifft_gpu_batch_free.argtypes = [P]
            L.clifft_gpu_sample_k.restype = ctypes.c_int
            L.clifft_gpu_sample_k.argtypes = [P, ctypes.POINTER(SampleArgs), ctypes.c_uint32, ctypes.POINTER(Outputs)]
            L.clifft_gpu_expval_grad.restype = ctypes.c_int
            L.clifft_gpu_expval_grad.argtypes = [P, ctypes.POINTER(GradArgs), P, P]
            L.clifft_gpu_program_num_rot_params.restype = ctypes.c_uint32
            L.clifft_gpu_program_num_rot_params.argtypes = [P]
            L.clifft_gpu_backend_name.restype = ctypes.c_char_p
            L.clifft_gpu_last_error.restype = ctypes.c_char_p
            L.clifft_gpu_program_peak_rank.restype = ctypes.c_uint32
            L.clifft_gpu_program_peak_rank.argtypes = [P]
            L.clifft_gpu_program_device_bytes.restype = ctypes.c_uint64
            L.clifft_gpu_program_device_bytes.argtypes = [P]
            _lib = L
    return _lib


EXPORTED_SYMBOLS = (
    "clifft_gpu_load", "clifft_gpu_free", "clifft_gpu_sample", "clifft_gpu_backend_name",
    "clifft_gpu_last_error", "clifft_gpu_program_peak_rank", "clifft_gpu_program_device_bytes",
    "clifft_gpu_sample_noalloc", "clifft_gpu_batch_create", "clifft_gpu_batch_run", "clifft_gpu_batch_free",
    "clifft_gpu_expval_grad", "clifft_gpu_program_num_rot_params", "clifft_gpu_sample_k", "clifft_gpu_trim",
)
NOALLOC_SCRATCH_WORDS = 512  # CLIFFT_GPU_NOALLOC_SCRATCH_WORDS


def check(rc: int, what: str) -> None:
    if rc == 0:
        return
    msg = lib().clifft_gpu_last_error().decode(errors="replace")
    if rc == -1:
        raise ValueError(f"{what}: {msg}")
    if rc == -4:
        raise MemoryError(f"{what}: {msg}")
    raise RuntimeError(f"{what}: {STATUS.get(rc, rc)}: {msg}")


def backend_name() -> str:
    return lib().clifft_gpu_backend_name().decode()
