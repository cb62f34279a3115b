"""ctypes bindings for the CPU oracle and the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, by `__graft_entry__.smoke()` and
by the CPU-baseline leg of bench.py, always as the checker or as the timed CPU
baseline, never by the product package.

  * `run(...)`         -> oracle/_build/libsvm_oracle.so (svm_oracle.c), the
                          plain-C restatement of the reference executor;
  * `ref_*` functions  -> oracle/_ref/libclifft_ref.so, the reference's own
                          executor and bytecode passes built from its sources
                          by oracle/build_ref.sh (present only where the
                          reference tree was available at build time);
                          `ref_select_native()` switches the timing calls to
                          the -march=native build of the same sources when
                          this host can run it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libsvm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libclifft_ref.so")
REF_NATIVE_SO = os.path.join(HERE, "_ref", "libclifft_ref_native.so")

RNG_XOSHIRO = 0
RNG_PHILOX = 1
REFERENCE_DUST_EPS = 1e-18

P = ctypes.c_void_p


class OracleArgs(ctypes.Structure):
    _fields_ = [
        ("shots", ctypes.c_uint32), ("seed", ctypes.c_uint64), ("rng_kind", ctypes.c_uint32),
        ("first_shot", ctypes.c_uint64), ("dust_eps", ctypes.c_double),
        ("forced_meas", P), ("fault_offsets", P), ("fault_sites", P), ("fault_channels", P),
        ("readout_offsets", P), ("readout_entries", P),
    ]


class OracleOutputs(ctypes.Structure):
    _fields_ = [
        ("meas", P), ("det", P), ("obs", P), ("exp_vals", P), ("discarded", P),
        ("meas_prob", P), ("log_prob", P), ("reachable", P), ("final_k", P),
        ("final_gamma", P), ("final_px", P), ("final_pz", P), ("final_v", P),
        ("dust_clamps", ctypes.c_uint64),
    ]


_oracle = None
_ref = None


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_run.restype = ctypes.c_int
        lib.oracle_run.argtypes = [P, ctypes.POINTER(OracleArgs), ctypes.POINTER(OracleOutputs)]
        lib.oracle_last_error.restype = ctypes.c_char_p
        lib.oracle_philox4x32_10.argtypes = [P, P, P]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


_ref_path = REF_SO


def ref_select_native() -> bool:
    """Use the -march=native build for every later ref_* call if it exists
    and a child process can run a small sample with it (a host without the
    build host's instruction set dies of SIGILL there, not here). Returns
    whether the native build is now in use. Call before the first ref_* call."""
    global _ref_path
    if _ref is not None or not os.path.exists(REF_NATIVE_SO):
        return _ref_path == REF_NATIVE_SO
    probe = ("import sys; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
             "from oracle import pyoracle as O\n"
             "from clifft_b200.program import OP, Program, instr, p_u32x2\n"
             "import numpy as np\n"
             "code = [instr(OP['EXPAND'], 0), instr(OP['EXPAND_T'], 1), instr(OP['ARRAY_H'], 0),\n"
             "        instr(OP['ARRAY_CNOT'], 0, 1), instr(OP['MEAS_ACTIVE_DIAGONAL'], 1, 0, 0, p_u32x2(0, 0))]\n"
             "p = Program(num_qubits=2, peak_rank=2, num_measurements=1, total_meas_slots=1,\n"
             "            instructions=np.frombuffer(b''.join(code), np.uint8).reshape(-1, 32))\n"
             "O._ref_path = O.REF_NATIVE_SO\n"
             "O.ref_sample(p, 64, 1); O.ref_time_sample(p, 8, 1, 2, False, 1)\n") % (
        os.path.dirname(HERE), HERE)
    import sys
    ok = subprocess.run([sys.executable, "-c", probe], capture_output=True, timeout=120).returncode == 0
    if ok:
        _ref_path = REF_NATIVE_SO
    return ok


def ref_build_kind() -> str:
    return "native" if _ref_path == REF_NATIVE_SO else "generic"


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"reference harness not built: {REF_SO}")
        lib = ctypes.CDLL(_ref_path)
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_svm_backend.restype = ctypes.c_char_p
        lib.ref_sample.restype = ctypes.c_int
        lib.ref_sample.argtypes = [P, ctypes.c_uint32, ctypes.c_uint64, P, P, P, P]
        lib.ref_sample_k.restype = ctypes.c_int
        lib.ref_sample_k.argtypes = [P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, P, P, P, P]
        lib.ref_noise_site_probabilities.restype = ctypes.c_int64
        lib.ref_noise_site_probabilities.argtypes = [P, P, ctypes.c_uint64]
        lib.ref_sample_survivors.restype = ctypes.c_int64
        lib.ref_sample_survivors.argtypes = [P, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                                             P, P, P, P, P, P]
        lib.ref_time_sample.restype = ctypes.c_double
        lib.ref_time_sample.argtypes = [P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                        ctypes.c_int]
        lib.ref_time_sample_omp.restype = ctypes.c_double
        lib.ref_time_sample_omp.argtypes = [P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int]
        lib.ref_forced_run.restype = ctypes.c_int
        lib.ref_forced_run.argtypes = [P, ctypes.c_uint32] + [P] * 19
        lib.ref_run_passes.restype = P
        lib.ref_run_passes.argtypes = [P, ctypes.c_uint32]
        lib.ref_module_image.restype = P
        lib.ref_module_image.argtypes = [P]
        lib.ref_module_free.argtypes = [P]
        _ref = lib
    return _ref


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def philox_block(ctr: Sequence[int], key: Sequence[int]) -> np.ndarray:
    c = np.array(ctr, np.uint32)
    k = np.array(key, np.uint32)
    out = np.zeros(4, np.uint32)
    oracle_lib().oracle_philox4x32_10(c.ctypes.data, k.ctypes.data, out.ctypes.data)
    return out


def _csr(lists, dtype=np.uint32):
    off = np.zeros(len(lists) + 1, np.uint32)
    flat = []
    for i, l in enumerate(lists):
        flat.extend(l)
        off[i + 1] = len(flat)
    return off, np.array(flat, dtype)


def run(prog, shots: int, seed: int = 0, rng: int = RNG_PHILOX, first_shot: int = 0,
        dust_eps: float = REFERENCE_DUST_EPS, forced_meas: Optional[np.ndarray] = None,
        faults: Optional[Sequence[Sequence[tuple]]] = None,
        readout_faults: Optional[Sequence[Sequence[int]]] = None,
        want_state: bool = False) -> Dict[str, np.ndarray]:
    """Run the oracle on `prog` (a clifft_b200.program.Program).

    faults[s] is a list of (site, channel) pairs for shot s (ascending sites);
    readout_faults[s] a list of readout-entry indices. Either one switches the
    shot to forced-fault mode (gap sampler bypassed)."""
    lib = oracle_lib()
    img = prog.image()
    slots = prog.total_meas_slots
    keep = []
    a = OracleArgs(shots=shots, seed=seed, rng_kind=rng, first_shot=first_shot, dust_eps=dust_eps)
    if forced_meas is not None:
        fm = np.ascontiguousarray(forced_meas, dtype=np.uint8).reshape(shots, slots)
        keep.append(fm)
        a.forced_meas = fm.ctypes.data
    if faults is not None or readout_faults is not None:
        fo, fs = _csr([[f[0] for f in sh] for sh in (faults or [[]] * shots)])
        _, fc = _csr([[f[1] for f in sh] for sh in (faults or [[]] * shots)])
        ro, re_ = _csr(readout_faults or [[]] * shots)
        keep += [fo, fs, fc, ro, re_]
        a.fault_offsets, a.fault_sites, a.fault_channels = fo.ctypes.data, _ptr(fs), _ptr(fc)
        a.readout_offsets, a.readout_entries = ro.ctypes.data, _ptr(re_)
    out = {
        "meas": np.zeros((shots, prog.num_measurements), np.uint8),
        "det": np.zeros((shots, prog.num_detectors), np.uint8),
        "obs": np.zeros((shots, prog.num_observables), np.uint8),
        "exp_vals": np.zeros((shots, prog.num_exp_vals), np.float64),
        "discarded": np.zeros(shots, np.uint8),
        "meas_prob": np.zeros((shots, slots), np.float64),
        "log_prob": np.zeros(shots, np.float64),
        "reachable": np.zeros(shots, np.uint8),
        "final_k": np.zeros(shots, np.uint32),
        "final_gamma": np.zeros((shots, 2), np.float64),
        "final_px": np.zeros((shots, prog.num_words), np.uint64),
        "final_pz": np.zeros((shots, prog.num_words), np.uint64),
    }
    if want_state:
        out["final_v"] = np.zeros((shots, 1 << prog.peak_rank, 2), np.float64)
    o = OracleOutputs()
    for key, arr in out.items():
        setattr(o, key, arr.ctypes.data if arr.size else None)
    rc = lib.oracle_run(ctypes.byref(img), ctypes.byref(a), ctypes.byref(o))
    if rc != 0:
        raise RuntimeError(lib.oracle_last_error().decode())
    out["dust_clamps"] = int(o.dust_clamps)
    if want_state:
        out["final_v"] = out["final_v"][..., 0] + 1j * out["final_v"][..., 1]
    return out


# ----------------------------------------------------------- reference side
def ref_backend() -> str:
    return ref_lib().ref_svm_backend().decode()


def ref_sample(prog, shots: int, seed: int) -> Dict[str, np.ndarray]:
    lib = ref_lib()
    out = {
        "meas": np.zeros((shots, prog.num_measurements), np.uint8),
        "det": np.zeros((shots, prog.num_detectors), np.uint8),
        "obs": np.zeros((shots, prog.num_observables), np.uint8),
        "exp_vals": np.zeros((shots, prog.num_exp_vals), np.float64),
    }
    rc = lib.ref_sample(ctypes.byref(prog.image()), shots, seed, *[_ptr(out[k]) for k in
                                                                     ("meas", "det", "obs", "exp_vals")])
    if rc != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return out


def ref_sample_k(prog, shots: int, k: int, seed: int) -> Dict[str, np.ndarray]:
    """The reference's clifft::sample_k (exactly k faults per shot)."""
    lib = ref_lib()
    out = {
        "meas": np.zeros((shots, prog.num_measurements), np.uint8),
        "det": np.zeros((shots, prog.num_detectors), np.uint8),
        "obs": np.zeros((shots, prog.num_observables), np.uint8),
        "exp_vals": np.zeros((shots, prog.num_exp_vals), np.float64),
    }
    rc = lib.ref_sample_k(ctypes.byref(prog.image()), shots, k, seed,
                          *[_ptr(out[x]) for x in ("meas", "det", "obs", "exp_vals")])
    if rc != 0:
        raise ValueError(lib.ref_last_error().decode())
    return out


def ref_noise_site_probabilities(prog) -> np.ndarray:
    lib = ref_lib()
    cap = 1 << 20
    buf = np.zeros(cap, np.float64)
    n = lib.ref_noise_site_probabilities(ctypes.byref(prog.image()), buf.ctypes.data, cap)
    if n < 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return buf[:n].copy()


def ref_sample_survivors(prog, shots: int, seed: int, keep_records: bool = False):
    lib = ref_lib()
    counts = np.zeros(3, np.uint64)
    ones = np.zeros(max(1, prog.num_observables), np.uint64)
    out = {
        "meas": np.zeros((shots, prog.num_measurements), np.uint8),
        "det": np.zeros((shots, prog.num_detectors), np.uint8),
        "obs": np.zeros((shots, prog.num_observables), np.uint8),
        "exp_vals": np.zeros((shots, prog.num_exp_vals), np.float64),
    }
    rows = lib.ref_sample_survivors(ctypes.byref(prog.image()), shots, seed, int(keep_records),
                                    counts.ctypes.data, ones.ctypes.data,
                                    *[_ptr(out[k]) for k in ("meas", "det", "obs", "exp_vals")])
    if rows < 0:
        raise RuntimeError(lib.ref_last_error().decode())
    res = {k: v[:rows] for k, v in out.items()}
    res.update(total_shots=int(counts[0]), passed_shots=int(counts[1]),
               logical_errors=int(counts[2]), observable_ones=ones[:prog.num_observables].copy())
    return res


def ref_time_sample(prog, shots: int, seed: int, threads: int, survivors: bool,
                    omp_threads: int = 1) -> float:
    """Wall seconds of the reference's clifft::sample (or sample_survivors) over
    `shots` shots split across `threads` host threads (distinct seeds), each
    thread's OpenMP team limited to `omp_threads` (the executor parallelises
    one shot's statevector loops with OpenMP at large k)."""
    lib = ref_lib()
    t = lib.ref_time_sample_omp(ctypes.byref(prog.image()), shots, seed, threads, int(survivors),
                                omp_threads)
    if t < 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return t


def ref_forced(prog, forced_meas: np.ndarray, faults=None, readout_faults=None) -> Dict[str, np.ndarray]:
    lib = ref_lib()
    slots = prog.total_meas_slots
    shots = int(np.shape(forced_meas)[0])
    fm = np.ascontiguousarray(forced_meas, dtype=np.uint8).reshape(shots, slots)
    if fm.size == 0:
        fm = np.zeros((shots, 1), np.uint8)
    fo = fs = fc = ro = re_ = None
    if faults is not None:
        fo, fs = _csr([[f[0] for f in sh] for sh in faults])
        _, fc = _csr([[f[1] for f in sh] for sh in faults])
    if readout_faults is not None:
        ro, re_ = _csr(readout_faults)
    out = {
        "meas": np.zeros((shots, slots), np.uint8),
        "det": np.zeros((shots, prog.num_detectors), np.uint8),
        "obs": np.zeros((shots, prog.num_observables), np.uint8),
        "exp_vals": np.zeros((shots, prog.num_exp_vals), np.float64),
        "meas_prob": np.zeros((shots, slots), np.float64),
        "log_prob": np.zeros(shots, np.float64),
        "reachable": np.zeros(shots, np.uint8),
        "discarded": np.zeros(shots, np.uint8),
        "final_k": np.zeros(shots, np.uint32),
        "final_gamma": np.zeros((shots, 2), np.float64),
        "final_px": np.zeros((shots, prog.num_words), np.uint64),
        "final_pz": np.zeros((shots, prog.num_words), np.uint64),
        "final_v": np.zeros((shots, 1 << prog.peak_rank, 2), np.float64),
    }
    order = ["meas", "det", "obs", "exp_vals", "meas_prob", "log_prob", "reachable", "discarded",
             "final_k", "final_gamma", "final_px", "final_pz", "final_v"]
    rc = lib.ref_forced_run(ctypes.byref(prog.image()), shots, fm.ctypes.data,
                            _ptr(fo), _ptr(fs), _ptr(fc), _ptr(ro), _ptr(re_),
                            *[out[k].ctypes.data if out[k].size else None for k in order])
    if rc != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    out["final_v"] = out["final_v"][..., 0] + 1j * out["final_v"][..., 1]
    return out


PASS_NOISE_BLOCK, PASS_MULTI_GATE, PASS_EXPAND_T, PASS_EXPAND_ROT = 1, 2, 4, 8
PASS_SWAP_MEAS, PASS_TILE_AXIS, PASS_SINGLE_AXIS = 16, 32, 64
PASS_ALL = 127


def ref_passes(prog, mask: int = PASS_ALL):
    """Run the reference's own bytecode passes (registry order) over `prog`."""
    from clifft_b200.program import Program, ProgramImage
    lib = ref_lib()
    h = lib.ref_run_passes(ctypes.byref(prog.image()), mask)
    if not h:
        raise RuntimeError(lib.ref_last_error().decode())
    try:
        img = ctypes.cast(lib.ref_module_image(h), ctypes.POINTER(ProgramImage)).contents
        out = Program.from_image(img, name=prog.name)
    finally:
        lib.ref_module_free(h)
    return out
