"""C ABI surface without a GPU: the library loads, exports every symbol the
header declares, and rejects malformed programs with ValueError before any
device work (clifft_gpu_load validates on the host)."""

import ctypes
import os
import re

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200 import _native as N
from clifft_b200.program import OP, Program, instr, p_u32x2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "clifft_gpu.h")).read()
    return sorted(set(re.findall(r"\b(clifft_gpu_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    names = declared_symbols()
    assert set(names) == set(N.EXPORTED_SYMBOLS)
    for name in names:
        assert hasattr(lib, name), name


def test_backend_name_without_device_reports_unavailable():
    name = cb.backend_name()
    assert name.startswith("cuda:sm_100a") or name.startswith("unavailable:")


def prog_of(*ins, peak=2, slots=1, **kw):
    return Program(num_qubits=4, peak_rank=peak, num_measurements=slots, total_meas_slots=slots,
                   instructions=np.frombuffer(b"".join(ins), np.uint8).reshape(-1, 32).copy(), **kw)


@pytest.mark.parametrize("ins,msg", [
    ((instr(OP["ARRAY_H"], 0),), "dormant"),
    ((instr(OP["EXPAND"], 1),), "EXPAND must target"),
    ((instr(OP["EXPAND"], 0), instr(OP["EXPAND"], 1), instr(OP["MEAS_ACTIVE_DIAGONAL"], 0,
                                                                  payload=p_u32x2(0, 0))), "active_k-1"),
    ((instr(OP["EXPAND"], 0), instr(OP["EXPAND"], 1), instr(OP["ARRAY_CNOT"], 1, 1)), "distinct"),
    ((instr(OP["MEAS_DORMANT_STATIC"], 3, payload=p_u32x2(5, 0)),), "classical index"),
    ((instr(OP["ARRAY_U2"], 0, payload=p_u32x2(0, 0)),), "U2"),
    ((instr(OP["NOISE"], payload=p_u32x2(0, 0)),), "noise site"),
    ((instr(60),), "unknown opcode"),
    ((instr(OP["EXPAND"], 0), instr(OP["EXPAND"], 1), instr(OP["EXPAND"], 2)), "peak_rank"),
])
def test_load_rejects_malformed_bytecode(ins, msg):
    with pytest.raises(ValueError, match=msg):
        cb.load(prog_of(*ins))


def test_sample_rejects_postselected_program():
    p = prog_of(instr(OP["MEAS_DORMANT_STATIC"], 0, payload=p_u32x2(0, 0)), has_postselection=1)
    with pytest.raises(ValueError, match="post-selected"):
        cb.sample(p, 10)


def test_program_npz_roundtrip(tmp_path):
    from clifft_b200 import workloads as W
    p = W.lower(W.config1(), postselect_all=True)
    path = tmp_path / "p.npz"
    p.save(str(path))
    q = Program.load(str(path))
    for name in ("instructions", "noise_channel_x", "detector_targets", "noise_hazards"):
        assert np.array_equal(getattr(p, name), getattr(q, name))
    assert q.has_postselection == 1 and q.peak_rank == p.peak_rank
