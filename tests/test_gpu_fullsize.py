"""Full-size workloads, checked through properties that do not depend on an
oracle run of the same size:

  * k = 24 (2^24 amplitudes per shot): under forced outcomes every launch
    shape (128 / 256 / 512-thread CTAs, 256 / 512 + a copy warp) and fused vs one-pass-per-opcode
    execution give the same records and FP64 probabilities to 1e-12, and the
    FP32 statevector stays within 1e-5 of FP64 on every probability;
  * the 10^6-shot post-selected memory grid: the survivor fraction and the
    logical-error rate of the FP32 executor match the reference's own
    sample_survivors within 5 sigma;
  * edge cases: zero shots, a program without measurements, one shot.
"""

from __future__ import annotations

import math
import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import Program
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


def _load(name):
    return Program.load(os.path.join(PROGRAMS, f"{name}.npz"))


def _forced(prog, shots, seed):
    r = cb.run(prog, shots, seed, precision="fp64")
    bits = cb.api._unpack(r["meas_words"], prog.num_measurements)
    fm = np.zeros((shots, prog.total_meas_slots), np.uint8)
    fm[:, :prog.num_measurements] = bits
    return fm


def test_k24_shapes_fusion_and_precision():
    prog = _load("cfg3")
    assert prog.peak_rank == 24
    fm = _forced(prog, 4, 9)
    runs = {}
    for group in (128, 256, 288, 512, 544):
        for fusion in (True, False):
            if group != 256 and not fusion:
                continue
            runs[(group, fusion)] = cb.run(prog, 4, 0, precision="fp64", forced_meas=fm, trace=True,
                                           group_threads=group, fusion=fusion)
    base = runs[(256, True)]
    assert np.all(base["survived"] == 1)
    for key, r in runs.items():
        assert np.array_equal(r["meas_words"], base["meas_words"]), key
        assert np.array_equal(r["final_k"], base["final_k"]), key
        assert np.array_equal(r["final_px"], base["final_px"]) and np.array_equal(r["final_pz"], base["final_pz"])
        np.testing.assert_allclose(r["meas_prob"], base["meas_prob"], rtol=0, atol=1e-12, err_msg=str(key))
    f32 = cb.run(prog, 4, 0, precision="fp32", forced_meas=fm, trace=True)
    np.testing.assert_allclose(f32["meas_prob"], base["meas_prob"], rtol=0, atol=1e-5)
    assert np.array_equal(f32["meas_words"], base["meas_words"])


def test_memory_grid_million_shots_vs_reference_survivors():
    prog = _load("cfg1")
    n_gpu = 1_000_000
    r = cb.sample_survivors(prog, n_gpu, seed=21, precision="fp32")
    n_ref = 400_000
    ref = O.ref_sample_survivors(prog, n_ref, 22)
    p_ref = ref["passed_shots"] / n_ref
    p_gpu = r.passed_shots / n_gpu
    p = (p_ref * n_ref + p_gpu * n_gpu) / (n_ref + n_gpu)
    assert abs(p_ref - p_gpu) <= 5 * math.sqrt(p * (1 - p) * (1 / n_ref + 1 / n_gpu))
    l_ref = ref["logical_errors"] / max(ref["passed_shots"], 1)
    l_gpu = r.logical_errors / max(r.passed_shots, 1)
    q = (l_ref + l_gpu) / 2
    assert abs(l_ref - l_gpu) <= 5 * math.sqrt(max(q * (1 - q), 1e-6) *
                                               (1 / max(ref["passed_shots"], 1) + 1 / max(r.passed_shots, 1)))


def test_edge_cases():
    prog = _load("cfg0")
    r0 = cb.run(prog, 0, 1, precision="fp32")
    assert r0["meas_words"].shape[0] == 0 and r0["kernel_launches"] == 0
    one = cb.sample(prog, 1, seed=3, precision="fp64")
    assert one.measurements.shape == (1, prog.num_measurements)
    ev = _load("cfg4")  # no measurements, expectation values only
    assert ev.num_measurements == 0
    r = cb.run(ev, 5, 1, precision="fp64")
    assert r["exp_vals"].shape == (5, ev.num_exp_vals) and np.all(np.abs(r["exp_vals"]) <= 1.0)
    assert np.allclose(r["exp_vals"], r["exp_vals"][0])  # no randomness without measurements
