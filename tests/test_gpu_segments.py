"""Survivor compaction between POSTSELECT segments: a run cut into segments
(shots alive at a cut carried over, the rest dropped) returns the same records
and counters as one launch, and the FP64 run matches the oracle's streams."""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import Program
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_segmented_survivor_run_equals_one_launch(precision):
    prog = Program.load(os.path.join(PROGRAMS, "cfg1.npz"))
    shots = 600_000  # several resident waves: the segmented path is taken
    seg = cb.run(prog, shots, 31, precision=precision, survivors=True)
    one = cb.run(prog, shots, 31, precision=precision, survivors=True, segments=False)
    assert seg["kernel_launches"] > one["kernel_launches"]  # segments ran as separate launches
    for key in ("meas_words", "det_words", "obs_words", "survived"):
        assert np.array_equal(seg[key], one[key]), key
    assert seg["passed_shots"] == one["passed_shots"] and seg["logical_errors"] == one["logical_errors"]
    assert np.array_equal(seg["observable_ones"], one["observable_ones"])
    assert seg["algorithmic_bytes"] == one["algorithmic_bytes"]


def test_segmented_fp64_matches_oracle_streams():
    prog = Program.load(os.path.join(PROGRAMS, "cfg1.npz"))
    shots = 400_000
    g = cb.run(prog, shots, 7, precision="fp64", survivors=True)
    assert g["kernel_launches"] > 1
    o = O.run(prog, shots, seed=7, rng=O.RNG_PHILOX)
    keep = o["discarded"] == 0
    assert np.array_equal(g["survived"].astype(bool), keep)
    gm = cb.api._unpack(g["meas_words"], prog.num_measurements)
    assert np.array_equal(gm[keep], o["meas"][keep])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_segmented_warp_tile_run_equals_one_launch(precision):
    # peak k = 13: one warp per shot with a global statevector, streamed
    # through the warp's 4 KiB tiles; shots alive at a cut carry 2^k
    # amplitudes between segment launches
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from _programs import random_program
    prog = random_program(21, n=18, length=400, max_k=13, postselect=True, expand_bias=0.2)
    assert prog.peak_rank == 13
    shots = 12_000  # > 4 resident waves of 16 warps on every SM
    seg = cb.run(prog, shots, 19, precision=precision, survivors=True, group_threads=32)
    one = cb.run(prog, shots, 19, precision=precision, survivors=True, group_threads=32, segments=False)
    assert seg["state_in_smem"] == 0 and seg["fused"]
    assert seg["kernel_launches"] > one["kernel_launches"]
    for key in ("meas_words", "det_words", "obs_words", "survived", "exp_vals"):
        assert np.array_equal(seg[key], one[key]), key
    assert seg["passed_shots"] == one["passed_shots"] > 0
    if precision == "fp64":
        n = 300  # per-shot Philox streams: the first shots of the run equal an oracle run of n shots
        o = O.run(prog, n, seed=19, rng=O.RNG_PHILOX)
        keep = o["discarded"] == 0
        assert np.array_equal(seg["survived"][:n].astype(bool), keep)
        gm = cb.api._unpack(seg["meas_words"][:n], prog.num_measurements)
        assert np.array_equal(gm[keep], o["meas"][keep])
