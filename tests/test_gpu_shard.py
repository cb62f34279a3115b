"""The GPU shard of a multi-GPU run: sampling global shots [a, b) through
`first_shot` gives exactly the rows of a single call over [0, N)."""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200 import shard
from clifft_b200.program import Program

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_shards_concatenate_to_one_call(precision):
    prog = Program.load(os.path.join(PROGRAMS, "cfg1.npz"))
    total, seed, world = 5001, 23, 3
    whole = shard.gpu_sampler(prog, total, seed, 0, precision, True)
    parts = [shard.gpu_sampler(prog, n, seed, first, precision, True)
             for first, n in (shard.shard_range(total, world, r) for r in range(world))]
    merged = shard.merge(parts)
    for key in ("meas_words", "det_words", "obs_words", "survived"):
        assert np.array_equal(merged[key], whole[key]), key
    assert merged["passed_shots"] == whole["passed_shots"]
    assert np.array_equal(merged["observable_ones"], whole["observable_ones"])


def test_sample_sharded_without_process_group_is_one_shard():
    prog = Program.load(os.path.join(PROGRAMS, "cfg0.npz"))
    r = shard.sample_sharded(prog, 1000, 5, precision="fp64")
    direct = cb.run(prog, 1000, 5, precision="fp64")
    assert np.array_equal(r["meas_words"], direct["meas_words"])
