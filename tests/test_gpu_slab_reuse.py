"""Statevector slabs across program uploads: a program uploaded again after
others ran (and were released) samples the same records, and clifft_gpu_trim
is safe to call at any point. Each shot initialises its own state, so records
must not depend on what device memory held before."""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import Program

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


@pytest.mark.parametrize("name,group", [("cfg2_36", 0), ("dense_k20", 288)])
def test_parked_slab_serves_the_next_upload(name, group):
    path = os.path.join(PROGRAMS, f"{name}.npz")
    shots = 300
    first = Program.load(path)
    want = cb.run(first, shots, 21, precision="fp32", group_threads=group)
    first._device_program.free()
    other = Program.load(os.path.join(PROGRAMS, "cfg2_01.npz"))
    cb.run(other, 64, 3, precision="fp32")  # other statevectors in device memory
    other._device_program.free()
    again = Program.load(path)
    got = cb.run(again, shots, 21, precision="fp32", group_threads=group)
    for key in ("meas_words", "det_words", "obs_words", "survived"):
        assert np.array_equal(got[key], want[key]), key
    again._device_program.free()
    cb.trim()
    last = Program.load(path)
    after = cb.run(last, shots, 21, precision="fp32", group_threads=group)
    assert np.array_equal(after["meas_words"], want["meas_words"])
