"""Launch-shape autotuning (group_threads == 0): the first large call of a
(precision, mode) pair times candidate shapes on its own shots and keeps the
fastest on the program handle; results are those of any fixed shape."""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import Program

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


def _prog(name):
    return Program.load(os.path.join(PROGRAMS, f"{name}.npz"))


@pytest.mark.parametrize("name", ["cfg2_36", "cfg0"])
def test_autotune_picks_a_candidate_and_matches_fixed_shapes(name):
    prog = _prog(name)
    shots = 4096
    fixed = cb.run(prog, shots, 21, precision="fp64", autotune=False)
    first = cb.run(prog, shots, 21, precision="fp64")
    assert first["kernel_launches"] > 1  # trial launches ran
    again = cb.run(prog, shots, 21, precision="fp64")
    assert again["kernel_launches"] == 1  # cached for this program content
    assert again["group_threads"] == first["group_threads"]
    for r in (first, again):
        assert np.array_equal(r["meas_words"], fixed["meas_words"])
        assert np.array_equal(r["survived"], fixed["survived"])
        np.testing.assert_allclose(r["exp_vals"], fixed["exp_vals"], atol=1e-12)


def test_tuning_is_shared_by_handles_of_the_same_program():
    a = _prog("cfg2_12")
    cb.run(a, 4096, 3, precision="fp32")
    b = _prog("cfg2_12")  # a second upload of the same content
    r = cb.run(b, 4096, 3, precision="fp32")
    assert r["kernel_launches"] == 1


def test_small_calls_do_not_tune():
    prog = _prog("cfg2_20")
    r = cb.run(prog, 200, 1, precision="fp32")
    assert r["kernel_launches"] == 1


def test_tune_cache_file_is_written_and_read_by_a_later_process(tmp_path):
    import subprocess
    import sys
    cache = tmp_path / "tune.txt"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, %r); import clifft_b200 as cb; from clifft_b200.program import Program; "
            "p = Program.load(%r); r = cb.run(p, 4096, 1, precision='fp32'); print(r['kernel_launches'])"
            % (root, os.path.join(PROGRAMS, "cfg2_15.npz")))
    env = dict(os.environ, CLIFFT_GPU_TUNE_CACHE=str(cache))
    first = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    assert int(first.stdout.split()[-1]) > 1 and cache.read_text().strip()
    second = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, check=True)
    assert int(second.stdout.split()[-1]) == 1  # shape read from the file, no trials
