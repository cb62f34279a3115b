"""Pins the C oracle restatement to the reference executor built from its own
sources (oracle/_ref/libclifft_ref.so): bit-identical sampling streams,
survivor counts and forced replays on random programs, raw and after the
reference's bytecode passes. Skipped where the reference harness was not built."""

import numpy as np
import pytest

from _programs import random_forced_inputs, random_program
from oracle import pyoracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")


@pytest.mark.parametrize("seed", range(16))
@pytest.mark.parametrize("passes", [0, O.PASS_ALL])
def test_sampling_stream_matches_reference(seed, passes):
    p = random_program(seed, n=10, length=180, max_k=6, postselect=(seed % 4 == 3))
    q = O.ref_passes(p, passes) if passes else p
    o = O.run(q, 200, seed=seed, rng=O.RNG_XOSHIRO)
    if q.has_postselection:
        r = O.ref_sample_survivors(q, 200, seed, keep_records=True)
        keep = o["discarded"] == 0
        assert r["passed_shots"] == int(keep.sum())
        assert np.array_equal(r["meas"], o["meas"][keep])
        assert np.array_equal(r["obs"], o["obs"][keep])
    else:
        r = O.ref_sample(q, 200, seed)
        for key in ("meas", "det", "obs"):
            assert np.array_equal(r[key], o[key]), key
        np.testing.assert_allclose(r["exp_vals"], o["exp_vals"], atol=1e-12)


@pytest.mark.parametrize("seed", range(12))
def test_forced_replay_matches_reference(seed):
    q = O.ref_passes(random_program(seed + 50, n=10, length=180, max_k=6), O.PASS_ALL)
    o = O.run(q, 30, seed=seed, rng=O.RNG_PHILOX)
    fm = np.zeros((30, q.total_meas_slots), np.uint8)
    fm[:, :q.num_measurements] = o["meas"]
    fm[::6] ^= 1
    faults, ros = random_forced_inputs(q, 30, seed)
    r = O.ref_forced(q, fm, faults, ros)
    f = O.run(q, 30, forced_meas=fm, faults=faults, readout_faults=ros, want_state=True)
    for key in ("reachable", "final_k", "final_px", "final_pz", "det", "obs"):
        assert np.array_equal(r[key], f[key]), key
    np.testing.assert_allclose(r["log_prob"], f["log_prob"], atol=1e-10)
    np.testing.assert_allclose(r["final_gamma"], f["final_gamma"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(r["final_v"], f["final_v"], atol=1e-10)
    np.testing.assert_allclose(r["exp_vals"], f["exp_vals"], atol=1e-10)
    assert np.array_equal(np.isnan(r["meas_prob"]), np.isnan(f["meas_prob"]))
    np.testing.assert_allclose(np.nan_to_num(r["meas_prob"]), np.nan_to_num(f["meas_prob"]), atol=1e-12)


def test_workload_programs_match_reference():
    from clifft_b200 import workloads as W
    p = O.ref_passes(W.lower(W.config0()), O.PASS_ALL)
    r = O.ref_sample(p, 1000, 7)
    o = O.run(p, 1000, seed=7, rng=O.RNG_XOSHIRO)
    assert np.array_equal(r["meas"], o["meas"])
    p1 = O.ref_passes(W.lower(W.config1(), postselect_all=True), O.PASS_ALL)
    r1 = O.ref_sample_survivors(p1, 3000, 3)
    o1 = O.run(p1, 3000, seed=3, rng=O.RNG_XOSHIRO)
    assert r1["passed_shots"] == int((o1["discarded"] == 0).sum())
