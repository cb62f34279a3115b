"""The oracle against golden fixtures recorded from the reference executor
(tests/golden/make_golden.py). Runs where the reference tree is absent."""

import glob
import os

import numpy as np
import pytest

from golden.make_golden import load_case, unflatten
from oracle import pyoracle as O

CASES = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def test_fixtures_present():
    assert len(CASES) >= 10


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c)[:-4] for c in CASES])
def test_oracle_matches_golden(path):
    prog, d = load_case(path)
    seed = int(d["sample_seed"])
    o = O.run(prog, 256, seed=seed, rng=O.RNG_XOSHIRO)
    if "sample_meas" in d:
        assert np.array_equal(o["meas"], d["sample_meas"])
        assert np.array_equal(o["det"], d["sample_det"])
        assert np.array_equal(o["obs"], d["sample_obs"])
        np.testing.assert_allclose(o["exp_vals"], d["sample_exp_vals"], atol=1e-12)
    else:
        keep = o["discarded"] == 0
        assert int(keep.sum()) == int(d["surv_passed_shots"])
        assert np.array_equal(o["meas"][keep], d["surv_meas"])
    faults, ros = unflatten(d)
    f = O.run(prog, d["forced_meas_in"].shape[0], forced_meas=d["forced_meas_in"], faults=faults,
              readout_faults=ros, want_state=True)
    for key in ("reachable", "final_k", "final_px", "final_pz"):
        assert np.array_equal(f[key], d[f"forced_{key}"]), key
    np.testing.assert_allclose(f["log_prob"], d["forced_log_prob"], atol=1e-10)
    np.testing.assert_allclose(f["final_v"][:, :d["forced_final_v"].shape[1]], d["forced_final_v"],
                               atol=1e-10)
    np.testing.assert_allclose(f["final_gamma"], d["forced_final_gamma"], rtol=1e-10, atol=1e-10)
