"""k-fault importance sampling (clifft_gpu_sample_k) against the reference's
clifft::sample_k: stratum validation, survivor fractions, and detector /
observable statistics of the k = 1 / 2 strata in both the Poisson-binomial
(DP) and the uniform-subset modes, within 5-sigma binomial bounds."""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import Program
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


def _grid():
    return Program.load(os.path.join(PROGRAMS, "cfg1.npz"))


def _uniform_grid():
    """The memory grid with every fault site at total probability 15 * 2^-14
    exactly (channels rescaled), so both samplers use uniform k-subsets."""
    p = _grid()
    d = p.to_npz_dict()
    off = p.noise_site_offsets.astype(np.int64)
    cp = p.noise_channel_prob.copy()
    for i in range(len(off) - 1):
        n = off[i + 1] - off[i]
        assert 15 % n == 0
        cp[off[i]:off[i + 1]] = (15 // n) * 2.0 ** -14
    d["noise_channel_prob"] = cp
    d["readout_prob"] = np.full_like(p.readout_prob, 15 * 2.0 ** -14)
    q = Program.from_npz_dict(d)
    pr = cb.noise_site_probabilities(q)
    assert np.all(pr == pr[0])
    return q


def _no_postselect(p):
    d = p.to_npz_dict()
    ins = p.instructions.copy()
    ins[ins[:, 0] == cb.OP["POSTSELECT"], 0] = cb.OP["DETECTOR"]
    d["instructions"] = ins
    d["has_postselection"] = np.array(0)
    return Program.from_npz_dict(d)


def _close(a, b, n1, n2):
    p = (a * n1 + b * n2) / (n1 + n2)
    tol = 5 * np.sqrt(np.maximum(p * (1 - p), 1e-12) * (1 / n1 + 1 / n2)) + 1e-4
    return np.all(np.abs(a - b) <= tol), np.max(np.abs(a - b) - tol)


def test_noise_site_probabilities_match_reference():
    p = _grid()
    np.testing.assert_allclose(cb.noise_site_probabilities(p), O.ref_noise_site_probabilities(p), rtol=1e-12)


def test_stratum_validation():
    p = _grid()
    n = len(cb.noise_site_probabilities(p))
    with pytest.raises(ValueError, match="exceeds total fault sites"):
        cb.sample_k(_no_postselect(p), 10, n + 1, seed=1)
    d = p.to_npz_dict()
    cp = p.noise_channel_prob.copy()
    lo, hi = int(p.noise_site_offsets[0]), int(p.noise_site_offsets[1])
    cp[lo:hi] = 0.0
    cp[lo] = 1.0  # a site that always fires: the k = 0 stratum has no mass
    d["noise_channel_prob"] = cp
    q = _no_postselect(Program.from_npz_dict(d))
    with pytest.raises(ValueError, match="zero probability mass"):
        cb.sample_k(q, 10, 0, seed=1)


@pytest.mark.parametrize("k", [0, 1])
def test_survivor_fraction_matches_reference(k):
    # the grid's magic gates make detectors fire even in the fault-free stratum
    p = _grid()
    n_gpu, n_ref = 100_000, 50_000
    r = cb.sample_k_survivors(p, n_gpu, k, seed=3, keep_records=False)
    ref = O.ref_sample_k(_no_postselect(p), n_ref, k, 4)
    ok, worst = _close(np.array([r.passed_shots / n_gpu]),
                       np.array([(ref["det"].sum(axis=1) == 0).mean()]), n_gpu, n_ref)
    assert ok, worst


@pytest.mark.parametrize("mode,k", [("dp", 1), ("dp", 2), ("uniform", 2)])
def test_detector_statistics_match_reference_sample_k(mode, k):
    p = _no_postselect(_grid() if mode == "dp" else _uniform_grid())
    n_gpu, n_ref = 200_000, 100_000
    g = cb.sample_k(p, n_gpu, k, seed=11, precision="fp64")
    ref = O.ref_sample_k(p, n_ref, k, 12)
    ok, worst = _close(g.detectors.mean(axis=0), ref["det"].mean(axis=0), n_gpu, n_ref)
    assert ok, worst
    # number of fired detectors per shot: same histogram (first few bins)
    hg = np.bincount(g.detectors.sum(axis=1), minlength=8)[:8] / n_gpu
    hr = np.bincount(ref["det"].sum(axis=1), minlength=8)[:8] / n_ref
    ok, worst = _close(hg, hr, n_gpu, n_ref)
    assert ok, worst
    ok, worst = _close(g.observables.mean(axis=0), ref["obs"].mean(axis=0), n_gpu, n_ref)
    assert ok, worst


def test_sample_k_is_deterministic_and_shards():
    p = _no_postselect(_grid())
    a = cb.run(p, 3000, 5, precision="fp64", k_faults=2)
    b = cb.run(p, 3000, 5, precision="fp64", k_faults=2)
    assert np.array_equal(a["det_words"], b["det_words"])
    lo = cb.run(p, 1000, 5, precision="fp64", k_faults=2)
    hi = cb.run(p, 2000, 5, precision="fp64", k_faults=2, first_shot=1000)
    assert np.array_equal(np.concatenate([lo["det_words"], hi["det_words"]]), a["det_words"])
