"""GPU parity: the CUDA executor through the C ABI against the oracle and the
reference's golden fixtures.

Tolerances (stated per the parity contract):
  * records, detector / observable bits, reachability, final frame and k:
    bit-exact under forced outcomes and injected faults (FP64 and FP32);
  * FP64: every measurement probability, log probability, gamma*v amplitude
    and expectation value within 1e-10 of the reference / oracle;
  * FP32: every measurement probability within 1e-5, expectation values and
    normalised final amplitudes within 1e-4 (relative to the state norm);
  * free sampling: FP64 bit-identical to the oracle running the same Philox
    streams; FP32 identical except for shots whose outcome threshold lies within
    FP32 rounding of a draw (< 1% of shots); statistics vs the reference's own
    sampler by TVD < 4 sqrt((2^m - 1) / N) and per-bit 5-sigma bounds.
"""

import glob
import math
import os

import numpy as np
import pytest

import clifft_b200 as cb
from _programs import random_forced_inputs, random_program
from clifft_b200 import workloads as W
from golden.make_golden import load_case, unflatten
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

CASES = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
IDS = [os.path.basename(c)[:-4] for c in CASES]


@pytest.fixture(scope="module", autouse=True)
def device():
    name = cb.backend_name()
    assert name.startswith("cuda:sm_100a"), f"no sm_100 device: {name}"
    return name


def unpack(words, n):
    return cb.api._unpack(words, n)


def amplitudes(gamma, v):
    g = gamma[:, 0] + 1j * gamma[:, 1]
    return g[:, None] * v


def forced_gpu(prog, fm, faults, ros, precision, group=0):
    return cb.run(prog, fm.shape[0], 0, precision=precision, forced_meas=fm, faults=faults,
                  readout_faults=ros, trace=True, dump_shots=fm.shape[0], group_threads=group)


@pytest.mark.parametrize("path", CASES, ids=IDS)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_forced_parity_vs_reference_golden(path, precision):
    prog, d = load_case(path)
    fm = d["forced_meas_in"]
    faults, ros = unflatten(d)
    g = forced_gpu(prog, fm, faults, ros, precision)
    reach = d["forced_reachable"].astype(bool)
    assert np.array_equal(g["survived"].astype(bool), reach & (d["forced_discarded"] == 0))
    ok = reach & (d["forced_discarded"] == 0)
    meas = unpack(g["meas_words"], prog.num_measurements)
    assert np.array_equal(meas[ok], d["forced_meas"][ok][:, :prog.num_measurements])
    assert np.array_equal(unpack(g["obs_words"], prog.num_observables)[ok], d["forced_obs"][ok])
    assert np.array_equal(unpack(g["det_words"], prog.num_detectors)[ok], d["forced_det"][ok])
    assert np.array_equal(g["final_k"][reach], d["forced_final_k"][reach])
    assert np.array_equal(g["final_px"][reach], d["forced_final_px"][reach])
    assert np.array_equal(g["final_pz"][reach], d["forced_final_pz"][reach])
    ptol = 1e-10 if precision == "fp64" else 1e-5
    ref_p, gpu_p = d["forced_meas_prob"][reach], g["meas_prob"][reach]
    assert np.array_equal(np.isnan(ref_p), np.isnan(gpu_p))
    np.testing.assert_allclose(np.nan_to_num(gpu_p), np.nan_to_num(ref_p), atol=ptol)
    ra = amplitudes(d["forced_final_gamma"], d["forced_final_v"])[reach]
    ga = amplitudes(g["final_gamma"], g["final_v"])[reach][:, :ra.shape[1]]
    atol = 1e-10 if precision == "fp64" else 1e-4
    np.testing.assert_allclose(ga, ra, atol=atol * max(1.0, np.abs(ra).max(initial=0.0)))
    if prog.num_exp_vals:
        np.testing.assert_allclose(g["exp_vals"][ok], d["forced_exp_vals"][ok],
                                   atol=1e-10 if precision == "fp64" else 1e-4)


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_free_sampling_fp64_bit_identical_to_oracle_philox(path):
    prog, d = load_case(path)
    shots = 512
    g = cb.run(prog, shots, 1234, precision="fp64", survivors=bool(prog.has_postselection))
    o = O.run(prog, shots, seed=1234, rng=O.RNG_PHILOX)
    keep = o["discarded"] == 0
    assert np.array_equal(g["survived"].astype(bool), keep)
    assert np.array_equal(unpack(g["meas_words"], prog.num_measurements)[keep], o["meas"][keep])
    assert np.array_equal(unpack(g["det_words"], prog.num_detectors)[keep], o["det"][keep])
    assert np.array_equal(unpack(g["obs_words"], prog.num_observables)[keep], o["obs"][keep])
    np.testing.assert_allclose(g["exp_vals"][keep], o["exp_vals"][keep], atol=1e-10)


@pytest.mark.parametrize("seed", range(6))
def test_free_sampling_fp32_matches_oracle_streams(seed):
    prog = O.ref_passes(random_program(seed, n=10, length=200, max_k=7), O.PASS_ALL) \
        if O.ref_available() else random_program(seed, n=10, length=200, max_k=7)
    shots = 2000
    g = cb.run(prog, shots, 99 + seed, precision="fp32")
    o = O.run(prog, shots, seed=99 + seed, rng=O.RNG_PHILOX)
    gm = unpack(g["meas_words"], prog.num_measurements)
    mismatched = np.any(gm != o["meas"], axis=1).mean()
    assert mismatched < 0.01


@pytest.mark.parametrize("group", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512])
def test_launch_shape_independence(group):
    prog, d = load_case(os.path.join(os.path.dirname(__file__), "golden", "fuzz_k9.npz"))
    base = cb.run(prog, 300, 5, precision="fp64", group_threads=0)
    g = cb.run(prog, 300, 5, precision="fp64", group_threads=group)
    assert g["group_threads"] == group
    assert np.array_equal(base["meas_words"], g["meas_words"])
    np.testing.assert_allclose(base["exp_vals"], g["exp_vals"], atol=1e-12)
    # forced replay is shape independent to rounding
    o = O.run(prog, 40, seed=9, rng=O.RNG_PHILOX)
    fm = np.zeros((40, prog.total_meas_slots), np.uint8)
    fm[:, :prog.num_measurements] = o["meas"]
    f = forced_gpu(prog, fm, None, None, "fp64", group)
    ref = O.run(prog, 40, forced_meas=fm, want_state=True)
    np.testing.assert_allclose(np.nan_to_num(f["meas_prob"]), np.nan_to_num(ref["meas_prob"]), atol=1e-10)
    np.testing.assert_allclose(amplitudes(f["final_gamma"], f["final_v"]),
                               amplitudes(ref["final_gamma"], ref["final_v"]), atol=1e-10)


@pytest.mark.parametrize("group", [32, 128, 256, 288, 512, 544])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_large_k_global_state_forced_parity(precision, group):
    # k = 17: 2^17 amplitudes per shot in a global slab, one warp per shot
    # (L2/HBM sweeps) or one CTA per shot (bulk-copy tile engine)
    prog = random_program(7, n=20, length=170, max_k=17, noise=False, classical=False,
                          expand_bias=0.5)
    assert prog.peak_rank >= 16
    o = O.run(prog, 4, seed=3, rng=O.RNG_PHILOX)
    fm = np.zeros((4, prog.total_meas_slots), np.uint8)
    fm[:, :prog.num_measurements] = o["meas"]
    ref = O.run(prog, 4, forced_meas=fm, want_state=True)
    g = forced_gpu(prog, fm, None, None, precision, group)
    assert g["group_threads"] == group and not g["state_in_smem"]
    assert np.array_equal(g["survived"].astype(bool), ref["reachable"].astype(bool))
    assert np.array_equal(g["final_k"], ref["final_k"])
    ptol = 1e-10 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(np.nan_to_num(g["meas_prob"]), np.nan_to_num(ref["meas_prob"]), atol=ptol)
    ra = amplitudes(ref["final_gamma"], ref["final_v"])
    ga = amplitudes(g["final_gamma"], g["final_v"])
    np.testing.assert_allclose(ga, ra, atol=(1e-10 if precision == "fp64" else 1e-4))


def test_survivors_match_oracle_and_counters():
    prog = O.ref_passes(W.lower(W.config1(), postselect_all=True), O.PASS_ALL) \
        if O.ref_available() else W.lower(W.config1(), postselect_all=True)
    shots = 20000
    r = cb.sample_survivors(prog, shots, seed=11, keep_records=True, precision="fp64")
    o = O.run(prog, shots, seed=11, rng=O.RNG_PHILOX)
    keep = o["discarded"] == 0
    assert r.passed_shots == int(keep.sum())
    assert r.total_shots == shots and r.discards == shots - r.passed_shots
    assert np.array_equal(r.measurements, o["meas"][keep])
    assert np.array_equal(r.observables, o["obs"][keep])
    assert r.logical_errors == int(np.any(o["obs"][keep], axis=1).sum())
    r32 = cb.sample_survivors(prog, shots, seed=11, precision="fp32")
    assert abs(r32.passed_shots - r.passed_shots) <= max(3, 0.002 * shots)


def test_free_sampling_tvd_vs_reference_histogram():
    # 6 measured bits: full outcome histogram, TVD bound of the reference's own
    # statistical tests (tests/python/test_statistical_equivalence.py:556-635)
    prog = None
    for s in range(200):
        p = random_program(300 + s, n=8, length=60, max_k=5, noise=True, classical=False,
                           expvals=False, readout=False)
        if 4 <= p.num_measurements <= 8:
            prog = p
            break
    assert prog is not None
    n_ref, n_gpu = 200_000, 200_000
    ref = O.run(prog, n_ref, seed=5, rng=O.RNG_XOSHIRO)["meas"]
    gpu = cb.sample(prog, n_gpu, seed=6, precision="fp32").measurements
    m = prog.num_measurements
    w = 1 << np.arange(m)
    h_ref = np.bincount(ref @ w, minlength=1 << m) / n_ref
    h_gpu = np.bincount(gpu @ w, minlength=1 << m) / n_gpu
    tvd = 0.5 * np.abs(h_ref - h_gpu).sum()
    assert tvd < 4 * math.sqrt(((1 << m) - 1) / min(n_ref, n_gpu))


def test_cfg0_marginals_vs_reference_sampler():
    prog = W.lower(W.config0())
    n = 100_000
    ref = O.run(prog, 20_000, seed=42, rng=O.RNG_XOSHIRO)["meas"].mean(0)
    res = cb.sample(prog, n, seed=1, precision="fp64")
    assert res.measurements.shape == (n, prog.num_measurements)
    gpu = res.measurements.mean(0)
    sigma = np.sqrt(np.maximum(ref * (1 - ref), 1e-4) * (1 / 20_000 + 1 / n))
    assert np.all(np.abs(gpu - ref) < 5 * sigma + 1e-9)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-4)])
def test_expectation_values_cfg4(precision, tol):
    c, _ = W.config4()
    prog = W.lower(c)
    o = O.run(prog, 1, seed=0)
    g = cb.run(prog, 4, 0, precision=precision)
    np.testing.assert_allclose(g["exp_vals"], np.repeat(o["exp_vals"], 4, axis=0), atol=tol)


def test_record_probabilities_match_oracle():
    prog = random_program(21, n=10, length=150, max_k=6, noise=False, classical=False)
    o = O.run(prog, 64, seed=2, rng=O.RNG_PHILOX)
    rec = o["meas"].copy()
    rec[::4] ^= 1
    lp = cb.record_probabilities(prog, rec)
    f = O.run(prog, 64, forced_meas=rec)
    reach = f["reachable"].astype(bool)
    assert np.all(lp[~reach] == np.finfo(np.float64).min)
    np.testing.assert_allclose(lp[reach], f["log_prob"][reach], atol=1e-10)


@pytest.mark.parametrize("group", [32, 128, 256, 288, 512, 544])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fused_tile_sweeps_match_unfused(precision, group):
    # k = 16 with the reference's U2 / U4 / MULTI nodes: fused blocks perform
    # each amplitude's arithmetic in the same order as one sweep per opcode
    # (micro-ops, EXPAND copies, the H that folds an X-basis measurement, the
    # b = 1 half kept by relabelling instead of copying), so the final
    # amplitudes agree bit for bit. A fused block sums a measurement's
    # half-norms in another order than the measurement's own pass (and an
    # X-basis measurement sums |(x +- y) / sqrt2|^2, rounded to the
    # statevector's precision, where the pass sums |x +- y|^2), so
    # probabilities and gamma agree to FP64 rounding in FP64 (1e-13) and to
    # 1e-8 in FP32.
    # (A warp per shot streams 4 KiB tiles through two buffers, 128 / 256 /
    # 512-thread CTAs 32 KiB tiles through two / three / four; 288 / 544-thread
    # CTAs compute with 256 / 512 threads while their last warp issues the
    # copies.)
    prog, d = load_case(os.path.join(os.path.dirname(__file__), "golden", "fuzz_k16.npz"))
    fm = d["forced_meas_in"]
    faults, ros = unflatten(d)
    n = fm.shape[0]
    kw = dict(precision=precision, forced_meas=fm, faults=faults, readout_faults=ros, trace=True,
              dump_shots=n, group_threads=group)  # fusion is a feature of one-shot groups (tile engine)
    a = cb.run(prog, n, 0, fusion=True, **kw)
    b = cb.run(prog, n, 0, fusion=False, **kw)
    assert a["fused"] and not b["fused"]
    assert a["streamed_bytes"] < b["streamed_bytes"]
    assert a["algorithmic_bytes"] == b["algorithmic_bytes"]
    assert np.array_equal(a["survived"], b["survived"])
    assert np.array_equal(a["meas_words"], b["meas_words"])
    assert np.array_equal(a["final_k"], b["final_k"])
    assert np.array_equal(a["final_v"], b["final_v"])
    tol = 1e-13 if precision == "fp64" else 1e-8
    np.testing.assert_allclose(a["final_gamma"], b["final_gamma"], rtol=tol, atol=0)
    pa, pb = np.nan_to_num(a["meas_prob"], nan=-1.0), np.nan_to_num(b["meas_prob"], nan=-1.0)
    np.testing.assert_allclose(pa, pb, rtol=0, atol=tol)
    fa = cb.run(prog, 64, 3, precision=precision, fusion=True)
    fb = cb.run(prog, 64, 3, precision=precision, fusion=False)
    assert np.array_equal(fa["meas_words"], fb["meas_words"])


def test_resident_cap_gives_the_same_records():
    # max_resident bounds the statevectors held at once (shots then run in
    # waves); per-shot Philox streams make the records independent of it
    prog = O.ref_passes(random_program(7, n=20, length=170, max_k=17, noise=False, classical=False,
                                       expand_bias=0.5), O.PASS_ALL) if O.ref_available() else \
        random_program(7, n=20, length=170, max_k=17, noise=False, classical=False, expand_bias=0.5)
    a = cb.run(prog, 600, 9, precision="fp64", group_threads=256)
    b = cb.run(prog, 600, 9, precision="fp64", group_threads=256, max_resident=40)
    assert np.array_equal(a["meas_words"], b["meas_words"])
    np.testing.assert_allclose(a["exp_vals"], b["exp_vals"], atol=1e-12)
