"""Parity of the benchmarked programs against the reference executor.

The programs the benchmark times (tests/golden/programs: the k = 24 program
cfg3, the k = 16 / 18 seed programs cfg2_36 / cfg2_01, the noisy memory grid
cfg1 and the k = 8 program cfg0) are replayed shot by shot through the
reference's own executor (oracle/_ref, built from src/clifft/svm/*.cc and
src/clifft/api/record_probabilities.cc) under the same forced outcomes and
injected faults as the GPU run (forced replay as in
src/clifft/api/record_probabilities.cc:96-191, forced kernels
src/clifft/svm/svm_forced_kernels.cc:112-304).

Tolerances:
  * records, detector / observable bits, survival, final frame and k: bit-exact
    in both precisions;
  * every measurement probability: 1e-10 (FP64 statevector), 1e-5 (FP32);
  * amplitudes at peak rank (a prefix of the program that ends where k first
    reaches its peak): gamma*v within 1e-10 of the reference in FP64; in FP32
    every normalised amplitude within 1e-5 of the reference's largest
    amplitude, relative L2 error below 1e-5 and overlap 1 - |<a|b>| below 1e-9.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import ACTIVE_MEAS, Program
from oracle import pyoracle as O

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_available(), reason="reference executor (oracle/_ref) not built")]

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")
PTOL = {"fp64": 1e-10, "fp32": 1e-5}


def _load(name):
    return Program.load(os.path.join(PROGRAMS, f"{name}.npz"))


def _faults(prog, shots, seed):
    """Up to three injected noise events and one readout flip per shot."""
    rng = np.random.default_rng(seed)
    off = prog.noise_site_offsets
    nsites = len(off) - 1
    faults, ros = [], []
    for _ in range(shots):
        sites = sorted(rng.choice(nsites, size=min(nsites, int(rng.integers(0, 4))), replace=False).tolist()) \
            if nsites else []
        faults.append([(s, int(rng.integers(0, off[s + 1] - off[s]))) for s in sites])
        nro = len(prog.readout_meas_idx)
        ros.append(sorted(rng.choice(nro, size=min(nro, int(rng.integers(0, 2))), replace=False).tolist())
                   if nro else [])
    return faults, ros


def _outcomes(prog, shots, seed, faults, ros):
    """Outcomes of a free FP64 run under the injected faults: a trajectory
    the forced replay can follow."""
    r = cb.run(prog, shots, seed, precision="fp64", faults=faults, readout_faults=ros)
    bits = cb.api._unpack(r["meas_words"], prog.num_measurements)
    fm = np.zeros((shots, prog.total_meas_slots), np.uint8)
    fm[:, :prog.num_measurements] = bits
    return fm


def _prefix(prog, n):
    d = prog.to_npz_dict()
    d["instructions"] = prog.instructions[:n].copy()
    return Program.from_npz_dict(d)


def _peak_cut(prog):
    """Index of the first active measurement after k first reaches the peak
    (the prefix before it ends with the state at peak rank)."""
    hist = prog.active_k_history()
    ops = prog.opcodes.tolist()
    first = int(np.argmax(hist == prog.peak_rank))
    for pc in range(first, len(ops)):
        if ops[pc] in ACTIVE_MEAS:
            return pc
    return len(ops)


@pytest.mark.parametrize("name,shots", [("cfg3", 2), ("cfg2_36", 6), ("cfg2_01", 4), ("cfg1", 24), ("cfg0", 24)])
def test_benchmarked_program_forced_parity_vs_reference(name, shots):
    prog = _load(name)
    noisy = len(prog.noise_site_offsets) > 1 or len(prog.readout_meas_idx) > 0
    faults, ros = _faults(prog, shots, 11) if noisy else (None, None)
    fm = _outcomes(prog, shots, 5, faults, ros)
    ref = O.ref_forced(prog, fm, faults, ros)
    reach = ref["reachable"].astype(bool)
    ok = reach & (ref["discarded"] == 0)
    assert reach.all(), "a trajectory of the GPU run is unreachable in the reference"
    for precision in ("fp64", "fp32"):
        g = cb.run(prog, shots, 0, precision=precision, forced_meas=fm, faults=faults, readout_faults=ros,
                   trace=True)
        assert np.array_equal(g["survived"].astype(bool), ok), precision
        meas = cb.api._unpack(g["meas_words"], prog.num_measurements)
        assert np.array_equal(meas[ok], ref["meas"][ok][:, :prog.num_measurements]), precision
        assert np.array_equal(cb.api._unpack(g["det_words"], prog.num_detectors)[ok], ref["det"][ok])
        assert np.array_equal(cb.api._unpack(g["obs_words"], prog.num_observables)[ok], ref["obs"][ok])
        assert np.array_equal(g["final_k"], ref["final_k"]), precision
        assert np.array_equal(g["final_px"], ref["final_px"]) and np.array_equal(g["final_pz"], ref["final_pz"])
        rp, gp = ref["meas_prob"], g["meas_prob"]
        assert np.array_equal(np.isnan(rp), np.isnan(gp)), precision
        err = float(np.max(np.abs(np.nan_to_num(gp) - np.nan_to_num(rp)), initial=0.0))
        assert err <= PTOL[precision], f"{name} {precision}: largest probability error {err:.3e}"
        np.testing.assert_allclose(g["log_prob"][reach], ref["log_prob"][reach],
                                   atol=1e-9 if precision == "fp64" else 1e-3)


@pytest.mark.parametrize("name", ["cfg3", "cfg2_36", "cfg2_01"])
def test_amplitudes_at_peak_rank_vs_reference(name):
    prog = _load(name)
    pre = _prefix(prog, _peak_cut(prog))
    shots = 2
    fm = _outcomes(pre, shots, 3, None, None)
    ref = O.ref_forced(pre, fm)
    k = int(ref["final_k"][0])
    assert k == prog.peak_rank and np.all(ref["final_k"] == k)
    ra = (ref["final_gamma"][:, 0] + 1j * ref["final_gamma"][:, 1])[:, None] * ref["final_v"][:, :1 << k]
    del ref
    for precision in ("fp64", "fp32"):
        g = cb.run(pre, shots, 0, precision=precision, forced_meas=fm, trace=True, dump_shots=shots)
        assert np.array_equal(g["final_k"], np.full(shots, k))
        v = g["final_v"][:, :1 << k]
        ga = (g["final_gamma"][:, 0] + 1j * g["final_gamma"][:, 1])[:, None] * v
        del g, v
        for s in range(shots):
            a, b = ga[s], ra[s]
            nb = np.linalg.norm(b)
            if precision == "fp64":
                np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * np.abs(b).max())
                continue
            an, bn = a / np.linalg.norm(a), b / nb
            assert np.abs(an - bn).max() <= 1e-5 * np.abs(bn).max(), name
            assert np.linalg.norm(a - b) / nb <= 1e-5, name
            assert 1.0 - abs(np.vdot(an, bn)) <= 1e-9, name
        del ga
