"""Dense blocks on the tensor cores (CLIFFT_GPU_TENSOR_DENSE) against the
reference executor.

With the flag, a fused block's run of micro-ops on at most four tile-local
bits that holds an H / U2 / U4 is composed into one 16 x 16 complex matrix
(one per shot: the frame-dependent node matrices of
src/clifft/svm/svm_kernels.inl:1087-1531 are chosen first) and applied as
3xTF32 MMAs. The arithmetic differs from the CUDA-core path, so the checks
are tolerances, not bit equality:

  * forced replay (src/clifft/api/record_probabilities.cc:96-191) of the
    dense k = 20 program and of a dense k = 16 program: records, final k and
    frame bit-exact, every measurement probability within 1e-5 of the
    reference's, log probability within 1e-3;
  * amplitudes at peak rank: every normalised amplitude within 1e-4 of the
    reference's largest, relative L2 error below 1e-5, and different from the
    CUDA-core FP32 path (the tensor-core path ran);
  * free sampling: the records of the dense path equal the CUDA-core path's
    except where a draw falls within rounding of a branch threshold (< 1 %);
  * configured programs (CNOT / CZ / SWAP / phase gates only) form no dense
    run: the flag leaves their results bit-identical.
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
GROUPS = [256, 288, 512]


def _load(name):
    return Program.load(os.path.join(PROGRAMS, f"{name}.npz"))


def _dense_k16():
    from _programs import random_program
    return O.ref_passes(random_program(501, n=20, length=700, max_k=16, noise=False, classical=False,
                                       expvals=False, readout=False, expand_bias=0.2), O.PASS_ALL)


def _outcomes(prog, shots, seed):
    r = cb.run(prog, shots, seed, precision="fp64")
    fm = np.zeros((shots, prog.total_meas_slots), np.uint8)
    fm[:, :prog.num_measurements] = cb.api._unpack(r["meas_words"], prog.num_measurements)
    return fm


def _peak_prefix(prog):
    hist = prog.active_k_history()
    ops = prog.opcodes.tolist()
    first = int(np.argmax(hist == prog.peak_rank))
    cut = next((pc for pc in range(first, len(ops)) if ops[pc] in ACTIVE_MEAS), len(ops))
    d = prog.to_npz_dict()
    d["instructions"] = prog.instructions[:cut].copy()
    return Program.from_npz_dict(d)


@pytest.mark.parametrize("group", GROUPS)
@pytest.mark.parametrize("which", ["dense_k20", "dense_k16"])
def test_dense_forced_parity_vs_reference(which, group):
    prog = _load(which) if which == "dense_k20" else _dense_k16()
    assert prog.peak_rank == (20 if which == "dense_k20" else 16)
    shots = 4
    fm = _outcomes(prog, shots, 5)
    ref = O.ref_forced(prog, fm)
    assert ref["reachable"].all()
    g = cb.run(prog, shots, 0, precision="fp32", forced_meas=fm, trace=True, group_threads=group,
               tensor_dense=True)
    assert np.all(g["survived"] == 1)
    assert np.array_equal(cb.api._unpack(g["meas_words"], prog.num_measurements),
                          ref["meas"][:, :prog.num_measurements])
    assert np.array_equal(g["final_k"], ref["final_k"])
    assert np.array_equal(g["final_px"], ref["final_px"]) and np.array_equal(g["final_pz"], ref["final_pz"])
    rp, gp = ref["meas_prob"], g["meas_prob"]
    assert np.array_equal(np.isnan(rp), np.isnan(gp))
    err = float(np.max(np.abs(np.nan_to_num(gp) - np.nan_to_num(rp)), initial=0.0))
    assert err <= 1e-5, f"{which} group {group}: largest probability error {err:.3e}"
    np.testing.assert_allclose(g["log_prob"], ref["log_prob"], atol=1e-3)


@pytest.mark.parametrize("group", [256, 288])
def test_dense_amplitudes_at_peak_rank_vs_reference(group):
    pre = _peak_prefix(_load("dense_k20"))
    shots = 2
    fm = _outcomes(pre, shots, 3)
    ref = O.ref_forced(pre, fm)
    k = int(ref["final_k"][0])
    assert k == 20
    ra = (ref["final_gamma"][:, 0] + 1j * ref["final_gamma"][:, 1])[:, None] * ref["final_v"][:, :1 << k]
    del ref
    out = {}
    for dense in (True, False):
        g = cb.run(pre, shots, 0, precision="fp32", forced_meas=fm, trace=True, dump_shots=shots,
                   group_threads=group, tensor_dense=dense)
        assert np.array_equal(g["final_k"], np.full(shots, k))
        out[dense] = (g["final_gamma"][:, 0] + 1j * g["final_gamma"][:, 1])[:, None] * g["final_v"][:, :1 << k]
        del g
    assert not np.array_equal(out[True], out[False]), "the dense path left the CUDA-core arithmetic unchanged"
    for s in range(shots):
        a, b = out[True][s], ra[s]
        an, bn = a / np.linalg.norm(a), b / np.linalg.norm(b)
        assert np.abs(an - bn).max() <= 1e-4 * np.abs(bn).max()
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5


def test_dense_free_sampling_matches_the_cuda_core_path():
    prog = _load("dense_k20")
    shots = 296
    a = cb.run(prog, shots, 17, precision="fp32", group_threads=288, tensor_dense=True)
    b = cb.run(prog, shots, 17, precision="fp32", group_threads=288)
    ma = cb.api._unpack(a["meas_words"], prog.num_measurements)
    mb = cb.api._unpack(b["meas_words"], prog.num_measurements)
    rows = np.any(ma != mb, axis=1)
    assert rows.mean() < 0.01, f"{rows.sum()} of {shots} shots differ"


@pytest.mark.parametrize("name", ["cfg2_36", "cfg3"])
def test_configured_programs_form_no_dense_run(name):
    prog = _load(name)
    shots = 4
    a = cb.run(prog, shots, 9, precision="fp32", group_threads=288, trace=True, tensor_dense=True)
    b = cb.run(prog, shots, 9, precision="fp32", group_threads=288, trace=True)
    for key in ("meas_words", "meas_prob", "log_prob", "final_gamma"):
        assert np.array_equal(a[key], b[key]), key
