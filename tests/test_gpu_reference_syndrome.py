"""compute_reference_syndrome on the GPU.

The reference computes the noiseless reference syndrome by stripping the
noise from its HIR and lowering again without post-selection or expected
parities, then sampling one shot with seed 0
(src/clifft/api/reference_syndrome.cc:9-30). The GPU backend runs the compiled
program once in forced-fault mode with no faults, detectors and observables
without their expected parities and POSTSELECT recorded in its detector slot
(CLIFFT_GPU_RAW_PARITY).

Checked here:
  * known answers on a one-measurement program whose record is 1: each
    detector / post-selection / observable flavour reports parity 1 whatever
    its expected parity says;
  * the noisy memory grid (240 post-selected detectors): the result equals
    the oracle's noise-free shot of the program rewritten the way the
    reference lowers it (POSTSELECT as DETECTOR, expected parities cleared).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import FLAG_EXPECTED_ONE, FLAG_IDENTITY, FLAG_SIGN, OP, Program, instr, p_u32x2
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")


def _kat_program(det_op, det_flags, expected_obs):
    code = [instr(OP["MEAS_DORMANT_STATIC"], 0, 0, FLAG_SIGN | FLAG_IDENTITY, p_u32x2(0, 0)),
            instr(OP[det_op], 0, 0, det_flags, p_u32x2(0, 0)),
            instr(OP["OBSERVABLE"], 0, 0, 0, p_u32x2(0, 0))]
    return Program(num_qubits=1, peak_rank=0, num_measurements=1, total_meas_slots=1,
                   num_detectors=1, num_observables=1,
                   has_postselection=int(det_op == "POSTSELECT"),
                   instructions=np.frombuffer(b"".join(code), np.uint8).reshape(-1, 32),
                   detector_offsets=np.array([0, 1], np.uint32), detector_targets=np.array([0], np.uint32),
                   observable_offsets=np.array([0, 1], np.uint32), observable_targets=np.array([0], np.uint32),
                   expected_observables=np.array(expected_obs, np.uint8))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("det_op,det_flags,expected_obs", [
    ("DETECTOR", 0, []),
    ("DETECTOR", FLAG_EXPECTED_ONE, [1]),
    ("POSTSELECT", FLAG_EXPECTED_ONE, [1]),
])
def test_reference_syndrome_known_answers(det_op, det_flags, expected_obs, precision):
    prog = _kat_program(det_op, det_flags, expected_obs)
    ref = cb.compute_reference_syndrome(prog, precision=precision)
    assert ref["detectors"].tolist() == [1]
    assert ref["observables"].tolist() == [1]
    # the ordinary sampler still applies the expected parities
    plain = cb.run(prog, 4, 0, precision=precision)
    assert np.all(plain["survived"] == 1)
    if det_op == "DETECTOR":
        want = 0 if det_flags & FLAG_EXPECTED_ONE else 1
        assert np.all(cb.api._unpack(plain["det_words"], 1)[:, 0] == want)
    assert np.all(cb.api._unpack(plain["obs_words"], 1)[:, 0] == (1 ^ (expected_obs[0] if expected_obs else 0)))


def _as_reference_lowers_it(prog):
    """The program as the reference lowers it for the reference syndrome:
    every POSTSELECT a DETECTOR of the same list and slot, no expected
    parities, no post-selection."""
    d = prog.to_npz_dict()
    ins = prog.instructions.copy()
    ops = ins[:, 0]
    ins[ops == OP["POSTSELECT"], 0] = OP["DETECTOR"]
    det = ins[:, 0] == OP["DETECTOR"]
    ins[det, 2] &= np.uint8(~FLAG_EXPECTED_ONE & 0xFF)
    d["instructions"] = ins
    d["has_postselection"] = 0
    d["expected_observables"] = np.zeros_like(prog.expected_observables)
    return Program.from_npz_dict(d)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_reference_syndrome_of_the_memory_grid(precision):
    prog = Program.load(os.path.join(PROGRAMS, "cfg1.npz"))
    assert prog.has_postselection
    ref = cb.compute_reference_syndrome(prog, precision=precision)
    o = O.run(_as_reference_lowers_it(prog), 1, seed=0, rng=O.RNG_PHILOX, faults=[[]], readout_faults=[[]])
    assert np.array_equal(ref["detectors"], o["det"][0])
    assert np.array_equal(ref["observables"], o["obs"][0])
    assert ref["detectors"].shape == (prog.num_detectors,)
