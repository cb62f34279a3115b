"""Known-answer tests of the executor's numerical rules on the GPU, restated
from the reference's own tests, in both precisions:

  * zero-probability branches are deterministic and leave a finite gamma and a
    unit physical norm (tests/test_svm.cc:1445-1570);
  * lazy renormalisation rescues gamma from underflow and overflow
    (tests/test_svm.cc:1572-1611, SchrodingerState::scale_magnitude,
    src/clifft/svm/svm.h:177-186). Here the drift is produced by the
    executor's own dynamics rather than by planting gamma = 1e-150: hundreds of
    EXPAND / H / deterministic-measurement cycles shrink gamma by 1/sqrt(2) a
    cycle; forced low-probability outcomes grow it by 1/sin(phi) a cycle;
  * the dust clamp of sample_branch (src/clifft/svm/svm_internal.h:46,65-79)
    fires on T^4 interference (tests/test_svm.cc:1975-2024).

Two rules differ in the FP32 statevector, by design:
  * renormalisation window: |gamma| outside [1e-20, 1e20] (FP64 keeps the
    reference's [1e-100, 1e100]); the physical state gamma * v is unchanged by
    either, which the tests check against the reference executor;
  * dust threshold: 1e-9 * total (FP64 keeps 1e-18 * total). FP32 rounding
    leaves |v0 + v1|^2 ~ 1e-14 * total after T^4, above the FP64 threshold:
    with the reference's threshold the FP32 executor would draw a random
    number there, shifting every later draw of the shot. The dust test shows
    both: with the default FP32 threshold the records equal the FP64 oracle's
    bit for bit; forced to 1e-18 they do not.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import clifft_b200 as cb
from clifft_b200.program import OP, Program, instr, p_f64x2, p_u32x2
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PRECISIONS = ["fp64", "fp32"]
WINDOW = {"fp64": (1e-100, 1e100), "fp32": (1e-20, 1e20)}


def _program(code, n, peak, slots, u2=None):
    kw = {}
    if u2 is not None:
        kw["u2_data"] = np.asarray(u2, np.float64).reshape(-1, 40)
        kw["u2_out"] = np.tile(np.arange(4, dtype=np.uint8), (len(kw["u2_data"]), 1))
    return Program(num_qubits=n, peak_rank=peak, num_measurements=slots, total_meas_slots=slots,
                   instructions=np.frombuffer(b"".join(code), np.uint8).reshape(-1, 32), **kw)


def _meas(op, axis, slot, axis2=0):
    return instr(OP[op], axis, axis2, 0, p_u32x2(slot, 0))


MINUS = p_f64x2(-1.0, 0.0)


def _physical_norm(g):
    gam = g["final_gamma"][:, 0] + 1j * g["final_gamma"][:, 1]
    k = g["final_k"]
    return np.array([abs(gam[s]) ** 2 * np.sum(np.abs(g["final_v"][s, :1 << int(k[s])]) ** 2)
                     for s in range(len(k))])


ZERO_PROB = {
    # |->: prob_plus = 0 exactly, b_x = 1 (tests/test_svm.cc:1445-1467)
    "minus_interfere": ([instr(OP["EXPAND"], 0), instr(OP["ARRAY_ROT"], 0, payload=MINUS),
                         _meas("MEAS_ACTIVE_INTERFERE", 0, 0)], 1, 0),
    # |+>: prob_minus = 0, b_x = 0 (:1469-1489)
    "plus_interfere": ([instr(OP["EXPAND"], 0), _meas("MEAS_ACTIVE_INTERFERE", 0, 0)], 0, 0),
    # |0>: prob_1 = 0, b = 0 (:1491-1510)
    "zero_diagonal": ([instr(OP["EXPAND"], 0), instr(OP["ARRAY_H"], 0), _meas("MEAS_ACTIVE_DIAGONAL", 0, 0)], 0, 0),
    # |1>: prob_0 = 0, b = 1 (:1512-1531)
    "one_diagonal": ([instr(OP["EXPAND"], 0), instr(OP["ARRAY_ROT"], 0, payload=MINUS), instr(OP["ARRAY_H"], 0),
                      _meas("MEAS_ACTIVE_DIAGONAL", 0, 0)], 1, 0),
    # k = 3, axis 2 exactly |-> over every state of axes 0, 1 (:1533-1570)
    "multi_axis_interfere": ([instr(OP["EXPAND"], 0), instr(OP["EXPAND_T"], 1), instr(OP["ARRAY_H"], 1),
                              instr(OP["ARRAY_CNOT"], 1, 0), instr(OP["ARRAY_T"], 0), instr(OP["EXPAND"], 2),
                              instr(OP["ARRAY_ROT"], 2, payload=MINUS), _meas("MEAS_ACTIVE_INTERFERE", 2, 0)], 1, 2),
}


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("case", sorted(ZERO_PROB))
def test_zero_probability_branches_are_deterministic(case, precision):
    code, want, final_k = ZERO_PROB[case]
    peak = 3 if case == "multi_axis_interfere" else 1
    prog = _program(code, 3, peak, 1)
    shots = 256
    for seed in (1, 7, 1234):
        g = cb.run(prog, shots, seed, precision=precision, trace=True, dump_shots=shots)
        assert np.all(cb.api._unpack(g["meas_words"], 1)[:, 0] == want), (case, seed)
        assert np.all(g["final_k"] == final_k)
        assert np.all(np.isfinite(g["final_gamma"]))
        assert g["dust_clamps"] == 0
        np.testing.assert_allclose(_physical_norm(g), 1.0, atol=1e-9 if precision == "fp64" else 1e-5)
        assert np.all(g["meas_prob"][:, 0] == 1.0)


def _underflow_program(cycles):
    code = []
    for c in range(cycles):
        code += [instr(OP["EXPAND"], 0), instr(OP["ARRAY_H"], 0), _meas("MEAS_ACTIVE_DIAGONAL", 0, c)]
    code.append(instr(OP["EXPAND"], 0))
    return _program(code, 2, 1, cycles)


def _overflow_program(cycles, phi):
    # EXPAND, H, then a rotation by phi: the |1> branch has probability sin^2(phi)
    c, s = math.cos(phi), math.sin(phi)
    node = []
    for _ in range(4):  # the same 2x2 matrix for every incoming frame state, gamma factor 1
        node += [c, 0.0, -s, 0.0, s, 0.0, c, 0.0, 1.0, 0.0]
    code = []
    for k in range(cycles):
        code += [instr(OP["EXPAND"], 0), instr(OP["ARRAY_H"], 0), instr(OP["ARRAY_U2"], 0, payload=p_u32x2(0, 0)),
                 _meas("MEAS_ACTIVE_DIAGONAL", 0, k)]
    code.append(instr(OP["EXPAND"], 0))
    return _program(code, 2, 1, cycles, u2=node)


def _check_renormalised(prog, fm, precision):
    shots = fm.shape[0]
    g = cb.run(prog, shots, 0, precision=precision, forced_meas=fm, trace=True, dump_shots=shots)
    assert np.all(g["survived"] == 1)
    gam = g["final_gamma"][:, 0] + 1j * g["final_gamma"][:, 1]
    lo, hi = WINDOW[precision]
    assert np.all((np.abs(gam) >= lo) & (np.abs(gam) <= hi)), np.abs(gam)
    v = g["final_v"][:, :2]
    assert np.all(np.isfinite(v))
    ga = gam[:, None] * v
    o = O.run(prog, shots, forced_meas=fm, want_state=True)
    oa = (o["final_gamma"][:, 0] + 1j * o["final_gamma"][:, 1])[:, None] * o["final_v"][:, :2]
    tol = 1e-10 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(ga, oa, rtol=0, atol=tol * np.abs(oa).max())
    if O.ref_available():
        r = O.ref_forced(prog, fm)
        ra = (r["final_gamma"][:, 0] + 1j * r["final_gamma"][:, 1])[:, None] * r["final_v"][:, :2]
        np.testing.assert_allclose(ga, ra, rtol=0, atol=tol * np.abs(ra).max())
        np.testing.assert_allclose(g["log_prob"], r["log_prob"], rtol=1e-9 if precision == "fp64" else 1e-5)
    return gam


@pytest.mark.parametrize("precision", PRECISIONS)
def test_lazy_renormalisation_rescues_gamma_from_underflow(precision):
    # 700 cycles: without renormalisation |gamma| = 2^-350.5 (below 1e-100)
    # while v[0] = 2^350 (beyond FP32's range)
    cycles = 700
    prog = _underflow_program(cycles)
    fm = np.zeros((4, cycles), np.uint8)
    gam = _check_renormalised(prog, fm, precision)
    # |+> at the end: gamma * v = (1, 1) / sqrt(2)
    free = cb.run(prog, 64, 3, precision=precision)
    assert np.all(cb.api._unpack(free["meas_words"], cycles) == 0)
    assert np.all(np.abs(gam) > 2.0 ** -350)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_lazy_renormalisation_rescues_gamma_from_overflow(precision):
    # forced |1> outcomes of probability sin^2(1e-3) = 1e-6 (above both dust
    # thresholds): gamma grows ~707x a cycle, to ~1e114 after 40 cycles
    cycles = 40
    prog = _overflow_program(cycles, 1e-3)
    fm = np.ones((4, cycles), np.uint8)
    g = cb.run(prog, 4, 0, precision=precision, forced_meas=fm, trace=True)
    np.testing.assert_allclose(g["meas_prob"], math.sin(1e-3) ** 2, rtol=1e-9 if precision == "fp64" else 1e-5)
    _check_renormalised(prog, fm, precision)


def _t4_program():
    # EXPAND_T then T^3 on axis 0: v = (1, e^{i pi}) up to rounding dust, an
    # X-basis measurement that is analytically deterministic (b_x = 1), then a
    # dormant random measurement that consumes the shot's next draw
    code = [instr(OP["EXPAND_T"], 0)] + [instr(OP["ARRAY_T"], 0)] * 3
    code += [_meas("MEAS_ACTIVE_INTERFERE", 0, 0), _meas("MEAS_DORMANT_RANDOM", 1, 1)]
    return _program(code, 2, 1, 2)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_t4_interference_dust_is_clamped(precision):
    prog = _t4_program()
    shots = 4096
    o = O.run(prog, shots, seed=42, rng=O.RNG_PHILOX)
    assert o["dust_clamps"] == shots  # the FP64 oracle sees dust on every shot
    g = cb.run(prog, shots, 42, precision=precision)
    assert g["dust_clamps"] == shots
    meas = cb.api._unpack(g["meas_words"], 2)
    assert np.all(meas[:, 0] == 1)
    assert np.array_equal(meas, o["meas"])  # no draw was consumed by the clamped branch
    if O.ref_available():
        r = O.ref_sample(prog, 2000, 42)
        assert np.all(r["meas"][:, 0] == 1)


def test_fp32_with_the_fp64_dust_threshold_consumes_a_draw():
    # the divergence the FP32 threshold exists for: FP32 dust (~1e-14 * total)
    # passes the FP64 threshold of 1e-18 * total, so the clamped branch draws
    # a random number and the next measurement reads a different draw
    prog = _t4_program()
    shots = 4096
    o = O.run(prog, shots, seed=42, rng=O.RNG_PHILOX)
    g = cb.run(prog, shots, 42, precision="fp32", dust_eps=1e-18)
    assert g["dust_clamps"] == 0
    meas = cb.api._unpack(g["meas_words"], 2)
    assert np.mean(meas[:, 0] == 1) > 0.999
    assert np.mean(meas[:, 1] != o["meas"][:, 1]) > 0.2
