"""Random valid SVM bytecode for parity tests (in the spirit of the reference's
tests/test_fuzz.cc): every opcode the executor accepts, emitted only where the
executor's invariants allow it (array ops on active axes, EXPAND on axis k,
active measurements on axis k-1, SWAP-measure with f <= k-1, pool indices in
range). Runs of single-axis and two-axis ops are emitted back to back so the
reference's TileAxisFusion / SingleAxisFusion passes find U4 / U2 candidates.
"""

from __future__ import annotations

import math
from typing import List

import numpy as np

from clifft_b200.program import (FLAG_EXPECTED_ONE, FLAG_IDENTITY, FLAG_SIGN, OP, Program, instr,
                                 p_f64x2, p_u32x2, p_u64)


def random_program(seed: int, n: int = 10, length: int = 160, max_k: int = 6,
                   noise: bool = True, classical: bool = True, expvals: bool = True,
                   postselect: bool = False, readout: bool = True, expand_bias: float = 0.12,
                   measure: bool = True, active_expvals: bool = False) -> Program:
    rng = np.random.default_rng(seed)
    W = (n + 63) // 64
    k = 0
    peak = 0
    code: List[bytes] = []
    slots = 0
    pauli, expm, sites, hz, ro, dets, obs_l = [], [], [], [], [], [], []
    acc = 0.0
    ndet = nobs = nexp = 0

    def rbits():
        v = 0
        for q in range(n):
            if rng.random() < 0.5:
                v |= 1 << q
        return v

    def rmask():
        return rbits(), rbits()

    def words(v):
        return [(v >> (64 * w)) & 0xFFFFFFFFFFFFFFFF for w in range(W)]

    def emit(*a, **kw):
        code.append(instr(*a, **kw))

    while len(code) < length:
        r = rng.random()
        if (r < 0.12 or rng.random() < expand_bias - 0.12) and k < max_k:
            kind = rng.integers(0, 5)
            if rng.random() < 0.3:
                emit(OP["FRAME_H"], k)
            if kind == 0:
                emit(OP["EXPAND"], k)
            elif kind == 1:
                emit(OP["EXPAND_T"], k)
            elif kind == 2:
                emit(OP["EXPAND_T_DAG"], k)
            else:
                a = rng.uniform(-1, 1)
                emit(OP["EXPAND_ROT"], k, payload=p_f64x2(math.cos(a * math.pi), math.sin(a * math.pi)))
            k += 1
            peak = max(peak, k)
        elif r < 0.30 and k >= 1:
            # single-axis run (U2 candidate)
            a = int(rng.integers(0, k))
            for _ in range(int(rng.integers(1, 5))):
                c = rng.integers(0, 7)
                if c == 0:
                    emit(OP["ARRAY_H"], a)
                elif c == 1:
                    emit(OP["ARRAY_S"], a)
                elif c == 2:
                    emit(OP["ARRAY_S_DAG"], a)
                elif c == 3:
                    emit(OP["ARRAY_T"], a)
                elif c == 4:
                    emit(OP["ARRAY_T_DAG"], a)
                elif c == 5:
                    t = rng.uniform(-1, 1)
                    emit(OP["ARRAY_ROT"], a, payload=p_f64x2(math.cos(t * math.pi), math.sin(t * math.pi)))
                else:
                    emit(OP["FRAME_S"], a)
        elif r < 0.45 and k >= 2:
            # two-axis run (U4 candidate)
            a, b = (int(v) for v in rng.choice(k, size=2, replace=False))
            for _ in range(int(rng.integers(1, 6))):
                c = rng.integers(0, 6)
                if c == 0:
                    emit(OP["ARRAY_CNOT"], a, b)
                elif c == 1:
                    emit(OP["ARRAY_CZ"], a, b)
                elif c == 2:
                    emit(OP["ARRAY_SWAP"], a, b)
                elif c == 3:
                    emit(OP["ARRAY_H"], a if rng.random() < 0.5 else b)
                elif c == 4:
                    emit(OP["ARRAY_T"], a if rng.random() < 0.5 else b)
                else:
                    emit(OP["ARRAY_CNOT"], b, a)
        elif r < 0.50 and k >= 2:
            piv = int(rng.integers(0, k))
            m = int(rng.integers(1, 1 << k)) & ~(1 << piv)
            if m:
                emit(OP["ARRAY_MULTI_CNOT"] if rng.random() < 0.5 else OP["ARRAY_MULTI_CZ"], piv,
                     payload=p_u64(m))
        elif r < 0.58:
            # frame ops anywhere
            a, b = (int(v) for v in rng.choice(n, size=2, replace=False))
            c = rng.integers(0, 6)
            op = ["FRAME_CNOT", "FRAME_CZ", "FRAME_H", "FRAME_S", "FRAME_S_DAG", "FRAME_SWAP"][c]
            # frame opcodes only conjugate p_x / p_z, so any pair of axes is valid
            if c in (0, 1, 5):
                emit(OP[op], a, b)
            else:
                emit(OP[op], a)
        elif r < 0.62:
            a = int(rng.integers(0, n))
            c = rng.integers(0, 3)
            if c == 2:
                t = rng.uniform(-1, 1)
                emit(OP["ARRAY_ROT"], a, payload=p_f64x2(math.cos(t * math.pi), math.sin(t * math.pi)))
            else:
                emit(OP["ARRAY_T"] if c == 0 else OP["ARRAY_T_DAG"], a)
        elif r < 0.74 and measure:
            # measurement
            sign = FLAG_SIGN if rng.random() < 0.3 else 0
            c = rng.integers(0, 5)
            if c <= 1 and k >= 1:
                if c == 0 and k >= 2 and rng.random() < 0.5:
                    f = int(rng.integers(0, k))
                    emit(OP["SWAP_MEAS_INTERFERE"], f, k - 1, sign, p_u32x2(slots, 0))
                else:
                    emit(OP["MEAS_ACTIVE_DIAGONAL"] if c == 1 else OP["MEAS_ACTIVE_INTERFERE"], k - 1,
                         0, sign, p_u32x2(slots, 0))
                k -= 1
            elif c == 2 and k < n:
                emit(OP["MEAS_DORMANT_STATIC"], int(rng.integers(k, n)), 0, sign, p_u32x2(slots, 0))
            elif c == 3 and k < n:
                emit(OP["MEAS_DORMANT_RANDOM"], int(rng.integers(k, n)), 0, sign, p_u32x2(slots, 0))
            else:
                emit(OP["MEAS_DORMANT_STATIC"], 0, 0, sign | FLAG_IDENTITY, p_u32x2(slots, 0))
            slots += 1
        elif r < 0.80 and noise:
            chans = []
            for _ in range(int(rng.integers(1, 4))):
                x, z = rmask()
                chans.append((float(rng.uniform(0.01, 0.3)), x, z))
            psum = sum(c[0] for c in chans)
            if psum > 0.95:
                chans = [(c[0] * 0.9 / psum, c[1], c[2]) for c in chans]
            sites.append(chans)
            ps = 0.0
            for c in chans:
                ps += c[0]
            acc += -math.log1p(-min(ps, 1.0 - 2.0 ** -53))
            hz.append(acc)
            emit(OP["NOISE"], payload=p_u32x2(len(sites) - 1, 0))
        elif r < 0.85 and classical and slots > 0:
            c = rng.integers(0, 4)
            if c == 0:
                x, z = rmask()
                pauli.append((x, z, int(rng.integers(0, 2))))
                emit(OP["APPLY_PAULI"], payload=p_u32x2(len(pauli) - 1, int(rng.integers(0, slots))))
            elif c == 1 and readout:
                ro.append((int(rng.integers(0, slots)), float(rng.uniform(0.05, 0.5))))
                emit(OP["READOUT_NOISE"], payload=p_u32x2(len(ro) - 1, 0))
            elif c == 2:
                tg = [int(v) for v in rng.choice(slots, size=min(slots, int(rng.integers(1, 4))), replace=False)]
                dets.append(tg)
                fl = FLAG_EXPECTED_ONE if rng.random() < 0.2 else 0
                op = OP["POSTSELECT"] if postselect and rng.random() < 0.5 else OP["DETECTOR"]
                emit(op, 0, 0, fl, p_u32x2(len(dets) - 1, ndet))
                ndet += 1
            else:
                tg = [int(v) for v in rng.choice(slots, size=min(slots, int(rng.integers(1, 3))), replace=False)]
                obs_l.append(tg)
                emit(OP["OBSERVABLE"], payload=p_u32x2(len(obs_l) - 1, int(rng.integers(0, 2))))
                nobs = max(nobs, 2)
        elif r < 0.90 and expvals:
            x, z = rmask()
            if active_expvals:
                x &= (1 << k) - 1  # X / Y only on active axes: a non-zero expectation
            expm.append((x, z, int(rng.integers(0, 2))))
            emit(OP["EXP_VAL"], payload=p_u32x2(len(expm) - 1, nexp))
            nexp += 1

    def mk(lst):
        x = np.array([words(m[0]) for m in lst], np.uint64).reshape(-1, W)
        z = np.array([words(m[1]) for m in lst], np.uint64).reshape(-1, W)
        s = np.array([m[2] for m in lst], np.uint8)
        return x, z, s

    px, pz, ps_ = mk(pauli)
    ex, ez, es = mk(expm)
    offs, cp, cx, cz = [0], [], [], []
    for s in sites:
        for prob, x, z in s:
            cp.append(prob)
            cx.append(words(x))
            cz.append(words(z))
        offs.append(len(cp))

    def csr(lists):
        o, t = [0], []
        for l in lists:
            t.extend(l)
            o.append(len(t))
        return np.array(o, np.uint32), np.array(t, np.uint32)

    do, dt = csr(dets)
    oo, ot = csr(obs_l)
    has_ps = any(c[0] == OP["POSTSELECT"] for c in code)
    return Program(
        num_qubits=n, peak_rank=peak, num_measurements=slots, total_meas_slots=slots,
        num_detectors=ndet, num_observables=nobs, num_exp_vals=nexp, has_postselection=int(has_ps),
        instructions=np.frombuffer(b"".join(code), np.uint8).reshape(-1, 32).copy(),
        pauli_x=px, pauli_z=pz, pauli_sign=ps_, exp_val_x=ex, exp_val_z=ez, exp_val_sign=es,
        noise_site_offsets=np.array(offs, np.uint32), noise_channel_prob=np.array(cp, np.float64),
        noise_channel_x=np.array(cx, np.uint64).reshape(-1, W),
        noise_channel_z=np.array(cz, np.uint64).reshape(-1, W),
        noise_hazards=np.array(hz, np.float64),
        readout_meas_idx=np.array([r[0] for r in ro], np.uint32),
        readout_prob=np.array([r[1] for r in ro], np.float64),
        detector_offsets=do, detector_targets=dt, observable_offsets=oo, observable_targets=ot,
        expected_observables=np.array([1, 0][:nobs], np.uint8),
        name=f"fuzz_s{seed}_n{n}_k{max_k}")


def random_forced_inputs(prog: Program, shots: int, seed: int, fault_rate: float = 0.3):
    """Forced faults (site, channel) per shot and readout flips per shot."""
    rng = np.random.default_rng(seed)
    ns = prog.noise_site_offsets.shape[0] - 1
    nr = prog.readout_meas_idx.shape[0]
    faults, ros = [], []
    for _ in range(shots):
        f = []
        for s in range(ns):
            if rng.random() < fault_rate:
                nch = int(prog.noise_site_offsets[s + 1] - prog.noise_site_offsets[s])
                f.append((s, int(rng.integers(0, nch))))
        faults.append(f)
        ros.append([e for e in range(nr) if rng.random() < fault_rate])
    return faults, ros
