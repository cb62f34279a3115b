"""Seeded synthetic near-Clifford circuits and a small lowering to SVM bytecode.

The reference compiles Stim-format circuit text with Stim (parse -> trace ->
lower, src/python/bindings.cc:829-883). Stim v1.15.0 is not available offline,
so this module stands in for that compiler: it builds the seeded circuits the
benchmark configurations describe and lowers them to reference-format bytecode
with the same construction the reference backend uses:

  * Clifford gates are absorbed into a virtual frame W (no bytecode), kept as
    the map P -> W^dag P W on physical Paulis (a 2n-row tableau of
    phase-tracked virtual Paulis i^r X^x Z^z);
  * every non-Clifford rotation and measurement pulls its Pauli back through W
    and localizes it with the reference's greedy pivot rule
    (src/clifft/backend/backend.cc:404-506: X-support pivot preferring dormant
    axes, CNOT fan-out, CZ clean-up, S for Y; pure-Z pivot preferring active
    axes), emitting FRAME_* ops for dormant controls and ARRAY_* ops inside the
    active block (backend.cc:303-350);
  * routing to an active Z follows backend.cc:361-389 (SWAP to axis k,
    FRAME_H + EXPAND for a dormant X; ARRAY_H for an active X);
  * T / T_DAG / ROT emission, measurement opcode choice (dormant static /
    random, SWAP to k-1 then active diagonal / interfere) and the virtual H after
    an X-basis measurement follow backend.cc:680-805;
  * noise channels are mapped into the virtual frame and hazards accumulate
    -log1p(-min(p, 1 - 2^-53)) (backend.cc:840-868); resets lower to a
    measurement plus a conditional APPLY_PAULI.

The output is therefore a valid reference-format CompiledModule whose
instruction mix and active-dimension trajectory follow the reference lowering.
It is not byte-identical to what Stim-backed `clifft.compile` would emit (the
frontend's peephole and squeeze passes are not replicated), which is why every
executor comparison in this repository runs both executors on the same
bytecode.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .program import (FLAG_EXPECTED_ONE, FLAG_IDENTITY, FLAG_SIGN, OP, Program, instr,
                      p_f64x2, p_u32x2)

INV_SQRT2 = math.sqrt(2.0) / 2.0

# --------------------------------------------------------------------------
# Phase-tracked Pauli algebra on python ints: (r, x, z) means i^r X^x Z^z.
# --------------------------------------------------------------------------
Pauli = Tuple[int, int, int]


def _popc(v: int) -> int:
    return bin(v).count("1")


def pmul(a: Pauli, b: Pauli) -> Pauli:
    """(i^ra X^xa Z^za)(i^rb X^xb Z^zb): moving Z^za past X^xb costs (-1)^(za.xb)."""
    return ((a[0] + b[0] + 2 * _popc(a[2] & b[1])) & 3, a[1] ^ b[1], a[2] ^ b[2])


def stim_sign(p: Pauli) -> bool:
    """Sign of p written as +-(product of per-qubit X/Y/Z), Y = iXZ."""
    ph = (p[0] - _popc(p[1] & p[2])) & 3
    assert ph in (0, 2), "non-Hermitian Pauli"
    return ph == 2


def conj_h(p: Pauli, a: int) -> Pauli:
    r, x, z = p
    bx, bz = (x >> a) & 1, (z >> a) & 1
    if bx and bz:
        r += 2
    m = 1 << a
    x = (x & ~m) | (bz << a)
    z = (z & ~m) | (bx << a)
    return (r & 3, x, z)


def conj_s(p: Pauli, a: int, dag: bool = False) -> Pauli:
    r, x, z = p
    if (x >> a) & 1:
        r += 3 if dag else 1
        z ^= 1 << a
    return (r & 3, x, z)


def conj_cnot(p: Pauli, c: int, t: int) -> Pauli:
    r, x, z = p
    if (x >> c) & 1:
        x ^= 1 << t
    if (z >> t) & 1:
        z ^= 1 << c
    return (r, x, z)


def conj_cz(p: Pauli, a: int, b: int) -> Pauli:
    r, x, z = p
    xa, xb = (x >> a) & 1, (x >> b) & 1
    if xa and xb:
        r += 2
    if xa:
        z ^= 1 << b
    if xb:
        z ^= 1 << a
    return (r & 3, x, z)


def conj_swap(p: Pauli, a: int, b: int) -> Pauli:
    r, x, z = p

    def sw(v):
        ba, bb = (v >> a) & 1, (v >> b) & 1
        if ba != bb:
            v ^= (1 << a) | (1 << b)
        return v
    return (r, sw(x), sw(z))


# --------------------------------------------------------------------------
# Circuit description
# --------------------------------------------------------------------------
@dataclass
class Gate:
    kind: str                 # H S S_DAG CX CZ T T_DAG RZ M MR R DEP1 DEP2 XERR DET OBS EXPVAL
    qubits: Tuple[int, ...] = ()
    arg: float = 0.0
    targets: Tuple[int, ...] = ()      # DET / OBS: measurement indices
    pauli: str = ""                    # EXPVAL: per-qubit letters for `qubits`


@dataclass
class Circuit:
    num_qubits: int
    gates: List[Gate] = field(default_factory=list)
    name: str = ""

    def add(self, kind, *qubits, arg=0.0, targets=(), pauli=""):
        self.gates.append(Gate(kind, tuple(qubits), arg, tuple(targets), pauli))


# --------------------------------------------------------------------------
# Lowering
# --------------------------------------------------------------------------
class Lowerer:
    def __init__(self, n: int):
        self.n = n
        self.W = max(1, (n + 63) // 64)
        # rows: images of X_q and Z_q under P -> W^dag P W
        self.rx: List[Pauli] = [(0, 1 << q, 0) for q in range(n)]
        self.rz: List[Pauli] = [(0, 0, 1 << q) for q in range(n)]
        self.k = 0
        self.peak = 0
        self.code: List[bytes] = []
        self.pauli_masks: List[Tuple[int, int, int]] = []
        self.exp_masks: List[Tuple[int, int, int]] = []
        self.noise_sites: List[List[Tuple[float, int, int]]] = []
        self.hazards: List[float] = []
        self.hazard_acc = 0.0
        self.det_lists: List[Sequence[int]] = []
        self.obs_lists: List[Sequence[int]] = []
        self.num_meas = 0
        self.num_det = 0
        self.num_obs = 0
        self.num_exp = 0
        self.global_weight = 1.0 + 0.0j
        self.postselect = False

    # ---- frame bookkeeping ------------------------------------------------
    def _virtual(self, fn, *args):
        self.rx = [fn(p, *args) for p in self.rx]
        self.rz = [fn(p, *args) for p in self.rz]

    def image_of(self, xs: int, zs: int) -> Pauli:
        """W^dag (X^xs Z^zs) W for a physical Pauli given as bit masks."""
        acc: Pauli = (0, 0, 0)
        q = 0
        while xs >> q:
            if (xs >> q) & 1:
                acc = pmul(acc, self.rx[q])
            q += 1
        q = 0
        while zs >> q:
            if (zs >> q) & 1:
                acc = pmul(acc, self.rz[q])
            q += 1
        return acc

    def emit(self, b: bytes):
        self.code.append(b)

    # ---- emit helpers (backend.cc:303-350) -------------------------------
    def e_cnot(self, c, t):
        self._virtual(conj_cnot, c, t)
        if c >= self.k:
            self.emit(instr(OP["FRAME_CNOT"], c, t))
        else:
            assert t < self.k
            self.emit(instr(OP["ARRAY_CNOT"], c, t))

    def e_cz(self, a, b):
        self._virtual(conj_cz, a, b)
        if a >= self.k or b >= self.k:
            self.emit(instr(OP["FRAME_CZ"], a, b))
        else:
            self.emit(instr(OP["ARRAY_CZ"], a, b))

    def e_s(self, v):
        self._virtual(conj_s, v)
        self.emit(instr(OP["ARRAY_S"] if v < self.k else OP["FRAME_S"], v))

    def e_swap(self, a, b):
        if a == b:
            return
        assert (a < self.k) == (b < self.k)
        self._virtual(conj_swap, a, b)
        self.emit(instr(OP["ARRAY_SWAP"] if a < self.k else OP["FRAME_SWAP"], a, b))

    # ---- localization (backend.cc:404-506) -------------------------------
    def localize(self, p: Pauli) -> Tuple[int, str, Pauli]:
        r, x, z = p
        k = self.k
        assert x or z
        if x:
            dorm = x >> k
            pivot = (k + (dorm & -dorm).bit_length() - 1) if dorm else (x & -x).bit_length() - 1
            rest = x & ~(1 << pivot)
            while rest:
                q = (rest & -rest).bit_length() - 1
                self.e_cnot(pivot, q)
                p = conj_cnot(p, pivot, q)
                rest &= rest - 1
            rest = z & ~(1 << pivot)
            while rest:
                q = (rest & -rest).bit_length() - 1
                self.e_cz(pivot, q)
                p = conj_cz(p, pivot, q)
                rest &= rest - 1
            if (p[2] >> pivot) & 1:
                self.e_s(pivot)
                p = conj_s(p, pivot)
            basis = "X"
        else:
            act = z & ((1 << k) - 1)
            pivot = (act & -act).bit_length() - 1 if act else (z & -z).bit_length() - 1
            rest = z & ~(1 << pivot)
            while rest:
                q = (rest & -rest).bit_length() - 1
                self.e_cnot(q, pivot)
                p = conj_cnot(p, q, pivot)
                rest &= rest - 1
            basis = "Z"
        assert p[1] in (0, 1 << pivot) and p[2] in (0, 1 << pivot)
        return pivot, basis, p

    def route_to_active_z(self, pivot: int, basis: str, p: Pauli) -> Tuple[int, Pauli]:
        dormant = pivot >= self.k
        if dormant and basis == "Z":
            return pivot, p
        if dormant:
            nxt = self.k
            if pivot != nxt:
                self.e_swap(pivot, nxt)
                p = conj_swap(p, pivot, nxt)
                pivot = nxt
            self._virtual(conj_h, pivot)
            p = conj_h(p, pivot)
            self.emit(instr(OP["FRAME_H"], pivot))
            self.emit(instr(OP["EXPAND"], pivot))
            self.k += 1
            self.peak = max(self.peak, self.k)
            return pivot, p
        if basis == "X":
            self._virtual(conj_h, pivot)
            p = conj_h(p, pivot)
            self.emit(instr(OP["ARRAY_H"], pivot))
        return pivot, p

    # ---- circuit ops ------------------------------------------------------
    def clifford(self, g: Gate):
        q = g.qubits
        if g.kind == "H":
            a = q[0]
            self.rx[a], self.rz[a] = self.rz[a], self.rx[a]
        elif g.kind in ("S", "S_DAG"):
            a = q[0]
            xz = pmul(self.rx[a], self.rz[a])
            # S^dag X S = -iXZ ; S X S^dag = +iXZ
            self.rx[a] = ((xz[0] + (3 if g.kind == "S" else 1)) & 3, xz[1], xz[2])
        elif g.kind == "CX":
            c, t = q
            self.rx[c] = pmul(self.rx[c], self.rx[t])
            self.rz[t] = pmul(self.rz[c], self.rz[t])
        elif g.kind == "CZ":
            a, b = q
            self.rx[a] = pmul(self.rx[a], self.rz[b])
            self.rx[b] = pmul(self.rz[a], self.rx[b])
        else:
            raise ValueError(g.kind)

    def rotation(self, q: int, kind: str, alpha: float = 0.0):
        p = self.rz[q]
        sign0 = stim_sign(p)
        pivot, basis, p = self.localize(p)
        pivot, p = self.route_to_active_z(pivot, basis, p)
        sign = stim_sign(p)
        if kind in ("T", "T_DAG"):
            dagger = kind == "T_DAG"
            if sign:
                self.global_weight *= complex(INV_SQRT2, -INV_SQRT2 if dagger else INV_SQRT2)
            flip = sign ^ dagger
            self.emit(instr(OP["ARRAY_T_DAG"] if flip else OP["ARRAY_T"], pivot))
        else:
            if sign != sign0:
                corr = alpha * math.pi * (-1.0 if sign0 else 1.0)
                self.global_weight *= complex(math.cos(corr), math.sin(corr))
            a = -alpha if sign else alpha
            self.emit(instr(OP["ARRAY_ROT"], pivot,
                            payload=p_f64x2(math.cos(a * math.pi), math.sin(a * math.pi))))

    def measure(self, q: int, hidden: bool = False) -> int:
        idx = self.num_meas
        self.num_meas += 1
        p = self.rz[q]
        if p[1] == 0 and p[2] == 0:
            self.emit(instr(OP["MEAS_DORMANT_STATIC"], 0, 0,
                            FLAG_IDENTITY | (FLAG_SIGN if stim_sign(p) else 0), p_u32x2(idx, 0)))
            return idx
        pivot, basis, p = self.localize(p)
        sign = stim_sign(p)
        fl = FLAG_SIGN if sign else 0
        if pivot >= self.k:
            op = OP["MEAS_DORMANT_STATIC"] if basis == "Z" else OP["MEAS_DORMANT_RANDOM"]
            self.emit(instr(op, pivot, 0, fl, p_u32x2(idx, 0)))
            if basis == "X":
                self._virtual(conj_h, pivot)
        else:
            top = self.k - 1
            if pivot != top:
                self.e_swap(pivot, top)
                pivot = top
            op = OP["MEAS_ACTIVE_DIAGONAL"] if basis == "Z" else OP["MEAS_ACTIVE_INTERFERE"]
            self.emit(instr(op, pivot, 0, fl, p_u32x2(idx, 0)))
            if basis == "X":
                self._virtual(conj_h, pivot)
            self.k -= 1
        return idx

    def reset_after(self, q: int, cond_idx: int):
        p = self.rx[q]
        h = len(self.pauli_masks)
        self.pauli_masks.append((p[1], p[2], int(stim_sign(p))))
        self.emit(instr(OP["APPLY_PAULI"], payload=p_u32x2(h, cond_idx)))

    def noise(self, channels: Sequence[Tuple[float, int, int]]):
        mapped = []
        for prob, xs, zs in channels:
            im = self.image_of(xs, zs)
            mapped.append((prob, im[1], im[2]))
        psum = 0.0
        for prob, _, _ in mapped:
            psum += prob
        site = len(self.noise_sites)
        self.noise_sites.append(mapped)
        self.emit(instr(OP["NOISE"], payload=p_u32x2(site, 0)))
        self.hazard_acc += -math.log1p(-min(psum, 1.0 - 2.0 ** -53))
        self.hazards.append(self.hazard_acc)

    def lower(self, circ: Circuit, postselect_all: bool = False) -> Program:
        self.postselect = postselect_all
        for g in circ.gates:
            kd = g.kind
            if kd in ("H", "S", "S_DAG", "CX", "CZ"):
                self.clifford(g)
            elif kd in ("T", "T_DAG"):
                self.rotation(g.qubits[0], kd)
            elif kd == "RZ":
                self.rotation(g.qubits[0], "RZ", g.arg / math.pi)
            elif kd == "M":
                self.measure(g.qubits[0])
            elif kd == "MR":
                i = self.measure(g.qubits[0])
                self.reset_after(g.qubits[0], i)
            elif kd == "DEP1":
                q = g.qubits[0]
                p = g.arg / 3.0
                self.noise([(p, 1 << q, 0), (p, 1 << q, 1 << q), (p, 0, 1 << q)])
            elif kd == "DEP2":
                a, b = g.qubits
                chans = []
                for pa in range(4):
                    for pb in range(4):
                        if pa == 0 and pb == 0:
                            continue
                        xs = ((pa in (1, 2)) << a) | ((pb in (1, 2)) << b)
                        zs = ((pa in (2, 3)) << a) | ((pb in (2, 3)) << b)
                        chans.append((g.arg / 15.0, xs, zs))
                self.noise(chans)
            elif kd == "XERR":
                self.noise([(g.arg, 1 << g.qubits[0], 0)])
            elif kd == "DET":
                lst = len(self.det_lists)
                self.det_lists.append(g.targets)
                op = OP["POSTSELECT"] if self.postselect else OP["DETECTOR"]
                self.emit(instr(op, payload=p_u32x2(lst, self.num_det)))
                self.num_det += 1
            elif kd == "OBS":
                lst = len(self.obs_lists)
                self.obs_lists.append(g.targets)
                self.emit(instr(OP["OBSERVABLE"], payload=p_u32x2(lst, int(g.arg))))
                self.num_obs = max(self.num_obs, int(g.arg) + 1)
            elif kd == "EXPVAL":
                xs = zs = 0
                for q, c in zip(g.qubits, g.pauli):
                    if c in "XY":
                        xs |= 1 << q
                    if c in "ZY":
                        zs |= 1 << q
                # the probe is the Hermitian product of per-qubit letters (Y = iXZ)
                im = self.image_of(xs, zs)
                im = ((im[0] + _popc(xs & zs)) & 3, im[1], im[2])
                h = len(self.exp_masks)
                self.exp_masks.append((im[1], im[2], int(stim_sign(im))))
                self.emit(instr(OP["EXP_VAL"], payload=p_u32x2(h, self.num_exp)))
                self.num_exp += 1
            else:
                raise ValueError(f"unknown gate {kd}")
        return self.program(circ.name)

    def program(self, name: str) -> Program:
        W = self.W

        def words(v: int) -> List[int]:
            return [(v >> (64 * w)) & 0xFFFFFFFFFFFFFFFF for w in range(W)]

        def masks(lst):
            x = np.array([words(m[0]) for m in lst], np.uint64).reshape(-1, W)
            z = np.array([words(m[1]) for m in lst], np.uint64).reshape(-1, W)
            s = np.array([m[2] for m in lst], np.uint8)
            return x, z, s

        px, pz, ps = masks(self.pauli_masks)
        ex, ez, es = masks(self.exp_masks)
        offs, cp, cx, cz = [0], [], [], []
        for site in self.noise_sites:
            for prob, xs, zs in site:
                cp.append(prob)
                cx.append(words(xs))
                cz.append(words(zs))
            offs.append(len(cp))

        def csr(lists):
            o, t = [0], []
            for l in lists:
                t.extend(l)
                o.append(len(t))
            return np.array(o, np.uint32), np.array(t, np.uint32)

        do, dt = csr(self.det_lists)
        oo, ot = csr(self.obs_lists)
        code = np.frombuffer(b"".join(self.code), np.uint8).reshape(-1, 32).copy() \
            if self.code else np.zeros((0, 32), np.uint8)
        return Program(
            num_qubits=self.n, peak_rank=self.peak, num_measurements=self.num_meas,
            total_meas_slots=self.num_meas, num_detectors=self.num_det,
            num_observables=self.num_obs, num_exp_vals=self.num_exp,
            has_postselection=int(self.postselect and self.num_det > 0),
            instructions=code, pauli_x=px, pauli_z=pz, pauli_sign=ps,
            exp_val_x=ex, exp_val_z=ez, exp_val_sign=es,
            noise_site_offsets=np.array(offs, np.uint32),
            noise_channel_prob=np.array(cp, np.float64),
            noise_channel_x=np.array(cx, np.uint64).reshape(-1, W),
            noise_channel_z=np.array(cz, np.uint64).reshape(-1, W),
            noise_hazards=np.array(self.hazards, np.float64),
            detector_offsets=do, detector_targets=dt,
            observable_offsets=oo, observable_targets=ot,
            global_weight=self.global_weight, name=name)


def lower(circ: Circuit, postselect_all: bool = False) -> Program:
    return Lowerer(circ.num_qubits).lower(circ, postselect_all)


# --------------------------------------------------------------------------
# Seeded generators for the benchmark configurations
# --------------------------------------------------------------------------
def random_near_clifford(n: int, layers: int, t_count: int, seed: int,
                         meas_every: int = 25, meas_per_round: int = 4,
                         final_measure: bool = True, name: str = "") -> Circuit:
    """Layered random near-Clifford circuit.

    Each layer applies H or S (50/50) to every qubit with probability 0.3, then
    a CX on each pair of a uniformly random disjoint pairing with probability
    0.5. `t_count` T gates sit at uniformly random (layer, qubit) positions and
    act at the start of their layer. Every `meas_every` layers, M on
    `meas_per_round` distinct random qubits; optionally M on all qubits at the
    end. Randomness: numpy.random.default_rng(seed), drawn in the order T
    positions, then per layer (1-qubit gates, pairing, pair coins, mid-circuit
    measurement qubits).
    """
    rng = np.random.default_rng(seed)
    c = Circuit(n, name=name or f"near_clifford_n{n}_L{layers}_T{t_count}_s{seed}")
    t_layer = rng.integers(0, layers, size=t_count)
    t_qubit = rng.integers(0, n, size=t_count)
    t_at: Dict[int, List[int]] = {}
    for l, q in zip(t_layer.tolist(), t_qubit.tolist()):
        t_at.setdefault(l, []).append(q)
    for layer in range(layers):
        for q in t_at.get(layer, []):
            c.add("T", q)
        coins = rng.random(n)
        kinds = rng.integers(0, 2, size=n)
        for q in range(n):
            if coins[q] < 0.3:
                c.add("H" if kinds[q] == 0 else "S", q)
        perm = rng.permutation(n)
        pair_coins = rng.random(n // 2)
        for i in range(n // 2):
            if pair_coins[i] < 0.5:
                c.add("CX", int(perm[2 * i]), int(perm[2 * i + 1]))
        if meas_every and (layer + 1) % meas_every == 0 and (layer + 1) < layers:
            for q in rng.choice(n, size=meas_per_round, replace=False).tolist():
                c.add("M", q)
    if final_measure:
        for q in range(n):
            c.add("M", q)
    return c


def config0(seed: int = 42) -> Circuit:
    """16 qubits, 100 layers, 8 T, M on 4 qubits every 25 layers, final M; no noise."""
    return random_near_clifford(16, 100, 8, seed, name=f"cfg0_s{seed}")


def config2_circuits(seeds=range(100, 164)) -> List[Circuit]:
    """64 cfg0-style circuits on 32 qubits; T count ~ U{4..18} drawn from each seed."""
    out = []
    for s in seeds:
        t = int(np.random.default_rng(s + 10_000).integers(4, 19))
        out.append(random_near_clifford(32, 100, t, s, name=f"cfg2_s{s}_T{t}"))
    return out


def config3(seed: int = 42) -> Circuit:
    """64 qubits, 400 layers, 24 T gates."""
    return random_near_clifford(64, 400, 24, seed, name=f"cfg3_s{seed}")


def memory_grid(rows: int = 7, cols: int = 7, rounds: int = 10, t_count: int = 12,
                p: float = 1e-3, seed: int = 7) -> Circuit:
    """Noisy memory-style grid circuit.

    n = rows*cols qubits; odd-index qubits are measured and reset each round.
    Each round: CX on every nearest-neighbour edge (control = lower index) in
    an order fixed by the seed, DEPOLARIZE2(p) after each CX; magic gates at
    `t_count` random (round, qubit) positions, each a T in the X basis
    (H, T, H; DEPOLARIZE1(p) after each 1-qubit gate) so it acts non-trivially
    on the computational-basis memory; X_ERROR(p) before every measurement;
    MR on the odd qubits; DETECTOR per measured qubit comparing it with its
    previous-round measurement (round 0: with the reset value). One observable:
    parity of the last round's measurements of the odd qubits in row 0.
    """
    rng = np.random.default_rng(seed)
    n = rows * cols
    c = Circuit(n, name=f"memory_grid_{rows}x{cols}_r{rounds}_T{t_count}_s{seed}")
    edges = []
    for r in range(rows):
        for q in range(cols):
            i = r * cols + q
            if q + 1 < cols:
                edges.append((i, i + 1))
            if r + 1 < rows:
                edges.append((i, i + cols))
    order = rng.permutation(len(edges))
    t_round = rng.integers(0, rounds, size=t_count)
    t_qubit = rng.integers(0, n, size=t_count)
    anc = [q for q in range(n) if q % 2 == 1]
    prev: Dict[int, int] = {}
    meas = 0
    last_round: Dict[int, int] = {}
    for r in range(rounds):
        for e in order.tolist():
            a, b = edges[e]
            c.add("CX", a, b)
            c.add("DEP2", a, b, arg=p)
        for tr, tq in zip(t_round.tolist(), t_qubit.tolist()):
            if tr == r:
                for kd in ("H", "T", "H"):
                    c.add(kd, tq)
                    c.add("DEP1", tq, arg=p)
        for q in anc:
            c.add("XERR", q, arg=p)
        for q in anc:
            c.add("MR", q)
            tg = (prev[q], meas) if q in prev else (meas,)
            prev[q] = meas
            last_round[q] = meas
            meas += 1
            c.add("DET", targets=tg)
    c.add("OBS", targets=tuple(last_round[q] for q in anc if q < cols), arg=0)
    return c


def config1(seed: int = 7) -> Circuit:
    return memory_grid(seed=seed)


def config4(seed: int = 3, n: int = 40, layers: int = 120, n_rot: int = 32,
            n_obs: int = 16, rot_layers: int = 10) -> Tuple[Circuit, np.ndarray]:
    """Measurement-free, noise-free rotation circuit with `n_obs` weight-4 probes.

    Rotation positions are uniform over (layer, qubit) with the layer drawn from
    the first `rot_layers` Clifford layers: a rotation placed after full
    scrambling almost always opens a new active axis (32 rotations -> k ~ 30),
    while placing them among the first 10 layers gives the peak k ~ 14 this
    workload is specified with. Positions and angles theta ~ U(0, 2 pi) come from
    default_rng(seed); the Clifford layers from default_rng(seed + 1) with the
    layer recipe of `random_near_clifford`; the probes (4 distinct random qubits,
    uniform X/Y/Z letters) from default_rng(seed + 2). Returns the circuit and
    the angle vector (in circuit order of the rotations).
    """
    rng = np.random.default_rng(seed)
    pos_layer = rng.integers(0, min(rot_layers, layers), size=n_rot)
    pos_q = rng.integers(0, n, size=n_rot)
    theta = rng.uniform(0.0, 2.0 * math.pi, size=n_rot)
    rot_at: Dict[int, List[int]] = {}
    for i, l in enumerate(pos_layer.tolist()):
        rot_at.setdefault(l, []).append(i)
    crng = np.random.default_rng(seed + 1)
    c = Circuit(n, name=f"cfg4_n{n}_L{layers}_R{n_rot}_s{seed}")
    order = []
    for layer in range(layers):
        for i in rot_at.get(layer, []):
            c.add("RZ", int(pos_q[i]), arg=float(theta[i]))
            order.append(i)
        coins = crng.random(n)
        kinds = crng.integers(0, 2, size=n)
        for q in range(n):
            if coins[q] < 0.3:
                c.add("H" if kinds[q] == 0 else "S", q)
        perm = crng.permutation(n)
        pair_coins = crng.random(n // 2)
        for i in range(n // 2):
            if pair_coins[i] < 0.5:
                c.add("CX", int(perm[2 * i]), int(perm[2 * i + 1]))
    prng = np.random.default_rng(seed + 2)
    for _ in range(n_obs):
        qs = prng.choice(n, size=4, replace=False)
        letters = "".join("XYZ"[int(v)] for v in prng.integers(0, 3, size=4))
        c.add("EXPVAL", *[int(q) for q in qs], pauli=letters)
    return c, theta[np.array(order, dtype=np.int64)]


def active_probes(program, seed: int = 0):
    """`program` with every EXP_VAL mask redrawn as a low-weight Pauli (X / Y
    on one or two axes, Z on up to two) on the axes active at that
    instruction, in the compiled frame basis. Random weight-4 probes in the
    circuit basis of a scrambled Clifford circuit read 0, and so do their
    derivatives (their X / Y support lands on dormant axes); these probes have
    non-trivial values and slopes, so gradient checks and timings exercise the
    whole backward pass."""
    import numpy as np
    from .program import OP, Program
    rng = np.random.default_rng(seed)
    hist = program.active_k_history()
    ex, ez, es = program.exp_val_x.copy(), program.exp_val_z.copy(), program.exp_val_sign.copy()
    for pc in np.nonzero(program.opcodes == OP["EXP_VAL"])[0]:
        cp = int(program.instructions[pc, 8:12].copy().view(np.uint32)[0])
        k = int(hist[pc])
        xs = rng.choice(k, size=int(rng.integers(1, 3)), replace=False)
        zs = rng.choice(k, size=int(rng.integers(0, 3)), replace=False)
        ex[cp] = 0
        ez[cp] = 0
        ex[cp, 0] = np.uint64(sum(1 << int(a) for a in xs))
        ez[cp, 0] = np.uint64(sum(1 << int(a) for a in zs))
        es[cp] = rng.integers(0, 2)
    d = program.to_npz_dict()
    d["exp_val_x"], d["exp_val_z"], d["exp_val_sign"] = ex, ez, es
    return Program.from_npz_dict(d)
