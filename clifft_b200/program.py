"""Host-side container for a compiled Clifft program.

`Program` holds the reference's `CompiledModule` (src/clifft/backend/backend.h:324-344)
as numpy arrays in exactly the layout of `clifft_program_image`
(include/clifft_program_image.h): 32-byte instructions copied byte for byte
(backend.h:95-163), Pauli-mask arenas as parallel x/z word arrays
(src/clifft/util/pauli_arena.h:63-110), noise sites and target lists as CSR, and
FusedU2Node / FusedU4Node (backend.h:224-253) as flat complex tables.

The same image feeds the CUDA backend's C ABI, the CPU oracle and the
reference harness, so one `Program` object is what every layer agrees on.
"""

from __future__ import annotations

import ctypes
import struct
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# Opcode numbering of `enum class Opcode` (src/clifft/backend/backend.h:25-86).
OPCODES = [
    "FRAME_CNOT", "FRAME_CZ", "FRAME_H", "FRAME_S", "FRAME_S_DAG", "FRAME_SWAP",
    "ARRAY_CNOT", "ARRAY_CZ", "ARRAY_SWAP", "ARRAY_MULTI_CNOT", "ARRAY_MULTI_CZ",
    "ARRAY_H", "ARRAY_S", "ARRAY_S_DAG", "ARRAY_T", "ARRAY_T_DAG", "ARRAY_ROT",
    "ARRAY_U2", "ARRAY_U4",
    "EXPAND", "EXPAND_T", "EXPAND_T_DAG", "EXPAND_ROT",
    "MEAS_DORMANT_STATIC", "MEAS_DORMANT_RANDOM", "MEAS_ACTIVE_DIAGONAL",
    "MEAS_ACTIVE_INTERFERE", "SWAP_MEAS_INTERFERE",
    "MEAS_DORMANT_STATIC_FORCED", "MEAS_DORMANT_RANDOM_FORCED",
    "MEAS_ACTIVE_DIAGONAL_FORCED", "MEAS_ACTIVE_INTERFERE_FORCED",
    "SWAP_MEAS_INTERFERE_FORCED",
    "APPLY_PAULI", "NOISE", "NOISE_BLOCK", "READOUT_NOISE", "DETECTOR", "POSTSELECT",
    "OBSERVABLE", "EXP_VAL",
]
OP = {name: i for i, name in enumerate(OPCODES)}

# Instruction flag bits (backend.h:97-101).
FLAG_SIGN = 0x01
FLAG_HIDDEN = 0x02
FLAG_IDENTITY = 0x04
FLAG_EXPECTED_ONE = 0x08

ACTIVE_MEAS = {
    OP["MEAS_ACTIVE_DIAGONAL"], OP["MEAS_ACTIVE_INTERFERE"], OP["SWAP_MEAS_INTERFERE"],
    OP["MEAS_ACTIVE_DIAGONAL_FORCED"], OP["MEAS_ACTIVE_INTERFERE_FORCED"],
    OP["SWAP_MEAS_INTERFERE_FORCED"],
}
EXPANDS = {OP["EXPAND"], OP["EXPAND_T"], OP["EXPAND_T_DAG"], OP["EXPAND_ROT"]}


def instr(opcode: int, axis_1: int = 0, axis_2: int = 0, flags: int = 0,
          payload: bytes = b"") -> bytes:
    """Pack one 32-byte instruction (field offsets of backend.h:103-160)."""
    head = struct.pack("<BBBBHH", opcode, 0, flags, 0, axis_1, axis_2)
    return head + payload.ljust(24, b"\0")


def p_u32x2(a: int, b: int) -> bytes:
    return struct.pack("<II", a, b)


def p_f64x2(re: float, im: float) -> bytes:
    return struct.pack("<dd", re, im)


def p_u64(v: int) -> bytes:
    return struct.pack("<Q", v)


class ProgramImage(ctypes.Structure):
    """ctypes mirror of `clifft_program_image`."""

    _fields_ = [
        ("num_qubits", ctypes.c_uint32),
        ("peak_rank", ctypes.c_uint32),
        ("num_measurements", ctypes.c_uint32),
        ("total_meas_slots", ctypes.c_uint32),
        ("num_detectors", ctypes.c_uint32),
        ("num_observables", ctypes.c_uint32),
        ("num_exp_vals", ctypes.c_uint32),
        ("has_postselection", ctypes.c_uint32),
        ("num_instructions", ctypes.c_uint32),
        ("instructions", ctypes.c_void_p),
        ("num_words", ctypes.c_uint32),
        ("num_pauli_masks", ctypes.c_uint32),
        ("pauli_x", ctypes.c_void_p),
        ("pauli_z", ctypes.c_void_p),
        ("pauli_sign", ctypes.c_void_p),
        ("num_exp_val_masks", ctypes.c_uint32),
        ("exp_val_x", ctypes.c_void_p),
        ("exp_val_z", ctypes.c_void_p),
        ("exp_val_sign", ctypes.c_void_p),
        ("num_noise_sites", ctypes.c_uint32),
        ("noise_site_offsets", ctypes.c_void_p),
        ("num_noise_channels", ctypes.c_uint32),
        ("noise_channel_prob", ctypes.c_void_p),
        ("noise_channel_x", ctypes.c_void_p),
        ("noise_channel_z", ctypes.c_void_p),
        ("noise_hazards", ctypes.c_void_p),
        ("num_readout_noise", ctypes.c_uint32),
        ("readout_meas_idx", ctypes.c_void_p),
        ("readout_prob", ctypes.c_void_p),
        ("num_detector_lists", ctypes.c_uint32),
        ("detector_offsets", ctypes.c_void_p),
        ("detector_targets", ctypes.c_void_p),
        ("num_observable_lists", ctypes.c_uint32),
        ("observable_offsets", ctypes.c_void_p),
        ("observable_targets", ctypes.c_void_p),
        ("num_u2", ctypes.c_uint32),
        ("u2_data", ctypes.c_void_p),
        ("u2_out", ctypes.c_void_p),
        ("num_u4", ctypes.c_uint32),
        ("u4_data", ctypes.c_void_p),
        ("u4_out", ctypes.c_void_p),
        ("num_expected_observables", ctypes.c_uint32),
        ("expected_observables", ctypes.c_void_p),
        ("global_weight_re", ctypes.c_double),
        ("global_weight_im", ctypes.c_double),
    ]


_ARRAY_FIELDS = {
    # name: (dtype, columns or None)
    "instructions": (np.uint8, 32),
    "pauli_x": (np.uint64, "W"), "pauli_z": (np.uint64, "W"), "pauli_sign": (np.uint8, None),
    "exp_val_x": (np.uint64, "W"), "exp_val_z": (np.uint64, "W"), "exp_val_sign": (np.uint8, None),
    "noise_site_offsets": (np.uint32, None), "noise_channel_prob": (np.float64, None),
    "noise_channel_x": (np.uint64, "W"), "noise_channel_z": (np.uint64, "W"),
    "noise_hazards": (np.float64, None),
    "readout_meas_idx": (np.uint32, None), "readout_prob": (np.float64, None),
    "detector_offsets": (np.uint32, None), "detector_targets": (np.uint32, None),
    "observable_offsets": (np.uint32, None), "observable_targets": (np.uint32, None),
    "u2_data": (np.float64, 40), "u2_out": (np.uint8, 4),
    "u4_data": (np.float64, 544), "u4_out": (np.uint8, 16),
    "expected_observables": (np.uint8, None),
}
_META_FIELDS = ("num_qubits", "peak_rank", "num_measurements", "total_meas_slots",
                "num_detectors", "num_observables", "num_exp_vals", "has_postselection")


@dataclass
class Program:
    """A compiled program: bytecode + constant pool + metadata."""

    num_qubits: int
    peak_rank: int
    num_measurements: int
    total_meas_slots: int
    num_detectors: int = 0
    num_observables: int = 0
    num_exp_vals: int = 0
    has_postselection: int = 0
    instructions: np.ndarray = field(default_factory=lambda: np.zeros((0, 32), np.uint8))
    pauli_x: Optional[np.ndarray] = None
    pauli_z: Optional[np.ndarray] = None
    pauli_sign: Optional[np.ndarray] = None
    exp_val_x: Optional[np.ndarray] = None
    exp_val_z: Optional[np.ndarray] = None
    exp_val_sign: Optional[np.ndarray] = None
    noise_site_offsets: Optional[np.ndarray] = None
    noise_channel_prob: Optional[np.ndarray] = None
    noise_channel_x: Optional[np.ndarray] = None
    noise_channel_z: Optional[np.ndarray] = None
    noise_hazards: Optional[np.ndarray] = None
    readout_meas_idx: Optional[np.ndarray] = None
    readout_prob: Optional[np.ndarray] = None
    detector_offsets: Optional[np.ndarray] = None
    detector_targets: Optional[np.ndarray] = None
    observable_offsets: Optional[np.ndarray] = None
    observable_targets: Optional[np.ndarray] = None
    u2_data: Optional[np.ndarray] = None
    u2_out: Optional[np.ndarray] = None
    u4_data: Optional[np.ndarray] = None
    u4_out: Optional[np.ndarray] = None
    expected_observables: Optional[np.ndarray] = None
    global_weight: complex = 1.0 + 0.0j
    name: str = ""

    def __post_init__(self) -> None:
        W = self.num_words
        for fname, (dt, cols) in _ARRAY_FIELDS.items():
            a = getattr(self, fname)
            ncol = W if cols == "W" else cols
            if a is None:
                a = np.zeros((0,) if ncol is None else (0, ncol), dtype=dt)
            a = np.ascontiguousarray(np.asarray(a, dtype=dt))
            if ncol is not None:
                a = a.reshape(-1, ncol)
            setattr(self, fname, a)
        for off in ("noise_site_offsets", "detector_offsets", "observable_offsets"):
            if getattr(self, off).size == 0:
                setattr(self, off, np.zeros(1, np.uint32))
        self._image = None
        self._keep = None

    # ------------------------------------------------------------------ sizes
    @property
    def num_words(self) -> int:
        return max(1, (self.num_qubits + 63) // 64) if self.num_qubits > 0 else 1

    @property
    def num_instructions(self) -> int:
        return int(self.instructions.shape[0])

    @property
    def opcodes(self) -> np.ndarray:
        return self.instructions[:, 0]

    @property
    def axis_1(self) -> np.ndarray:
        return self.instructions[:, 4:6].copy().view(np.uint16).reshape(-1)

    @property
    def axis_2(self) -> np.ndarray:
        return self.instructions[:, 6:8].copy().view(np.uint16).reshape(-1)

    def active_k_history(self) -> np.ndarray:
        """k before each instruction. The trajectory is outcome independent
        (EXPAND* adds an axis, active measurements remove one), which is what
        the reference records in SourceMap::active_k_history
        (src/clifft/backend/source_map.h)."""
        k = 0
        out = np.zeros(self.num_instructions, np.int32)
        for i, op in enumerate(self.opcodes.tolist()):
            out[i] = k
            if op in EXPANDS:
                k += 1
            elif op in ACTIVE_MEAS:
                k -= 1
        return out

    # --------------------------------------------------------------- C image
    def image(self) -> ProgramImage:
        """ctypes image pointing into this object's arrays (kept alive here)."""
        if self._image is not None:
            return self._image
        img = ProgramImage()
        keep = []
        for m in _META_FIELDS:
            setattr(img, m, int(getattr(self, m)))
        img.num_instructions = self.num_instructions
        img.num_words = self.num_words

        def ptr(a):
            keep.append(a)
            return a.ctypes.data if a.size else None

        for fname in _ARRAY_FIELDS:
            setattr(img, fname, ptr(getattr(self, fname)))
        img.num_pauli_masks = self.pauli_sign.shape[0]
        img.num_exp_val_masks = self.exp_val_sign.shape[0]
        img.num_noise_sites = self.noise_site_offsets.shape[0] - 1
        img.num_noise_channels = self.noise_channel_prob.shape[0]
        img.num_readout_noise = self.readout_meas_idx.shape[0]
        img.num_detector_lists = self.detector_offsets.shape[0] - 1
        img.num_observable_lists = self.observable_offsets.shape[0] - 1
        img.num_u2 = self.u2_out.shape[0]
        img.num_u4 = self.u4_out.shape[0]
        img.num_expected_observables = self.expected_observables.shape[0]
        img.global_weight_re = float(np.real(self.global_weight))
        img.global_weight_im = float(np.imag(self.global_weight))
        self._image, self._keep = img, keep
        return img

    @classmethod
    def from_image(cls, img: ProgramImage, name: str = "") -> "Program":
        """Deep-copy a C image (e.g. one returned by the reference harness)."""
        W = img.num_words

        def arr(p, n, dt, cols=None):
            cnt = n * (cols or 1)
            if cnt == 0 or not p:
                return np.zeros((0,) if cols is None else (0, cols), dt)
            a = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                      shape=(cnt,)).copy()
            return a if cols is None else a.reshape(n, cols)

        ns, nc = img.num_noise_sites, img.num_noise_channels
        return cls(
            num_qubits=img.num_qubits, peak_rank=img.peak_rank,
            num_measurements=img.num_measurements, total_meas_slots=img.total_meas_slots,
            num_detectors=img.num_detectors, num_observables=img.num_observables,
            num_exp_vals=img.num_exp_vals, has_postselection=img.has_postselection,
            instructions=arr(img.instructions, img.num_instructions, np.uint8, 32),
            pauli_x=arr(img.pauli_x, img.num_pauli_masks, np.uint64, W),
            pauli_z=arr(img.pauli_z, img.num_pauli_masks, np.uint64, W),
            pauli_sign=arr(img.pauli_sign, img.num_pauli_masks, np.uint8),
            exp_val_x=arr(img.exp_val_x, img.num_exp_val_masks, np.uint64, W),
            exp_val_z=arr(img.exp_val_z, img.num_exp_val_masks, np.uint64, W),
            exp_val_sign=arr(img.exp_val_sign, img.num_exp_val_masks, np.uint8),
            noise_site_offsets=arr(img.noise_site_offsets, ns + 1, np.uint32),
            noise_channel_prob=arr(img.noise_channel_prob, nc, np.float64),
            noise_channel_x=arr(img.noise_channel_x, nc, np.uint64, W),
            noise_channel_z=arr(img.noise_channel_z, nc, np.uint64, W),
            noise_hazards=arr(img.noise_hazards, ns, np.float64),
            readout_meas_idx=arr(img.readout_meas_idx, img.num_readout_noise, np.uint32),
            readout_prob=arr(img.readout_prob, img.num_readout_noise, np.float64),
            detector_offsets=arr(img.detector_offsets, img.num_detector_lists + 1, np.uint32),
            detector_targets=arr(img.detector_targets,
                                 int(arr(img.detector_offsets, img.num_detector_lists + 1,
                                         np.uint32)[-1]), np.uint32),
            observable_offsets=arr(img.observable_offsets, img.num_observable_lists + 1, np.uint32),
            observable_targets=arr(img.observable_targets,
                                   int(arr(img.observable_offsets, img.num_observable_lists + 1,
                                           np.uint32)[-1]), np.uint32),
            u2_data=arr(img.u2_data, img.num_u2, np.float64, 40),
            u2_out=arr(img.u2_out, img.num_u2, np.uint8, 4),
            u4_data=arr(img.u4_data, img.num_u4, np.float64, 544),
            u4_out=arr(img.u4_out, img.num_u4, np.uint8, 16),
            expected_observables=arr(img.expected_observables, img.num_expected_observables,
                                     np.uint8),
            global_weight=complex(img.global_weight_re, img.global_weight_im),
            name=name,
        )

    # ------------------------------------------------------------ persistence
    def to_npz_dict(self) -> dict:
        d = {m: np.array(getattr(self, m)) for m in _META_FIELDS}
        for fname in _ARRAY_FIELDS:
            d[fname] = getattr(self, fname)
        d["global_weight"] = np.array([np.real(self.global_weight), np.imag(self.global_weight)])
        d["name"] = np.array(self.name)
        return d

    def save(self, path: str) -> None:
        np.savez_compressed(path, **self.to_npz_dict())

    @classmethod
    def from_npz_dict(cls, d) -> "Program":
        kw = {m: int(d[m]) for m in _META_FIELDS}
        for fname in _ARRAY_FIELDS:
            kw[fname] = d[fname]
        gw = d["global_weight"]
        kw["global_weight"] = complex(float(gw[0]), float(gw[1]))
        kw["name"] = str(d["name"]) if "name" in d else ""
        return cls(**kw)

    @classmethod
    def load(cls, path: str) -> "Program":
        with np.load(path, allow_pickle=False) as d:
            return cls.from_npz_dict(d)

    def with_instructions(self, instructions: np.ndarray, peak_rank: Optional[int] = None) -> "Program":
        d = self.to_npz_dict()
        d["instructions"] = instructions
        if peak_rank is not None:
            d["peak_rank"] = np.array(peak_rank)
        return Program.from_npz_dict(d)

    def summary(self) -> dict:
        ops = self.opcodes
        hist = {OPCODES[o]: int(c) for o, c in zip(*np.unique(ops, return_counts=True))}
        kh = self.active_k_history()
        return {"name": self.name, "n": self.num_qubits, "peak_rank": self.peak_rank,
                "instructions": self.num_instructions, "meas_slots": self.total_meas_slots,
                "detectors": self.num_detectors, "max_k": int(kh.max(initial=0)), "ops": hist}
