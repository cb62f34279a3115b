"""Expectation values and their adjoint gradients (clifft_gpu_expval_grad).

Parameters are the program's rotation instructions (ARRAY_ROT, EXPAND_ROT) in
program order; parameter j is the phase angle phi_j (radians) of its payload
(cos phi_j, sin phi_j). For an RZ(theta) lowered to one such instruction,
phi = theta (the payload is e^{i theta}, the global phase dropped).

    ev, g = expval_grad(program, phases)   # (B, E), (B, E, P)
    ev = ExpVal.apply(phases_tensor, program)   # differentiable in torch
"""

from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import _native as N
from . import api
from .program import OP, Program

_ROT_OPS = (OP["ARRAY_ROT"], OP["EXPAND_ROT"])


def rot_instructions(program: Program) -> np.ndarray:
    """Instruction indices of the rotation parameters, in parameter order."""
    return np.nonzero(np.isin(program.opcodes, _ROT_OPS))[0]


def rot_phases(program: Program) -> np.ndarray:
    """The program's own rotation phases phi_j = atan2(sin, cos) of each payload."""
    ins = program.instructions[rot_instructions(program)]
    cs = ins[:, 8:16].copy().view(np.float64).reshape(-1)
    sn = ins[:, 16:24].copy().view(np.float64).reshape(-1)
    return np.arctan2(sn, cs)


def with_rot_phases(program: Program, phases: np.ndarray) -> Program:
    """A copy of `program` whose rotation payloads are (cos phi_j, sin phi_j)."""
    idx = rot_instructions(program)
    phases = np.asarray(phases, np.float64).reshape(-1)
    if phases.shape[0] != idx.shape[0]:
        raise ValueError(f"expected {idx.shape[0]} phases, got {phases.shape[0]}")
    ins = program.instructions.copy()
    ins[idx, 8:16] = np.cos(phases).astype(np.float64).view(np.uint8).reshape(-1, 8)
    ins[idx, 16:24] = np.sin(phases).astype(np.float64).view(np.uint8).reshape(-1, 8)
    return program.with_instructions(ins)


def num_rot_params(program: Program) -> int:
    return int(N.lib().clifft_gpu_program_num_rot_params(api.load(program).handle))


def expval_grad(program: Program, phases: Optional[np.ndarray] = None, *, precision: str = "fp64",
                batch: Optional[int] = None) -> Tuple[np.ndarray, np.ndarray]:
    """(exp_vals (B, E), grads (B, E, P)) for B parameter vectors (rows of
    `phases`, shape (B, P)); phases=None uses the program's payloads (B = batch or 1)."""
    if precision not in api._PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(api._PRECISIONS)}")
    dp = api.load(program)
    npar = int(N.lib().clifft_gpu_program_num_rot_params(dp.handle))
    if phases is not None:
        ph = np.ascontiguousarray(np.asarray(phases, np.float64).reshape(-1, npar) if npar else
                                  np.zeros((int(np.shape(phases)[0]), 0)))
        b = ph.shape[0]
    else:
        ph = None
        b = int(batch or 1)
    ev = np.zeros((b, program.num_exp_vals), np.float64)
    g = np.zeros((b, program.num_exp_vals, npar), np.float64)
    a = N.GradArgs(batch=b, precision=api._PRECISIONS[precision], flags=0,
                   phases=ph.ctypes.data if (ph is not None and ph.size) else None)
    N.check(N.lib().clifft_gpu_expval_grad(dp.handle, ctypes.byref(a), ev.ctypes.data,
                                           g.ctypes.data if g.size else None), "clifft_gpu_expval_grad")
    return ev, g


def _torch_function():
    import torch

    class ExpVal(torch.autograd.Function):
        """<P_e>(phi) for a batch of phase vectors phi (B, P), float64, on the
        current CUDA device or the host; backward contracts the adjoint
        gradients computed in the same call."""

        @staticmethod
        def forward(ctx, phases, program, precision="fp64"):
            dp = api.load(program)
            npar = int(N.lib().clifft_gpu_program_num_rot_params(dp.handle))
            x = phases.detach().to(dtype=torch.float64).reshape(-1, npar).contiguous()
            dev = torch.device("cuda", torch.cuda.current_device())
            xd = x.to(dev)
            b = xd.shape[0]
            ev = torch.zeros((b, program.num_exp_vals), dtype=torch.float64, device=dev)
            g = torch.zeros((b, program.num_exp_vals, max(npar, 1)), dtype=torch.float64, device=dev)
            a = N.GradArgs(batch=b, precision=api._PRECISIONS[precision], flags=N.CLIFFT_GPU_DEVICE_PTRS,
                           phases=xd.data_ptr() if npar else None,
                           stream=torch.cuda.current_stream().cuda_stream)
            N.check(N.lib().clifft_gpu_expval_grad(dp.handle, ctypes.byref(a), ev.data_ptr(), g.data_ptr()),
                    "clifft_gpu_expval_grad")
            ctx.save_for_backward(g[..., :npar])
            ctx.in_device = phases.device
            return ev.to(phases.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            go = grad_out.to(device=g.device, dtype=torch.float64)
            return torch.einsum("be,bep->bp", go, g).to(ctx.in_device), None, None

    return ExpVal


_EXPVAL = None


def __getattr__(name):
    global _EXPVAL
    if name == "ExpVal":
        if _EXPVAL is None:
            _EXPVAL = _torch_function()
        return _EXPVAL
    raise AttributeError(name)
