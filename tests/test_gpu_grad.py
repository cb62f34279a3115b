"""Adjoint gradients of expectation values (clifft_gpu_expval_grad).

Checks: the forward values equal the sampling executor's and the reference
executor's EXP_VAL outputs; d<P>/dphi equals FP64 central differences
(h = 1e-4) of the reference executor run on phase-shifted payloads, within
1e-6; the FP32-statevector gradient is within 1e-4 of the FP64 one; batches
of phase vectors; every array / expansion opcode on random measurement-free
programs; the torch.autograd.Function contracts the same gradients.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import clifft_b200 as cb
from _programs import random_program
from clifft_b200 import grad as GR
from clifft_b200.program import Program
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

PROGRAMS = os.path.join(os.path.dirname(__file__), "golden", "programs")
H = 1e-4
FD_TOL = 1e-6


def _cfg4():
    return Program.load(os.path.join(PROGRAMS, "cfg4.npz"))


def _active_probes(prog, seed=0):
    from clifft_b200.workloads import active_probes
    return active_probes(prog, seed)


def _cpu_expvals(prog):
    if O.ref_available():
        return O.ref_sample(prog, 1, 0)["exp_vals"][0]
    return O.run(prog, 1, seed=0)["exp_vals"][0]


def _central_differences(prog, phases, params):
    out = []
    for j in params:
        up, dn = phases.copy(), phases.copy()
        up[j] += H
        dn[j] -= H
        ep = _cpu_expvals(GR.with_rot_phases(prog, up))
        em = _cpu_expvals(GR.with_rot_phases(prog, dn))
        out.append((ep - em) / (2 * H))
    return np.stack(out, axis=-1)  # (E, len(params))


@pytest.mark.parametrize("probes", ["circuit", "active"])
def test_cfg4_values_and_gradients_match_reference_central_differences(probes):
    prog = _cfg4() if probes == "circuit" else _active_probes(_cfg4())
    phases = GR.rot_phases(prog)
    assert GR.num_rot_params(prog) == phases.shape[0] == 32
    ev, g = GR.expval_grad(prog, None, precision="fp64")
    assert ev.shape == (1, prog.num_exp_vals) and g.shape == (1, prog.num_exp_vals, 32)
    np.testing.assert_allclose(ev[0], cb.run(prog, 1, 0, precision="fp64")["exp_vals"][0], atol=1e-10)
    np.testing.assert_allclose(ev[0], _cpu_expvals(prog), atol=1e-10)
    fd = _central_differences(prog, phases, range(32))
    np.testing.assert_allclose(g[0], fd, atol=FD_TOL)
    if probes == "active":
        assert np.abs(ev).max() > 1e-2 and np.abs(g).max() > 1e-3  # non-trivial values and slopes


def test_fp32_statevector_gradient_within_1e4_of_fp64():
    prog = _active_probes(_cfg4())
    _, g64 = GR.expval_grad(prog, None, precision="fp64")
    e32, g32 = GR.expval_grad(prog, None, precision="fp32")
    np.testing.assert_allclose(g32, g64, atol=1e-4)
    np.testing.assert_allclose(e32[0], cb.run(prog, 1, 0, precision="fp64")["exp_vals"][0], atol=1e-4)


def test_batch_of_phase_vectors():
    prog = _active_probes(_cfg4(), seed=1)
    rng = np.random.default_rng(3)
    phases = rng.uniform(0.0, 2 * np.pi, size=(6, 32))
    ev, g = GR.expval_grad(prog, phases, precision="fp64")
    for b in (0, 5):
        q = GR.with_rot_phases(prog, phases[b])
        np.testing.assert_allclose(ev[b], cb.run(q, 1, 0, precision="fp64")["exp_vals"][0], atol=1e-10)
        fd = _central_differences(prog, phases[b], (0, 7, 19, 31))
        np.testing.assert_allclose(g[b][:, (0, 7, 19, 31)], fd, atol=FD_TOL)


@pytest.mark.parametrize("seed", range(8))
def test_random_programs_every_array_opcode(seed):
    prog = random_program(100 + seed, n=9, length=180, max_k=7, noise=False, classical=False,
                          expvals=True, measure=False, expand_bias=0.3, active_expvals=True)
    if prog.num_exp_vals == 0:
        pytest.skip("no EXP_VAL emitted")
    ev, g = GR.expval_grad(prog, None, precision="fp64")
    np.testing.assert_allclose(ev[0], _cpu_expvals(prog), atol=1e-10)
    npar = g.shape[2]
    if npar:
        fd = _central_differences(prog, GR.rot_phases(prog), range(npar))
        np.testing.assert_allclose(g[0], fd, atol=FD_TOL)


def test_torch_autograd_function():
    import torch
    prog = _active_probes(_cfg4(), seed=2)
    rng = np.random.default_rng(5)
    phases = torch.tensor(rng.uniform(0, 2 * np.pi, size=(3, 32)), dtype=torch.float64, requires_grad=True)
    ev = GR.ExpVal.apply(phases, prog)
    w = torch.tensor(rng.normal(size=(3, prog.num_exp_vals)), dtype=torch.float64)
    (ev * w).sum().backward()
    _, g = GR.expval_grad(prog, phases.detach().numpy(), precision="fp64")
    np.testing.assert_allclose(phases.grad.numpy(), np.einsum("be,bep->bp", w.numpy(), g), atol=1e-12)


def test_rejects_programs_with_measurements():
    prog = Program.load(os.path.join(PROGRAMS, "cfg0.npz"))
    with pytest.raises(ValueError, match="measurement-free"):
        GR.expval_grad(prog, None)
