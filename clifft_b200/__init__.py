"""clifft_b200 -- B200-native (sm_100a) backend for Clifft's Schrodinger VM.

The package executes the reference compiler's bytecode (a `Program`, the flat
form of clifft::CompiledModule) on the GPU through the C ABI declared in
include/clifft_gpu.h:

    import clifft_b200 as cb
    res = cb.sample(program, shots=100_000, seed=1)            # clifft.sample
    res = cb.sample_survivors(program, 10**6, keep_records=True)  # clifft.sample_survivors
    lp  = cb.record_probabilities(program, records)            # clifft.record_probabilities
    res = cb.sample_k(program, shots=10**5, k=2)                # clifft.sample_k
    ref = cb.compute_reference_syndrome(program)                # clifft.compute_reference_syndrome
"""

from .program import OP, OPCODES, Program
from ._sample_result import SampleResult
from .api import (DeviceProgram, compute_reference_syndrome, load, noise_site_probabilities,
                  record_probabilities, run, sample, sample_k, sample_k_survivors, sample_survivors, trim)
from ._native import backend_name

__all__ = [
    "OP", "OPCODES", "Program", "SampleResult", "DeviceProgram", "load", "run", "sample",
    "sample_survivors", "sample_k", "sample_k_survivors", "noise_site_probabilities",
    "record_probabilities", "compute_reference_syndrome", "trim", "backend_name",
]
