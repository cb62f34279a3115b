"""Result type returned by the sampling calls.

Same attribute contract as the reference's `clifft.SampleResult`
(src/python/clifft/_sample_result.py:11-86): uint8 record arrays of shape
(rows, count), float64 exp_vals, survivor counters (None for plain sampling)
and tuple unpacking into (measurements, detectors, observables).
"""

from __future__ import annotations

from typing import Iterator, Optional

import numpy as np


class SampleResult:
    __slots__ = ("measurements", "detectors", "observables", "exp_vals", "total_shots",
                 "passed_shots", "discards", "logical_errors", "observable_ones", "stats")

    def __init__(self, measurements: np.ndarray, detectors: np.ndarray, observables: np.ndarray,
                 total_shots: Optional[int] = None, passed_shots: Optional[int] = None,
                 logical_errors: Optional[int] = None,
                 observable_ones: Optional[np.ndarray] = None,
                 exp_vals: Optional[np.ndarray] = None, stats: Optional[dict] = None) -> None:
        self.measurements = measurements
        self.detectors = detectors
        self.observables = observables
        self.exp_vals = (exp_vals if exp_vals is not None
                         else np.empty((measurements.shape[0], 0), dtype=np.float64))
        self.total_shots = total_shots
        self.passed_shots = passed_shots
        self.discards = (None if total_shots is None or passed_shots is None
                         else total_shots - passed_shots)
        self.logical_errors = logical_errors
        self.observable_ones = observable_ones
        self.stats = stats or {}

    def __iter__(self) -> Iterator[np.ndarray]:
        yield self.measurements
        yield self.detectors
        yield self.observables

    def __repr__(self) -> str:
        parts = [f"shots={self.measurements.shape[0]}",
                 f"measurements={self.measurements.shape[1]}"]
        if self.total_shots is not None:
            parts.append(f"total_shots={self.total_shots}")
        if self.passed_shots is not None:
            parts.append(f"passed_shots={self.passed_shots}")
        return f"SampleResult({', '.join(parts)})"
