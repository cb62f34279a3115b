"""Result type returned by the sampling calls.

Interface kept from the reference's `clifft.SampleResult`
(src/python/clifft/_sample_result.py:11-86), which callers unpack and index:
`measurements`, `detectors` and `observables` are uint8 arrays of shape
(rows, count); `exp_vals` is float64 (rows, num_exp_vals); iterating yields
the three record arrays in that order; `total_shots`, `passed_shots`,
`discards` and `logical_errors` are the survivor counters (None after plain
sampling), `observable_ones` counts surviving shots per observable.
"""

from __future__ import annotations

from typing import Iterator, Optional, Tuple

import numpy as np


class SampleResult:
    """Records of one sampling call, held as a (measurements, detectors,
    observables) triple plus the survivor counters the call reported.

    `stats` carries this backend's launch telemetry (kernel time, launch
    shape, bytes streamed); it is not part of the reference's interface."""

    def __init__(self, measurements: np.ndarray, detectors: np.ndarray, observables: np.ndarray,
                 total_shots: Optional[int] = None, passed_shots: Optional[int] = None,
                 logical_errors: Optional[int] = None,
                 observable_ones: Optional[np.ndarray] = None,
                 exp_vals: Optional[np.ndarray] = None, stats: Optional[dict] = None) -> None:
        records = tuple(np.asarray(a) for a in (measurements, detectors, observables))
        rows = {a.shape[0] for a in records}
        if len(rows) != 1:
            raise ValueError(f"record arrays disagree on the number of rows: {sorted(rows)}")
        self._records: Tuple[np.ndarray, np.ndarray, np.ndarray] = records
        (n_rows,) = rows
        self.exp_vals = np.zeros((n_rows, 0), np.float64) if exp_vals is None else np.asarray(exp_vals)
        self.total_shots = total_shots
        self.passed_shots = passed_shots
        self.logical_errors = logical_errors
        self.observable_ones = observable_ones
        self.stats = dict(stats) if stats else {}

    @property
    def measurements(self) -> np.ndarray:
        return self._records[0]

    @property
    def detectors(self) -> np.ndarray:
        return self._records[1]

    @property
    def observables(self) -> np.ndarray:
        return self._records[2]

    @property
    def discards(self) -> Optional[int]:
        """Shots dropped by post-selection; None unless both survivor counters are set."""
        if self.total_shots is None or self.passed_shots is None:
            return None
        return self.total_shots - self.passed_shots

    def __iter__(self) -> Iterator[np.ndarray]:
        return iter(self._records)

    def __repr__(self) -> str:
        rows, n_meas = self.measurements.shape[0], self.measurements.shape[1]
        text = f"{rows} rows of {n_meas} measurements"
        if self.total_shots is not None:
            text += f", {self.passed_shots} of {self.total_shots} shots kept"
        return f"<SampleResult: {text}>"
