"""Beam descriptions (host data only; nothing here touches the GPU library).

pyuvdata is not a dependency, so beams are given as

* :class:`GridBeam`  -- a beam tabulated on a regular (za, az) grid, the array a
  ``UVBeam`` holds after ``_prepare_coordinate_data`` (gpu/beams.py:15-19):
  ``data`` (nax, nfeed, nza, naz), complex E-field or real power;
* :class:`GaussianBeam` -- an achromatic Gaussian power beam in zenith angle.

The interpolation plugin that evaluates them on the device is
``matvis_b200.beams.B200BeamInterpolator``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class GridBeam:
    """A beam on a regular az/za grid (radians); ``za[0]`` must be 0."""

    data: np.ndarray
    az: np.ndarray
    za: np.ndarray
    beam_type: str = "efield"
    _dev: dict = field(default_factory=dict, repr=False, compare=False)

    def __post_init__(self):
        self.data = np.asarray(self.data)
        self.az = np.asarray(self.az, dtype=np.float64)
        self.za = np.asarray(self.za, dtype=np.float64)
        if self.data.ndim != 4:
            raise ValueError("GridBeam.data must have shape (nax, nfeed, nza, naz)")
        if self.data.shape[-2:] != (len(self.za), len(self.az)):
            raise ValueError("GridBeam.data grid shape does not match (za, az)")
        if self.beam_type not in ("efield", "power"):
            raise ValueError("beam_type must be 'efield' or 'power'")
        if abs(self.za[0]) > 1e-12:
            raise ValueError("za grid must start at 0 (za / dza is the row coordinate)")

    @property
    def daz(self) -> float:
        return float(np.diff(self.az)[0])

    @property
    def dza(self) -> float:
        return float(np.diff(self.za)[0])

    @property
    def azmin(self) -> float:
        return float(np.min(self.az))

    @property
    def Nfeeds(self) -> int:
        return self.data.shape[1]

    def power_grid(self, feed: int = 0) -> np.ndarray:
        """Single-feed power pattern (1, 1, nza, naz): sum over vector axes of |E|^2."""
        if self.beam_type == "power":
            return np.real(self.data[:1, :1]).astype(np.float64)
        return np.sum(np.abs(self.data[:, feed : feed + 1]) ** 2, axis=0, keepdims=True)


@dataclass
class GaussianBeam:
    """Achromatic Gaussian power beam: E-field amplitude exp(-za^2 / (2 sigma^2))."""

    sigma: float
    beam_type: str = "power"
