"""Coordinate rotation plugin and horizon selection.

Mirrors ``matvis.core.coords.CoordinateRotation`` (core/coords.py:20-179): the
``_methods`` registry filled by ``__init_subclass__``, ``setup``, ``rotate(t)``
filling ``all_coords_topo`` and ``select_chunk(chunk, t)`` returning the
above-horizon coordinates, fluxes and count.  Coordinates stay in float64 on the
device at both precisions (the reference stores float32 at precision=1,
core/coords.py:84-97).

Two rotations are provided: the rigid LST rotation
``eci_to_enu_matrix(lst, lat) @ point_source_crd_eq(ra, dec)``
(coordinates.py:91-125, 174-200), with ``times`` given as LSTs in radians, and
the ERFA-style apparent place (cpu/coords.py:41-230) from per-time astrometry
parameters, with ``times`` in seconds.
"""

from __future__ import annotations

from abc import ABC, abstractmethod

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_handle
from .coordinates import (
    ENU_TO_ALTAZ,
    atioq_matrix,
    eci_to_enu_matrix,
    latitude_of,
    lsts_of,
    pack_astrom,
    point_source_crd_eq,
    radec_of,
)


class CoordinateRotation(ABC):
    """Equatorial -> topocentric rotation with horizon selection on the GPU."""

    _methods: dict = {}
    requires_gpu: bool = True

    def __init_subclass__(cls) -> None:
        CoordinateRotation._methods[cls.__name__] = cls
        return super().__init_subclass__()

    def __init__(
        self,
        flux,
        times,
        telescope_loc,
        skycoords,
        chunk_size: int | None = None,
        source_buffer: float = 0.55,
        precision: int = 1,
        gpu: bool = True,
        device=None,
    ):
        self.device = _lib.require_cuda(device)
        self.gpu = True
        self.precision = precision
        flux = np.asarray(flux)
        # core/coords.py:64: a (NSRCS, NFREQS, 2, 2) coherency is a polarised sky
        self._polarized = flux.ndim == 4
        if flux.ndim != 1 and not (self._polarized and flux.shape[2:] == (2, 2)):
            raise ValueError("flux must have shape (NSRCS,) or, for a polarised sky, (NSRCS, NFREQS, 2, 2)")
        self.flux_host = flux.astype(np.complex128 if self._polarized else np.float64)
        self.nsrc = len(flux)
        self.times = lsts_of(times)
        self.telescope_loc = telescope_loc
        self.latitude = latitude_of(telescope_loc)
        self.skycoords = skycoords
        ra, dec = radec_of(skycoords)
        if len(ra) != self.nsrc:
            raise ValueError("skycoords and flux must have the same length")
        self._ra, self._dec = ra, dec
        self.chunk_size = chunk_size or self.nsrc
        self.source_buffer = source_buffer
        # core/coords.py:77-82
        if self.chunk_size > 1000:
            self.nsrc_alloc = int(self.chunk_size * self.source_buffer)
        else:
            self.nsrc_alloc = self.chunk_size

    def setup(self):
        dev = self.device
        self.flux = torch.as_tensor(self.flux_host, device=dev)
        self.all_coords_topo = torch.zeros((3, self.nsrc), dtype=torch.float64, device=dev)
        self.coords_above_horizon = torch.zeros((3, self.nsrc_alloc), dtype=torch.float64, device=dev)
        self.flux_above_horizon = torch.zeros((self.nsrc_alloc,) + tuple(self.flux_host.shape[1:]),
                                              dtype=self.flux.dtype, device=dev)
        if self._polarized:
            self.radec = torch.as_tensor(np.stack([self._ra, self._dec]), dtype=torch.float64, device=dev)
            self.frame_rotation = torch.zeros((self.nsrc_alloc, 2), dtype=torch.float64, device=dev)
        self.kept_index = torch.zeros((max(self.nsrc_alloc, 1),), dtype=torch.int32, device=dev)
        self.n_above = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        nbytes = _lib.lib.mvb_horizon_ws_bytes(self.chunk_size)
        self._ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)

    def enqueue_select(self, chunk: int, stream=None, t: int = 0):
        """Enqueue the selection of one chunk; the count stays on the device (``n_above``).

        For a polarised sky the gathered coherency is also rotated from the
        (ra, dec) frame to the (alt, az) frame of time ``t`` (core/coords.py:128-147)."""
        c0 = chunk * self.chunk_size
        c1 = min((chunk + 1) * self.chunk_size, self.nsrc)
        c1 = max(c0, c1)
        sh = stream_handle(stream)
        scalar = not self._polarized
        check(
            _lib.lib.mvb_horizon_compact(
                ptr(self.all_coords_topo), self.nsrc, min(c0, self.nsrc), min(c1, self.nsrc),
                ptr(self.flux) if scalar else None, ptr(self.coords_above_horizon), ptr(self.kept_index),
                ptr(self.flux_above_horizon) if scalar else None, ptr(self.n_above), self.nsrc_alloc,
                ptr(self.status), ptr(self._ws), self._ws.numel(), sh,
            )
        )
        if self._polarized:
            r_avg = np.ascontiguousarray(ENU_TO_ALTAZ @ self.rigid_rotation(t))
            check(_lib.lib.mvb_coherency_rotation(
                ptr(self.radec), self.nsrc, ptr(self.kept_index), ptr(self.coords_above_horizon), self.nsrc_alloc,
                ptr(self.n_above), self.nsrc_alloc, r_avg.ctypes.data_as(_lib.c_void_p), ptr(self.frame_rotation),
                sh))
            check(_lib.lib.mvb_rotate_coherency(
                ptr(self.frame_rotation), ptr(self.kept_index), ptr(self.n_above), ptr(self.flux), self.nsrc,
                self.flux_host.shape[1], ptr(self.flux_above_horizon), self.nsrc_alloc, sh))

    def rigid_rotation(self, t: int) -> np.ndarray:
        """The rigid ICRS -> ENU rotation of time t (the frame of the coherency rotation)."""
        raise NotImplementedError

    def select_chunk(self, chunk: int, t: int):
        """Above-horizon sources of one chunk at time t; core/coords.py:99-150.

        Returns (coords (3, nsrc_alloc), flux (nsrc_alloc,), n); the count ``n`` is
        read back to the host (one synchronisation, as in the reference).
        """
        self.status.zero_()
        self.enqueue_select(chunk, t=t)
        n = int(self.n_above.item())
        if int(self.status.item()) & _lib.MVB_DEV_OVERFLOW:
            raise ValueError(
                f"nsrc_alloc ({self.nsrc_alloc}) is too small for the number of "
                f"sources above horizon ({n}). Try increasing source_buffer."
            )
        return self.coords_above_horizon, self.flux_above_horizon, n

    @abstractmethod
    def rotate(self, t: int):
        """Fill ``all_coords_topo`` for time index t."""


class CoordinateRotationLST(CoordinateRotation):
    """Rigid LST rotation of all sources, FP64 on the GPU (``mvb_rotate``)."""

    def setup(self):
        super().setup()
        self.eci = torch.as_tensor(np.ascontiguousarray(point_source_crd_eq(self._ra, self._dec)), device=self.device)

    def rotation_matrix(self, t: int) -> np.ndarray:
        return np.ascontiguousarray(eci_to_enu_matrix(self.times[t], self.latitude), dtype=np.float64)

    def rigid_rotation(self, t: int) -> np.ndarray:
        return self.rotation_matrix(t)

    def enqueue_rotate(self, t: int, stream=None):
        R = self.rotation_matrix(t)
        check(
            _lib.lib.mvb_rotate(
                ptr(self.eci), self.nsrc, R.ctypes.data_as(_lib.c_void_p), ptr(self.all_coords_topo),
                stream_handle(stream),
            )
        )

    def rotate(self, t: int):
        self.enqueue_rotate(t)


class CoordinateRotationERFA(CoordinateRotation):
    """ERFA-style apparent place on the GPU (the reference's CoordinateRotationERFA /
    GPUCoordinateRotationERFA, cpu/coords.py:41-230, gpu/coords.py:37-53).

    pyerfa is not a dependency, so the per-time astrometry parameters (the
    ``apco`` output: eh, em, v, bm1, bpn, eral, xpl, ypl, sphi, cphi) are given as
    ``astrom`` (one dict per time).  ``times`` are the times in seconds (for
    ``update_bcrs_every``).  Light deflection, aberration and BPN run per source in
    ``mvb_bcrs`` and are cached until ``update_bcrs_every`` seconds have passed;
    the CIRS -> ENU rotation runs in ``mvb_rotate``.
    """

    def __init__(self, update_bcrs_every: float = 0.0, *args, astrom=None, **kwargs):
        super().__init__(*args, **kwargs)
        if astrom is None or len(astrom) != len(self.times):
            raise ValueError("CoordinateRotationERFA needs one astrom parameter dict per time (pyerfa apco output)")
        self.astrom = list(astrom)
        self.update_bcrs_every = float(update_bcrs_every)
        self._time_of_last_evaluation = None

    def setup(self):
        super().setup()
        self.eci = torch.as_tensor(np.ascontiguousarray(point_source_crd_eq(self._ra, self._dec)), device=self.device)
        self._bcrs = torch.zeros_like(self.eci)

    def enqueue_rotate(self, t: int, stream=None):
        sh = stream_handle(stream)
        last = self._time_of_last_evaluation
        # cpu/coords.py:194-215: refresh when more than update_bcrs_every seconds passed
        if last is None or self.times[t] - self.times[last] > self.update_bcrs_every:
            a = pack_astrom(self.astrom[t])
            check(_lib.lib.mvb_bcrs(ptr(self.eci), self.nsrc, a.ctypes.data_as(_lib.c_void_p), ptr(self._bcrs), sh))
            self._time_of_last_evaluation = t
        R = np.ascontiguousarray(atioq_matrix(self.astrom[t]))
        check(_lib.lib.mvb_rotate(ptr(self._bcrs), self.nsrc, R.ctypes.data_as(_lib.c_void_p),
                                  ptr(self.all_coords_topo), sh))

    def rigid_rotation(self, t: int) -> np.ndarray:
        # BPN then CIRS -> ENU; light deflection and aberration enter per source
        return atioq_matrix(self.astrom[t]) @ np.asarray(self.astrom[t]["bpn"], dtype=np.float64).reshape(3, 3)

    def rotate(self, t: int):
        self.enqueue_rotate(t)
