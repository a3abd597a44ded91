"""Beams and the beam-interpolation plugin.

Mirrors ``matvis.core.beams`` (``BeamInterpolator``, ``_wrangle_beams``;
core/beams.py:35-208) and ``matvis.gpu.beams.GPUBeamInterpolator``
(gpu/beams.py:22-124).  pyuvdata is not a dependency: beams are the
:class:`~matvis_b200.beam_models.GridBeam` and
:class:`~matvis_b200.beam_models.GaussianBeam` descriptions (re-exported here).

Interpolation runs in ``mvb_beam_interp`` / ``mvb_beam_gaussian``.
"""

from __future__ import annotations

from abc import ABC, abstractmethod

import numpy as np
import torch

from . import _lib, devcache
from ._lib import check, ptr, stream_handle
from .beam_models import GaussianBeam, GridBeam  # noqa: F401  (re-exported)


def _wrangle_beams(beam_idx, beam_list, polarized, nant, freq):
    """Checks of core/beams.py:35-99 (no frequency interpolation: grids are achromatic)."""
    beam_list = list(beam_list)
    nbeam = len(beam_list)
    if beam_idx is None and nbeam not in (1, nant):
        raise ValueError("If number of beams provided is not 1 or nant, beam_idx must be provided.")
    if beam_idx is not None:
        beam_idx = np.asarray(beam_idx)
        if beam_idx.shape != (nant,):
            raise ValueError("beam_idx must be length nant")
        if not all(0 <= i < nbeam for i in beam_idx):
            raise ValueError("beam_idx contains indices greater than the number of beams")
    if polarized and any(getattr(b, "beam_type", None) != "efield" for b in beam_list):
        raise ValueError("beam type must be efield if using polarized=True")
    return beam_list, nbeam, beam_idx


def resolve_beam_idx(beam_idx, nbeam: int, nant: int) -> np.ndarray:
    """Explicit per-antenna beam index (None: beam a for antenna a, or beam 0)."""
    if beam_idx is not None:
        return np.asarray(beam_idx, dtype=np.int32)
    if nbeam == nant:
        return np.arange(nant, dtype=np.int32)
    return np.zeros(nant, dtype=np.int32)


def gpu_beam_interpolation(beam, daz, dza, azmin, az, za, beam_at_src=None, order: int = 1, device=None):
    """Order-1 interpolation of grids at (az, za); mirrors gpu/beams.py:127-200.

    ``beam`` (nbeam, nax, nfeed, nza, naz) real (power, sqrt applied) or complex;
    returns (nbeam, nfeed, nax, nsrc) complex on the device (complex128 for
    float64 / complex128 grids, complex64 otherwise).
    """
    if order != 1:
        raise ValueError("only order=1 interpolation is implemented")
    dev = _lib.require_cuda(device)
    b = np.asarray(beam.cpu() if isinstance(beam, torch.Tensor) else beam)
    if b.dtype in (np.dtype("float32"), np.dtype("complex64")):
        ctype = torch.complex64
    elif b.dtype in (np.dtype("float64"), np.dtype("complex128")):
        ctype = torch.complex128
    else:
        raise ValueError(f"Got {b.dtype} as the dtype for beam, which is unrecognized")
    nbeam, nax, nfeed, nza, naz = b.shape
    if np.iscomplexobj(b):
        grids, kind = torch.as_tensor(np.ascontiguousarray(b.astype(np.complex64)), device=dev), 0
    else:
        grids, kind = torch.as_tensor(np.ascontiguousarray(b.astype(np.float32)), device=dev), 1
    params = np.stack(
        [np.broadcast_to(np.asarray(daz, dtype=np.float64), (nbeam,)),
         np.broadcast_to(np.asarray(dza, dtype=np.float64), (nbeam,)),
         np.broadcast_to(np.asarray(azmin, dtype=np.float64), (nbeam,))], axis=1)
    params = torch.as_tensor(np.ascontiguousarray(params), device=dev)
    azza = torch.as_tensor(np.stack([np.asarray(az, np.float64), np.asarray(za, np.float64)]), device=dev).contiguous()
    nsrc = azza.shape[1]
    out = beam_at_src
    if out is None:
        out = torch.zeros((nbeam, nfeed, nax, nsrc), dtype=ctype, device=dev)
    elif tuple(out.shape) != (nbeam, nfeed, nax, nsrc):
        raise ValueError("beam_at_src has the wrong shape")
    check(
        _lib.lib.mvb_beam_interp_azza(
            ptr(grids), kind, nbeam, nax, nfeed, nza, naz, ptr(params), ptr(azza), nsrc, nsrc, ptr(out),
            1 if out.dtype == torch.complex128 else 0, stream_handle(),
        )
    )
    return out


class BeamInterpolator(ABC):
    """Base class of beam interpolators (core/beams.py:102-208)."""

    def __init__(self, beam_list, beam_idx, polarized, nant, freq, nsrc, spline_opts=None, precision=1):
        self.beam_list, self.nbeam, self.beam_idx = _wrangle_beams(
            beam_idx=beam_idx, beam_list=beam_list, polarized=polarized, nant=nant, freq=freq
        )
        self.polarized = polarized
        self.nant = nant
        self.freq = freq
        self.spline_opts = spline_opts or {}
        self.nfeed = self.nax = 2 if polarized else 1
        if precision not in (1, 2):
            raise ValueError("precision must be 1 or 2")
        self.precision = precision
        self.complex_dtype = torch.complex64 if precision == 1 else torch.complex128
        self.nsrc = nsrc

    def setup(self):  # noqa: B027
        self.interpolated_beam = torch.zeros((self.nbeam, self.nfeed, self.nax, self.nsrc), dtype=self.complex_dtype)

    @abstractmethod
    def interp(self, tx, ty, out):
        """Fill ``out`` (nbeam, nfeed, nax, nsrc) with the beam at (tx, ty)."""

    def __call__(self, tx, ty, check: bool = True):
        self.interp(tx, ty, self.interpolated_beam)
        if check:
            sm = self.interpolated_beam.sum()
            if torch.isinf(sm).any() or torch.isnan(sm).any():
                raise ValueError("Beam interpolation resulted in an invalid value")
        return self.interpolated_beam


def is_chromatic(beams) -> bool:
    """True when a beam carries several frequencies (a beamfits beam)."""
    return any(hasattr(b, "at_frequency") for b in beams)


def beams_at_frequency(beams, freq: float) -> list:
    """Beams at one frequency: beamfits beams are interpolated to ``freq`` and
    re-gridded (core/beams.py:82-93); grid and analytic beams pass unchanged."""
    return [b.to_grid_beam(freq) if hasattr(b, "at_frequency") else b for b in beams]


class B200BeamInterpolator(BeamInterpolator):
    """Beam interpolation on the B200 (``mvb_beam_interp`` / ``mvb_beam_gaussian``).

    Replaces ``GPUBeamInterpolator`` (gpu/beams.py:22-124): the gridded path uses
    the same order-1 scheme with the same edge rule; analytic beams are evaluated
    on the device instead of on the host.
    """

    def __init__(self, *args, device=None, **kwargs):
        super().__init__(*args, **kwargs)
        self.device = _lib.require_cuda(device)

    def setup(self):
        dev = self.device
        kinds = {isinstance(b, GridBeam) for b in self.beam_list}
        if len(kinds) > 1:
            raise ValueError(
                "GPUBeamInterpolator only supports beam_lists with either all UVBeam or all AnalyticBeam objects."
            )
        self.use_interp = isinstance(self.beam_list[0], GridBeam)
        self.beam_index = resolve_beam_idx(self.beam_idx, self.nbeam, self.nant)
        self.beam_index_dev = torch.as_tensor(self.beam_index, dtype=torch.int32, device=dev)
        if self.use_interp:
            shapes = {b.data.shape[-2:] for b in self.beam_list}
            if len(shapes) > 1:
                raise ValueError("all gridded beams must share one (nza, naz) grid shape")
            nza, naz = shapes.pop()
            if self.polarized:
                grids = np.stack([b.data[: self.nax, : self.nfeed] for b in self.beam_list]).astype(np.complex64)
                if grids.shape[1:3] != (self.nax, self.nfeed):
                    raise ValueError("polarized gridded beams need nax = nfeed = 2")
                self.grid_kind = 0
            else:
                grids = np.stack([b.power_grid() for b in self.beam_list]).astype(np.float32)
                self.grid_kind = 1
            self.nza, self.naz = nza, naz
            params = np.array([[b.daz, b.dza, b.azmin] for b in self.beam_list], dtype=np.float64)
            grids = np.ascontiguousarray(grids)
            # equal grids share one device copy across jobs (served form)
            key = ("beam", devcache.device_key(dev), devcache.digest(grids, params))
            self.grids, self.params = devcache.CACHE.get(
                key, lambda: (torch.as_tensor(grids, device=dev), torch.as_tensor(params, device=dev)))
        else:
            if self.polarized:
                raise ValueError("beam type must be efield if using polarized=True")
            self.sigmas = torch.as_tensor([float(b.sigma) for b in self.beam_list], dtype=torch.float64, device=dev)
        self.interpolated_beam = torch.zeros(
            (self.nbeam, self.nfeed, self.nax, self.nsrc), dtype=self.complex_dtype, device=dev
        )
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._coord_ws = None  # made at the first launch, or handed over by the engine

    def launch(self, crd: torch.Tensor, ld: int, n_dev, nsrc: int, out: torch.Tensor, stream=None, status=None):
        """Enqueue the interpolation at crd (SoA float64, leading dimension ld)."""
        out_c128 = 1 if out.dtype == torch.complex128 else 0
        nout = out.shape[-1]
        sh = stream_handle(stream)
        if self.use_interp:
            # per-source grid coordinates, computed once for all the planes
            if self._coord_ws is None or self._coord_ws.numel() < 2 * self.nbeam * nout:
                self._coord_ws = torch.empty(2 * self.nbeam * nout, dtype=torch.float64, device=self.device)
            ws = self._coord_ws
            check(
                _lib.lib.mvb_beam_interp(
                    ptr(self.grids), self.grid_kind, self.nbeam, self.nax, self.nfeed, self.nza, self.naz,
                    ptr(self.params), ptr(crd), ld, ptr(n_dev), nsrc, ptr(out), out_c128, nout, ptr(status),
                    ptr(ws), ws.numel() * 8, sh,
                )
            )
        else:
            check(
                _lib.lib.mvb_beam_gaussian(
                    ptr(self.sigmas), self.nbeam, ptr(crd), ld, ptr(n_dev), nsrc, ptr(out), out_c128, nout, sh
                )
            )

    def interp(self, tx, ty, out):
        """Beam at direction cosines (tx, ty) (device float64, length <= nsrc)."""
        tx = torch.as_tensor(tx, dtype=torch.float64, device=self.device)
        ty = torch.as_tensor(ty, dtype=torch.float64, device=self.device)
        n = tx.shape[0]
        ld = ty.data_ptr() - tx.data_ptr()
        if ld % 8 == 0 and ld // 8 >= n and tx.is_contiguous() and ty.is_contiguous():
            crd, ldn = tx, ld // 8  # already SoA rows of one buffer
        else:
            crd = torch.stack([tx, ty]).contiguous()
            ldn = n
        self.launch(crd, ldn, None, n, out)
