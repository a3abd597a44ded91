"""Z-matrix plugin (mirrors ``matvis.core.getz.ZMatrixCalc``, core/getz.py:13-105).

Z is produced directly in the layout the Hermitian-product kernel reads (a
:class:`ZPanel`): split-precision real planes for the tensor-core modes, or a
plain complex64 matrix for the pair-list product.  Columns are ordered
k = src * nax + ax (the source sum does not depend on the order).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_handle


class ZPanel:
    """Device Z in split-plane (or plain complex64) layout.

    ``data``: (Kcap / KB, Mpad / 128, planes, 128, KB) for the tensor-core modes
    -- the Hermitian product's shared-memory image of each (64-byte k-block,
    128-row block), the 16-byte chunks of every row in 64-byte swizzled order,
    so that one operand of a product stage is one contiguous bulk copy -- and
    (M, Kcap) complex64 for the plain mode.
    ``n_dev`` / ``n_host`` give the valid source count; the valid K extent is
    that count times ``nax``.
    """

    def __init__(self, mode: int, nant: int, nfeed: int, nax: int, nsrc_cap: int, device, data=None):
        self.mode = mode
        self.nant, self.nfeed, self.nax = nant, nfeed, nax
        self.M = nant * nfeed
        self.nsrc_cap = nsrc_cap
        self.Mpad, self.Kcap = _lib.zpanel_shape(mode, self.M, nax * nsrc_cap)
        shape = self.data_shape(mode, self.M, self.Mpad, self.Kcap)
        if data is None:
            data = torch.zeros(shape, dtype=_lib.zpanel_dtype(mode), device=device)
        elif tuple(data.shape) != shape or data.dtype != _lib.zpanel_dtype(mode) or not data.is_contiguous():
            raise ValueError("panel storage has the wrong shape or type")
        self.data = data
        self.n_dev = None
        self.n_host = 0
        #: power-of-two factor the panel holds Z multiplied by (fp16x3 mode)
        self.scale = 1.0

    @staticmethod
    def data_shape(mode: int, M: int, Mpad: int, Kcap: int) -> tuple:
        if mode == _lib.Z_C64:
            return (M, Kcap)
        kb = _lib.zpanel_kblock(mode)
        return (Kcap // kb, Mpad // _lib.TILE, _lib.zpanel_planes(mode), _lib.TILE, kb)

    @classmethod
    def group(cls, n: int, mode: int, nant: int, nfeed: int, nax: int, nsrc_cap: int, device) -> list["ZPanel"]:
        """``n`` panels of one shape in one allocation, consecutive in memory (the
        operands of one grouped tau/Z and product launch; the byte distance
        between panels is ``panels[0].nbytes``)."""
        M = nant * nfeed
        Mpad, Kcap = _lib.zpanel_shape(mode, M, nax * nsrc_cap)
        store = torch.zeros((n,) + cls.data_shape(mode, M, Mpad, Kcap), dtype=_lib.zpanel_dtype(mode), device=device)
        return [cls(mode, nant, nfeed, nax, nsrc_cap, device, data=store[g]) for g in range(n)]

    @property
    def nbytes(self) -> int:
        return self.data.numel() * self.data.element_size()

    @property
    def shape(self):
        return (self.M, self.nax * self.nsrc_cap)

    def to_complex(self) -> torch.Tensor:
        """Reassemble Z (M, nax * n_host) as complex128 (inspection and tests)."""
        n = self.n_host if self.n_dev is None else int(self.n_dev.item())
        k = n * self.nax
        if self.mode == _lib.Z_C64:
            return self.data[:, :k].to(torch.complex128)
        nkb, nblk, p, rows, kb = self.data.shape
        # undo the 64-byte swizzle: chunk c of row r sits at chunk c ^ ((r >> 1) & 3)
        r = torch.arange(rows, device=self.data.device)[:, None]
        c = torch.arange(kb, device=self.data.device)[None, :]
        epc = kb // 4
        idx = (((c // epc) ^ ((r >> 1) & 3)) * epc + c % epc).expand(nkb, nblk, p, rows, kb)
        d = torch.gather(self.data, 4, idx).permute(2, 1, 3, 0, 4).reshape(p, nblk * rows, nkb * kb)
        d = d[:, : self.M, :k].to(torch.float64)
        re = d[0::2].sum(0) / self.scale
        im = d[1::2].sum(0) / self.scale
        return torch.complex(re, im)


class ZMatrixCalc:
    """Builds Z = A * sqrt(I) * exp(tau) on the device."""

    def __init__(self, nant, nfeed, nax, nsrc, ctype=None, gpu: bool = True, mode: int | str = _lib.GEMM_F16_3,
                 device=None):
        self.device = _lib.require_cuda(device)
        self.nant, self.nfeed, self.nax, self.nsrc = nant, nfeed, nax, nsrc
        self.ctype = ctype
        self.mode = _lib.GEMM_MODES[mode] if isinstance(mode, str) else int(mode)
        self.gpu = True

    def setup(self):
        self.z = ZPanel(self.mode, self.nant, self.nfeed, self.nax, self.nsrc, self.device)
        self._sflux = torch.zeros(max(self.nsrc, 1), dtype=torch.float32, device=self.device)

    def __call__(self, sqrt_flux, beam, exptau, beam_idx) -> ZPanel:
        """Z from exptau, sqrt flux and the interpolated beam; core/getz.py:52-105."""
        dev = self.device
        beam = torch.as_tensor(beam, device=dev)
        exptau = torch.as_tensor(exptau, device=dev)
        n = min(exptau.shape[1], self.nsrc)
        sf = torch.as_tensor(sqrt_flux, device=dev)[:n].to(torch.float32)
        self._sflux[:n].copy_(sf)
        bidx = None if beam_idx is None else torch.as_tensor(np.asarray(beam_idx), dtype=torch.int32, device=dev)
        if bidx is None and beam.shape[0] not in (1, self.nant):
            raise ValueError("beam_idx must be provided when nbeam is not 1 or nant")
        if bidx is None and beam.shape[0] == self.nant and self.nant > 1:
            bidx = torch.arange(self.nant, dtype=torch.int32, device=dev)
        b64 = beam.to(torch.complex64).contiguous()
        e_c128 = 1 if exptau.dtype == torch.complex128 else 0
        exptau = exptau.contiguous()
        if self.mode == _lib.GEMM_F16_3:
            # |Z| <= max |exptau| * max sqrt_flux * max |beam|, |exptau| = 1
            bound = float(sf.abs().max().item()) * float(b64.abs().max().item()) if n else 0.0
            self.z.scale = _lib.f16_scale(bound)
        check(
            _lib.lib.mvb_z_from_exptau(
                ptr(exptau), e_c128, exptau.shape[1], self.nant, n, ptr(self._sflux), ptr(b64), b64.shape[-1],
                b64.shape[0], ptr(bidx), self.nfeed, self.nax, self.mode, self.z.scale, ptr(self.z.data), self.z.Mpad,
                self.z.Kcap, stream_handle(),
            )
        )
        self.z.n_dev = None
        self.z.n_host = n
        return self.z

    def fused(self, antpos: torch.Tensor, freq: float, crd: torch.Tensor, ld: int, n_dev, nsrc: int,
              sflux: torch.Tensor, sidx, beam: torch.Tensor, beam_idx: torch.Tensor, stream=None,
              scale: float = 1.0) -> ZPanel:
        """Fused tau + Z (``mvb_tau_z``): no exptau round trip, count read on the device."""
        self.z.scale = scale
        check(
            _lib.lib.mvb_tau_z(
                ptr(antpos), self.nant, float(freq), ptr(crd), ld, ptr(n_dev), nsrc, ptr(sflux), ptr(sidx),
                ptr(beam), beam.shape[-1], beam.shape[0], ptr(beam_idx), self.nfeed, self.nax, self.mode, scale,
                ptr(self.z.data), self.z.Mpad, self.z.Kcap, stream_handle(stream),
            )
        )
        self.z.n_dev = n_dev
        self.z.n_host = nsrc
        return self.z
