"""Phase-term plugin (mirrors ``matvis.core.tau.TauCalculator``, core/tau.py:16-71).

``exptau = exp(+2 pi i nu / c * D . X)`` (the sign the reference code uses);
the phase in cycles is reduced mod 1 in FP64 on the device before the sincos.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_handle

#: Speed of light (m/s), SI-defined.
SPEED_OF_LIGHT = 299792458.0


class TauCalculator:
    """Computes exptau (nant, nsrc) with ``mvb_exptau``."""

    def __init__(self, antpos, freq: float, nsrc: int, precision: int = 1, gpu: bool = True, device=None):
        self.device = _lib.require_cuda(device)
        self.antpos_host = np.ascontiguousarray(np.asarray(antpos, dtype=np.float64))
        if self.antpos_host.ndim != 2 or self.antpos_host.shape[1] != 3:
            raise ValueError("antpos must have shape (NANTS, 3).")
        self.nant = len(self.antpos_host)
        self.freq = float(freq)
        self.nsrc = nsrc
        self.precision = precision
        self.ctype = torch.complex64 if precision == 1 else torch.complex128
        self.gpu = True

    def setup(self):
        self.antpos = torch.as_tensor(self.antpos_host, device=self.device)
        self.exptau = torch.zeros((self.nant, self.nsrc), dtype=self.ctype, device=self.device)

    def __call__(self, crdtop) -> torch.Tensor:
        crd = torch.as_tensor(crdtop, dtype=torch.float64, device=self.device)
        if crd.shape[0] != 3:
            raise ValueError("crdtop must have shape (3, NSRCS)")
        crd = crd.contiguous()
        n = min(crd.shape[1], self.nsrc)
        check(
            _lib.lib.mvb_exptau(
                ptr(self.antpos), self.nant, self.freq, ptr(crd), crd.shape[1], n, ptr(self.exptau),
                1 if self.ctype == torch.complex128 else 0, stream_handle(),
            )
        )
        return self.exptau
