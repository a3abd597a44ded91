"""Source-summing plugins (mirror ``matvis.core.matprod.MatProd`` and its backends).

* :class:`B200MatMul` -- upper-triangle Hermitian product on the tcgen05 tensor
  cores (``mvb_herk`` + ``mvb_herk_reduce``); replaces CPUMatMul / GPUMatMul
  (cpu/matprod.py:8-32, gpu/matprod.py:10-63).
* :class:`B200VectorDot` -- per-pair sums from shared-memory stages of the panel
  (``mvb_vecdot_staged``; ``mvb_vecdot`` for arrays too large to stage);
  replaces CPUVectorDot / GPUVectorDot (cpu/matprod.py:35-53, gpu/matprod.py:66-98).

Output layout (npairs, nfeed, nfeed) with out[i, p, q] pairing feed q of ant1 with
feed p of ant2, the reference's transposed feed convention (tests/test_matprod.py:57-65).
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, stream_handle
from .getz import ZPanel


def choose_k_chunk(n_tiles: int, kvalid: int, num_sms: int = 148, lo: int = 1024, hi: int = 8192) -> int:
    """k-slice length of the Hermitian product.

    Enough slices that every SM gets about two work units, no shorter than
    ``lo`` columns (partial-tile traffic) and no longer than ``hi`` (FP32
    accumulation length in TMEM before the FP64 reduction).
    """
    want_units = 2 * num_sms
    slices = max(1, -(-want_units // max(n_tiles, 1)))
    kc = -(-max(kvalid, 1) // slices)
    kc = -(-kc // _lib.K_ALIGN) * _lib.K_ALIGN
    return int(min(max(kc, lo), hi))


#: Per-column costs measured on one B200 on a config-3 slice (K = 1.0e6 columns,
#: the seeded 5,000 pairs at F = 2): mvb_vecdot_staged took 5.64 ms, i.e.
#: 2.8e-13 s per (pair x F^2 x column), mvb_vecdot (one warp per pair, for
#: arrays too large to stage) 11.83 ms, 5.9e-13 s; mvb_herk in fp16x3 took
#: 6.51 ms for 21 tiles of 128 x 128, i.e. 1.03e-10 s per (tile x split product
#: x column), with TF32 operands at half that rate.  Break-even at F = 2, 21
#: tiles: ~5,750 pairs (staged).
VECDOT_STAGED_S_PER_PAIR_COL = 2.8e-13
VECDOT_S_PER_PAIR_COL = 5.9e-13
HERK_S_PER_TILE_PRODUCT_COL = 1.03e-10


def pair_product(nant: int, nfeed: int, npairs: int, gemm_mode="fp16x3") -> str:
    """Which kernel computes an explicit pair list fastest on the device.

    Returns ``"herk"`` when the tensor-core Hermitian product over all pairs
    followed by a gather of the listed pairs (mvb_herk + mvb_herk_reduce with a
    pair list) is predicted faster than per-pair sums (mvb_vecdot_staged, or
    mvb_vecdot where the array's rows do not fit its shared-memory stages),
    else ``"vecdot"``.  Both give the reference's VectorDot output
    out[i, p, q] = sum_k Z[aj F + p, k] conj(Z[ai F + q, k]) (cpu/matprod.py:48-51);
    the per-column cost of each kernel is the measured one above, so the choice
    does not depend on the source count.  Lists above ~5,750 pairs of a
    350-antenna two-feed array go to the Hermitian product; shorter ones
    (redundant-baseline sets of compact arrays, sparse pair selections) stay on
    per-pair sums.
    """
    T = -(-int(nant) * int(nfeed) // _lib.TILE)
    mode = _lib.GEMM_MODES[gemm_mode] if isinstance(gemm_mode, str) else int(gemm_mode)
    rate = 2.0 if mode == _lib.GEMM_TF32_3 else 1.0
    herk = T * (T + 1) // 2 * _lib.GEMM_PRODUCTS[mode] * rate * HERK_S_PER_TILE_PRODUCT_COL
    per = VECDOT_STAGED_S_PER_PAIR_COL if _lib.lib.mvb_vecdot_stage_columns(int(nant), int(nfeed)) > 0 \
        else VECDOT_S_PER_PAIR_COL
    vecdot = int(npairs) * int(nfeed) ** 2 * per
    return "herk" if herk < vecdot else "vecdot"


class AntpairsOutOfRange(IndexError, ValueError):
    """A pair list names an antenna outside [0, nant).  An IndexError, as the
    reference's gather ``vis[ant1_idx, ant2_idx]`` raises (cpu/matprod.py:29-30),
    and a ValueError, as for the other argument checks."""


def _pairs_tensor(antpairs, device):
    if antpairs is None:
        return None
    a = np.ascontiguousarray(np.asarray(antpairs, dtype=np.int32).reshape(-1, 2))
    return torch.as_tensor(a, device=device)


class MatProd(ABC):
    """Abstract source-summing operation; core/matprod.py:11-115."""

    def __init__(self, nchunks: int, nfeed: int, nant: int, antpairs, precision=1, device=None):
        if antpairs is None:
            self.all_pairs = True
            idx = np.arange(nant)
            self.antpairs = np.stack(np.meshgrid(idx, idx, indexing="ij"), axis=-1).reshape(-1, 2)  # i slow
        else:
            self.all_pairs = False
            self.antpairs = np.asarray(antpairs)
            if self.antpairs.size and (self.antpairs.ndim != 2 or self.antpairs.shape[1] != 2):
                raise ValueError("antpairs must have shape (npairs, 2)")
            self.antpairs = self.antpairs.reshape(-1, 2)
            if self.antpairs.size and (self.antpairs.min() < 0 or self.antpairs.max() >= nant):
                raise AntpairsOutOfRange(f"antpairs name antennas outside [0, {nant})")
        self.device = _lib.require_cuda(device)
        self.nchunks = nchunks
        self.nfeed = nfeed
        self.nant = nant
        self.npairs = len(self.antpairs)
        self.precision = precision
        self.ctype = torch.complex64 if precision == 1 else torch.complex128
        self.ant1_idx = self.antpairs[:, 0] if self.npairs else np.zeros(0, int)
        self.ant2_idx = self.antpairs[:, 1] if self.npairs else np.zeros(0, int)
        self.status = None

    def allocate_vis(self):
        self.vis = torch.zeros((self.nchunks, self.npairs, self.nfeed, self.nfeed), dtype=self.ctype, device=self.device)

    def setup(self):
        self.allocate_vis()
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._pairs_dev = torch.as_tensor(
            np.ascontiguousarray(self.antpairs.astype(np.int32).reshape(-1, 2)), device=self.device
        )

    @abstractmethod
    def compute(self, z, out):
        """Sum over sources of one (time, chunk) into ``out`` (npairs, nfeed, nfeed)."""

    def __call__(self, z, chunk: int):
        self.compute(z, out=self.vis[chunk])
        return self.vis[chunk]

    def sum_chunks(self, out):
        """Sum the chunks into ``out`` (host array or device tensor), in chunk
        order with FP64 accumulation (``mvb_chunk_sum``)."""
        tot = self.vis[0]
        if self.nchunks > 1:
            tot = torch.empty_like(self.vis[0])
            check(_lib.lib.mvb_chunk_sum(ptr(self.vis), self.nchunks, tot.numel(),
                                         1 if tot.dtype == torch.complex128 else 0, ptr(tot), stream_handle()))
        if self.status is not None:
            _lib.check_status_word(self.status, type(self).__name__)
        if isinstance(out, torch.Tensor):
            out.copy_(tot)
        else:
            out[:] = tot.cpu().numpy()

    # -- helpers -------------------------------------------------------------
    def _as_panel(self, z, mode: int) -> ZPanel:
        if isinstance(z, ZPanel):
            if z.mode != mode:
                raise ValueError(f"Z panel mode {z.mode} does not match this product's mode {mode}")
            return z
        zt = torch.as_tensor(z, device=self.device)
        if not torch.is_complex(zt) or zt.ndim != 2:
            raise TypeError(f"invalid Z: expected a complex (nant*nfeed, K) matrix, got {zt.dtype} {tuple(zt.shape)}")
        if zt.shape[0] != self.nant * self.nfeed:
            raise ValueError("Z must have nant * nfeed rows")
        if zt.dtype not in (torch.complex64, torch.complex128):
            zt = zt.to(torch.complex128)
        zt = zt.contiguous()
        M, K = zt.shape
        key = (mode, K)
        panel = getattr(self, "_packed", {}).get(key)
        if panel is None:
            panel = ZPanel(mode, self.nant, self.nfeed, 1, K, self.device)
            self._packed = {key: panel}
        c128 = 1 if zt.dtype == torch.complex128 else 0
        scale = 1.0
        if mode == _lib.GEMM_F16_3:
            mx = torch.zeros(1, dtype=torch.float32, device=self.device)
            check(_lib.lib.mvb_absmax(ptr(zt), c128, M * K, ptr(mx), stream_handle()))
            scale = _lib.f16_scale(float(mx.item()) * (1 + 2**-10))
        panel.scale = scale
        check(
            _lib.lib.mvb_z_pack(
                ptr(zt), c128, M, K, K, mode, scale, ptr(panel.data), panel.Mpad, panel.Kcap, stream_handle(),
            )
        )
        panel.n_dev = None
        panel.n_host = K
        return panel


class B200MatMul(MatProd):
    """Hermitian product V = conj(Z) Z^T, upper-triangle tiles on the tensor cores."""

    def __init__(self, nchunks, nfeed, nant, antpairs, precision=1, gemm_mode: str | int = "fp16x3",
                 k_chunk: int | None = None, device=None, drain_ksteps: int = 0):
        super().__init__(nchunks, nfeed, nant, antpairs, precision=precision, device=device)
        #: k-steps per TMEM block before the drain to FP32 registers (0: the mode's default)
        self.drain_ksteps = int(drain_ksteps)
        self.mode = _lib.GEMM_MODES[gemm_mode] if isinstance(gemm_mode, str) else int(gemm_mode)
        if self.mode not in (_lib.GEMM_BF16_3, _lib.GEMM_BF16_6, _lib.GEMM_TF32_3, _lib.GEMM_F16_3):
            raise ValueError(f"unknown gemm_mode {gemm_mode!r}")
        self.k_chunk = k_chunk
        self._ws = None

    def workspace(self, panel: ZPanel, k_chunk: int, ngroup: int = 1) -> torch.Tensor:
        """Partial-tile workspace for ``ngroup`` panels of ``panel``'s shape (kept
        and grown as needed)."""
        nbytes = ngroup * _lib.lib.mvb_herk_ws_bytes(panel.Mpad, panel.Kcap, k_chunk)
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = None
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self._ws

    def enqueue_grouped(self, panels: list[ZPanel], out: torch.Tensor, accumulate: bool = False, stream=None,
                        k_chunk=None):
        """Products of consecutive panels of one allocation (``ZPanel.group``) in
        one launch, all with panels[0]'s column count; panel g's visibilities go
        to ``out[g]`` (``out`` indexed along its first dimension, any stride)."""
        ng = len(panels)
        p0 = panels[0]
        if ng == 1:
            return self.enqueue(p0, out[0], accumulate=accumulate, stream=stream, k_chunk=k_chunk)
        stride = panels[1].data.data_ptr() - p0.data.data_ptr()
        if any(p.data.data_ptr() - p0.data.data_ptr() != g * stride for g, p in enumerate(panels)):
            raise ValueError("grouped panels must be equally spaced in one allocation")
        kc = k_chunk or self.resolve_k_chunk(p0)
        ws = self.workspace(p0, kc, ng)
        sh = stream_handle(stream)
        check(
            _lib.lib.mvb_herk_grouped(
                ptr(p0.data), stride, ng, self.mode, p0.Mpad, p0.Kcap, ptr(p0.n_dev), p0.n_host, p0.nax, kc,
                self.drain_ksteps, ptr(ws), ws.numel(), ptr(self.status), sh,
            )
        )
        self.reduce_grouped(panels, out, accumulate=accumulate, stream=stream, k_chunk=kc)

    def batch_group(self, panels: list[ZPanel], k_chunk: int) -> _lib.HerkGroup:
        """The ``mvb_herk_batch`` entry for the products of ``panels`` (consecutive
        panels of one allocation, all with panels[0]'s column count): run in a
        batch with other jobs' groups, its partial tiles equal those of
        enqueue_grouped's product, and ``reduce_grouped`` then writes the same
        visibilities."""
        p0 = panels[0]
        ng = len(panels)
        stride = panels[1].data.data_ptr() - p0.data.data_ptr() if ng > 1 else 0
        ws = self.workspace(p0, k_chunk, ng)
        return _lib.HerkGroup(z=p0.data.data_ptr(), z_stride=stride, ngroup=ng, Mpad=p0.Mpad, Kcap=p0.Kcap,
                              n_dev=None if p0.n_dev is None else p0.n_dev.data_ptr(), n_host=p0.n_host,
                              kmul=p0.nax, k_chunk=k_chunk, ws=ws.data_ptr(), ws_bytes=ws.numel(),
                              status=self.status.data_ptr())

    def reduce_grouped(self, panels: list[ZPanel], out: torch.Tensor, accumulate: bool = False, stream=None,
                       k_chunk=None):
        """The reduction of the grouped product of ``panels`` (after mvb_herk_grouped
        or a batch holding their group): panel g's visibilities to ``out[g]``."""
        p0 = panels[0]
        kc = k_chunk or self.resolve_k_chunk(p0)
        ws = self.workspace(p0, kc, len(panels))
        pairs = None if self.all_pairs else self._pairs_dev
        check(
            _lib.lib.mvb_herk_reduce_grouped(
                ptr(ws), ws.numel(), len(panels), p0.Mpad, p0.Kcap, ptr(p0.n_dev), p0.n_host, p0.nax, kc, self.nant,
                self.nfeed, ptr(pairs), self.npairs, ptr(out), out.stride(0) * out.element_size(),
                1 if out.dtype == torch.complex128 else 0, 1.0 / p0.scale**2, int(accumulate), stream_handle(stream),
            )
        )

    def resolve_k_chunk(self, panel: ZPanel) -> int:
        if self.k_chunk is not None:
            return int(self.k_chunk)
        T = panel.Mpad // _lib.TILE
        sm = torch.cuda.get_device_properties(self.device).multi_processor_count
        kvalid = panel.n_host * panel.nax if panel.n_dev is None else panel.Kcap
        return choose_k_chunk(T * (T + 1) // 2, kvalid, sm, hi=4096)

    def enqueue(self, panel: ZPanel, out: torch.Tensor, accumulate: bool = False, stream=None, k_chunk=None):
        kc = k_chunk or self.resolve_k_chunk(panel)
        ws = self.workspace(panel, kc)
        sh = stream_handle(stream)
        kmul = panel.nax
        check(
            _lib.lib.mvb_herk(
                ptr(panel.data), self.mode, panel.Mpad, panel.Kcap, ptr(panel.n_dev), panel.n_host, kmul, kc,
                self.drain_ksteps, ptr(ws), ws.numel(), ptr(self.status), sh,
            )
        )
        pairs = None if self.all_pairs else self._pairs_dev
        check(
            _lib.lib.mvb_herk_reduce(
                ptr(ws), ws.numel(), panel.Mpad, panel.Kcap, ptr(panel.n_dev), panel.n_host, kmul, kc, self.nant,
                self.nfeed,
                ptr(pairs), self.npairs, ptr(out), 1 if out.dtype == torch.complex128 else 0, 1.0 / panel.scale**2,
                int(accumulate), sh,
            )
        )

    def compute(self, z, out):
        panel = self._as_panel(z, self.mode)
        self.enqueue(panel, out)
        return out


def vecdot_plan(antpairs, nant: int, nfeed: int) -> np.ndarray:
    """Bundles of the staged pair kernel for a host pair list (``mvb_vecdot_plan``):
    int32 (nbundles, 8) rows {i, j0, j1, j2, pair0, pair1, pair2, flip bits},
    nbundles a multiple of 32; pair -1 marks a filler step."""
    pairs = np.ascontiguousarray(np.asarray(antpairs, dtype=np.int32).reshape(-1, 2))
    npairs = len(pairs)
    buf = np.zeros(max(int(_lib.lib.mvb_vecdot_plan_bytes(npairs, nfeed)), 32) // 4, dtype=np.int32)
    nb = ctypes.c_int64(0)
    check(_lib.lib.mvb_vecdot_plan(pairs.ctypes.data if npairs else None, npairs, int(nant), int(nfeed),
                                   buf.ctypes.data, buf.nbytes, ctypes.byref(nb)))
    return buf[: 8 * nb.value].reshape(-1, 8).copy()


class B200VectorDot(MatProd):
    """Per-pair source sums for explicit pair lists.

    ``kernel="staged"`` (the default wherever the array's rows fit the
    shared-memory stages, ``mvb_vecdot_stage_columns``): the panel is read from
    HBM once and every pair runs from shared memory (``mvb_vecdot_staged``, pair
    bundles planned once at :meth:`setup`); ``kernel="warp"``: one warp per (k-slice,
    pair) reading both rows through L2 (``mvb_vecdot``)."""

    def __init__(self, nchunks, nfeed, nant, antpairs, precision=1, k_chunk: int = 4096, device=None,
                 kernel: str = "auto"):
        super().__init__(nchunks, nfeed, nant, antpairs, precision=precision, device=device)
        if kernel not in ("auto", "staged", "warp"):
            raise ValueError(f"kernel must be 'auto', 'staged' or 'warp', not {kernel!r}")
        staged_ok = _lib.lib.mvb_vecdot_stage_columns(nant, nfeed) > 0
        if kernel == "staged" and not staged_ok:
            raise ValueError(f"{nant} x {nfeed} rows do not fit the staged kernel's shared memory")
        self.kernel = "staged" if kernel in ("auto", "staged") and staged_ok else "warp"
        self.mode = _lib.Z_C64
        self.k_chunk = int(k_chunk)
        if self.k_chunk % 16:
            raise ValueError("k_chunk must be a multiple of 16")
        self._ws = None
        self._plan_dev = None
        self.nbundles = 0

    def setup(self):
        super().setup()
        if self.kernel == "staged":
            plan = vecdot_plan(self.antpairs, self.nant, self.nfeed)
            self.nbundles = len(plan)
            self._plan_dev = torch.as_tensor(plan, device=self.device)

    def enqueue(self, panel: ZPanel, out: torch.Tensor, accumulate: bool = False, stream=None):
        c128 = 1 if out.dtype == torch.complex128 else 0
        if self.kernel == "staged":
            if self._plan_dev is None:
                self.setup()
            nbytes = _lib.lib.mvb_vecdot_staged_ws_bytes(self.nbundles, self.nfeed, panel.Kcap, self.k_chunk)
        else:
            nbytes = _lib.lib.mvb_vecdot_ws_bytes(self.npairs, self.nfeed, panel.Kcap, self.k_chunk)
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = None
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        if self.kernel == "staged":
            check(
                _lib.lib.mvb_vecdot_staged(
                    ptr(panel.data), panel.Kcap, ptr(panel.n_dev), panel.n_host, panel.nax, self.nfeed, self.nant,
                    ptr(self._plan_dev), self.nbundles, self.npairs, self.k_chunk, ptr(self._ws), self._ws.numel(),
                    ptr(out), c128, int(accumulate), ptr(self.status), stream_handle(stream),
                )
            )
            return
        check(
            _lib.lib.mvb_vecdot(
                ptr(panel.data), panel.Kcap, ptr(panel.n_dev), panel.n_host, panel.nax, self.nfeed,
                ptr(self._pairs_dev), self.npairs, self.k_chunk, ptr(self._ws), self._ws.numel(), ptr(out),
                c128, int(accumulate), stream_handle(stream),
            )
        )

    def compute(self, z, out):
        panel = self._as_panel(z, self.mode)
        self.enqueue(panel, out)
        return out
