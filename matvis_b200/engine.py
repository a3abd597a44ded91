"""Batched visibility engine: every (frequency, time) slice of a job on one GPU.

The reference runs ``simulate`` once per frequency (wrapper.py:180-199) and,
inside it, rotation -> horizon selection -> beam -> tau -> Z -> product per time
and chunk with a device synchronisation after each stage (cpu/cpu.py:247-272,
gpu/gpu.py:197-254).  Here one job is one stream of launches:

    for t:      mvb_rotate -> (per chunk) mvb_horizon_compact -> mvb_beam_*
      for each group of G frequencies:
                mvb_tau_z_grouped -> mvb_herk_grouped -> mvb_herk_reduce_grouped
                (G panels, one launch each; a beamfits beam, which changes with
                frequency, or a pair list on mvb_vecdot goes one frequency at a time:
                [mvb_beam_*] -> mvb_tau_z -> mvb_herk + mvb_herk_reduce or mvb_vecdot)

Rotation, selection and (for an achromatic beam) beam interpolation depend on
time only and are done once per time for all frequencies.  The above-horizon count never leaves the device:
every later kernel reads it from ``n_above`` and sizes its work from it, so the
whole job can be captured once as a CUDA graph and replayed.
"""

from __future__ import annotations

import os
import queue
import threading
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, replace

import numpy as np
import torch

from . import _lib, devcache
from .beams import B200BeamInterpolator, GridBeam, beams_at_frequency, is_chromatic
from .coordinates import (
    ENU_TO_ALTAZ,
    atioq_matrix,
    bcrs_refresh_plan,
    eci_to_enu_matrix,
    pack_astrom,
    point_source_crd_eq,
)
from .getz import ZMatrixCalc, ZPanel
from . import autotune
from .autotune import KD_CANDIDATES, tune_product
from .matprod import B200MatMul, B200VectorDot, choose_k_chunk, pair_product

#: k-slice of the Hermitian product without autotuning: the tuner's choice for
#: the HERA-350-like slice in fp16x3 (product + reduction 1.36 ms at 4096
#: columns; shorter slices mean more partial tiles to reduce).  The number of
#: slices is still fitted to whole waves of SMs on the device.
DEFAULT_K_CHUNK = 4096

#: Frequencies per grouped launch (tau/Z, product and reduction of that many
#: frequencies of a time step in one launch each, on as many Z panels) unless
#: the job sets ``freq_group``; fewer when the job has fewer frequencies or the
#: device memory (``fit_freq_group``) allows fewer.
DEFAULT_FREQ_GROUP = 8


@dataclass
class JobSpec:
    antpos: np.ndarray  # (A, 3) metres
    eci: np.ndarray  # (3, N) unit vectors
    fluxes: np.ndarray  # (N, Nf) Stokes I, or (N, Nf, 2, 2) coherency (polarised sky)
    freqs: np.ndarray  # (Nf,) Hz
    lsts: np.ndarray  # (Nt,) radians
    latitude: float  # radians
    beams: list
    beam_idx: np.ndarray | None = None
    polarized: bool = False
    antpairs: np.ndarray | None = None
    precision: int = 1
    gemm_mode: str = "fp16x3"
    matprod: str = "MatMul"  # or "VectorDot"
    #: kernel for a VectorDot pair list: "auto" (measured cost model), "vecdot" or "herk"
    pair_product: str = "auto"
    k_chunk: int | None = None
    source_buffer: float = 1.0
    nchunks: int = 1
    #: ERFA-style apparent place: one astrom dict per time (else the LST rotation)
    astrom: list | None = None
    update_bcrs_every: float = 0.0
    time_s: np.ndarray | None = None
    #: (2, N) ra / dec in radians for the polarised sky's frame rotation (else from eci)
    radec: np.ndarray | None = None
    #: frequencies per grouped launch (None: DEFAULT_FREQ_GROUP; 1: one frequency per launch)
    freq_group: int | None = None
    #: name of a sky model shared by several jobs: jobs with the same key (and sky
    #: shape) share one device copy of the source directions and fluxes
    sky_key: str | None = None


def _norm_matprod(name: str) -> str:
    n = str(name)
    for p in ("B200", "GPU", "CPU"):
        if n.startswith(p):
            n = n[len(p):]
    if n in ("MatMul",):
        return "MatMul"
    if n in ("VectorDot", "VectorLoop"):
        return "VectorDot"
    raise ValueError(f"unknown matprod_method {name!r}")


def _pinned(src: np.ndarray) -> torch.Tensor:
    """A page-locked host copy of ``src`` for an asynchronous upload (filled by
    host threads when large; torch's pinned-block cache keeps the block until the
    copy that reads it has run).  Pageable when the host refuses to pin."""
    src = np.ascontiguousarray(src)
    try:
        t = torch.empty(src.shape, dtype=torch.from_numpy(src[:0]).dtype, pin_memory=True)
    except RuntimeError:
        return torch.from_numpy(src)
    d, s_ = t.numpy().reshape(-1), src.reshape(-1)
    nthreads = min(os.cpu_count() or 1, 8)
    if src.nbytes < (8 << 20) or nthreads < 2:
        np.copyto(d, s_)
        return t
    step = -(-s_.size // nthreads)
    with ThreadPoolExecutor(nthreads) as ex:
        list(ex.map(lambda lo: np.copyto(d[lo:lo + step], s_[lo:lo + step]), range(0, s_.size, step)))
    return t


def _repack_coherency(c: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(N, Nf, 2, 2) complex coherency -> (Nf, N, 4) float32 [C00, C11, Re C01,
    Im C01] and the (N, Nf) float64 trace max(C00 + C11, 0); source chunks on
    host threads (plain copies and one addition: the values do not depend on
    the split)."""
    n, nf = c.shape[:2]
    coh = np.empty((nf, n, 4), dtype=np.float32)
    trace = np.empty((n, nf), dtype=np.float64)

    def work(lo):
        hi = min(lo + step, n)
        cb = c[lo:hi]
        coh[:, lo:hi, 0] = cb[..., 0, 0].real.T
        coh[:, lo:hi, 1] = cb[..., 1, 1].real.T
        coh[:, lo:hi, 2] = cb[..., 0, 1].real.T
        coh[:, lo:hi, 3] = cb[..., 0, 1].imag.T
        np.maximum(cb[..., 0, 0].real + cb[..., 1, 1].real, 0.0, out=trace[lo:hi])

    nthreads = min(os.cpu_count() or 1, 16)
    step = max(-(-n // nthreads), 1)
    if n * nf < (1 << 16) or nthreads < 2:
        step = max(n, 1)
        work(0)
    else:
        with ThreadPoolExecutor(nthreads) as ex:
            list(ex.map(work, range(0, n, step)))
    return coh, trace


def _resolve_product(spec: JobSpec) -> tuple[str, str | None]:
    """(kernel family, pair kernel): a VectorDot request runs on the Hermitian
    product with a pair gather when ``pair_product`` says so (or, on "auto", when
    the measured cost model predicts it faster); the output is the same."""
    method = _norm_matprod(spec.matprod)
    if method != "VectorDot":
        return method, None
    choice = str(spec.pair_product)
    if choice not in ("auto", "vecdot", "herk"):
        raise ValueError(f"pair_product must be 'auto', 'vecdot' or 'herk', not {choice!r}")
    nant = len(spec.antpos)
    nfeed = 2 if spec.polarized else 1
    npairs = nant * nant if spec.antpairs is None else len(spec.antpairs)
    if choice == "auto":
        choice = pair_product(nant, nfeed, npairs, spec.gemm_mode)
    return ("MatMul" if choice == "herk" else "VectorDot"), choice


class VisEngine:
    """Device-resident state and launch sequence of one job."""

    def __init__(self, spec: JobSpec, device=None):
        self.spec = spec
        self.device = _lib.require_cuda(device)
        s = spec
        self.antpos_host = np.ascontiguousarray(np.asarray(s.antpos, dtype=np.float64))
        self.nant = self.antpos_host.shape[0]
        self.nfeed = self.nax = 2 if s.polarized else 1
        self.eci_host = np.ascontiguousarray(np.asarray(s.eci, dtype=np.float64))
        self.nsrc = self.eci_host.shape[1]
        self.freqs = np.asarray(s.freqs, dtype=np.float64)
        self.lsts = np.asarray(s.lsts, dtype=np.float64)
        fl = np.asarray(s.fluxes)
        self.pol_sky = fl.ndim == 4
        if fl.shape[:2] != (self.nsrc, len(self.freqs)) or (self.pol_sky and fl.shape[2:] != (2, 2)) or \
                fl.ndim not in (2, 4):
            raise ValueError("The `fluxes` array must have shape (NSRCS, NFREQS) or (NSRCS, NFREQS, 2, 2).")
        if self.pol_sky:
            if not s.polarized:
                raise ValueError("a polarised sky (coherency fluxes) needs polarized=True")
            # per frequency and source: C00, C11, Re C01, Im C01 (float32, 16 bytes);
            # Stokes I = trace C for the Z scale bound
            self.coh_host, self.flux_host = _repack_coherency(np.asarray(fl, dtype=np.complex128))
            if s.radec is not None:
                self.radec_host = np.ascontiguousarray(np.asarray(s.radec, dtype=np.float64).reshape(2, self.nsrc))
            else:
                e = self.eci_host
                self.radec_host = np.ascontiguousarray(np.stack([np.arctan2(e[1], e[0]), np.arcsin(np.clip(e[2], -1, 1))]))
        else:
            # Stokes I (N, Nf); sqrt(0.5 I) (cpu/cpu.py:188) is formed on the device,
            # frequency-major float32, by mvb_flux_sqrt_half at upload
            self.flux_host = np.ascontiguousarray(fl, dtype=np.float64)
        self.method, self.pair_kernel = _resolve_product(s)
        self.nchunks = max(1, int(s.nchunks))
        self.chunk_size = int(np.ceil(self.nsrc / self.nchunks)) if self.nsrc else 1
        if not 0 < s.source_buffer <= 1:
            raise ValueError("source_buffer must satisfy 0 < source_buffer <= 1")
        self.cap = int(self.chunk_size * s.source_buffer) if self.chunk_size > 1000 else self.chunk_size
        self.cap = max(self.cap, 1)
        self.ctype = torch.complex64 if s.precision == 1 else torch.complex128
        if s.astrom is not None:
            if len(s.astrom) != len(self.lsts):
                raise ValueError("astrom must hold one parameter dict per time")
            self.rot = np.stack([atioq_matrix(a) for a in s.astrom])
            if s.time_s is None and s.update_bcrs_every > 0:
                raise ValueError("update_bcrs_every needs time_s (the times in seconds)")
            # without time_s every time step refreshes the apparent-place directions
            self.bcrs_plan = ([True] * len(self.lsts) if s.time_s is None
                              else bcrs_refresh_plan(s.time_s, s.update_bcrs_every))
            self.astrom_packed = [pack_astrom(a) for a in s.astrom]
        else:
            self.rot = (np.stack([eci_to_enu_matrix(l, s.latitude) for l in self.lsts]) if len(self.lsts)
                        else np.zeros((0, 3, 3)))
            self.bcrs_plan = None
        if self.pol_sky:
            # rigid ICRS -> alt/az-cartesian rotation per time for the coherency frame
            if s.astrom is not None:
                rigid = [atioq_matrix(a) @ np.asarray(a["bpn"], dtype=np.float64).reshape(3, 3) for a in s.astrom]
            else:
                rigid = list(self.rot)
            self.ravg = [np.ascontiguousarray(ENU_TO_ALTAZ @ r) for r in rigid]
        # a beamfits beam is interpolated to every frequency of the job on the host
        # (re-gridded per frequency, core/beams.py:82-93) and on the device per slice
        self.chromatic = is_chromatic(s.beams)
        self.beams_per_freq = ([beams_at_frequency(s.beams, f) for f in self.freqs] if self.chromatic
                               else [list(s.beams)])
        self.fgroup = freq_group_of(s, self.method, self.chromatic)
        self.zscale = 1.0
        if self.method == "MatMul" and _lib.GEMM_MODES.get(s.gemm_mode, s.gemm_mode) == _lib.GEMM_F16_3:
            # |Z| <= max sqrt(0.5 I) * max |beam| (bilinear weights are convex, |exptau| = 1); for a
            # polarised sky |sum_x beam_x L_xy| <= sqrt(2) max|beam| sqrt(trace C) = 2 max|beam| sqrt(I / 2)
            smax = float(np.sqrt(0.5 * max(float(self.flux_host.max(initial=0.0)), 0.0)))
            bmax = max((beam_bound(b) for b in self.beams_per_freq), default=1.0)
            zmax = smax * bmax * (2.0 if self.pol_sky else 1.0)
            self.zscale = _lib.f16_scale(zmax * (1 + 2**-10))
        self._graph = None
        self._allocated = False
        self._uploaded = False
        #: the autotuner's decision for this job (set by capture())
        self.tuned: dict | None = None

    # ------------------------------------------------------------------ setup
    def allocate(self):
        dev = self.device
        s = self.spec
        A, N = self.nant, self.nsrc
        # at least one source slot, so that an empty sky still hands the kernels
        # valid pointers (they read nothing when the source count is 0)
        Na = max(N, 1)
        self.eci = torch.zeros((3, Na), dtype=torch.float64, device=dev)
        self.antpos = torch.empty((A, 3), dtype=torch.float64, device=dev)
        self.sflux = torch.zeros((len(self.freqs), Na), dtype=torch.float32, device=dev)
        self.topo = torch.zeros((3, Na), dtype=torch.float64, device=dev)
        self.bcrs = torch.zeros((3, Na), dtype=torch.float64, device=dev) if self.bcrs_plan is not None else None
        if self.pol_sky:
            self.coh = torch.zeros((len(self.freqs), Na, 4), dtype=torch.float32, device=dev)
            self.radec = torch.zeros((2, Na), dtype=torch.float64, device=dev)
            self.rot2 = torch.zeros((self.cap, 2), dtype=torch.float64, device=dev)
        self.crd = torch.zeros((3, self.cap), dtype=torch.float64, device=dev)
        self.kept = torch.zeros((self.cap,), dtype=torch.int32, device=dev)
        self.n_above = torch.zeros(1, dtype=torch.int32, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ws_compact = torch.empty(_lib.lib.mvb_horizon_ws_bytes(self.chunk_size), dtype=torch.uint8, device=dev)
        # one interpolator per frequency for a beamfits beam, all writing one beam buffer
        self.bmfuncs = []
        for i, bl in enumerate(self.beams_per_freq):
            bf = B200BeamInterpolator(beam_list=bl, beam_idx=s.beam_idx, polarized=s.polarized, nant=A,
                                      freq=float(self.freqs[i]) if len(self.freqs) else 0.0, nsrc=self.cap,
                                      precision=1, device=dev)
            bf.setup()
            if self.bmfuncs:
                # the per-frequency interpolators run in turn on one stream: one
                # output and one coordinate workspace serve them all
                bf.interpolated_beam = self.bmfuncs[0].interpolated_beam
            self.bmfuncs.append(bf)
        if self.bmfuncs[0].use_interp:
            ws = torch.empty(2 * self.bmfuncs[0].nbeam * max(self.cap, 1), dtype=torch.float64, device=dev)
            for bf in self.bmfuncs:
                bf._coord_ws = ws
        self.bmfunc = self.bmfuncs[0]
        if self.method == "MatMul":
            self.matprod = B200MatMul(1, self.nfeed, A, s.antpairs, precision=s.precision, gemm_mode=s.gemm_mode,
                                      k_chunk=s.k_chunk, device=dev)
            zmode = self.matprod.mode
        else:
            pairs = s.antpairs if s.antpairs is not None else np.array([(i, j) for i in range(A) for j in range(A)])
            self.matprod = B200VectorDot(1, self.nfeed, A, pairs, precision=s.precision,
                                         k_chunk=s.k_chunk or 4096, device=dev)
            zmode = _lib.Z_C64
        self.matprod.setup()
        self.matprod.status = self.status
        self.zcalc = ZMatrixCalc(A, self.nfeed, self.nax, self.cap, mode=zmode, device=dev)
        if self.fgroup > 1:
            # G panels of one allocation: the operands of one grouped launch
            self.panels = ZPanel.group(self.fgroup, zmode, A, self.nfeed, self.nax, self.cap, dev)
            self.zcalc.z = self.panels[0]
        else:
            self.zcalc.setup()
            self.panels = [self.zcalc.z]
        self.freqs_dev = torch.as_tensor(self.freqs, dtype=torch.float64, device=dev)
        self.npairs = self.matprod.npairs
        self.vis = torch.zeros((len(self.freqs), len(self.lsts), self.npairs, self.nfeed, self.nfeed), dtype=self.ctype,
                               device=dev)
        if self.method == "MatMul":
            panel = self.zcalc.z
            self.k_chunk = int(s.k_chunk) if s.k_chunk else DEFAULT_K_CHUNK
            if not s.k_chunk and not self.matprod.drain_ksteps:
                # a choice the autotuner made earlier in this process for this shape
                # (about half the sky above the horizon)
                hit = autotune.cached_choice(self.matprod.mode, panel.Mpad, self.nsrc // 2 * self.nax,
                                             torch.device(dev).index or 0)
                if hit is not None:
                    self.k_chunk, self.matprod.drain_ksteps = hit
                    self.tuned = {"k_chunk": hit[0], "drain_ksteps": hit[1], "cached": True}
            self.matprod.workspace(panel, self.k_chunk, self.fgroup)
        self._allocated = True

    def upload(self, stream=None):
        """Host -> device copies of the job inputs (pinned staging when possible)."""
        if not self._allocated:
            self.allocate()
        N = self.nsrc
        self.antpos.copy_(_pinned(self.antpos_host), non_blocking=True)
        key = self.spec.sky_key
        if key is not None and not self.pol_sky and N:
            # a named sky shared with other jobs: one device copy (read-only here)
            ck = ("sky", devcache.device_key(self.eci.device), str(key), tuple(self.eci.shape),
                  tuple(self.freqs.tolist()))
            self.eci, self.sflux = devcache.CACHE.get(ck, self._upload_sky)
            self._uploaded = True
            return
        # every copy is asynchronous on the current stream, from page-locked staging
        if N:
            self.eci[:, :N].copy_(_pinned(self.eci_host), non_blocking=True)
        if self.pol_sky:
            self.sflux.zero_()  # not read: the polarised writer takes the coherency
        elif N:
            self._fill_sflux(self.sflux)
        if self.pol_sky and N:
            self.coh[:, :N].copy_(_pinned(self.coh_host), non_blocking=True)
            self.radec[:, :N].copy_(_pinned(self.radec_host), non_blocking=True)
        self._uploaded = True

    def _fill_sflux(self, sflux: torch.Tensor):
        """sqrt(0.5 I) per frequency and source from the host Stokes I (on the device)."""
        fl = torch.empty(self.flux_host.shape, dtype=torch.float64, device=sflux.device)
        fl.copy_(_pinned(self.flux_host), non_blocking=True)
        _lib.check(_lib.lib.mvb_flux_sqrt_half(_lib.ptr(fl), self.nsrc, len(self.freqs), _lib.ptr(sflux),
                                               _lib.stream_handle()))

    def _upload_sky(self) -> tuple[torch.Tensor, torch.Tensor]:
        eci = torch.zeros_like(self.eci)
        eci[:, :self.nsrc].copy_(_pinned(self.eci_host), non_blocking=True)
        sflux = torch.zeros_like(self.sflux)
        self._fill_sflux(sflux)
        return eci, sflux

    def h2d_bytes(self) -> int:
        n = self.eci_host.nbytes + self.antpos_host.nbytes + (0 if self.pol_sky else self.flux_host.nbytes)
        if self.pol_sky:
            n += self.coh_host.nbytes + self.radec_host.nbytes
        return n

    # ----------------------------------------------------------------- launch
    def enqueue(self, stream=None):
        """Enqueue every kernel of the job on ``stream`` (no host synchronisation)."""
        for t in range(len(self.lsts)):
            self.enqueue_time(t, stream)

    def enqueue_time(self, t: int, stream=None, after=None):
        """Enqueue the kernels of time index t (all chunks and frequencies).

        ``after(f0, g)``, if given, is called once the launches that complete
        frequencies f0 .. f0 + g - 1 of this time are enqueued (for a results
        copy that can start as soon as they have run)."""
        L = _lib.lib
        sh = _lib.stream_handle(stream)
        chk = _lib.check
        A = self.nant
        F, X = self.nfeed, self.nax
        panel = self.zcalc.z
        for c in range(self.nchunks):
            beam = self.chunk_prologue(t, c, stream)
            last = c == self.nchunks - 1
            if self.fgroup > 1:
                for f0 in range(0, len(self.freqs), self.fgroup):
                    g = self.tau_z_group(t, f0, beam, stream)
                    self.matprod.enqueue_grouped(self.panels[:g], self.vis[f0:f0 + g, t], accumulate=c > 0,
                                                 stream=stream, k_chunk=self.k_chunk)
                    if last and after is not None:
                        after(f0, g)
                continue
            for f in range(len(self.freqs)):
                if self.chromatic:
                    self.bmfuncs[f].launch(self.crd, self.cap, self.n_above, self.cap, beam, stream=stream,
                                           status=self.status)
                if self.pol_sky:
                    chk(L.mvb_tau_z_pol(
                        _lib.ptr(self.antpos), A, float(self.freqs[f]), _lib.ptr(self.crd), self.cap,
                        _lib.ptr(self.n_above), self.cap, _lib.ptr(self.coh[f]), _lib.ptr(self.kept),
                        _lib.ptr(self.rot2), _lib.ptr(beam), beam.shape[-1], beam.shape[0],
                        _lib.ptr(self.bmfunc.beam_index_dev), self.zcalc.mode, self.zscale, _lib.ptr(panel.data),
                        panel.Mpad, panel.Kcap, sh))
                else:
                    chk(L.mvb_tau_z(
                        _lib.ptr(self.antpos), A, float(self.freqs[f]), _lib.ptr(self.crd), self.cap,
                        _lib.ptr(self.n_above), self.cap, _lib.ptr(self.sflux[f]), _lib.ptr(self.kept),
                        _lib.ptr(beam), beam.shape[-1], beam.shape[0], _lib.ptr(self.bmfunc.beam_index_dev), F, X,
                        self.zcalc.mode, self.zscale, _lib.ptr(panel.data), panel.Mpad, panel.Kcap, sh))
                panel.n_dev = self.n_above
                panel.n_host = self.cap
                panel.scale = self.zscale
                out = self.vis[f, t]
                if self.method == "MatMul":
                    self.matprod.enqueue(panel, out, accumulate=c > 0, stream=stream, k_chunk=self.k_chunk)
                else:
                    self.matprod.enqueue(panel, out, accumulate=c > 0, stream=stream)
                if last and after is not None:
                    after(f, 1)

    def chunk_prologue(self, t: int, c: int, stream=None) -> torch.Tensor:
        """The kernels of time t and source chunk c that every frequency shares:
        for c = 0 the apparent-place refresh and the rotation; then the horizon
        selection of the chunk, the beam (an achromatic one: once for all
        frequencies) and the polarised sky's frame rotation.  Returns the beam
        buffer."""
        L = _lib.lib
        sh = _lib.stream_handle(stream)
        chk = _lib.check
        if c == 0:
            R = np.ascontiguousarray(self.rot[t])
            src = self.eci
            if self.bcrs_plan is not None:
                if self.bcrs_plan[t]:
                    a = self.astrom_packed[t]
                    chk(L.mvb_bcrs(_lib.ptr(self.eci), self.nsrc, a.ctypes.data_as(_lib.c_void_p),
                                   _lib.ptr(self.bcrs), sh))
                src = self.bcrs
            chk(L.mvb_rotate(_lib.ptr(src), self.nsrc, R.ctypes.data_as(_lib.c_void_p), _lib.ptr(self.topo), sh))
        c0 = min(c * self.chunk_size, self.nsrc)
        c1 = min((c + 1) * self.chunk_size, self.nsrc)
        chk(L.mvb_horizon_compact(
            _lib.ptr(self.topo), self.nsrc, c0, c1, None, _lib.ptr(self.crd), _lib.ptr(self.kept), None,
            _lib.ptr(self.n_above), self.cap, _lib.ptr(self.status), _lib.ptr(self.ws_compact),
            self.ws_compact.numel(), sh))
        beam = self.bmfunc.interpolated_beam
        if not self.chromatic:  # time-only: once for all frequencies
            self.bmfunc.launch(self.crd, self.cap, self.n_above, self.cap, beam, stream=stream, status=self.status)
        if self.pol_sky:
            chk(L.mvb_coherency_rotation(
                _lib.ptr(self.radec), self.nsrc, _lib.ptr(self.kept), _lib.ptr(self.crd), self.cap,
                _lib.ptr(self.n_above), self.cap, self.ravg[t].ctypes.data_as(_lib.c_void_p), _lib.ptr(self.rot2),
                sh))
        return beam

    def tau_z_group(self, t: int, f0: int, beam: torch.Tensor, stream=None) -> int:
        """One grouped tau/Z launch: frequencies f0 .. f0 + g - 1 (g = fgroup or
        what is left) of the current chunk into ``panels[:g]``.  Returns g."""
        L = _lib.lib
        sh = _lib.stream_handle(stream)
        A, F, X = self.nant, self.nfeed, self.nax
        g = min(self.fgroup, len(self.freqs) - f0)
        p0 = self.panels[0]
        zstride = p0.nbytes
        if self.pol_sky:
            _lib.check(L.mvb_tau_z_pol_grouped(
                _lib.ptr(self.antpos), A, _lib.ptr(self.freqs_dev[f0:]), g, _lib.ptr(self.crd), self.cap,
                _lib.ptr(self.n_above), self.cap, _lib.ptr(self.coh[f0]), self.coh.shape[1], _lib.ptr(self.kept),
                _lib.ptr(self.rot2), _lib.ptr(beam), beam.shape[-1], beam.shape[0],
                _lib.ptr(self.bmfunc.beam_index_dev), self.zcalc.mode, self.zscale, _lib.ptr(p0.data), zstride,
                p0.Mpad, p0.Kcap, sh))
        else:
            _lib.check(L.mvb_tau_z_grouped(
                _lib.ptr(self.antpos), A, _lib.ptr(self.freqs_dev[f0:]), g, _lib.ptr(self.crd), self.cap,
                _lib.ptr(self.n_above), self.cap, _lib.ptr(self.sflux[f0]), self.sflux.shape[1],
                _lib.ptr(self.kept), _lib.ptr(beam), beam.shape[-1], beam.shape[0],
                _lib.ptr(self.bmfunc.beam_index_dev), F, X, self.zcalc.mode, self.zscale, _lib.ptr(p0.data),
                zstride, p0.Mpad, p0.Kcap, sh))
        for p in self.panels[:g]:
            p.n_dev = self.n_above
            p.n_host = self.cap
            p.scale = self.zscale
        return g

    @property
    def batchable(self) -> bool:
        """Whether the job's products can share a launch with other jobs'
        (mvb_herk_batch): the Hermitian product with an achromatic beam."""
        return self.method == "MatMul" and not self.chromatic

    def device_bytes(self) -> int:
        """Device memory this job holds once allocated."""
        if not self._allocated:
            return estimate_device_bytes(self.spec)
        tensors = [self.eci, self.antpos, self.sflux, self.topo, self.crd, self.kept, self.ws_compact, self.vis,
                   self.zcalc.z.data, self.bmfunc.interpolated_beam]
        n = sum(t.numel() * t.element_size() for t in tensors) + (len(self.panels) - 1) * self.zcalc.z.nbytes
        ws = getattr(self.matprod, "_ws", None)
        return n + (ws.numel() if ws is not None else 0)

    def launches_per_run(self) -> int:
        # per frequency (or per group of fgroup frequencies): tau/Z, then the product
        # and its reduction (mvb_herk[_grouped] + reduce, or vecdot_kernel + its slice reduction)
        per_f = 3
        nlaunch = len(self.freqs) if self.fgroup <= 1 else -(-len(self.freqs) // self.fgroup)
        # a gridded beam is two launches (grid coordinates, then the planes), an analytic one one
        bl = 1 if all(hasattr(b, "sigma") for b in self.spec.beams) else 2
        # count + scatter + beam (+ frame), per frequency (+ its beam for a beamfits beam)
        per_chunk = 2 + bl * int(not self.chromatic) + (per_f + bl * int(self.chromatic)) * nlaunch + int(self.pol_sky)
        n = len(self.lsts) * (1 + self.nchunks * per_chunk)
        return n + (sum(self.bcrs_plan) if self.bcrs_plan is not None else 0)

    def run(self, check: bool = True) -> torch.Tensor:
        """Run the job on the current stream; returns the device visibilities."""
        if not self._uploaded:
            self.upload()
        self.status.zero_()
        if self._graph is not None:
            self._graph.replay()
        else:
            self.enqueue()
        if check:
            torch.cuda.current_stream().synchronize()
            _lib.check_status_word(self.status, "VisEngine")
        return self.vis

    def run_to_host(self, out: np.ndarray | None = None) -> np.ndarray:
        """Run the job and return the visibilities in host memory (``out`` if given).

        As soon as the kernels of a group of frequencies of a time step have
        run, a helper thread copies those visibilities into ``out`` on its own
        stream, so the device -> host copy, and the first touch of freshly
        allocated host pages (slower than the copy itself), overlap the compute
        that follows; only the last group's copy runs after the compute.
        """
        if not self._uploaded:
            self.upload()
        shape = tuple(self.vis.shape)
        dtype = np.complex64 if self.ctype == torch.complex64 else np.complex128
        if out is None:
            out = np.empty(shape, dtype=dtype)
        elif out.shape != shape or out.dtype != dtype or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous {dtype.__name__} array of shape {shape}")
        host = torch.from_numpy(out)
        nf, nt = shape[:2]
        dev = self.vis.device
        self.status.zero_()
        main = torch.cuda.current_stream(dev)
        side = torch.cuda.Stream(device=dev)
        steps: queue.Queue = queue.Queue()
        errors: list[BaseException] = []

        page = 4096 // out.itemsize

        def copier():
            try:
                torch.cuda.set_device(dev)
                with torch.cuda.stream(side):
                    while (item := steps.get()) is not None:
                        t, f0, g, done = item
                        # touch the destination pages while the group still computes, so
                        # that the copy after it is not held up by first-touch page faults
                        for f in range(f0, f0 + g):
                            out[f, t].reshape(-1)[::page] = 0
                        side.wait_event(done)
                        for f in range(f0, f0 + g):
                            host[f, t].copy_(self.vis[f, t])
            except BaseException as exc:  # re-raised on the calling thread
                errors.append(exc)
                while steps.get() is not None:
                    pass

        worker = threading.Thread(target=copier, name="mvb-d2h", daemon=True)
        worker.start()
        try:
            for t in range(nt):
                def after(f0, g, t=t):
                    done = torch.cuda.Event()
                    done.record(main)
                    steps.put((t, f0, g, done))

                self.enqueue_time(t, after=after)
        finally:
            steps.put(None)
            worker.join()
        main.synchronize()
        if errors:
            raise errors[0]
        _lib.check_status_word(self.status, "VisEngine")
        return out

    def capture(self):
        """Capture the launch sequence as one CUDA graph (run once uncaptured first)."""
        if not self._uploaded:
            self.upload()
        self.enqueue()  # warm-up: function attributes, lazy module loading
        torch.cuda.synchronize()
        if self.method == "MatMul" and not self.spec.k_chunk:
            # the panel holds the last slice: time the (k-slice, drain interval) candidates on it
            panel, scratch = self.zcalc.z, torch.empty_like(self.vis[0, 0])
            mp = self.matprod
            kd0 = mp.drain_ksteps

            def run(kc, kd, st):
                mp.drain_ksteps = kd
                mp.enqueue(panel, scratch, accumulate=False, stream=st, k_chunk=kc)

            try:
                self.k_chunk, kd = tune_product(panel, mp.mode, self.status, run=run,
                                                kd_candidates=(kd0,) if kd0 else KD_CANDIDATES)
            finally:
                mp.drain_ksteps = kd0
            mp.drain_ksteps = kd
            self.tuned = dict(autotune.last_choice) or {"k_chunk": self.k_chunk, "drain_ksteps": kd, "cached": True}
            mp.workspace(self.zcalc.z, self.k_chunk, self.fgroup)
            torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.enqueue(stream=s)
        torch.cuda.current_stream().wait_stream(s)
        self._graph = g
        return g

    def result(self, polarized: bool | None = None) -> torch.Tensor:
        pol = self.spec.polarized if polarized is None else polarized
        return self.vis if pol else self.vis[..., 0, 0]


def job_from_arrays(*, ants, fluxes, ra, dec, freqs, lsts, latitude, beams, **kw) -> JobSpec:
    """JobSpec from the simulate_vis-style inputs (ants dict, ra/dec in radians)."""
    if isinstance(ants, dict):
        antpos = np.array([ants[k] for k in ants.keys()], dtype=np.float64)
    else:
        antpos = np.asarray(ants, dtype=np.float64)
    kw.setdefault("radec", np.stack([np.asarray(ra, dtype=np.float64), np.asarray(dec, dtype=np.float64)]))
    return JobSpec(antpos=antpos, eci=point_source_crd_eq(ra, dec), fluxes=np.asarray(fluxes), freqs=np.asarray(freqs),
                   lsts=np.asarray(lsts), latitude=float(latitude), beams=list(beams), **kw)


def estimate_device_bytes(spec: JobSpec) -> int:
    """HBM footprint of a job (admission control): inputs, per-time buffers, Z panel,
    product workspace and the output."""
    A = len(spec.antpos)
    N = np.asarray(spec.eci).shape[1]
    Nf, Nt = len(spec.freqs), len(spec.lsts)
    F = X = 2 if spec.polarized else 1
    nch = max(1, int(spec.nchunks))
    chunk = int(np.ceil(N / nch)) if N else 1
    cap = max(1, int(chunk * spec.source_buffer) if chunk > 1000 else chunk)
    npairs = len(spec.antpairs) if spec.antpairs is not None else A * A
    csize = 8 if spec.precision == 1 else 16
    method, _ = _resolve_product(spec)
    if method == "MatMul":
        mode = _lib.GEMM_MODES[spec.gemm_mode] if isinstance(spec.gemm_mode, str) else int(spec.gemm_mode)
    else:
        mode = _lib.Z_C64
    mpad, kcap = _lib.zpanel_shape(mode, A * F, cap * X)
    G = freq_group_of(spec, method, is_chromatic(spec.beams))
    panel = G * _lib.lib.mvb_zpanel_bytes(mode, mpad, kcap)
    if method == "MatMul":
        T = mpad // _lib.TILE
        kc = spec.k_chunk or choose_k_chunk(T * (T + 1) // 2, kcap)
        ws = G * _lib.lib.mvb_herk_ws_bytes(mpad, kcap, kc)
    elif _lib.lib.mvb_vecdot_stage_columns(A, F) > 0:
        # the staged pair kernel: bundles of up to 3 pairs, ~0.85 filled, in warps of 32
        nb = -(-(int(npairs / 3 / 0.85) + 8) // 32) * 32
        ws = _lib.lib.mvb_vecdot_staged_ws_bytes(nb, F, kcap, spec.k_chunk or 4096) + 32 * nb
    else:
        ws = _lib.lib.mvb_vecdot_ws_bytes(npairs, F, kcap, spec.k_chunk or 4096)
    nbeam = len(spec.beams)
    pol_sky = np.ndim(spec.fluxes) == 4
    extra = (16 * Nf * N + 16 * N + 16 * cap) if pol_sky else 0  # coherency, ra/dec, frame rotations
    beam = 8 * nbeam * F * X * cap + 16 * nbeam * cap  # interpolated beams, per-source grid coordinates
    return int(24 * N + 8 * 3 * A + 4 * Nf * N + 24 * N + 28 * cap + beam + panel + ws
               + Nf * Nt * npairs * F * F * csize + extra)


def freq_group_of(spec: JobSpec, method: str, chromatic: bool) -> int:
    """Frequencies per grouped launch for this job: 1 for a pair list on per-pair
    sums (no grouped form) and for a beamfits beam (its beam changes with
    frequency), else ``spec.freq_group`` (default DEFAULT_FREQ_GROUP), at most
    the job's frequency count."""
    if method != "MatMul" or chromatic:
        return 1
    g = DEFAULT_FREQ_GROUP if spec.freq_group is None else int(spec.freq_group)
    if g < 1:
        raise ValueError("freq_group must be at least 1")
    return max(1, min(g, len(spec.freqs)))


def fit_freq_group(spec: JobSpec, budget: float) -> JobSpec:
    """``spec`` with the largest frequency group (at most its own) whose job fits
    ``budget`` bytes; a group of 1 when none does (``plan_job`` then batches)."""
    method, _ = _resolve_product(spec)
    g = freq_group_of(spec, method, is_chromatic(spec.beams))
    while g > 1 and estimate_device_bytes(replace(spec, freq_group=g)) > budget:
        g //= 2
    return replace(spec, freq_group=g)


def plan_job(spec: JobSpec, budget: float, max_chunks: int = 100) -> tuple[int, int]:
    """(frequencies per batch, source chunks) for ``spec`` to fit ``budget`` bytes of HBM.

    The output and the per-frequency fluxes grow with the number of frequencies,
    so a job larger than the budget runs as contiguous frequency batches of equal
    size, as few as fit (the reference runs one frequency per ``simulate`` call,
    wrapper.py:180-199, each sized to the free memory, gpu/gpu.py:99-110).  If a
    single frequency still does not fit, its sources are split into more chunks,
    up to ``max_chunks`` (the reference's cap, _utils.py:124-209); past that the
    plan is returned as is and the allocation itself reports the shortfall.
    """
    nf = len(spec.freqs)
    ch0 = max(1, int(spec.nchunks))
    fl = np.asarray(spec.fluxes)

    def fits(nfb: int, ch: int) -> bool:
        sub = replace(spec, freqs=np.asarray(spec.freqs)[:nfb], fluxes=fl[:, :nfb], nchunks=ch)
        return estimate_device_bytes(sub) <= budget

    if nf == 0 or not np.isfinite(budget) or fits(nf, ch0):
        return max(nf, 1), ch0
    if fits(1, ch0):
        lo, hi = 1, nf  # fits(lo) and not fits(hi): the largest batch that fits
        while hi - lo > 1:
            mid = (lo + hi) // 2
            lo, hi = (mid, hi) if fits(mid, ch0) else (lo, mid)
        nbatch = -(-nf // lo)
        return -(-nf // nbatch), ch0
    top = max(ch0, min(int(max_chunks), max(np.asarray(spec.eci).shape[1], 1)))
    for ch in range(ch0 + 1, top + 1):
        if fits(1, ch):
            return 1, ch
    return 1, top


def beam_bound(beams) -> float:
    """Upper bound of |interpolated beam| over all beams (grid maximum; 1 for Gaussians)."""
    b = 0.0
    for bm in beams:
        if isinstance(bm, GridBeam):
            d = bm.data if bm.beam_type == "efield" else np.sqrt(np.abs(bm.data))
            b = max(b, float(np.abs(d).max()))
        else:
            b = max(b, 1.0)
    return b
