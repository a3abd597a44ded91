"""``simulate`` (one frequency) and ``simulate_vis`` (all frequencies).

Keyword-compatible with ``matvis.cpu.simulate`` / ``matvis.gpu.simulate``
(cpu/cpu.py:35-277, gpu/gpu.py:57-256) and ``matvis.simulate_vis``
(wrapper.py:25-200), with these input conventions (astropy and pyuvdata are not
dependencies):

* ``times`` are local sidereal times in radians and ``telescope_loc`` is the
  latitude in radians (or an object with ``.lat``); the rotation is the rigid
  LST rotation (``coord_method="CoordinateRotationLST"``), or the ERFA-style
  apparent place (``coord_method="CoordinateRotationERFA"``) from per-time
  astrometry parameters given in ``coord_method_params``;
* ``fluxes`` is Stokes I (NSRCS, NFREQS), or, with ``polarized=True``, a
  (NSRCS, NFREQS, 2, 2) coherency for a polarised sky;
* beams are :class:`~matvis_b200.beams.GridBeam` / :class:`~matvis_b200.beams.GaussianBeam`
  or a beamfits beam (:func:`~matvis_b200.beamfits.read_beamfits`), interpolated to
  each frequency;
* ``skycoords`` is an (ra, dec) pair in radians or an object with ``.ra``/``.dec``;
* ``matprod_method="VectorDot"`` with a pair list runs the per-pair kernel or,
  where a measured cost model predicts it faster, the tensor-core Hermitian
  product with a pair gather (same output); ``pair_product`` ("auto", "vecdot",
  "herk") overrides the choice.

Both run the batched engine (``engine.VisEngine``): every time and frequency of
the call is one launch sequence on the GPU, with device-side source counts, and
each time step's visibilities are copied to the host while later steps compute.
"""

from __future__ import annotations

import logging
from dataclasses import replace

import numpy as np
import torch

from . import _lib
from ._utils import get_desired_chunks
from .beams import beams_at_frequency
from .coordinates import latitude_of, lsts_of, point_source_crd_eq, radec_of
from .engine import JobSpec, VisEngine, _norm_matprod, fit_freq_group, plan_job


logger = logging.getLogger(__name__)

_UNAVAILABLE_COORD = ("CoordinateRotationAstropy",)
_ERFA_COORD = ("CoordinateRotationERFA", "GPUCoordinateRotationERFA")


def _validate_inputs(precision, polarized, antpos, times, I_sky):
    """core/__init__.py:11-32."""
    assert precision in {1, 2}
    nax = nfeed = 2 if polarized else 1
    nant, ncrd = antpos.shape
    assert ncrd == 3, "antpos must have shape (NANTS, 3)."
    ntimes = len(times)
    assert I_sky.ndim == 1, "I_sky must have shape (NSRCS,)."
    return nax, nfeed, nant, ntimes


def _check_coord_method(coord_method, params=None):
    """Rotation keywords for the JobSpec: {} for the LST rotation, the astrom
    parameters for the ERFA-style one."""
    if coord_method in _UNAVAILABLE_COORD:
        raise NotImplementedError(
            f"{coord_method} needs astropy's transform machinery, which this build does not ship; use "
            "coord_method='CoordinateRotationLST' (times = LSTs in radians) or 'CoordinateRotationERFA' with "
            "coord_method_params={'astrom': [...], 'time_s': [...], 'update_bcrs_every': seconds}"
        )
    if coord_method in _ERFA_COORD:
        params = dict(params or {})
        if "astrom" not in params:
            raise ValueError("CoordinateRotationERFA needs coord_method_params['astrom'] (one pyerfa apco dict per time)")
        return {"astrom": list(params["astrom"]), "time_s": params.get("time_s"),
                "update_bcrs_every": float(params.get("update_bcrs_every", 0.0))}
    if coord_method != "CoordinateRotationLST":
        raise ValueError(f"unknown coord_method {coord_method!r}")
    return {}


def simulate(
    *,
    antpos,
    freq: float,
    times,
    skycoords,
    telescope_loc,
    I_sky,
    beam_list,
    antpairs=None,
    precision: int = 1,
    polarized: bool = False,
    beam_idx=None,
    beam_spline_opts=None,
    max_progress_reports: int = 100,
    matprod_method: str = "B200MatMul",
    pair_product: str = "auto",
    coord_method: str = "CoordinateRotationLST",
    max_memory=np.inf,
    min_chunks: int = 1,
    source_buffer: float = 1.0,
    memory_buffer: float = 0.9,
    coord_method_params=None,
    gemm_mode: str = "fp16x3",
    k_chunk: int | None = None,
    device=None,
):
    """Visibilities at one frequency for all times; returns (Nt, Npairs, F, F) or (Nt, Npairs)."""
    if not 0 < source_buffer <= 1:
        raise ValueError("source_buffer must satisfy 0 < source_buffer <= 1")
    if not 0 < memory_buffer <= 1:
        raise ValueError("memory_buffer must satisfy 0 < memory_buffer <= 1")
    rot_kw = _check_coord_method(coord_method, coord_method_params)
    dev = _lib.require_cuda(device)
    antpos = np.asarray(antpos, dtype=np.float64)
    I_sky = np.asarray(I_sky)
    lsts = lsts_of(times)
    nax, nfeed, nant, ntimes = _validate_inputs(precision, polarized, antpos, lsts, I_sky)
    ra, dec = radec_of(skycoords)
    free = torch.cuda.mem_get_info(dev)[0]
    nchunks, _ = get_desired_chunks(min(max_memory, free), min_chunks, beam_list, nax, nfeed, nant, len(I_sky),
                                    precision, source_buffer=source_buffer, memory_buffer=memory_buffer)
    spec = JobSpec(
        antpos=antpos, eci=point_source_crd_eq(ra, dec), fluxes=I_sky[:, None], freqs=np.array([float(freq)]),
        lsts=lsts, latitude=latitude_of(telescope_loc), beams=beams_at_frequency(beam_list, freq), beam_idx=beam_idx,
        polarized=polarized,
        antpairs=antpairs, precision=precision, gemm_mode=gemm_mode, matprod=_norm_matprod(matprod_method),
        pair_product=pair_product, k_chunk=k_chunk, source_buffer=source_buffer, nchunks=nchunks, **rot_kw,
    )
    eng = VisEngine(spec, device=dev)
    out = eng.run_to_host()[0]
    return out if polarized else out[:, :, 0, 0]


def simulate_vis(
    ants,
    fluxes,
    ra,
    dec,
    freqs,
    times,
    beams,
    telescope_loc,
    polarized: bool = False,
    precision: int = 1,
    use_feed: str = "x",
    use_gpu: bool = True,
    beam_spline_opts=None,
    beam_idx=None,
    antpairs=None,
    source_buffer: float = 1.0,
    coord_method: str = "CoordinateRotationLST",
    coord_method_params=None,
    matprod_method: str = "MatMul",
    pair_product: str = "auto",
    gemm_mode: str = "fp16x3",
    k_chunk: int | None = None,
    freq_group: int | None = None,
    min_chunks: int = 1,
    max_memory=np.inf,
    memory_buffer: float = 0.9,
    device=None,
    **backend_kwargs,
):
    """All frequencies and times; returns (Nf, Nt, Npairs, F, F) or (Nf, Nt, Npairs).

    ``ants``: {index: (x, y, z)} in metres; ``fluxes``: (NSRCS, NFREQS);
    ``ra``/``dec`` radians; ``freqs`` Hz; ``times`` LSTs (radians).

    The job is sized against ``memory_buffer`` x min(``max_memory``, the device's
    free memory): one batched job when it fits (with ``freq_group`` frequencies
    per grouped launch, fewer if memory is short: ``engine.fit_freq_group``),
    else contiguous frequency batches (and, if one frequency does not fit, more
    source chunks), each written into its slice of one host array
    (``engine.plan_job``).  ``beam_spline_opts`` and
    ``max_progress_reports`` are accepted for the reference's keyword set and
    have no effect; any other keyword is an error, as in the reference.
    """
    unknown = set(backend_kwargs) - {"max_progress_reports"}
    if unknown:
        raise TypeError(f"simulate_vis() got unexpected keyword arguments {sorted(unknown)}")
    if not 0 < memory_buffer <= 1:
        raise ValueError("memory_buffer must satisfy 0 < memory_buffer <= 1")
    if not use_gpu:
        raise ValueError("matvis_b200 runs on the GPU only (use_gpu=False has no CPU path here)")
    rot_kw = _check_coord_method(coord_method, coord_method_params)
    fluxes = np.asarray(fluxes)
    ra = np.asarray(ra, dtype=np.float64)
    dec = np.asarray(dec, dtype=np.float64)
    freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
    assert fluxes.shape[:2] == (ra.size, freqs.size) and fluxes.ndim in (2, 4), \
        "The `fluxes` array must have shape (NSRCS, NFREQS) or, for a polarised sky, (NSRCS, NFREQS, 2, 2)."
    antpos = np.array([ants[k] for k in ants.keys()], dtype=np.float64)
    if not 0 < source_buffer <= 1:
        raise ValueError("source_buffer must satisfy 0 < source_buffer <= 1")
    common = dict(
        antpos=antpos, eci=point_source_crd_eq(ra, dec), radec=np.stack([ra, dec]), lsts=lsts_of(times),
        latitude=latitude_of(telescope_loc),
        beam_idx=beam_idx, polarized=polarized, antpairs=antpairs, precision=precision, gemm_mode=gemm_mode,
        matprod=_norm_matprod(matprod_method), pair_product=pair_product, k_chunk=k_chunk, source_buffer=source_buffer,
        nchunks=max(1, int(min_chunks)), freq_group=freq_group, **rot_kw,
    )
    # frequency-dependent (beamfits) beams are interpolated per frequency inside the
    # one batched job (the reference re-interpolates per frequency, wrapper.py:180-199)
    spec = JobSpec(fluxes=fluxes, freqs=freqs, beams=list(beams), **common)
    dev = _lib.require_cuda(device)
    # memory the caching allocator holds but does not use is free for this job too
    free = torch.cuda.mem_get_info(dev)[0] + torch.cuda.memory_reserved(dev) - torch.cuda.memory_allocated(dev)
    budget = min(max_memory, free) * memory_buffer
    spec = fit_freq_group(spec, budget)
    nfb, nchunks = plan_job(spec, budget)
    if nfb >= freqs.size and nchunks == spec.nchunks:
        vis = VisEngine(spec, device=dev).run_to_host()
        return vis if polarized else vis[..., 0, 0]
    logger.info("simulate_vis: %d frequencies in batches of %d, %d source chunks", freqs.size, nfb, nchunks)
    vis = None
    for f0 in range(0, freqs.size, nfb):
        sub = replace(spec, fluxes=fluxes[:, f0 : f0 + nfb], freqs=freqs[f0 : f0 + nfb], nchunks=nchunks)
        eng = VisEngine(sub, device=dev)
        eng.allocate()
        if vis is None:
            vis = np.empty((freqs.size,) + tuple(eng.vis.shape[1:]),
                           dtype=np.complex64 if precision == 1 else np.complex128)
        eng.run_to_host(out=vis[f0 : f0 + len(sub.freqs)])
        del eng
    return vis if polarized else vis[..., 0, 0]
