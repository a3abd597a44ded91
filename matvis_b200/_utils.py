"""Chunk planning and dtypes (mirrors the reference's ``_utils.py:124-319``).

The byte model is the reference's; the free memory it is given here is the
device's free HBM (``torch.cuda.mem_get_info``), as in gpu/gpu.py:99-110.
"""

from __future__ import annotations

import logging

import numpy as np

logger = logging.getLogger(__name__)


def get_dtypes(precision: int):
    """(real, complex) numpy dtypes for precision 1 or 2; _utils.py:291-319."""
    if precision == 1:
        return np.float32, np.complex64
    return np.float64, np.complex128


def get_required_chunks(freemem, nax, nfeed, nant, nsrc, nbeam, nbeampix, precision, source_buffer=1.0,
                        memory_buffer=0.9) -> int:
    """Number of source chunks for the data to fit ``freemem`` bytes; _utils.py:124-209."""
    if not (0 < memory_buffer <= 1.0):
        raise ValueError("memory_buffer must be in the range (0, 1]")
    rsize = 4 * precision
    csize = 2 * rsize
    total = freemem
    ch = 0
    while total >= freemem * memory_buffer and ch < 100:
        ch += 1
        nchunk = int(nsrc // ch * source_buffer)
        sizes = {
            "antpos": nant * 3 * rsize,
            "flux": nsrc * rsize,
            "beam": nbeampix * nfeed * nax * csize,
            "crd_eq": 3 * nsrc * rsize,
            "eq2top": 3 * 3 * rsize,
            "crd_top": 3 * nsrc * rsize,
            "crd_chunk": 3 * nchunk * rsize,
            "flux_chunk": nchunk * rsize,
            "exptau": nant * nchunk * csize,
            "beam_interp": nbeam * nfeed * nax * nchunk * csize,
            "zmat": nchunk * nfeed * nant * nax * csize,
            "vis": ch * nfeed * nant * nfeed * nant * csize,
        }
        total = sum(sizes.values())
    return max(ch, 1)


def get_desired_chunks(freemem, min_chunks, beam_list, nax, nfeed, nant, nsrc, precision, source_buffer=1.0,
                       memory_buffer=0.9):
    """(nchunks, sources per chunk); _utils.py:212-288."""
    nbeampix = sum(b.data.shape[-2] * b.data.shape[-1] for b in beam_list if hasattr(b, "data"))
    nchunks = min(
        max(
            min_chunks,
            get_required_chunks(freemem, nax, nfeed, nant, nsrc, len(beam_list), nbeampix, precision, source_buffer,
                                memory_buffer),
        ),
        max(nsrc, 1),
    )
    return nchunks, int(np.ceil(nsrc / nchunks))
