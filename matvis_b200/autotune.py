"""Autotuner for the Hermitian product's k-slice length.

The k-slice (``k_chunk``) sets how many source columns one work unit of
``mvb_herk`` accumulates before its partial tile is written: short slices give
more units (better balance across the SMs) but more partial-tile traffic and a
longer FP64 reduction; long slices the reverse.  Every candidate keeps the
accumulation error below 1e-6 (each 32-byte k-step is summed in a fresh TMEM
block and slices are reduced in FP64), so the choice is speed only.

``tune_k_chunk`` times each candidate on the job's own Z panel (a few launches,
CUDA events on a side stream) -- the product together with its reduction when
the caller passes ``run``, since shorter slices also mean more partial tiles to
reduce -- and caches the winner per (mode, Mpad, K bucket) for the life of the
process.
"""

from __future__ import annotations

import torch

from . import _lib

CANDIDATES = (1024, 2048, 4096)
_cache: dict[tuple, int] = {}


def _bucket(k: int) -> int:
    b = 1
    while b < k:
        b <<= 1
    return b


def tune_k_chunk(panel, mode: int, status: torch.Tensor, reps: int = 3, candidates=CANDIDATES, run=None) -> int:
    """Fastest k_chunk for this panel shape (panel.n_dev / n_host give the valid K).

    ``run(k_chunk, stream)``, if given, enqueues everything that depends on the
    k-slice (product and reduction); otherwise the product alone is timed."""
    kvalid = panel.n_host * panel.nax if panel.n_dev is None else int(panel.n_dev.item()) * panel.nax
    key = (mode, panel.Mpad, _bucket(max(kvalid, 1)), torch.cuda.current_device())
    if key in _cache:
        return _cache[key]
    cands = [c for c in candidates if c <= max(kvalid, candidates[0])] or [candidates[0]]
    ws = None
    if run is None:
        nbytes = max(_lib.lib.mvb_herk_ws_bytes(panel.Mpad, panel.Kcap, c) for c in cands)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=panel.data.device)
    s = torch.cuda.Stream(device=panel.data.device)
    s.wait_stream(torch.cuda.current_stream())
    best, best_ms = cands[0], float("inf")
    with torch.cuda.stream(s):
        for c in cands:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            for r in range(reps + 1):
                if r == 1:
                    e0.record(s)
                if run is not None:
                    run(c, s)
                    continue
                _lib.check(_lib.lib.mvb_herk(_lib.ptr(panel.data), mode, panel.Mpad, panel.Kcap, _lib.ptr(panel.n_dev),
                                             panel.n_host, panel.nax, c, 0, _lib.ptr(ws), ws.numel(), _lib.ptr(status),
                                             _lib.stream_handle(s)))
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            if ms < best_ms:
                best, best_ms = c, ms
    torch.cuda.current_stream().wait_stream(s)
    _cache[key] = best
    return best
