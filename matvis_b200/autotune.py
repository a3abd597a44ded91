"""Autotuner for the Hermitian product: k-slice length and drain interval, timed
on the job's own Z panel; frequencies per grouped launch sized to memory.

* ``k_chunk`` -- how many source columns one work unit of ``mvb_herk``
  accumulates before its partial tile is written: short slices give more units
  (better balance across the SMs) but more partial-tile traffic and a longer
  FP64 reduction; long slices the reverse.
* ``drain_ksteps`` (KD) -- how many 32-byte k-steps the tensor core sums in one
  TMEM block before the epilogue adds the block to FP32 registers.  Fewer drains
  leave the UMMAs more of the SM, but the accumulator is truncated toward zero
  at every instruction, so the error grows with KD.  The block's products are
  issued in ascending magnitude (cross terms first), and the errors measured on a
  whole config-2 slice against the FP64 oracle (``MEASURED_ERROR``) decide which
  KD are candidates: those under ``ERROR_BUDGET``.
* frequencies per grouped launch (``fit_freq_group`` in the engine): the job time
  measured the same for 1 to 16 frequencies per launch (1.69-1.72 s for the
  config-2 job), so the group is sized by memory, not timed.

``tune_product`` times every candidate pair (a few launches each, CUDA events
on a side stream) -- the product together with its reduction when the caller
passes ``run`` -- and caches the winner per (mode, Mpad, K bucket, device) for
the life of the process; ``cached_choice`` hands it to later jobs of the same
shape that are not captured (``simulate_vis``).  ``last_choice`` reports the
latest decision.
"""

from __future__ import annotations

import torch

from . import _lib

KC_CANDIDATES = (1024, 2048, 4096, 8192)
KD_CANDIDATES = (1, 2, 4)
#: max |V - V_oracle| / sqrt(|V_ii| |V_jj|) measured on a whole config-2 slice
#: (196,608 sources, 350 antennas, complex128 output, k_chunk 4096) per split
#: mode and drain interval; product time per slice in the comment (one B200)
MEASURED_ERROR = {
    _lib.GEMM_F16_3: {1: 2.00e-7, 2: 3.04e-7, 4: 5.62e-7},   # 1.32 / 1.16 / 1.29 ms
    _lib.GEMM_TF32_3: {1: 1.75e-7, 2: 2.42e-7, 4: 3.83e-7},  # 2.61 / 2.14 / 2.56 ms
    _lib.GEMM_BF16_6: {1: 1.23e-7, 2: 1.66e-7, 4: 3.39e-7},  # 2.06 / 1.92 / 2.26 ms
    _lib.GEMM_BF16_3: {1: 3.5e-6, 2: 3.5e-6, 4: 3.5e-6},     # the 2-term bf16 split itself misses the bar
}
#: largest accepted measured error of a drain interval (the bar is 1e-6)
ERROR_BUDGET = 6e-7
_cache: dict[tuple, tuple[int, int]] = {}
#: the latest decision: candidates timed (ms per launch) and the winner
last_choice: dict = {}


def _bucket(k: int) -> int:
    b = 1
    while b < k:
        b <<= 1
    return b


def drain_candidates(mode: int, kd_candidates=KD_CANDIDATES) -> list[int]:
    """Drain intervals whose measured error fits ERROR_BUDGET (0 = the mode's
    default, always allowed); the lowest-error one if none does."""
    meas = MEASURED_ERROR.get(mode, {})
    ok = [d for d in kd_candidates if d == 0 or meas.get(d, float("inf")) <= ERROR_BUDGET]
    return ok or [min(meas, key=meas.get, default=1)]


def tune_product(panel, mode: int, status: torch.Tensor, run=None, reps: int = 3, kc_candidates=KC_CANDIDATES,
                 kd_candidates=KD_CANDIDATES) -> tuple[int, int]:
    """Fastest (k_chunk, drain_ksteps) for this panel shape (panel.n_dev / n_host
    give the valid K).

    ``run(k_chunk, drain_ksteps, stream)``, if given, enqueues everything that
    depends on the two (product and reduction); otherwise the product alone is
    timed."""
    global last_choice
    kvalid = panel.n_host * panel.nax if panel.n_dev is None else int(panel.n_dev.item()) * panel.nax
    kcs = [c for c in kc_candidates if c <= max(kvalid, kc_candidates[0])] or [kc_candidates[0]]
    kds = drain_candidates(mode, kd_candidates)
    key = (mode, panel.Mpad, _bucket(max(kvalid, 1)), torch.cuda.current_device(), tuple(kcs), tuple(kds))
    if key in _cache:
        return _cache[key]
    ws = None
    if run is None:
        nbytes = max(_lib.lib.mvb_herk_ws_bytes(panel.Mpad, panel.Kcap, c) for c in kcs)
        ws = torch.empty(nbytes, dtype=torch.uint8, device=panel.data.device)
    s = torch.cuda.Stream(device=panel.data.device)
    s.wait_stream(torch.cuda.current_stream())
    best, best_ms = (kcs[0], kds[0]), float("inf")
    timed = {}
    with torch.cuda.stream(s):
        for kd in kds:
            for c in kcs:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                for r in range(reps + 1):
                    if r == 1:
                        e0.record(s)
                    if run is not None:
                        run(c, kd, s)
                        continue
                    _lib.check(_lib.lib.mvb_herk(_lib.ptr(panel.data), mode, panel.Mpad, panel.Kcap,
                                                 _lib.ptr(panel.n_dev), panel.n_host, panel.nax, c, kd, _lib.ptr(ws),
                                                 ws.numel(), _lib.ptr(status), _lib.stream_handle(s)))
                e1.record(s)
                e1.synchronize()
                ms = e0.elapsed_time(e1) / reps
                timed[f"k_chunk={c},drain_ksteps={kd}"] = round(ms, 4)
                if ms < best_ms:
                    best, best_ms = (c, kd), ms
    torch.cuda.current_stream().wait_stream(s)
    _cache[key] = best
    last_choice = {"k_chunk": best[0], "drain_ksteps": best[1], "ms": round(best_ms, 4), "timed_ms": timed,
                   "shape": {"Mpad": panel.Mpad, "K": kvalid, "mode": mode}}
    return best


def cached_choice(mode: int, Mpad: int, kvalid: int, device: int) -> tuple[int, int] | None:
    """A (k_chunk, drain_ksteps) already tuned in this process for this shape
    (mode, Mpad, K bucket, device), or None."""
    b = _bucket(max(int(kvalid), 1))
    for key, choice in _cache.items():
        if key[:4] == (mode, Mpad, b, device):
            return choice
    return None


def tune_k_chunk(panel, mode: int, status: torch.Tensor, reps: int = 3, candidates=KC_CANDIDATES, run=None) -> int:
    """k-slice length alone (the mode's default drain interval)."""
    r = None if run is None else (lambda c, kd, st: run(c, st))
    return tune_product(panel, mode, status, run=r, reps=reps, kc_candidates=candidates, kd_candidates=(0,))[0]
