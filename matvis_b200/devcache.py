"""Device copies shared by the jobs of one process (the served form's caches).

Two kinds of read-only device data recur across jobs:

* beam grids: every polarised job of a served stream may use the same gridded
  beams.  They are keyed by content (a BLAKE2 digest of the grid bytes, a few
  hundred kilobytes per beam), so equal grids share one device copy however
  the caller built them;
* skies: a caller that serves many jobs on one sky model (different arrays,
  times or frequencies) names it with ``JobSpec.sky_key``; jobs with the same
  key share the device copy of the source directions and fluxes.  The key is
  the caller's promise that the arrays are equal; nothing is re-checked.

Entries are evicted least-recently-used beyond a byte budget; an entry a running
job still holds stays alive through that job's reference (torch frees it when
the last holder lets go), so eviction never invalidates a job.
"""

from __future__ import annotations

import hashlib
import threading
from collections import OrderedDict

import numpy as np
import torch

#: bytes of device memory the cache keeps (per process, all devices together)
MAX_BYTES = 4 << 30


class DeviceCache:
    """LRU map key -> tuple of device tensors, bounded by their bytes."""

    def __init__(self, max_bytes: int = MAX_BYTES):
        self.max_bytes = int(max_bytes)
        self._d: OrderedDict = OrderedDict()
        self._bytes = 0
        self._lock = threading.Lock()
        self.hits = 0
        self.misses = 0

    @staticmethod
    def _size(value) -> int:
        return sum(t.numel() * t.element_size() for t in value)

    def get(self, key, make):
        """The cached tensors for ``key`` (a tuple), built by ``make()`` on the
        current stream on a miss.  Any stream that receives them waits for the
        copies that made them, and each tensor is recorded on that stream, so
        the caching allocator does not reuse its memory while the stream still
        reads it."""
        with self._lock:
            hit = self._d.get(key)
            if hit is not None:
                self._d.move_to_end(key)
                self.hits += 1
        if hit is None:
            value = tuple(make())
            ready = torch.cuda.Event()
            ready.record()
            with self._lock:
                self.misses += 1
                if key not in self._d:
                    self._d[key] = (value, ready)
                    self._bytes += self._size(value)
                    while self._bytes > self.max_bytes and len(self._d) > 1:
                        _, (old, _) = self._d.popitem(last=False)
                        self._bytes -= self._size(old)
                hit = self._d[key]
        value, ready = hit
        cur = torch.cuda.current_stream(value[0].device if value else None)
        cur.wait_event(ready)
        for t in value:
            t.record_stream(cur)
        return value

    def clear(self):
        with self._lock:
            self._d.clear()
            self._bytes = 0

    @property
    def nbytes(self) -> int:
        return self._bytes


CACHE = DeviceCache()


def digest(*arrays) -> str:
    """Content key of host arrays (shape, dtype and bytes)."""
    h = hashlib.blake2b(digest_size=20)
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str((a.shape, a.dtype.str)).encode())
        h.update(memoryview(a).cast("B"))
    return h.hexdigest()


def device_key(device) -> str:
    d = torch.device(device)
    return f"{d.type}:{d.index if d.index is not None else torch.cuda.current_device()}"
