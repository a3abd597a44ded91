"""Multi-GPU partitioning of a job: independent (frequency) shards, no exchange.

The path shards naturally: every (frequency, time) slice is independent
(wrapper.py:180 and cpu/cpu.py:247 loops), so ranks take disjoint frequency
ranges, run them with no data-path collective, and the results are gathered to
rank 0 on the host.  One process per GPU; ``torch.distributed`` carries only
the gather and the timing reduction.
"""

from __future__ import annotations

import numpy as np


def frequency_shards(nfreq: int, world: int) -> list[tuple[int, int]]:
    """Contiguous [f0, f1) ranges, sizes differing by at most one, rank order."""
    if world <= 0:
        raise ValueError("world must be positive")
    base, extra = divmod(nfreq, world)
    out, f0 = [], 0
    for r in range(world):
        f1 = f0 + base + (1 if r < extra else 0)
        out.append((f0, f1))
        f0 = f1
    return out


def shard_spec(spec, rank: int, world: int):
    """The JobSpec restricted to this rank's frequency range (may be empty)."""
    from dataclasses import replace

    f0, f1 = frequency_shards(len(spec.freqs), world)[rank]
    return replace(spec, freqs=np.asarray(spec.freqs)[f0:f1], fluxes=np.asarray(spec.fluxes)[:, f0:f1]), (f0, f1)


def gather_frequency_shards(local: np.ndarray, rank: int, world: int, nfreq: int, group=None):
    """Gather per-rank (nf_r, ...) arrays to rank 0 as (nfreq, ...); other ranks get None."""
    import torch.distributed as dist

    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0, group=group)
    if rank != 0:
        return None
    out = np.concatenate([p for p in parts if p is not None and len(p)], axis=0)
    if out.shape[0] != nfreq:
        raise RuntimeError(f"gathered {out.shape[0]} frequencies, expected {nfreq}")
    return out


def run_sharded(spec, rank: int, world: int, device=None):
    """Run this rank's frequency shard on its GPU and gather the visibilities to rank 0."""
    from .engine import VisEngine

    local_spec, (f0, f1) = shard_spec(spec, rank, world)
    if f1 > f0:
        local = VisEngine(local_spec, device=device).run().cpu().numpy()
    else:
        nfeed = 2 if spec.polarized else 1
        npairs = len(spec.antpairs) if spec.antpairs is not None else len(spec.antpos) ** 2
        local = np.zeros((0, len(spec.lsts), npairs, nfeed, nfeed), dtype=np.complex64)
    return gather_frequency_shards(local, rank, world, len(spec.freqs))
