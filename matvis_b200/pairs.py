"""Redundant-baseline pair selection (``get_redundancies``, cli.py:273-290).

The selection runs in the native library (``mvb_redundant_pairs``); the result
is the ``antpairs`` list the drivers take, e.g. for the per-pair
``B200VectorDot`` product.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def get_redundancies(bls, ndecimals: int = 2) -> list[list[int]]:
    """One representative pair (i, j), i < j, per redundant baseline class.

    ``bls``: (nant, nant, 2) baselines with ``bls[i, j] = pos[j, :2] - pos[i, :2]``
    (an object with ``.value`` is unwrapped).  Same result and order as the
    reference's function.
    """
    bls = np.ascontiguousarray(np.asarray(getattr(bls, "value", bls), dtype=np.float64))
    if bls.ndim != 3 or bls.shape[0] != bls.shape[1] or bls.shape[2] != 2:
        raise ValueError("bls must have shape (nant, nant, 2)")
    nant = bls.shape[0]
    cap = max(1, nant * (nant - 1) // 2)
    out = np.zeros((cap, 2), dtype=np.int32)
    n = ctypes.c_int64(0)
    _lib.check(_lib.lib.mvb_redundant_pairs(bls.ctypes.data_as(ctypes.c_void_p), nant, int(ndecimals),
                                            out.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n)))
    return out[: n.value].tolist()


def baselines(antpos) -> np.ndarray:
    """(nant, nant, 2) east/north baselines ``pos[j] - pos[i]`` (cli.py:316)."""
    antpos = np.asarray(getattr(antpos, "value", antpos), dtype=np.float64)
    return antpos[np.newaxis, :, :2] - antpos[:, np.newaxis, :2]


def redundant_antpairs(antpos, ndecimals: int = 2) -> np.ndarray:
    """``antpairs`` (npairs, 2) int array of the redundant representatives."""
    return np.asarray(get_redundancies(baselines(antpos), ndecimals), dtype=np.int64).reshape(-1, 2)
