"""Bundle plan of the staged pair kernel (host code, no GPU).

``mvb_vecdot_plan`` orders a pair list into bundles {i, j0, j1, j2, pair0,
pair1, pair2, flip bits}: up to three pairs sharing the conjugated antenna i.
The staged kernel computes acc[p, q] = sum_k Z[j, p, k] conj(Z[i, q, k]) per
bundle step, and a flipped step stands for out[q, p] = conj(acc[p, q]).  These
tests check the plan's structure (each pair once; the 8 lanes of a
shared-memory wavefront on distinct antenna residues mod 8, for i and for each
step's j) and, by evaluating the bundles with numpy, that the plan reproduces
the reference's VectorDot output (cpu/matprod.py:35-53).
"""

import numpy as np
import pytest

from matvis_b200 import _lib
from matvis_b200.matprod import vecdot_plan
from oracle import oracle as orc

C = 8


def _steps(plan):
    """(bundle, step) rows: i, j, pair, flip."""
    i = np.repeat(plan[:, 0], 3)
    j = plan[:, 1:4].ravel()
    pair = plan[:, 4:7].ravel()
    flip = ((plan[:, 7:8] >> np.arange(3)) & 1).ravel()
    return i, j, pair, flip


def _check_structure(plan, pairs, nant):
    assert plan.shape[1] == 8 and len(plan) % 32 == 0
    i, j, pair, flip = _steps(plan)
    real = pair >= 0
    assert np.array_equal(np.sort(pair[real]), np.arange(len(pairs)))
    assert ((plan[:, :4] >= 0) & (plan[:, :4] < nant)).all()
    p = np.asarray(pairs).reshape(-1, 2)[pair[real]]
    f = flip[real].astype(bool)
    assert np.array_equal(np.where(f[:, None], p[:, ::-1], p), np.column_stack([i[real], j[real]]))
    if nant >= C:
        # lane c of every phase of 8 bundles holds an i of residue c; each step's j residues are distinct
        assert np.array_equal(plan[:, 0] % C, np.arange(len(plan)) % C)
        for s in range(3):
            for row in plan[:, 1 + s].reshape(-1, C) % C:
                assert len(set(row.tolist())) == C


def _emulate(plan, z, nant, nfeed, npairs):
    """The staged kernel's arithmetic in FP64: step sums, then the reduction's un-flip."""
    zz = z.reshape(nant, nfeed, -1)
    out = np.zeros((npairs, nfeed, nfeed), complex)
    for i, j, pair, flip in zip(*_steps(plan)):
        if pair < 0:
            continue
        acc = zz[j].dot(zz[i].conj().T)  # acc[p, q]
        if flip:
            acc = acc.T.conj()
        if i == j:
            acc[np.diag_indices(nfeed)] = acc[np.diag_indices(nfeed)].real
        out[pair] = acc
    return out


@pytest.mark.parametrize("nfeed", [1, 2])
@pytest.mark.parametrize("nant,npairs", [(350, 5000), (37, 63), (7, 40), (3, 5), (120, 1)])
def test_plan_structure_and_emulation(nant, npairs, nfeed):
    rng = np.random.default_rng(nant * 10 + nfeed)
    pairs = rng.integers(0, nant, size=(npairs, 2))
    plan = vecdot_plan(pairs, nant, nfeed)
    _check_structure(plan, pairs, nant)
    K = 33
    z = rng.normal(size=(nant * nfeed, K)) + 1j * rng.normal(size=(nant * nfeed, K))
    ref = orc.vectordot_vis(z, nant, nfeed, pairs)
    np.testing.assert_allclose(_emulate(plan, z, nant, nfeed, npairs), ref, rtol=1e-12, atol=1e-12)


def test_plan_fill_on_seeded_lists():
    """Useful pair steps / all steps on the seeded 5,000-pair list of a 350-antenna
    array and on all 61,425 pairs (autos included)."""
    from matvis_b200 import workloads as wl

    cfg = wl.config3(nsrc=10)
    pairs = np.asarray(cfg["antpairs"])
    nant = len(cfg["antpos"])
    plan = vecdot_plan(pairs, nant, 2)
    _check_structure(plan, pairs, nant)
    assert len(pairs) / (3 * len(plan)) >= 0.85
    iu, ju = np.triu_indices(nant)
    allp = np.column_stack([iu, ju])
    plan = vecdot_plan(allp, nant, 2)
    _check_structure(plan, allp, nant)
    assert len(allp) / (3 * len(plan)) >= 0.95


def test_plan_duplicates_autos_and_one_class():
    # every pair in one residue class pair: the plan still holds each once
    pairs = np.array([[0, 8], [8, 16], [16, 0], [0, 0], [8, 8], [0, 8], [0, 8]])
    plan = vecdot_plan(pairs, 24, 2)
    _check_structure(plan, pairs, 24)
    # the worst case for the plan's size: one antenna pair repeated (one lane per step)
    for n in (1, 2, 3, 4, 299, 300, 301):
        pairs = np.tile([[0, 8]], (n, 1))
        plan = vecdot_plan(pairs, 16, 2)
        _check_structure(plan, pairs, 16)
        assert len(plan) <= 8 * (n // 3 + 2) + 24


def test_plan_empty_and_errors():
    assert vecdot_plan(np.zeros((0, 2), int), 10, 2).shape == (0, 8)
    with pytest.raises(ValueError, match="outside"):
        vecdot_plan(np.array([[0, 10]]), 10, 2)
    with pytest.raises(ValueError, match="outside"):
        vecdot_plan(np.array([[-1, 3]]), 10, 1)
    import ctypes

    n = ctypes.c_int64(0)
    buf = np.zeros(8, np.int32)
    assert _lib.lib.mvb_vecdot_plan(np.array([0, 1], np.int32).ctypes.data, 1, 4, 2, buf.ctypes.data, 4,
                                    ctypes.byref(n)) == _lib.MVB_ERR_ARG


def test_stage_columns_and_workspace():
    # the widest stage of which two fit in shared memory; none past ~2,400 rows
    assert _lib.lib.mvb_vecdot_stage_columns(350, 2) == 16
    assert _lib.lib.mvb_vecdot_stage_columns(37, 1) == 16
    assert _lib.lib.mvb_vecdot_stage_columns(1000, 1) == 8
    assert _lib.lib.mvb_vecdot_stage_columns(1600, 1) == 8
    assert _lib.lib.mvb_vecdot_stage_columns(1000, 2) == 4
    assert _lib.lib.mvb_vecdot_stage_columns(4000, 2) == 0
    assert _lib.lib.mvb_vecdot_stage_columns(0, 2) == 0
    # up to 31 k-slices beyond ceil(Kcap / min(k_chunk, 1024))
    assert _lib.lib.mvb_vecdot_staged_ws_bytes(64, 2, 4096, 4096) == (4 + 31) * 64 * 3 * 8 * 8
    rc = _lib.lib.mvb_vecdot_staged(None, 0, None, 0, 1, 2, 10, None, 0, 0, 16, None, 0, None, 0, 0, None, None)
    assert rc == _lib.MVB_ERR_ARG
