"""The allocation-free horizon selection, ``mvb_horizon_compact_static``.

It serves callers that cannot allocate device memory at the moment they select
sources: pipelines that plan all device memory at start-up and forbid later
allocation (cudaMalloc / cudaFree can synchronise the whole device), and hosts
that are handed only a stream and buffers by another library.  Its scratch is a
static device array inside the library, so the results must equal those of the
workspace-taking ``mvb_horizon_compact`` exactly (the selection is bit-exact),
call after call, since every call reuses the same array.

This file is collected last so that, if it fails, a run stopping at the first
failure has already run every other test; it also passes alone in a fresh
process.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from matvis_b200 import _lib  # noqa: E402
from matvis_b200.coordinates import eci_to_enu_matrix, point_source_crd_eq  # noqa: E402

pytestmark = pytest.mark.gpu


def _select(topo, n, c0, c1, flux, cap, static: bool):
    dev = topo.device
    crd = torch.zeros((3, cap), dtype=torch.float64, device=dev)
    idx = torch.zeros((cap,), dtype=torch.int32, device=dev)
    fo = torch.full((cap,), -1.0, dtype=torch.float64, device=dev)
    nout = torch.zeros(1, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    sh = _lib.stream_handle()
    if static:
        rc = _lib.lib.mvb_horizon_compact_static(_lib.ptr(topo), n, c0, c1, _lib.ptr(flux), _lib.ptr(crd), _lib.ptr(idx),
                                                 _lib.ptr(fo), _lib.ptr(nout), cap, _lib.ptr(status), sh)
    else:
        ws = torch.empty(_lib.lib.mvb_horizon_ws_bytes(c1 - c0), dtype=torch.uint8, device=dev)
        rc = _lib.lib.mvb_horizon_compact(_lib.ptr(topo), n, c0, c1, _lib.ptr(flux), _lib.ptr(crd), _lib.ptr(idx),
                                          _lib.ptr(fo), _lib.ptr(nout), cap, _lib.ptr(status), _lib.ptr(ws), ws.numel(),
                                          sh)
    _lib.check(rc)
    torch.cuda.synchronize()
    k = int(nout.item())
    return k, idx[:k].cpu().numpy(), crd[:, :k].cpu().numpy(), fo.cpu().numpy(), int(status.item())


def test_static_scratch_matches_workspace_entry_point(device):
    rng = np.random.default_rng(2026)
    n = 300_000
    ra, dec = rng.uniform(0, 2 * np.pi, n), np.arcsin(rng.uniform(-1, 1, n))
    eci = torch.as_tensor(np.ascontiguousarray(point_source_crd_eq(ra, dec)), device=device)
    flux = torch.as_tensor(rng.uniform(0.1, 3.0, n), device=device)
    topo = torch.empty((3, n), dtype=torch.float64, device=device)
    lat = np.deg2rad(-30.72)
    # two calls in a row, different times and source ranges, sharing the static array
    for lst, c0, c1 in ((0.4, 0, n), (3.3, 12_345, 250_001)):
        R = np.ascontiguousarray(eci_to_enu_matrix(lst, lat))
        _lib.check(_lib.lib.mvb_rotate(_lib.ptr(eci), n, R.ctypes.data_as(_lib.c_void_p), _lib.ptr(topo),
                                       _lib.stream_handle()))
        cap = c1 - c0
        ref = _select(topo, n, c0, c1, flux, cap, static=False)
        got = _select(topo, n, c0, c1, flux, cap, static=True)
        assert got[0] == ref[0] and got[0] > 0
        np.testing.assert_array_equal(got[1], ref[1])
        np.testing.assert_array_equal(got[2], ref[2])
        np.testing.assert_array_equal(got[3], ref[3])
        assert got[4] == ref[4] == 0


def test_static_scratch_rejects_oversize_chunk(device):
    big = 4096 * 1024 + 1
    dummy = torch.zeros(3, dtype=torch.float64, device=device)
    nout = torch.zeros(1, dtype=torch.int32, device=device)
    # rejected on the host before any launch: nothing is read from the buffers
    rc = _lib.lib.mvb_horizon_compact_static(_lib.ptr(dummy), big, 0, big, None, _lib.ptr(dummy), _lib.ptr(nout),
                                             None, _lib.ptr(nout), 1, None, _lib.stream_handle())
    assert rc == _lib.MVB_ERR_ARG
    assert b"static limit" in _lib.lib.mvb_last_error()


def test_static_scratch_at_its_limit(device):
    """A chunk of exactly 4,194,304 sources (4,096 blocks: every slot of the static
    array) selects the same sources as the workspace entry point."""
    rng = np.random.default_rng(7)
    n = 4096 * 1024
    ra, dec = rng.uniform(0, 2 * np.pi, n), np.arcsin(rng.uniform(-1, 1, n))
    eci = torch.as_tensor(np.ascontiguousarray(point_source_crd_eq(ra, dec)), device=device)
    flux = torch.as_tensor(rng.uniform(0.1, 3.0, n), device=device)
    topo = torch.empty((3, n), dtype=torch.float64, device=device)
    R = np.ascontiguousarray(eci_to_enu_matrix(1.1, np.deg2rad(-30.72)))
    _lib.check(_lib.lib.mvb_rotate(_lib.ptr(eci), n, R.ctypes.data_as(_lib.c_void_p), _lib.ptr(topo),
                                   _lib.stream_handle()))
    ref = _select(topo, n, 0, n, flux, n, static=False)
    got = _select(topo, n, 0, n, flux, n, static=True)
    assert got[0] == ref[0] > n // 3
    np.testing.assert_array_equal(got[1], ref[1])
    np.testing.assert_array_equal(got[2], ref[2])
    np.testing.assert_array_equal(got[3], ref[3])
    assert got[4] == ref[4] == 0
