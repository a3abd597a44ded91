"""Failure paths of the device code that a test can reach without faulting the
GPU:

* every pipeline wait of the Hermitian product is bounded; with the limit
  shortened (mvb_set_wait_limit_ns) the product gives up, reports
  MVB_DEV_TIMEOUT through the status word (raised as MatvisB200Error with
  MVB_ERR_TIMEOUT), releases its tensor memory and returns, and the next
  product on the same device is correct;
* a pair list entry outside [0, nant) reaches the pair gather's device-side
  guard (the Python plugins reject it on the host first): its outputs are NaN
  and nothing outside the workspace is read;
* the chunk sum (MatProd.sum_chunks) adds in chunk order in FP64.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from matvis_b200 import _lib  # noqa: E402
from matvis_b200.matprod import B200MatMul  # noqa: E402

pytestmark = pytest.mark.gpu


def _random_z(nant, nfeed, K, seed):
    rng = np.random.default_rng(seed)
    z = rng.normal(size=(nant * nfeed, K)) + 1j * rng.normal(size=(nant * nfeed, K))
    return torch.as_tensor(z.astype(np.complex64), device="cuda")


def test_herk_wait_timeout_reports_and_recovers(device):
    nant, nfeed, K = 64, 2, 65536
    z = _random_z(nant, nfeed, K, 1)
    mp = B200MatMul(1, nfeed, nant, None, precision=2, gemm_mode="fp16x3", k_chunk=4096)
    mp.setup()
    ref = torch.zeros((nant * nant, nfeed, nfeed), dtype=torch.complex128, device=device)
    mp.compute(z, ref)
    torch.cuda.synchronize()
    _lib.check_status_word(mp.status, "first product")
    prev = _lib.lib.mvb_set_wait_limit_ns(1)
    try:
        out = torch.zeros_like(ref)
        mp.compute(z, out)
        torch.cuda.synchronize()
    finally:
        _lib.lib.mvb_set_wait_limit_ns(prev)
    assert int(mp.status.item()) & _lib.MVB_DEV_TIMEOUT
    with pytest.raises(_lib.MatvisB200Error) as exc:
        _lib.check_status_word(mp.status, "product with a 1 ns wait limit")
    assert exc.value.code == _lib.MVB_ERR_TIMEOUT
    # the limit is back to its default, and the device (its tensor memory included) is usable
    assert _lib.lib.mvb_set_wait_limit_ns(0) == prev
    mp.status.zero_()
    again = torch.zeros_like(ref)
    mp.compute(z, again)
    torch.cuda.synchronize()
    _lib.check_status_word(mp.status, "product after the timeout")
    assert torch.equal(again, ref)


def test_pair_gather_guards_out_of_range_entries(device):
    nant, nfeed, K = 40, 2, 8192
    z = _random_z(nant, nfeed, K, 2)
    mp = B200MatMul(1, nfeed, nant, None, precision=2, gemm_mode="tf32x3", k_chunk=2048)
    mp.setup()
    full = torch.zeros((nant * nant, nfeed, nfeed), dtype=torch.complex128, device=device)
    mp.compute(z, full)
    panel = mp._as_panel(z, mp.mode)
    ws = mp._ws
    pairs = torch.as_tensor(np.array([[0, 1], [0, 4000], [-1, 3], [5, 5], [39, 2]], dtype=np.int32), device=device)
    out = torch.zeros((5, nfeed, nfeed), dtype=torch.complex128, device=device)
    _lib.check(_lib.lib.mvb_herk_reduce(
        _lib.ptr(ws), ws.numel(), panel.Mpad, panel.Kcap, None, panel.n_host, panel.nax, 2048, nant, nfeed,
        _lib.ptr(pairs), 5, _lib.ptr(out), 1, 1.0 / panel.scale**2, 0, _lib.stream_handle()))
    torch.cuda.synchronize()
    o, f = out.cpu().numpy(), full.cpu().numpy()
    assert np.all(np.isnan(o[1].real)) and np.all(np.isnan(o[2].real))
    for row, (i, j) in ((0, (0, 1)), (3, (5, 5)), (4, (39, 2))):
        np.testing.assert_array_equal(o[row], f[i * nant + j])
    with pytest.raises(IndexError):
        B200MatMul(1, nfeed, nant, np.array([[0, nant]]))


@pytest.mark.parametrize("c128", [0, 1])
def test_chunk_sum_in_chunk_order(device, c128):
    rng = np.random.default_rng(3)
    dt = np.complex128 if c128 else np.complex64
    v = (rng.normal(size=(3, 257, 2, 2)) + 1j * rng.normal(size=(3, 257, 2, 2))).astype(dt)
    vd = torch.as_tensor(v, device=device)
    out = torch.empty_like(vd[0])
    _lib.check(_lib.lib.mvb_chunk_sum(_lib.ptr(vd), 3, out.numel(), c128, _lib.ptr(out), _lib.stream_handle()))
    want = v[0].astype(np.complex128)
    for c in (1, 2):
        want = want + v[c].astype(np.complex128)
    np.testing.assert_array_equal(out.cpu().numpy(), want.astype(dt))
