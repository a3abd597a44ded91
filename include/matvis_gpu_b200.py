"""Reference-side binding of libmatvis_b200.so for matvis's GPU backend.

A maintainer adding the library to matvis itself copies this file to
``src/matvis/gpu/_b200.py`` (beside ``gpu/_cublas.py``) and calls

* :func:`zdotz_upper` from ``GPUMatMul.compute`` (gpu/matprod.py:31-36) in
  place of ``_cublas.zdotz``, and
* :func:`set_bcrs` from ``GPUCoordinateRotationERFA._set_bcrs``
  (gpu/coords.py:37-53) in place of its deflection / aberration / BPN steps.

Device buffers are cupy arrays (matvis's GPU array library); only their raw
pointers cross the boundary.  The signatures below are those of
``include/matvis_b200.h``.
"""

import ctypes

import numpy as np

_p, _i, _i64, _sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_size_t
_f, _d = ctypes.c_float, ctypes.c_double

#: (restype, argtypes) of the entry points this binding calls
SIGNATURES = {
    "mvb_last_error": (ctypes.c_char_p, []),
    "mvb_zpanel_bytes": (_sz, [_i, _i64, _i64]),
    "mvb_z_pack": (_i, [_p, _i, _i64, _i64, _i64, _i, _f, _p, _i64, _i64, _p]),
    "mvb_herk_ws_bytes": (_sz, [_i64, _i64, _i]),
    "mvb_herk": (_i, [_p, _i, _i64, _i64, _p, _i64, _i, _i, _i, _p, _sz, _p, _p]),
    "mvb_herk_reduce": (_i, [_p, _sz, _i64, _i64, _p, _i64, _i, _i, _i, _i, _p, _i64, _p, _i, _d, _i, _p]),
    "mvb_bcrs": (_i, [_p, _i64, _p, _p, _p]),
}

#: mode 1 = 3-term bf16 split (6 products); the product's other modes are in the header
MVB_GEMM_BF16_6 = 1


def load(path: str = "libmatvis_b200.so") -> ctypes.CDLL:
    """Open the library and declare the signatures above."""
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def _check(lib, rc: int):
    if rc != 0:
        raise RuntimeError((lib.mvb_last_error() or b"").decode(errors="replace"))


def zdotz_upper(lib, z, nant: int, nfeed: int, out, mode: int = MVB_GEMM_BF16_6, k_chunk: int = 2048):
    """out[pair, p, q] for all nant^2 pairs (i slow) from z (nant*nfeed, K) complex,
    the reference's layout (cpu/matprod.py:21-30)."""
    import cupy as cp

    M, K = z.shape
    mpad, kcap = -(-M // 128) * 128, -(-K // 64) * 64
    # split planes in the product's stored shared-memory image (layout in matvis_b200.h)
    panel = cp.zeros(lib.mvb_zpanel_bytes(mode, mpad, kcap), dtype=cp.uint8)
    stream = cp.cuda.get_current_stream().ptr
    _check(lib, lib.mvb_z_pack(z.data.ptr, int(z.dtype == cp.complex128), M, K, K, mode, 1.0, panel.data.ptr, mpad,
                               kcap, stream))
    ws = cp.empty(lib.mvb_herk_ws_bytes(mpad, kcap, k_chunk), dtype=cp.uint8)
    status = cp.zeros(1, dtype=cp.int32)
    _check(lib, lib.mvb_herk(panel.data.ptr, mode, mpad, kcap, None, K, 1, k_chunk, 0, ws.data.ptr, ws.size,
                             status.data.ptr, stream))
    _check(lib, lib.mvb_herk_reduce(ws.data.ptr, ws.size, mpad, kcap, None, K, 1, k_chunk, nant, nfeed, None, 0,
                                    out.data.ptr, int(out.dtype == cp.complex128), 1.0, 0, stream))
    if int(status.get()[0]) != 0:
        raise RuntimeError(f"mvb_herk: device status 0x{int(status.get()[0]):x}")
    return out


def set_bcrs(lib, eci, bcrs, astrom: dict):
    """Deflected, aberrated and BPN-rotated source directions (SoA (3, N) float64
    cupy arrays) from one pyerfa ``apco`` parameter dict."""
    import cupy as cp

    a = np.concatenate([astrom["eh"], [astrom["em"], 1e-6], astrom["v"], [astrom["bm1"]],
                        np.ravel(astrom["bpn"])]).astype(np.float64)
    _check(lib, lib.mvb_bcrs(eci.data.ptr, eci.shape[1], a.ctypes.data, bcrs.data.ptr,
                             cp.cuda.get_current_stream().ptr))
