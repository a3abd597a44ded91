"""ctypes binding of ``libmatvis_b200.so`` (the C ABI declared in include/matvis_b200.h).

The library is the only compute path: importing this module without the built
library raises ``ImportError`` (build it with ``python matvis_b200/build.py``).
Device buffers are torch tensors; only their raw pointers cross the boundary.
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_float, c_int, c_int64, c_size_t, c_void_p
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libmatvis_b200.so"

MVB_OK = 0
MVB_ERR_ARG = 1
MVB_ERR_CUDA = 2
MVB_ERR_OVERFLOW = 3
MVB_ERR_NONFINITE = 4
MVB_ERR_TIMEOUT = 5
MVB_ERR_UNSUPPORTED = 6

MVB_DEV_OVERFLOW = 0x1
MVB_DEV_TIMEOUT = 0x2
MVB_DEV_NONFINITE = 0x4

GEMM_BF16_3 = 0
GEMM_BF16_6 = 1
GEMM_TF32_3 = 2
Z_C64 = 3
GEMM_F16_3 = 4

GEMM_MODES = {"bf16x3": GEMM_BF16_3, "bf16x6": GEMM_BF16_6, "tf32x3": GEMM_TF32_3, "fp16x3": GEMM_F16_3}
#: tensor-core products per complex multiply-accumulate term, per mode
GEMM_PRODUCTS = {GEMM_BF16_3: 3, GEMM_BF16_6: 6, GEMM_TF32_3: 3, GEMM_F16_3: 3}

K_ALIGN = 64
TILE = 128

_p = c_void_p
_SIGNATURES = {
    "mvb_version": (c_int, []),
    "mvb_last_error": (ctypes.c_char_p, []),
    "mvb_device_info": (c_int, [_p, _p, _p]),
    "mvb_rotate": (c_int, [_p, c_int64, _p, _p, _p]),
    "mvb_bcrs": (c_int, [_p, c_int64, _p, _p, _p]),
    "mvb_redundant_pairs": (c_int, [_p, c_int64, c_int, _p, c_int64, _p]),
    "mvb_flux_sqrt_half": (c_int, [_p, c_int64, c_int, _p, _p]),
    "mvb_coherency_rotation": (c_int, [_p, c_int64, _p, _p, c_int64, _p, c_int64, _p, _p, _p]),
    "mvb_rotate_coherency": (c_int, [_p, _p, _p, _p, c_int64, c_int, _p, c_int64, _p]),
    "mvb_tau_z_pol": (c_int, [_p, c_int, ctypes.c_double, _p, c_int64, _p, c_int64, _p, _p, _p, _p, c_int64, c_int,
                              _p, c_int, ctypes.c_float, _p, c_int64, c_int64, _p]),
    "mvb_horizon_ws_bytes": (c_size_t, [c_int64]),
    "mvb_horizon_compact": (
        c_int,
        [_p, c_int64, c_int64, c_int64, _p, _p, _p, _p, _p, c_int64, _p, _p, c_size_t, _p],
    ),
    "mvb_horizon_compact_static": (
        c_int,
        [_p, c_int64, c_int64, c_int64, _p, _p, _p, _p, _p, c_int64, _p, _p],
    ),
    "mvb_beam_interp": (
        c_int,
        [_p, c_int, c_int, c_int, c_int, c_int, c_int, _p, _p, c_int64, _p, c_int64, _p, c_int, c_int64, _p, _p,
         c_size_t, _p],
    ),
    "mvb_beam_interp_ws_bytes": (c_size_t, [c_int, c_int64]),
    "mvb_beam_interp_azza": (
        c_int, [_p, c_int, c_int, c_int, c_int, c_int, c_int, _p, _p, c_int64, c_int64, _p, c_int, _p]
    ),
    "mvb_beam_gaussian": (c_int, [_p, c_int, _p, c_int64, _p, c_int64, _p, c_int, c_int64, _p]),
    "mvb_exptau": (c_int, [_p, c_int, c_double, _p, c_int64, c_int64, _p, c_int, _p]),
    "mvb_zpanel_bytes": (c_size_t, [c_int, c_int64, c_int64]),
    "mvb_tau_z": (
        c_int,
        [_p, c_int, c_double, _p, c_int64, _p, c_int64, _p, _p, _p, c_int64, c_int, _p, c_int, c_int, c_int, c_float,
         _p, c_int64, c_int64, _p],
    ),
    "mvb_z_from_exptau": (
        c_int,
        [_p, c_int, c_int64, c_int, c_int64, _p, _p, c_int64, c_int, _p, c_int, c_int, c_int, c_float, _p, c_int64,
         c_int64, _p],
    ),
    "mvb_z_pack": (c_int, [_p, c_int, c_int64, c_int64, c_int64, c_int, c_float, _p, c_int64, c_int64, _p]),
    "mvb_absmax": (c_int, [_p, c_int, c_int64, _p, _p]),
    "mvb_herk_ws_bytes": (c_size_t, [c_int64, c_int64, c_int]),
    "mvb_herk": (c_int, [_p, c_int, c_int64, c_int64, _p, c_int64, c_int, c_int, c_int, _p, c_size_t, _p, _p]),
    "mvb_herk_reduce": (
        c_int,
        [_p, c_size_t, c_int64, c_int64, _p, c_int64, c_int, c_int, c_int, c_int, _p, c_int64, _p, c_int, c_double,
         c_int, _p],
    ),
    "mvb_set_wait_limit_ns": (ctypes.c_uint64, [ctypes.c_uint64]),
    "mvb_herk_grouped": (c_int, [_p, c_size_t, c_int, c_int, c_int64, c_int64, _p, c_int64, c_int, c_int, c_int, _p,
                                 c_size_t, _p, _p]),
    "mvb_herk_batch": (c_int, [_p, c_int, c_int, c_int, _p]),
    "mvb_herk_reduce_grouped": (
        c_int,
        [_p, c_size_t, c_int, c_int64, c_int64, _p, c_int64, c_int, c_int, c_int, c_int, _p, c_int64, _p, c_size_t,
         c_int, c_double, c_int, _p],
    ),
    "mvb_tau_z_grouped": (
        c_int,
        [_p, c_int, _p, c_int, _p, c_int64, _p, c_int64, _p, c_int64, _p, _p, c_int64, c_int, _p, c_int, c_int, c_int,
         c_float, _p, c_size_t, c_int64, c_int64, _p],
    ),
    "mvb_tau_z_pol_grouped": (
        c_int,
        [_p, c_int, _p, c_int, _p, c_int64, _p, c_int64, _p, c_int64, _p, _p, _p, c_int64, c_int, _p, c_int, c_float,
         _p, c_size_t, c_int64, c_int64, _p],
    ),
    "mvb_chunk_sum": (c_int, [_p, c_int64, c_int64, c_int, _p, _p]),
    "mvb_vecdot_ws_bytes": (c_size_t, [c_int64, c_int, c_int64, c_int]),
    "mvb_vecdot": (
        c_int,
        [_p, c_int64, _p, c_int64, c_int, c_int, _p, c_int64, c_int, _p, c_size_t, _p, c_int, c_int, _p],
    ),
    "mvb_vecdot_plan_bytes": (c_size_t, [c_int64, c_int]),
    "mvb_vecdot_plan": (c_int, [_p, c_int64, c_int, c_int, _p, c_size_t, _p]),
    "mvb_vecdot_stage_columns": (c_int, [c_int, c_int]),
    "mvb_vecdot_staged_ws_bytes": (c_size_t, [c_int64, c_int, c_int64, c_int]),
    "mvb_vecdot_staged": (
        c_int,
        [_p, c_int64, _p, c_int64, c_int, c_int, c_int, _p, c_int64, c_int64, c_int, _p, c_size_t, _p, c_int, c_int,
         _p, _p],
    ),
}


class HerkGroup(ctypes.Structure):
    """``mvb_herk_group`` of the C header: one panel group of mvb_herk_batch."""

    _fields_ = [("z", c_void_p), ("z_stride", c_size_t), ("ngroup", c_int), ("Mpad", c_int64), ("Kcap", c_int64),
                ("n_dev", c_void_p), ("n_host", c_int64), ("kmul", c_int), ("k_chunk", c_int), ("ws", c_void_p),
                ("ws_bytes", c_size_t), ("status", c_void_p)]


#: panels one mvb_herk_batch launch can hold
MAX_BATCH_PANELS = 32


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH.name} is not built; run `python matvis_b200/build.py` (needs nvcc). "
            "matvis_b200 has no CPU fallback."
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class MatvisB200Error(RuntimeError):
    """A non-OK status from the CUDA library."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[mvb status {code}] {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != MVB_OK:
        msg = (lib.mvb_last_error() or b"").decode(errors="replace")
        if rc == MVB_ERR_ARG:
            raise ValueError(msg)
        raise MatvisB200Error(rc, msg)


def ptr(t: torch.Tensor | None) -> c_void_p:
    """Raw device pointer of a tensor (None -> NULL)."""
    if t is None:
        return c_void_p(0)
    return c_void_p(t.data_ptr())


def stream_handle(stream: torch.cuda.Stream | None = None) -> c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("matvis_b200 needs a CUDA device (B200, sm_100a); none is visible")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if dev.type != "cuda":
        raise ValueError(f"matvis_b200 runs on CUDA devices only, got {dev}")
    return dev


def check_status_word(status: torch.Tensor, where: str) -> None:
    """Raise if a kernel OR-ed a failure bit into the device status word."""
    v = int(status.item())
    if v == 0:
        return
    if v & MVB_DEV_OVERFLOW:
        raise ValueError(f"{where}: more sources above the horizon than the allocated capacity (nsrc_alloc); "
                         "increase source_buffer")
    if v & MVB_DEV_NONFINITE:
        raise ValueError("Beam interpolation resulted in an invalid value")
    if v & MVB_DEV_TIMEOUT:
        raise MatvisB200Error(MVB_ERR_TIMEOUT, f"{where}: a bounded device wait ran out")
    raise MatvisB200Error(MVB_ERR_CUDA, f"{where}: device status 0x{v:x}")


def zpanel_shape(mode: int, M: int, K: int) -> tuple[int, int]:
    """(Mpad, Kcap) for a panel holding M rows and up to K columns."""
    mpad = -(-M // TILE) * TILE if mode != Z_C64 else M
    kcap = max(K_ALIGN, -(-K // K_ALIGN) * K_ALIGN)
    return mpad, kcap


def zpanel_dtype(mode: int) -> torch.dtype:
    return {GEMM_BF16_3: torch.bfloat16, GEMM_BF16_6: torch.bfloat16, GEMM_TF32_3: torch.float32,
            GEMM_F16_3: torch.float16, Z_C64: torch.complex64}[mode]


def zpanel_kblock(mode: int) -> int:
    """Elements per 64-byte k-block of a split-plane panel (stored
    [Kcap / KB][Mpad / 128][planes][128][KB], 16-byte chunks swizzled per row)."""
    return 64 // torch.empty((), dtype=zpanel_dtype(mode)).element_size()


def zpanel_planes(mode: int) -> int:
    return {GEMM_BF16_3: 4, GEMM_BF16_6: 6, GEMM_TF32_3: 4, GEMM_F16_3: 4, Z_C64: 1}[mode]


def f16_scale(maxabs: float) -> float:
    """Power-of-two scale s with max |s Z| < 2^15 (fp16 range), for the fp16x3 panel."""
    import math

    if not maxabs > 0 or not math.isfinite(maxabs):
        return 1.0
    e = math.floor(math.log2(2.0**14 / maxabs))
    return float(2.0 ** max(min(e, 100), -100))
