"""The C-ABI library loads and exports every symbol declared in include/*.h
(no compute calls: these run without a GPU)."""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "matvis_b200.h"
LIB = ROOT / "matvis_b200" / "libmatvis_b200.so"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mvb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("mvb_rotate", "mvb_horizon_compact", "mvb_beam_interp", "mvb_tau_z", "mvb_herk", "mvb_herk_reduce",
              "mvb_vecdot"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    if not LIB.exists():
        pytest.fail(f"{LIB} not built (python matvis_b200/build.py)")
    lib = ctypes.CDLL(str(LIB))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    from matvis_b200 import _lib

    missing = [s for s in declared_symbols() if s not in _lib._SIGNATURES]
    assert not missing, missing


def test_workspace_queries_without_gpu():
    from matvis_b200 import _lib

    assert _lib.lib.mvb_version() == 1
    assert _lib.lib.mvb_herk_ws_bytes(768, 393216, 2048) == 21 * (192 + 31) * 256 * 128 * 4 + 256  # up to 31 slices beyond ceil(K / k_chunk), and the unit counter
    assert _lib.lib.mvb_zpanel_bytes(_lib.GEMM_BF16_6, 768, 393216) == 6 * 768 * 393216 * 2
    assert _lib.lib.mvb_horizon_ws_bytes(196608) == 192 * 4
    assert _lib.lib.mvb_vecdot_ws_bytes(10, 2, 4096, 1024) == 4 * 10 * 4 * 2 * 8


def test_argument_errors_are_reported_without_gpu():
    """Argument validation happens on the host, before any CUDA call."""
    from matvis_b200 import _lib

    rc = _lib.lib.mvb_herk(None, 0, 768, 100, None, 0, 1, 64, 0, None, 0, None, None)
    assert rc == _lib.MVB_ERR_ARG
    assert b"mvb_herk" in _lib.lib.mvb_last_error()
    with pytest.raises(ValueError):
        _lib.check(rc)


def _null_call(name, size):
    """Every argument null or ``size``: pointers None, integers size, reals 1.0."""
    import ctypes as ct

    from matvis_b200 import _lib

    args = _lib._SIGNATURES[name][1]
    vals = [1.0 if a in (ct.c_double, ct.c_float) else None if a in (ct.c_void_p, ct.c_char_p) else size for a in args]
    return getattr(_lib.lib, name)(*vals)


def _status_entry_points():
    import ctypes as ct

    from matvis_b200 import _lib

    # mvb_vecdot_stage_columns returns a count, not a status
    return [n for n, (res, _) in _lib._SIGNATURES.items()
            if res is ct.c_int and n not in ("mvb_version", "mvb_device_info", "mvb_vecdot_stage_columns")]


@pytest.mark.parametrize("name", _status_entry_points())
def test_every_entry_point_rejects_null_buffers(name):
    """With non-zero sizes and null buffers every entry point returns
    MVB_ERR_ARG and names itself in mvb_last_error -- on the host, before any
    CUDA call (this runs without a GPU)."""
    from matvis_b200 import _lib

    assert _null_call(name, 1) == _lib.MVB_ERR_ARG
    assert _lib.lib.mvb_last_error().decode().startswith(name + ":")



def _c_to_ctypes(decl: str):
    decl = decl.strip()
    if "*" in decl:
        return "ptr"
    base = decl.replace("const", "").split()[0]
    return {"int": ctypes.c_int, "int64_t": ctypes.c_int64, "size_t": ctypes.c_size_t, "double": ctypes.c_double,
            "float": ctypes.c_float, "int32_t": ctypes.c_int32, "uint64_t": ctypes.c_uint64}[base]


def test_python_binding_matches_header_signatures():
    """Every ctypes signature has the header's argument count and types (a
    mismatch would pass garbage through the boundary without an error)."""
    from matvis_b200 import _lib

    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    decls = re.findall(r"^\s*([a-z_0-9 ]+?\**)\s*\b(mvb_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text, flags=re.M | re.S)
    assert len(decls) == len(declared_symbols())
    for ret, name, args in decls:
        res, argtypes = _lib._SIGNATURES[name]
        params = [] if args.strip() in ("", "void") else [a for a in args.split(",")]
        assert len(params) == len(argtypes), name
        for i, (p, t) in enumerate(zip(params, argtypes)):
            want = _c_to_ctypes(p)
            if want == "ptr":
                assert t in (ctypes.c_void_p, ctypes.c_char_p), (name, i, p)
            else:
                assert t is want, (name, i, p, t)
        want_ret = "ptr" if "*" in ret else _c_to_ctypes(ret)
        assert (res in (ctypes.c_void_p, ctypes.c_char_p)) if want_ret == "ptr" else res is want_ret, name


def test_reference_side_binding_matches_library():
    """The reference-side ctypes binding (include/matvis_gpu_b200.py, the module a
    maintainer adds to matvis) declares the library's own signatures, and loads
    the built library."""
    import importlib.util

    from matvis_b200 import _lib

    spec = importlib.util.spec_from_file_location("matvis_gpu_b200", ROOT / "include" / "matvis_gpu_b200.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert len(mod.SIGNATURES) >= 5
    for name, (res, args) in mod.SIGNATURES.items():
        assert (res, list(args)) == (_lib._SIGNATURES[name][0], list(_lib._SIGNATURES[name][1])), name
    lib = mod.load(str(LIB))
    assert lib.mvb_herk_ws_bytes(768, 4096, 2048) == _lib.lib.mvb_herk_ws_bytes(768, 4096, 2048)


def test_herk_reduce_applies_the_products_checks_without_gpu():
    """mvb_herk_reduce rejects, on the host, arguments the product would reject and
    a workspace smaller than the product's (nothing is read from the pointers)."""
    from matvis_b200 import _lib

    ws_need = _lib.lib.mvb_herk_ws_bytes(768, 4096, 2048)
    fake = ctypes.c_void_p(256)  # never dereferenced: every call below fails its checks first
    args = dict(ws=fake, ws_bytes=ws_need, Mpad=768, Kcap=4096, n_dev=None, n_host=2048, kmul=2, k_chunk=2048,
                nant=350, nfeed=2, pairs=None, npairs=0, out=fake, c128=0, vscale=1.0, acc=0, stream=None)
    for bad in (dict(ws_bytes=ws_need - 1), dict(k_chunk=2000), dict(Kcap=4000), dict(n_host=2049),
                dict(Mpad=700), dict(nfeed=3), dict(nant=385)):
        a = {**args, **bad}
        rc = _lib.lib.mvb_herk_reduce(*a.values())
        assert rc == _lib.MVB_ERR_ARG, bad
        assert _lib.lib.mvb_last_error().startswith(b"mvb_herk_reduce:")


def test_set_wait_limit_round_trip_without_gpu():
    from matvis_b200 import _lib

    prev = _lib.lib.mvb_set_wait_limit_ns(123)
    assert prev == 4_000_000_000
    assert _lib.lib.mvb_set_wait_limit_ns(0) == 123
    assert _lib.lib.mvb_set_wait_limit_ns(0) == prev


def test_pair_lists_are_range_checked_on_the_host():
    """A pair naming an antenna outside [0, nant) is refused before any device
    work (the reference's gather raises IndexError, cpu/matprod.py:29-30)."""
    import numpy as np

    from matvis_b200.matprod import AntpairsOutOfRange, B200MatMul, B200VectorDot

    for cls in (B200MatMul, B200VectorDot):
        for bad in ([[0, 3]], [[-1, 0]], [[2, 7], [0, 1]]):
            with pytest.raises(IndexError):
                cls(1, 2, 3, np.array(bad))
            with pytest.raises(ValueError):
                cls(1, 2, 3, np.array(bad))
    with pytest.raises(AntpairsOutOfRange):
        B200MatMul(1, 1, 3, np.array([[0, 3]]))
    with pytest.raises(ValueError, match="shape"):
        B200MatMul(1, 1, 3, np.array([[0, 1, 2]]))


def test_herk_group_struct_layout():
    """The ctypes mirror of mvb_herk_group has the C layout (x86-64 alignment):
    pointers and 64-bit fields on 8-byte boundaries, 88 bytes in all."""
    from matvis_b200 import _lib

    G = _lib.HerkGroup
    assert ctypes.sizeof(G) == 88
    assert [getattr(G, f).offset for f in ("z", "z_stride", "ngroup", "Mpad", "Kcap", "n_dev", "n_host", "kmul",
                                            "k_chunk", "ws", "ws_bytes", "status")] == [0, 8, 16, 24, 32, 40, 48, 56,
                                                                                         60, 64, 72, 80]
    text = HEADER.read_text()
    assert "} mvb_herk_group;" in text


def test_herk_batch_checks_without_gpu():
    """Every group is checked as mvb_herk_grouped checks it, and the panel total is
    bounded, before any CUDA call."""
    from matvis_b200 import _lib

    fake = 256
    need = _lib.lib.mvb_herk_ws_bytes(768, 4096, 2048)
    g = _lib.HerkGroup(z=fake, z_stride=0, ngroup=1, Mpad=768, Kcap=4096, n_dev=None, n_host=2048, kmul=2,
                       k_chunk=2048, ws=fake, ws_bytes=need - 16, status=fake)
    arr = (_lib.HerkGroup * 1)(g)
    assert _lib.lib.mvb_herk_batch(ctypes.cast(arr, ctypes.c_void_p), 1, _lib.GEMM_F16_3, 0, None) == _lib.MVB_ERR_ARG
    assert b"workspace" in _lib.lib.mvb_last_error()
    g.ws_bytes = 40 * need
    g.ngroup, g.z_stride = 33, _lib.lib.mvb_zpanel_bytes(_lib.GEMM_F16_3, 768, 4096)
    arr = (_lib.HerkGroup * 1)(g)
    assert _lib.lib.mvb_herk_batch(ctypes.cast(arr, ctypes.c_void_p), 1, _lib.GEMM_F16_3, 0, None) == _lib.MVB_ERR_ARG
    assert b"32 panels" in _lib.lib.mvb_last_error()
