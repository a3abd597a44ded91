"""Host-side logic that needs no GPU: chunk planning, sharding (2 gloo ranks),
synthetic generators, parameter plumbing."""

import os
import socket

import numpy as np
import pytest

from matvis_b200 import _utils, sharding, workloads
from matvis_b200.engine import JobSpec, _norm_matprod, _resolve_product
from matvis_b200.matprod import choose_k_chunk, pair_product
from oracle import oracle as orc

from .conftest import golden


def test_chunk_planning_matches_reference_table():
    for row in golden("chunks")["table"]:
        fm, nax, nfeed, nant, nsrc, nbeam, npix, prec, sb, mb, ch = row
        got = _utils.get_required_chunks(fm, int(nax), int(nfeed), int(nant), int(nsrc), int(nbeam), int(npix),
                                         int(prec), sb, mb)
        assert got == int(ch)
    with pytest.raises(ValueError):
        _utils.get_required_chunks(1, 1, 1, 1, 1, 1, 1, 1, 1.0, 0.0)



_CHUNK_KW = dict(freemem=10 * 1024**3, nax=2, nfeed=2, nant=4, nsrc=100, nbeam=2, nbeampix=0, precision=1)


def test_required_chunks_properties():
    """The properties the reference's own utils tests check (tests/test_utils.py:38-82)."""
    assert _utils.get_required_chunks(**_CHUNK_KW) >= 1
    assert _utils.get_required_chunks(**_CHUNK_KW, memory_buffer=0.1) >= \
        _utils.get_required_chunks(**_CHUNK_KW, memory_buffer=0.9)
    assert _utils.get_required_chunks(**{**_CHUNK_KW, "freemem": 10**18}, memory_buffer=1.0) == 1
    assert _utils.get_required_chunks(**_CHUNK_KW, memory_buffer=1.0) >= 1
    for bad in (1.1, 0.0, -0.5):
        with pytest.raises(ValueError, match="memory_buffer"):
            _utils.get_required_chunks(**_CHUNK_KW, memory_buffer=bad)
    # less memory never needs fewer chunks; the count stops at 100
    counts = [_utils.get_required_chunks(**{**_CHUNK_KW, "nsrc": 10**6, "freemem": fm}) for fm in
              (2**34, 2**30, 2**28, 2**26, 2**20)]
    assert counts == sorted(counts) and counts[-1] == 100

def test_desired_chunks_counts_grid_pixels():
    beams = workloads.dipole_beams(np.random.default_rng(0), 2, dgrid_deg=10.0)
    n, per = _utils.get_desired_chunks(2**40, 3, beams, 2, 2, 10, 1000, 1)
    assert n == 3 and per == 334


def test_get_dtypes():
    assert _utils.get_dtypes(1) == (np.float32, np.complex64)
    assert _utils.get_dtypes(2) == (np.float64, np.complex128)


def test_matprod_names():
    for n in ("MatMul", "CPUMatMul", "GPUMatMul", "B200MatMul"):
        assert _norm_matprod(n) == "MatMul"
    for n in ("VectorDot", "VectorLoop", "GPUVectorLoop", "CPUVectorDot"):
        assert _norm_matprod(n) == "VectorDot"
    with pytest.raises(ValueError):
        _norm_matprod("Einsum")


def test_pair_product_cost_model():
    """Measured break-even of the staged per-pair kernel against the Hermitian
    product with a pair gather: ~5,750 pairs for 350 two-feed antennas (21
    tiles); ~2,750 for arrays too large to stage (the warp kernel)."""
    assert pair_product(350, 2, 5000) == "vecdot"
    assert pair_product(350, 2, 7000) == "herk"
    assert pair_product(350, 2, 10649) == "herk"  # the redundant-baseline list of the 350-antenna array
    assert pair_product(350, 2, 350 * 351 // 2) == "herk"
    assert pair_product(37, 1, 63) == "vecdot"  # redundant-baseline representatives of a 37-element hexagon
    # TF32 operands and six split products double the product's cost
    assert pair_product(350, 2, 10000, "tf32x3") == "vecdot"
    assert pair_product(350, 2, 10000, "bf16x6") == "vecdot"
    assert pair_product(350, 2, 12000, "bf16x6") == "herk"
    # 4,000 two-feed antennas do not fit the stages: 2,016 tiles against the warp kernel (~264,000 pairs)
    assert pair_product(4000, 2, 200000) == "vecdot"
    assert pair_product(4000, 2, 300000) == "herk"


def test_resolve_product():
    def spec(**kw):
        base = dict(antpos=np.zeros((350, 3)), eci=np.zeros((3, 1)), fluxes=np.ones((1, 1)), freqs=np.ones(1),
                    lsts=np.zeros(1), latitude=0.0, beams=[], polarized=True)
        return JobSpec(**{**base, **kw})

    pairs = np.stack(np.triu_indices(350, 1), axis=1)
    assert _resolve_product(spec()) == ("MatMul", None)
    assert _resolve_product(spec(matprod="VectorDot", antpairs=pairs[:8000])) == ("MatMul", "herk")
    assert _resolve_product(spec(matprod="VectorDot", antpairs=pairs[:500])) == ("VectorDot", "vecdot")
    assert _resolve_product(spec(matprod="VectorDot", antpairs=pairs[:8000], pair_product="vecdot")) == \
        ("VectorDot", "vecdot")
    assert _resolve_product(spec(matprod="VectorDot", antpairs=pairs[:50], pair_product="herk")) == \
        ("MatMul", "herk")
    assert _resolve_product(spec(matprod="VectorDot")) == ("MatMul", "herk")  # all 350^2 pairs
    with pytest.raises(ValueError):
        _resolve_product(spec(matprod="VectorDot", pair_product="dense"))



def _plan_spec(nf=24, nsrc=200_000, nant=64, polarized=True, pol_sky=False):
    fl = np.ones((nsrc, nf, 2, 2)) if pol_sky else np.ones((nsrc, nf))
    return JobSpec(antpos=np.zeros((nant, 3)), eci=np.zeros((3, nsrc)), fluxes=fl, freqs=np.linspace(1e8, 2e8, nf),
                   lsts=np.zeros(6), latitude=0.0, beams=[], polarized=polarized)


@pytest.mark.parametrize("pol_sky", [False, True])
def test_plan_job_frequency_batches(pol_sky):
    """A job over the memory budget runs as the fewest equal frequency batches that fit."""
    from dataclasses import replace

    from matvis_b200.engine import estimate_device_bytes, plan_job

    spec = _plan_spec(pol_sky=pol_sky)
    full = estimate_device_bytes(spec)
    assert plan_job(spec, np.inf) == (24, 1)
    assert plan_job(spec, full) == (24, 1)

    def size(nfb, ch=1):
        return estimate_device_bytes(replace(spec, freqs=spec.freqs[:nfb], fluxes=spec.fluxes[:, :nfb], nchunks=ch))

    for frac in (0.999, 0.4, 0.1, 0.0):
        budget = size(1) + frac * (full - size(1))
        nfb, ch = plan_job(spec, budget)
        nbatch = -(-24 // nfb)
        assert ch == 1 and nfb < 24 and size(nfb) <= budget
        assert nfb == -(-24 // nbatch)  # batches as equal as the count allows
        assert size(-(-24 // (nbatch - 1))) > budget  # one batch fewer would not fit


def test_plan_job_source_chunks():
    """When one frequency alone does not fit, the sources are split into more chunks."""
    from dataclasses import replace

    from matvis_b200.engine import estimate_device_bytes, plan_job

    spec = _plan_spec(nf=3)
    one = replace(spec, freqs=spec.freqs[:1], fluxes=spec.fluxes[:, :1])
    budget = estimate_device_bytes(replace(one, nchunks=4))
    nfb, ch = plan_job(spec, budget)
    assert nfb == 1 and 1 < ch <= 4
    assert estimate_device_bytes(replace(one, nchunks=ch)) <= budget
    assert estimate_device_bytes(replace(one, nchunks=ch - 1)) > budget
    assert plan_job(spec, 1.0) == (1, 100)  # past the cap the plan stands and allocation reports it
    assert plan_job(_plan_spec(nf=3, nsrc=10), 1.0) == (1, 10)  # no more chunks than sources
    assert plan_job(replace(spec, nchunks=7), np.inf) == (3, 7)


def test_simulate_vis_keywords():
    """Reference keywords are accepted; an unknown keyword is a TypeError, as in the reference."""
    import inspect

    from matvis_b200.wrapper import simulate_vis

    params = inspect.signature(simulate_vis).parameters
    for name in ("max_memory", "memory_buffer", "min_chunks", "source_buffer", "beam_spline_opts", "coord_method",
                 "coord_method_params", "matprod_method"):
        assert name in params, name
    with pytest.raises(TypeError, match="bogus"):
        simulate_vis({0: (0, 0, 0)}, np.ones((1, 1)), np.zeros(1), np.zeros(1), np.ones(1), np.zeros(1), [], 0.0,
                     bogus=1)
    with pytest.raises(ValueError, match="memory_buffer"):
        simulate_vis({0: (0, 0, 0)}, np.ones((1, 1)), np.zeros(1), np.zeros(1), np.ones(1), np.zeros(1), [], 0.0,
                     memory_buffer=1.5)

@pytest.mark.parametrize("n", [1_000_000, 300_001, 131_072, 5])
def test_point_source_crd_eq_threads_bit_identical(n):
    """The threaded unit vectors equal the single numpy pass bit for bit (the
    horizon selection downstream is bit-exact against the oracle)."""
    from matvis_b200.coordinates import point_source_crd_eq

    rng = np.random.default_rng(n)
    ra, dec = rng.uniform(0, 2 * np.pi, n), np.arcsin(rng.uniform(-1, 1, n))
    one = np.asarray([np.cos(ra) * np.cos(dec), np.cos(dec) * np.sin(ra), np.sin(dec)])
    np.testing.assert_array_equal(point_source_crd_eq(ra, dec), one)
    np.testing.assert_array_equal(point_source_crd_eq(ra.reshape(-1, 1), dec.reshape(-1, 1)), one[:, :, None])


@pytest.mark.parametrize("mode", ["fp16x3", "bf16x6", "tf32x3"])
def test_panel_layout_round_trip(mode):
    """Z written element by element at the documented panel offsets (the
    product's swizzled shared-memory image) reads back through ZPanel.to_complex."""
    import torch

    from matvis_b200 import _lib
    from matvis_b200.getz import ZPanel

    m_, nax, nsrc = 200, 2, 150
    md = _lib.GEMM_MODES[mode]
    mpad, kcap = _lib.zpanel_shape(md, m_, nax * nsrc)
    kb, npl = _lib.zpanel_kblock(md), _lib.zpanel_planes(md)
    rng = np.random.default_rng(1)
    z = (rng.integers(-8, 8, (m_, nax * nsrc)) + 1j * rng.integers(-8, 8, (m_, nax * nsrc))).astype(np.complex128)
    flat = np.zeros(npl * mpad * kcap)
    e = kb // 4
    for m in range(m_):
        for k in range(nax * nsrc):
            c, r = k % kb, m % 128
            base = ((k // kb) * (mpad // 128) + m // 128) * npl * 128 * kb + r * kb + ((c // e) ^ ((r // 2) % 4)) * e + c % e
            flat[base] = z[m, k].real  # split term 0 carries the value, the others stay 0
            flat[base + 128 * kb] = z[m, k].imag
    panel = ZPanel.__new__(ZPanel)
    panel.mode, panel.M, panel.nax, panel.n_host, panel.n_dev, panel.scale = md, m_, nax, nsrc, None, 1.0
    panel.data = torch.as_tensor(flat.reshape(kcap // kb, mpad // 128, npl, 128, kb))
    np.testing.assert_array_equal(panel.to_complex().numpy(), z)


@pytest.mark.parametrize("n,nf", [(70001, 3), (5, 2), (0, 4)])
def test_repack_coherency(n, nf):
    """The threaded coherency repack equals the single-pass expressions exactly."""
    from matvis_b200.engine import _repack_coherency

    rng = np.random.default_rng(n)
    c = rng.normal(size=(n, nf, 2, 2)) + 1j * rng.normal(size=(n, nf, 2, 2))
    coh, trace = _repack_coherency(c)
    ref = np.stack([c[..., 0, 0].real, c[..., 1, 1].real, c[..., 0, 1].real, c[..., 0, 1].imag],
                   axis=-1).transpose(1, 0, 2).astype(np.float32)
    np.testing.assert_array_equal(coh, ref)
    np.testing.assert_array_equal(trace, np.maximum(c[..., 0, 0].real + c[..., 1, 1].real, 0.0))


def test_engine_interface():
    """The engine's public methods (the served form, simulate and bench call them)."""
    from matvis_b200.engine import VisEngine

    for name in ("allocate", "upload", "h2d_bytes", "enqueue", "enqueue_time", "run", "run_to_host", "capture",
                 "result", "device_bytes", "launches_per_run"):
        assert callable(getattr(VisEngine, name, None)), name


def test_choose_k_chunk():
    kc = choose_k_chunk(21, 196608, 148)
    assert kc % 64 == 0 and 1024 <= kc <= 8192
    assert choose_k_chunk(1, 100, 148) == 1024


def test_healpix_centres_equal_area():
    ra, dec = workloads.healpix_ring_centres(16)
    assert len(ra) == 12 * 16 * 16
    z = np.sin(dec)
    assert abs(z.mean()) < 1e-12  # symmetric about the equator
    # every ring of the equatorial belt has 4 nside pixels
    assert np.sum(np.isclose(z, 0.0)) == 4 * 16


def test_hex_array_spacing():
    a = workloads.hex_array(320, 14.6)
    assert a.shape == (320, 3)
    d = np.linalg.norm(a[:, None, :2] - a[None, :, :2], axis=-1)
    d[np.diag_indices(320)] = np.inf
    assert np.isclose(d.min(), 14.6)
    assert len(np.unique(np.round(a, 6), axis=0)) == 320


def test_powerlaw_flux_bounds():
    s = workloads.powerlaw_flux(np.random.default_rng(0), 100000)
    assert s.min() >= 0.05 and s.max() <= 100.0
    # N(>S) ~ S^-1.5: the fraction above 1 Jy
    frac = np.mean(s > 1.0)
    expect = (1.0**-1.5 - 100**-1.5) / (0.05**-1.5 - 100**-1.5)
    assert abs(frac - expect) < 0.01


def test_frequency_shards_cover_once():
    for nf in (1, 7, 64, 256):
        for w in (1, 2, 3, 8):
            sh = sharding.frequency_shards(nf, w)
            got = [f for a, b in sh for f in range(a, b)]
            assert got == list(range(nf))
            sizes = [b - a for a, b in sh]
            assert max(sizes) - min(sizes) <= 1


def test_cosine_metric_detects_error():
    rng = np.random.default_rng(0)
    z = rng.normal(size=(6, 50)) + 1j * rng.normal(size=(6, 50))
    v = orc.matmul_vis(z, 3, 2)
    assert orc.cosine_error_metric(v, v, 2) == 0
    w = v.copy()
    w[1, 0, 1] += 1e-3
    assert orc.cosine_error_metric(w, v, 2) > 1e-5


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _gather_worker(rank, world, port, nfreq, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        f0, f1 = sharding.frequency_shards(nfreq, world)[rank]
        # stand-in for the per-rank visibilities: each frequency slice filled with its index
        local = np.arange(f0, f1, dtype=np.float64)[:, None, None] * np.ones((1, 3, 4))
        out = sharding.gather_frequency_shards(local, rank, world, nfreq)
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nfreq", [5, 64])
def test_gather_two_gloo_ranks(nfreq):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, nfreq, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out.shape == (nfreq, 3, 4)
    np.testing.assert_array_equal(out[:, 0, 0], np.arange(nfreq))


def test_shard_spec_slices_fluxes():
    spec = JobSpec(antpos=np.zeros((2, 3)), eci=np.zeros((3, 4)), fluxes=np.arange(20.0).reshape(4, 5),
                   freqs=np.arange(5.0), lsts=np.zeros(1), latitude=0.0, beams=[])
    s1, (f0, f1) = sharding.shard_spec(spec, 1, 2)
    assert (f0, f1) == (3, 5)
    np.testing.assert_array_equal(s1.fluxes, spec.fluxes[:, 3:5])
    np.testing.assert_array_equal(s1.freqs, [3.0, 4.0])


def _golden_astrom(t):
    g = golden("erfa")
    return {k: (g[f"t{t}_{k}"] if g[f"t{t}_{k}"].ndim else float(g[f"t{t}_{k}"]))
            for k in ("eh", "em", "v", "bm1", "bpn", "eral", "xpl", "ypl", "sphi", "cphi")}


def test_atioq_matrix_reproduces_reference_topocentric():
    """The host 3x3 of the ERFA-style rotation against the reference's _atioq output."""
    from matvis_b200.coordinates import atioq_matrix

    g = golden("erfa")
    for t in range(3):
        a = _golden_astrom(t)
        np.testing.assert_allclose(atioq_matrix(a) @ g[f"t{t}_bcrs"], g[f"t{t}_topo"], rtol=0, atol=2e-15)


def test_pack_astrom_layout():
    from matvis_b200.coordinates import pack_astrom

    a = _golden_astrom(1)
    p = pack_astrom(a)
    assert p.shape == (18,) and p.dtype == np.float64 and p.flags["C_CONTIGUOUS"]
    np.testing.assert_array_equal(p[0:3], a["eh"])
    assert p[3] == a["em"] and p[4] == 1e-6 and p[8] == a["bm1"]
    np.testing.assert_array_equal(p[5:8], a["v"])
    np.testing.assert_array_equal(p[9:18], np.asarray(a["bpn"]).reshape(9))


def test_bcrs_refresh_plan_follows_update_interval():
    from matvis_b200.coordinates import bcrs_refresh_plan

    ts = np.array([0.0, 60.0, 120.0, 181.0, 240.0, 400.0])
    assert bcrs_refresh_plan(ts, 0.0) == [True] * 6
    # refresh strictly after 180 s since the last refresh
    assert bcrs_refresh_plan(ts, 180.0) == [True, False, False, True, False, True]
    assert bcrs_refresh_plan(ts, 1e9) == [True] + [False] * 5


def test_coord_method_keywords():
    from matvis_b200.wrapper import _check_coord_method

    assert _check_coord_method("CoordinateRotationLST") == {}
    with pytest.raises(NotImplementedError):
        _check_coord_method("CoordinateRotationAstropy")
    with pytest.raises(ValueError):
        _check_coord_method("CoordinateRotationERFA", {})
    with pytest.raises(ValueError):
        _check_coord_method("Nope")
    kw = _check_coord_method("GPUCoordinateRotationERFA", {"astrom": [{}], "time_s": [0.0], "update_bcrs_every": 5})
    assert kw["update_bcrs_every"] == 5.0 and kw["time_s"] == [0.0] and len(kw["astrom"]) == 1


def test_oracle_erfa_refresh_reuses_directions():
    """With a long update interval the oracle's ERFA path rotates the first
    time's apparent directions at every later time (cpu/coords.py:194-199)."""
    g = golden("erfa")
    eci = g["eci"]
    astrom = [_golden_astrom(t) for t in range(3)]
    b0 = orc.erfa_bcrs(eci, astrom[0])
    for t in range(3):
        topo = orc.rotate_fixed_order(orc.erfa_atioq_matrix(astrom[t]), b0)
        np.testing.assert_allclose(topo, orc.erfa_atioq_matrix(astrom[t]) @ b0, rtol=0, atol=4e-16)


@pytest.mark.parametrize("layout", ["hex37", "hex127_jitter", "hera350", "random40", "colocated", "line_half", "two",
                                    "one"])
@pytest.mark.parametrize("nd", [2, 0, -1])
def test_redundant_pairs_match_reference(layout, nd):
    """mvb_redundant_pairs against the reference's get_redundancies (cli.py:273-290)."""
    from matvis_b200.pairs import baselines, get_redundancies

    g = golden("redundancies")
    got = np.asarray(get_redundancies(baselines(g[f"{layout}_pos"]), ndecimals=nd), dtype=np.int64).reshape(-1, 2)
    np.testing.assert_array_equal(got, g[f"{layout}_nd{nd}"])


def test_redundant_pairs_errors_and_capacity():
    import ctypes

    from matvis_b200 import _lib
    from matvis_b200.pairs import get_redundancies

    with pytest.raises(ValueError):
        get_redundancies(np.zeros((3, 2, 2)))
    bls = np.zeros((3, 3, 2))
    bls[0, 1] = (1.0, 0.0)
    bls[0, 2] = (0.0, 1.0)
    bls[1, 2] = (np.nan, 0.0)
    with pytest.raises(ValueError):
        get_redundancies(bls)
    bls[1, 2] = (-1.0, 1.0)
    assert get_redundancies(bls) == [[0, 1], [0, 2], [1, 2]]
    out = np.zeros((1, 2), dtype=np.int32)
    n = ctypes.c_int64(0)
    rc = _lib.lib.mvb_redundant_pairs(bls.ctypes.data_as(ctypes.c_void_p), 3, 2, out.ctypes.data_as(ctypes.c_void_p),
                                      1, ctypes.byref(n))
    assert rc == _lib.MVB_ERR_OVERFLOW and n.value == 3 and out.tolist() == [[0, 1]]
    assert get_redundancies(np.zeros((0, 0, 2))) == []


def test_config5_job_stream_ranges():
    """The served-form stream: Poisson arrivals and per-job sizes in their stated ranges."""
    jobs = workloads.config5_jobs(njobs=300, rate_hz=20.0, nsrc_max=5000)
    t = np.array([a for a, _ in jobs])
    assert np.all(np.diff(t) > 0) and abs(np.mean(np.diff(t)) - 1 / 20.0) < 0.2 / 20.0
    for _, spec in jobs:
        nant, nsrc = len(spec.antpos), spec.eci.shape[1]
        assert 16 <= nant <= 512 and 1000 <= nsrc <= 5000
        assert 1 <= len(spec.freqs) <= 32 and 1 <= len(spec.lsts) <= 16
        assert spec.fluxes.shape == (nsrc, len(spec.freqs)) and np.all(np.diff(spec.freqs) >= 0)
        assert np.all(np.hypot(spec.antpos[:, 0], spec.antpos[:, 1]) <= 300.0)
        assert (len(spec.beams) == 1) and (spec.polarized == (not hasattr(spec.beams[0], "sigma")))
    assert 0 < sum(s.polarized for _, s in jobs) < len(jobs)


def test_latency_summary():
    from matvis_b200.serve import JobResult, latency_summary

    res = {i: JobResult(jid=i, vis=None, latency_s=0.1 * (i + 1), queue_s=0.01 * i, terms=1e9) for i in range(10)}
    res[10] = JobResult(jid=10, vis=None, latency_s=9.0, queue_s=0.0, terms=5e9, error="boom")
    s = latency_summary(res)
    assert s["jobs"] == 10 and s["errors"] == 1 and s["terms"] == 1e10
    assert s["p50_s"] == pytest.approx(0.55) and s["p99_s"] == pytest.approx(np.percentile(np.arange(1, 11) / 10, 99))
    assert s["mean_queue_s"] == pytest.approx(0.045)
    assert latency_summary({}) == {"jobs": 0}


def test_public_api_and_rotation_registry():
    """Every exported name resolves; rotation plugins register by class name
    (core/coords.py:32-38), including subclasses defined by a caller."""
    import matvis_b200 as mv
    from matvis_b200.coords import CoordinateRotation

    for name in mv.__all__:
        assert getattr(mv, name, None) is not None, name
    assert CoordinateRotation._methods["CoordinateRotationLST"] is mv.CoordinateRotationLST
    assert CoordinateRotation._methods["CoordinateRotationERFA"] is mv.CoordinateRotationERFA

    class CallerRotation(mv.CoordinateRotationLST):
        pass

    try:
        assert CoordinateRotation._methods["CallerRotation"] is CallerRotation
    finally:
        del CoordinateRotation._methods["CallerRotation"]


@pytest.mark.parametrize(("kwarg", "value", "errmsg"), [
    ("source_buffer", 0.0, "source_buffer must satisfy 0 < source_buffer <= 1"),
    ("source_buffer", 1.5, "source_buffer must satisfy 0 < source_buffer <= 1"),
    ("memory_buffer", 1.1, "memory_buffer must satisfy 0 < memory_buffer <= 1"),
])
def test_simulate_vis_buffer_validation(kwarg, value, errmsg):
    """The reference's wrapper validation (tests/test_wrapper.py:39-70), raised
    before any device work."""
    from matvis_b200.wrapper import simulate_vis

    kw = dict(ants={0: (0.0, 0.0, 0.0), 1: (14.6, 0.0, 0.0)}, fluxes=np.ones((15, 1)), ra=np.linspace(0, 1, 15),
              dec=np.full(15, -0.5), freqs=np.array([100e6]), times=np.zeros(5), beams=[], telescope_loc=-0.5)
    with pytest.raises(ValueError, match=errmsg):
        simulate_vis(**kw, **{kwarg: value})


def test_frequency_group_fits_memory():
    """fit_freq_group keeps the job's group when it fits, halves it while it does
    not, and falls back to one frequency per launch (then plan_job batches)."""
    from dataclasses import replace

    from matvis_b200 import workloads as wl
    from matvis_b200.engine import estimate_device_bytes, fit_freq_group, freq_group_of, job_from_arrays

    cfg = wl.subset(wl.config2(nfreq=16, ntimes=2), nsrc=3000, nfreq=16, ntimes=2, nant=40, seed=1)
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True)
    assert freq_group_of(spec, "MatMul", False) == 8
    assert freq_group_of(replace(spec, freq_group=32), "MatMul", False) == 16  # at most Nf
    assert freq_group_of(spec, "VectorDot", False) == 1 and freq_group_of(spec, "MatMul", True) == 1
    sizes = {g: estimate_device_bytes(replace(spec, freq_group=g)) for g in (1, 2, 4, 8)}
    assert sizes[1] < sizes[2] < sizes[4] < sizes[8]
    assert fit_freq_group(spec, sizes[8]).freq_group == 8
    assert fit_freq_group(spec, sizes[8] - 1).freq_group == 4
    assert fit_freq_group(spec, sizes[2]).freq_group == 2
    assert fit_freq_group(spec, 1.0).freq_group == 1


def test_autotuner_drain_candidates_stay_within_the_error_budget():
    """The drain interval is tuned only among intervals whose measured error (whole
    config-2 slice against the FP64 oracle) fits the budget: every interval for
    fp16x3, tf32x3 and bf16x6, none for bf16x3, which misses the bar at any
    interval and keeps its most accurate one."""
    from matvis_b200 import _lib
    from matvis_b200.autotune import ERROR_BUDGET, MEASURED_ERROR, drain_candidates

    for m in (_lib.GEMM_F16_3, _lib.GEMM_TF32_3, _lib.GEMM_BF16_6):
        assert drain_candidates(m) == [1, 2, 4]
    assert drain_candidates(_lib.GEMM_F16_3, (1, 2, 4, 8)) == [1, 2, 4]  # unmeasured intervals are not candidates
    assert max(MEASURED_ERROR[_lib.GEMM_F16_3].values()) <= ERROR_BUDGET
    assert drain_candidates(_lib.GEMM_BF16_3) == [1]
    assert drain_candidates(_lib.GEMM_F16_3, (0,)) == [0]
    assert ERROR_BUDGET < 1e-6
