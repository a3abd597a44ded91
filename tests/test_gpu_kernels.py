"""Kernel-level parity of the CUDA library against the FP64 oracle and the
reference-generated fixtures (run on a B200: ``pytest -m gpu``).

Tolerances (stated per test):
* rotation and horizon selection: bit-exact (coordinates and kept indices);
* beam interpolation: 1e-6 absolute against the FP64 result (grids are stored
  in float32 on the device, the weights and blend are FP64);
* exptau: 5e-7 absolute (complex64: FP64-reduced phase, FP32 sincospi),
  1e-12 (complex128);
* Hermitian product: max |dV| / sqrt(|V_ii| |V_jj|) <= 1e-6 for bf16x6 and
  tf32x3, <= 3e-5 for bf16x3; integer-valued Z is exact in every mode.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import matvis_b200 as mv  # noqa: E402
from matvis_b200 import _lib  # noqa: E402
from matvis_b200 import workloads  # noqa: E402
from oracle import oracle as orc  # noqa: E402

from .conftest import golden  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _cos_err(v, ref, nant, nfeed):
    return orc.cosine_error_metric(np.asarray(v).reshape(-1, nfeed, nfeed), np.asarray(ref).reshape(-1, nfeed, nfeed), nfeed)


# ---------------------------------------------------------------- rotation
@pytest.mark.parametrize("nsrc", [1, 1000, 4097, 196608])
def test_rotate_and_compact_bitexact(device, nsrc):
    rng = np.random.default_rng(nsrc)
    ra, dec = rng.uniform(0, 2 * np.pi, nsrc), np.arcsin(rng.uniform(-1, 1, nsrc))
    eci = orc.point_source_crd_eq(ra, dec)
    flux = np.sqrt(0.5 * rng.uniform(0.1, 10, nsrc))
    lat = np.deg2rad(-30.72)
    rot = mv.CoordinateRotationLST(flux=flux, times=np.array([0.3, 2.5]), telescope_loc=lat, skycoords=(ra, dec),
                                   source_buffer=1.0)
    rot.setup()
    for t, lst in enumerate(rot.times):
        rot.rotate(t)
        ref_top = orc.rotate_fixed_order(orc.eci_to_enu_matrix(lst, lat), eci)
        np.testing.assert_array_equal(rot.all_coords_topo.cpu().numpy(), ref_top)
        crd, fl, n = rot.select_chunk(0, t)
        rc, rf, rn, kept = orc.select_chunk(ref_top, flux, 0, nsrc, rot.nsrc_alloc)
        assert n == rn
        np.testing.assert_array_equal(rot.kept_index[:n].cpu().numpy(), kept)
        np.testing.assert_array_equal(crd[:, :n].cpu().numpy(), rc[:, :n])
        np.testing.assert_array_equal(fl.cpu().numpy(), rf)


def test_select_chunk_matches_reference_fixture(device):
    g = golden("coords")
    eci, flux = g["sel_eci"], g["sel_flux"]
    ra = np.arctan2(eci[1], eci[0])
    dec = np.arcsin(eci[2])
    rot = mv.CoordinateRotationLST(flux=flux, times=g["sel_lsts"], telescope_loc=float(g["sel_lat"]),
                                   skycoords=(ra, dec), chunk_size=int(g["sel_chunk_size"]), source_buffer=0.7)
    rot.setup()
    rot.eci.copy_(torch.as_tensor(eci))  # the fixture's exact unit vectors
    assert rot.nsrc_alloc == int(g["sel_alloc"])
    for t in range(len(g["sel_lsts"])):
        rot.rotate(t)
        for ch in range(2):
            crd, fl, n = rot.select_chunk(ch, t)
            assert n == int(g[f"sel_n_t{t}_c{ch}"])
            np.testing.assert_allclose(crd[:, :n].cpu().numpy(), g[f"sel_crd_t{t}_c{ch}"], rtol=0, atol=1e-15)
            np.testing.assert_array_equal(fl.cpu().numpy(), g[f"sel_flux_t{t}_c{ch}"])


def test_select_chunk_overflow_raises(device):
    n = 3000
    ra = np.zeros(n)
    dec = np.full(n, np.deg2rad(-30.72))  # all near zenith at lst 0
    rot = mv.CoordinateRotationLST(flux=np.ones(n), times=np.array([0.0]), telescope_loc=np.deg2rad(-30.72),
                                   skycoords=(ra, dec), source_buffer=0.5)
    rot.setup()
    rot.rotate(0)
    with pytest.raises(ValueError, match="nsrc_alloc"):
        rot.select_chunk(0, 0)


# ---------------------------------------------------------------- beams
@pytest.mark.parametrize("case", ["ident", "lin", "cplx", "pow"])
def test_bilinear_matches_reference(device, case):
    g = golden("bilinear")
    p = g[f"{case}_params"]
    beam = g[f"{case}_beam"]
    out = mv.beams.gpu_beam_interpolation(beam, p[:, 0], p[:, 1], p[:, 2], g[f"{case}_az"], g[f"{case}_za"])
    ref = g[f"{case}_out"]
    # grids are float32 on the device
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=0, atol=2e-6 * max(1.0, np.abs(ref).max()))


def test_bilinear_wrong_dtype(device):
    with pytest.raises(ValueError, match="as the dtype for beam, which is unrecognized"):
        mv.beams.gpu_beam_interpolation(np.ones((1, 1, 1, 3, 3), dtype=int), 1.0, 1.0, 0.0, [0.0], [0.0])


def test_beam_interpolator_enu_matches_oracle(device):
    rng = np.random.default_rng(3)
    beams = workloads.dipole_beams(rng, 2, dgrid_deg=2.0)
    n = 5000
    e = rng.uniform(-0.7, 0.7, n)
    nn = rng.uniform(-0.7, 0.7, n)
    bi = mv.B200BeamInterpolator(beam_list=beams, beam_idx=np.array([0, 1, 1]), polarized=True, nant=3, freq=1e8,
                                 nsrc=n, precision=2)
    bi.setup()
    out = bi(torch.as_tensor(e, device=DEV), torch.as_tensor(nn, device=DEV)).cpu().numpy()
    ob = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in beams]
    ref = orc.beam_response(ob, True, e, nn)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-6)


def test_beam_coordinate_workspace_matches_per_plane_path(device):
    """With a workspace the per-source grid coordinates are computed once for all
    planes; the result equals the per-plane recomputation (same FP64
    expressions) to the last bits of FP64, with the device's above-horizon count
    bounding the sources and the slots past it zero."""
    rng = np.random.default_rng(9)
    beams = workloads.dipole_beams(rng, 3, dgrid_deg=1.0)
    nout, n = 7000, 6123
    e = rng.uniform(-0.7, 0.7, nout)
    nn = rng.uniform(-0.7, 0.7, nout)
    bi = mv.B200BeamInterpolator(beam_list=beams, beam_idx=np.array([0, 1, 2]), polarized=True, nant=3, freq=1e8,
                                 nsrc=nout, precision=2)
    bi.setup()
    crd = torch.as_tensor(np.stack([e, nn]), device=DEV).contiguous()
    n_dev = torch.tensor([n], dtype=torch.int32, device=DEV)
    outs = []
    for ws in (None, torch.empty(2 * 3 * nout, dtype=torch.float64, device=DEV)):
        out = torch.full((3, 2, 2, nout), 7.0 + 7.0j, dtype=torch.complex128, device=DEV)
        _lib.check(_lib.lib.mvb_beam_interp(
            _lib.ptr(bi.grids), bi.grid_kind, 3, 2, 2, bi.nza, bi.naz, _lib.ptr(bi.params), _lib.ptr(crd), nout,
            _lib.ptr(n_dev), nout, _lib.ptr(out), 1, nout, None, _lib.ptr(ws), 0 if ws is None else ws.numel() * 8,
            _lib.stream_handle()))
        outs.append(out.cpu().numpy())
    np.testing.assert_allclose(outs[1], outs[0], rtol=1e-14, atol=1e-15)
    assert (outs[1][..., n:] == 0).all() and np.abs(outs[1][..., :n]).max() > 0.1
    with pytest.raises(ValueError, match="workspace"):
        _lib.check(_lib.lib.mvb_beam_interp(
            _lib.ptr(bi.grids), bi.grid_kind, 3, 2, 2, bi.nza, bi.naz, _lib.ptr(bi.params), _lib.ptr(crd), nout,
            None, nout, _lib.ptr(out), 1, nout, None, _lib.ptr(ws), 8, _lib.stream_handle()))


def test_hera_beamfits_beam_on_device_matches_oracle(device):
    """The reference's own HERA dipole file (tests/conftest.py:9-24), interpolated
    to 100.4 MHz and re-gridded on the host, then interpolated at 20,000 directions
    above the horizon by the device kernel against the oracle's FP64 bilinear on the
    same grid (1e-6 absolute: the device stores the grid in float32)."""
    from pathlib import Path

    fits = mv.read_beamfits(Path(__file__).resolve().parent / "golden" / "NF_HERA_Dipole_small.fits")
    g = fits.to_grid_beam(100.4e6)
    rng = np.random.default_rng(8)
    n = 20000
    r = np.sqrt(rng.uniform(0, 1, n))
    th = rng.uniform(0, 2 * np.pi, n)
    e, nn = r * np.cos(th), r * np.sin(th)
    bi = mv.B200BeamInterpolator(beam_list=[g], beam_idx=None, polarized=True, nant=2, freq=100.4e6, nsrc=n,
                                 precision=2)
    bi.setup()
    out = bi(torch.as_tensor(e, device=DEV), torch.as_tensor(nn, device=DEV)).cpu().numpy()
    ref = orc.beam_response([orc.GridBeam(data=g.data.astype(np.complex128), az=g.az, za=g.za)], True, e, nn)
    assert np.abs(ref).max() > 0.5
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-6)


def test_gaussian_beam(device):
    rng = np.random.default_rng(4)
    e, nn = rng.uniform(-0.6, 0.6, 1000), rng.uniform(-0.6, 0.6, 1000)
    bi = mv.B200BeamInterpolator(beam_list=[mv.GaussianBeam(0.2), mv.GaussianBeam(0.35)], beam_idx=np.array([0, 1]),
                                 polarized=False, nant=2, freq=1e8, nsrc=1000, precision=2)
    bi.setup()
    out = bi(torch.as_tensor(e, device=DEV), torch.as_tensor(nn, device=DEV)).cpu().numpy()
    ref = orc.beam_response([orc.GaussianPowerBeam(0.2), orc.GaussianPowerBeam(0.35)], False, e, nn)
    np.testing.assert_allclose(out, ref, rtol=1e-13, atol=1e-15)


# ---------------------------------------------------------------- tau / Z
@pytest.mark.parametrize("precision,tol", [(1, 5e-7), (2, 1e-12)])
def test_exptau_matches_reference(device, precision, tol):
    g = golden("tauz")
    tc = mv.TauCalculator(antpos=g["antpos"], freq=float(g["freq"]), nsrc=g["crd"].shape[1], precision=precision)
    tc.setup()
    out = tc(torch.as_tensor(g["crd"], device=DEV)).cpu().numpy()
    np.testing.assert_allclose(out, g["exptau"], rtol=0, atol=tol)


def test_exptau_long_baseline_phase():
    """1 km, 200 MHz: |phase| ~ 4e3 rad; the FP64 reduction keeps complex64 exact to ~1e-7."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(9)
    antpos = rng.uniform(-1000, 1000, (50, 3))
    crd = rng.normal(size=(3, 3000))
    crd /= np.linalg.norm(crd, axis=0)
    tc = mv.TauCalculator(antpos=antpos, freq=200e6, nsrc=3000, precision=1)
    tc.setup()
    out = tc(torch.as_tensor(crd, device=DEV)).cpu().numpy()
    np.testing.assert_allclose(out, orc.exptau(antpos, 200e6, crd), rtol=0, atol=5e-7)


@pytest.mark.parametrize("mode", ["bf16x3", "bf16x6", "tf32x3", "fp16x3"])
def test_z_from_exptau_matches_reference(device, mode):
    g = golden("tauz")
    zc = mv.ZMatrixCalc(nant=6, nfeed=2, nax=2, nsrc=g["exptau"].shape[1], mode=_lib.GEMM_MODES[mode])
    zc.setup()
    z = zc(g["sqrt_flux"], g["beam"], g["exptau"], g["beam_idx"])
    zz = z.to_complex().cpu().numpy()
    # panel column order is (src, ax); reference order is (ax, src)
    ref = g["z"].reshape(12, 2, -1).transpose(0, 2, 1).reshape(12, -1)
    tol = {"bf16x3": 2e-5, "bf16x6": 5e-7, "tf32x3": 5e-7, "fp16x3": 5e-7}[mode]
    np.testing.assert_allclose(zz, ref, rtol=0, atol=tol * np.abs(ref).max())


# ---------------------------------------------------------------- Hermitian product
@pytest.mark.parametrize("mode", ["bf16x3", "bf16x6", "tf32x3", "fp16x3"])
@pytest.mark.parametrize("nfeed", [1, 2])
@pytest.mark.parametrize("explicit", [False, True])
def test_matmul_arange_known_answer(device, mode, nfeed, explicit):
    """tests/test_matprod.py:45-65: integer-valued Z is reproduced exactly."""
    g = golden("matprod")
    nant, nsrc = 5, 15
    pairs = np.array([(i, j) for i in range(nant) for j in range(nant)]) if explicit else None
    for precision in (1, 2):
        mp = mv.B200MatMul(nchunks=1, nfeed=nfeed, nant=nant, antpairs=pairs, precision=precision, gemm_mode=mode)
        mp.setup()
        z = np.arange(nfeed * nant * nsrc, dtype=complex).reshape(nfeed * nant, nsrc) + 1j
        out = np.zeros((mp.npairs, nfeed, nfeed), dtype=np.complex64 if precision == 1 else np.complex128)
        mp(z, chunk=0)
        mp.sum_chunks(out)
        ref = g[f"arange_CPUMatMul_f{nfeed}_p{precision}_e{int(explicit)}_c1"]
        np.testing.assert_array_equal(out, ref)


def test_vectordot_arange_known_answer(device):
    g = golden("matprod")
    for nfeed in (1, 2):
        mp = mv.B200VectorDot(nchunks=1, nfeed=nfeed, nant=5, antpairs=None, precision=2)
        mp.setup()
        z = np.arange(nfeed * 5 * 15, dtype=complex).reshape(nfeed * 5, 15) + 1j
        out = np.zeros((25, nfeed, nfeed), dtype=complex)
        mp(z, 0)
        mp.sum_chunks(out)
        np.testing.assert_allclose(out, g[f"arange_CPUVectorDot_f{nfeed}_p2_e0_c1"], rtol=1e-7)


@pytest.mark.parametrize("mode,tol", [("bf16x6", 1e-6), ("tf32x3", 1e-6), ("fp16x3", 1e-6), ("bf16x3", 3e-5)])
# row counts whose last 128-row block holds 60 (700 rows), 64, 2, 72 and 128 rows
@pytest.mark.parametrize("nant,nfeed,K,k_chunk", [(350, 2, 20000, 2048), (64, 1, 777, 64), (129, 2, 4096, 1024),
                                                  (96, 2, 3000, 1024), (100, 2, 3000, 1024), (128, 1, 2000, 512)])
def test_matmul_random_vs_oracle(device, mode, tol, nant, nfeed, K, k_chunk):
    rng = np.random.default_rng(nant + K)
    M = nant * nfeed
    z = (rng.normal(size=(M, K)) + 1j * rng.normal(size=(M, K))) * rng.lognormal(0, 1, K)[None, :]
    mp = mv.B200MatMul(nchunks=1, nfeed=nfeed, nant=nant, antpairs=None, precision=2, gemm_mode=mode, k_chunk=k_chunk)
    mp.setup()
    out = torch.zeros((mp.npairs, nfeed, nfeed), dtype=torch.complex128, device=DEV)
    mp(z, 0)
    mp.sum_chunks(out)
    ref = orc.matmul_vis(z.astype(np.complex64).astype(np.complex128), nant, nfeed)
    err = _cos_err(out.cpu().numpy(), ref, nant, nfeed)
    assert err <= tol, f"{mode}: cosine error {err:.3e} > {tol}"


@pytest.mark.parametrize("mode", ["fp16x3", "bf16x6"])
def test_matmul_row_dynamic_range(device, mode):
    """Rows whose magnitude is 1 .. 1e-4 of the panel maximum.  fp16x3 scales the
    whole panel by one power of two, so a row keeps its ~22-bit split while its
    largest element stays above ~1e-5 of the maximum; the normalised error
    (by each row's own autocorrelation) stays <= 1e-6."""
    rng = np.random.default_rng(77)
    nant, K = 40, 6000
    z = rng.normal(size=(nant, K)) + 1j * rng.normal(size=(nant, K))
    z *= (10.0 ** -rng.integers(0, 5, nant))[:, None]
    mp = mv.B200MatMul(nchunks=1, nfeed=1, nant=nant, antpairs=None, precision=2, gemm_mode=mode, k_chunk=1024)
    mp.setup()
    out = torch.zeros((mp.npairs, 1, 1), dtype=torch.complex128, device=DEV)
    mp(z, 0)
    mp.sum_chunks(out)
    ref = orc.matmul_vis(z.astype(np.complex64).astype(np.complex128), nant, 1)
    err = _cos_err(out.cpu().numpy(), ref, nant, 1)
    assert err <= 1e-6, f"{mode}: cosine error {err:.3e}"


def test_matmul_sparse_pairs_vs_reference(device):
    g = golden("matprod")
    z, pairs = g["random_z"], g["random_pairs"]
    for mode in ("bf16x6", "tf32x3", "fp16x3"):
        mp = mv.B200MatMul(nchunks=1, nfeed=2, nant=7, antpairs=pairs, precision=2, gemm_mode=mode)
        mp.setup()
        out = np.zeros((len(pairs), 2, 2), dtype=complex)
        mp(z, 0)
        mp.sum_chunks(out)
        ref = g["random_CPUMatMul_sparse"]
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-6 * np.abs(ref).max())


def test_vectordot_random_vs_reference(device):
    g = golden("matprod")
    z, pairs = g["random_z"], g["random_pairs"]
    mp = mv.B200VectorDot(nchunks=1, nfeed=2, nant=7, antpairs=pairs, precision=2, k_chunk=64)
    mp.setup()
    out = np.zeros((len(pairs), 2, 2), dtype=complex)
    mp(z, 0)
    mp.sum_chunks(out)
    ref = g["random_CPUVectorDot_sparse"]
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-6 * np.abs(ref).max())


def _pair_err(v, ref, z, nant, nfeed, pairs):
    """max |dV| / sqrt(|V_jj^pp| |V_ii^qq|) for out[i, p, q] of pair (ai, aj) = (i, j)."""
    zz = z.reshape(nant, nfeed, -1)
    auto = (np.abs(zz) ** 2).sum(-1)
    den = np.sqrt(auto[pairs[:, 1]][:, :, None] * auto[pairs[:, 0]][:, None, :])
    return float(np.max(np.abs(np.asarray(v) - ref) / den)) if len(pairs) else 0.0


# nant x nfeed rows staged 16 (700, 37, 14, 3 rows), 8 (1000, 1600 rows) and 4 (2000 rows) columns at
# a time; odd K ends on a single column
@pytest.mark.parametrize("nant,nfeed,K,k_chunk,npairs", [(350, 2, 40000, 4096, 5000), (37, 1, 3001, 1024, 63),
                                                         (7, 2, 555, 64, 40), (3, 1, 100, 16, 5),
                                                         (1000, 1, 1501, 512, 2500), (1000, 2, 2048, 512, 3000),
                                                         (1600, 1, 999, 256, 2000)])
def test_vectordot_staged_vs_oracle(device, nant, nfeed, K, k_chunk, npairs):
    """Both pair kernels against the FP64 oracle (<= 1e-6 normalised), with
    autocorrelations (real one-feed autos) and a repeated pair in the list."""
    rng = np.random.default_rng(nant + K)
    pairs = rng.integers(0, nant, size=(npairs, 2))
    pairs[0] = (0, 0)
    pairs[-1] = pairs[len(pairs) // 2]
    M = nant * nfeed
    z = (rng.normal(size=(M, K)) + 1j * rng.normal(size=(M, K))) * rng.lognormal(0, 1, K)[None, :]
    ref = orc.vectordot_vis(z.astype(np.complex64).astype(np.complex128), nant, nfeed, pairs)
    outs = {}
    for kernel in ("staged", "warp"):
        mp = mv.B200VectorDot(nchunks=1, nfeed=nfeed, nant=nant, antpairs=pairs, precision=2, k_chunk=k_chunk,
                              kernel=kernel)
        mp.setup()
        assert mp.kernel == kernel
        out = torch.zeros((npairs, nfeed, nfeed), dtype=torch.complex128, device=DEV)
        mp(z, 0)
        mp.sum_chunks(out)
        o = outs[kernel] = out.cpu().numpy()
        err = _pair_err(o, ref, z, nant, nfeed, pairs)
        assert err <= 1e-6, f"{kernel}: normalised error {err:.3e}"
        autos = pairs[:, 0] == pairs[:, 1]
        for f in range(nfeed):
            assert (o[autos, f, f].imag == 0).all()
    # a repeated pair may sit in slots of either orientation: equal to rounding
    np.testing.assert_allclose(outs["staged"][-1], outs["staged"][len(pairs) // 2], rtol=1e-6)


def test_vectordot_staged_accumulate_complex64_and_fallback(device):
    rng = np.random.default_rng(5)
    nant, nfeed, K = 50, 2, 5000
    pairs = rng.integers(0, nant, size=(300, 2))
    z = rng.normal(size=(nant * nfeed, K)) + 1j * rng.normal(size=(nant * nfeed, K))
    mp = mv.B200VectorDot(nchunks=1, nfeed=nfeed, nant=nant, antpairs=pairs, precision=1, k_chunk=1024)
    mp.setup()
    assert mp.kernel == "staged"
    panel = mp._as_panel(z, mp.mode)
    out = torch.zeros((300, nfeed, nfeed), dtype=torch.complex64, device=DEV)
    mp.enqueue(panel, out)
    mp.enqueue(panel, out, accumulate=True)
    torch.cuda.synchronize()
    ref = orc.vectordot_vis(z.astype(np.complex64).astype(np.complex128), nant, nfeed, pairs)
    assert _pair_err(out.cpu().numpy().astype(np.complex128) / 2, ref, z, nant, nfeed, pairs) <= 1e-6
    # rows that do not fit two shared-memory stages: the warp kernel, or an error when asked for staging
    assert mv.B200VectorDot(1, 2, 4000, np.array([[0, 1]]), kernel="auto").kernel == "warp"
    with pytest.raises(ValueError, match="shared memory"):
        mv.B200VectorDot(1, 2, 4000, np.array([[0, 1]]), kernel="staged")


def test_vectordot_staged_positive_sums(device):
    """All-positive terms over a long K (autocorrelation-like): FP32 sums over one
    16-column stage, FP64 beyond, so the relative error stays near 1e-7."""
    rng = np.random.default_rng(2)
    nant, K = 40, 300000
    z = rng.uniform(0.5, 1.5, size=(nant, K)) * np.exp(1j * 0.01 * rng.normal(size=(nant, K)))
    pairs = np.column_stack([np.arange(nant), (np.arange(nant) + 1) % nant])
    pairs = np.concatenate([pairs, np.column_stack([np.arange(nant)] * 2)])
    mp = mv.B200VectorDot(nchunks=1, nfeed=1, nant=nant, antpairs=pairs, precision=2, k_chunk=16384)
    mp.setup()
    out = torch.zeros((len(pairs), 1, 1), dtype=torch.complex128, device=DEV)
    mp(z, 0)
    mp.sum_chunks(out)
    ref = orc.vectordot_vis(z.astype(np.complex64).astype(np.complex128), nant, 1, pairs)
    rel = np.abs(out.cpu().numpy() - ref) / np.abs(ref)
    assert rel.max() <= 1e-6, rel.max()


@pytest.mark.parametrize("mode", ["bf16x6", "fp16x3"])
@pytest.mark.parametrize("k_chunk", [512, 2048, 8192])
def test_herk_accumulation_positive_sums(device, k_chunk, mode):
    """All-positive terms (autocorrelation-like) over a long K: FP32 TMEM
    accumulation per k-slice, FP64 across slices."""
    rng = np.random.default_rng(1)
    M, K = 128, 65536
    z = rng.uniform(0.5, 1.5, size=(M, K)) * np.exp(1j * 0.01 * rng.normal(size=(M, K)))
    mp = mv.B200MatMul(nchunks=1, nfeed=1, nant=M, antpairs=None, precision=2, gemm_mode=mode, k_chunk=k_chunk)
    mp.setup()
    out = torch.zeros((M * M, 1, 1), dtype=torch.complex128, device=DEV)
    mp(z, 0)
    mp.sum_chunks(out)
    ref = orc.matmul_vis(z.astype(np.complex64).astype(np.complex128), M, 1)
    rel = np.abs(out.cpu().numpy() - ref) / np.abs(ref)
    print(f"{mode} k_chunk={k_chunk}: max rel {rel.max():.3e}, mean rel {rel.mean():.3e}")
    assert rel.max() < 2e-6


@pytest.mark.parametrize("N,nf", [(1, 1), (33, 3), (70001, 64), (1000, 33)])
def test_flux_sqrt_half_bitexact(device, N, nf):
    """sqrt(0.5 I) transposed to (Nf, N) float32 (cpu/cpu.py:188): FP64 square root
    rounded once to float32, as numpy does it."""
    rng = np.random.default_rng(N + nf)
    fl = rng.lognormal(0, 2, (N, nf))
    out = torch.empty((nf, N), dtype=torch.float32, device=DEV)
    src = torch.as_tensor(fl, device=DEV)
    _lib.check(_lib.lib.mvb_flux_sqrt_half(_lib.ptr(src), N, nf, _lib.ptr(out), None))
    np.testing.assert_array_equal(out.cpu().numpy(), np.sqrt(0.5 * fl).T.astype(np.float32))
