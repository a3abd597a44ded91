"""End-to-end parity of the batched engine / simulate_vis against the FP64 oracle
and against visibilities produced by the reference's own plugin classes.

Metric: max |V - V_ref| / sqrt(|V_ii^qq| |V_jj^pp|) over all outputs (the
Cauchy-Schwarz-normalised error), <= 1e-6 for the bf16x6 / tf32x3 products.
Sparse-pair outputs are compared elementwise with an absolute tolerance scaled
by the largest autocorrelation.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import matvis_b200 as mv  # noqa: E402
from matvis_b200 import workloads as wl  # noqa: E402
from matvis_b200.engine import VisEngine, job_from_arrays  # noqa: E402
from oracle import oracle as orc  # noqa: E402

from .conftest import golden  # noqa: E402

pytestmark = pytest.mark.gpu


def _oracle_job(cfg, matprod="MatMul", nchunks=1):
    beams = []
    for b in cfg["beams"]:
        if isinstance(b, mv.GaussianBeam):
            beams.append(orc.GaussianPowerBeam(sigma=b.sigma))
        else:
            beams.append(orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za, beam_type=b.beam_type))
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    return orc.simulate_vis(ants=ants, fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                            lsts=cfg["lsts"], latitude=cfg["latitude"], beams=beams, polarized=cfg["polarized"],
                            beam_idx=cfg.get("beam_idx"), antpairs=cfg.get("antpairs"), matprod=matprod,
                            nchunks=nchunks)


def _engine(cfg, **kw):
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg.get("beam_idx"),
                           polarized=cfg["polarized"], antpairs=cfg.get("antpairs"), **kw)
    return VisEngine(spec)


def _cos(v, ref, nfeed):
    return orc.cosine_error_metric(v.reshape(v.shape[:-2] + (nfeed, nfeed)) if v.ndim >= 3 else v[..., None, None],
                                   ref.reshape(ref.shape[:-2] + (nfeed, nfeed)) if ref.ndim >= 3 else ref[..., None, None],
                                   nfeed)


@pytest.mark.parametrize("mode", ["bf16x6", "tf32x3", "fp16x3"])
def test_config1_full_vs_oracle(device, mode):
    cfg = wl.config1()
    ref = _oracle_job(cfg)  # (Nf, Nt, Npairs)
    eng = _engine(cfg, precision=2, gemm_mode=mode)
    vis = eng.run().cpu().numpy()[..., 0, 0]
    err = orc.cosine_error_metric(vis[..., None, None], ref[..., None, None], 1)
    assert err <= 1e-6, err


def test_config1_graph_replay_identical(device):
    """Graph replays are bit-identical to each other and to the eager run with the
    same product parameters (k_chunk given, so capture() does not retune them)."""
    cfg = wl.config1()
    eng = _engine(cfg, precision=2, k_chunk=2048)
    v1 = eng.run().clone()
    eng.capture()
    assert eng.tuned is None and eng.k_chunk == 2048
    v2 = eng.run().clone()
    v3 = eng.run().clone()
    assert torch.equal(v1, v2) and torch.equal(v2, v3)


def test_tuned_graph_replays_are_identical(device):
    """With the autotuner choosing the product parameters, replays still agree bit
    for bit, and the tuned job meets the parity bar."""
    cfg = wl.config1()
    eng = _engine(cfg, precision=2)
    v1 = eng.run().clone()
    eng.capture()
    v2 = eng.run().clone()
    v3 = eng.run().clone()
    assert torch.equal(v2, v3)
    assert _cos(v2.cpu().numpy(), v1.cpu().numpy(), 1) <= 1e-6


@pytest.mark.parametrize("mode", ["bf16x6", "tf32x3", "fp16x3"])
def test_config2_subset_vs_oracle(device, mode):
    """HERA-350-like array and beams, 20k sources, 2 frequencies x 2 times."""
    cfg = wl.subset(wl.config2(nfreq=64, ntimes=16), nsrc=20000, nfreq=2, ntimes=2, seed=1)
    ref = _oracle_job(cfg)
    eng = _engine(cfg, precision=1, gemm_mode=mode)
    vis = eng.run().cpu().numpy()
    err = orc.cosine_error_metric(vis, ref, 2)
    print(f"config2 subset {mode}: cosine error {err:.3e}")
    assert err <= 1e-6


def test_pipeline_unpolarized_reference_fixture(device):
    g = golden("pipeline")
    ants = {i: tuple(p) for i, p in enumerate(g["a_antpos"])}
    vis = mv.simulate_vis(ants, g["a_fluxes"], g["a_ra"], g["a_dec"], g["a_freqs"], g["a_lsts"],
                          [mv.GaussianBeam(float(g["a_sigma"]))], float(g["a_lat"]), precision=2)
    ref = g["a_vis"]
    assert vis.shape == ref.shape
    err = orc.cosine_error_metric(vis[..., None, None], ref[..., None, None], 1)
    assert err <= 1e-6, err


@pytest.mark.parametrize("method,name", [("MatMul", "all"), ("MatMul", "sparse"), ("VectorDot", "sparse")])
def test_pipeline_polarized_reference_fixture(device, method, name):
    g = golden("pipeline")
    grids, p = g["b_grids"], g["b_grid_params"]
    naz, nza = grids.shape[-1], grids.shape[-2]
    beams = [mv.GridBeam(data=grids[b].astype(np.complex64), az=p[b, 2] + p[b, 0] * np.arange(naz),
                         za=p[b, 1] * np.arange(nza)) for b in range(grids.shape[0])]
    ants = {i: tuple(x) for i, x in enumerate(g["b_antpos"])}
    pairs = None if name == "all" else g["b_pairs"]
    vis = mv.simulate_vis(ants, g["b_fluxes"], g["b_ra"], g["b_dec"], g["b_freqs"], g["b_lsts"], beams,
                          float(g["b_lat"]), polarized=True, precision=2, beam_idx=g["b_beam_idx"], antpairs=pairs,
                          matprod_method=method, min_chunks=2)
    ref = g[f"b_vis_CPU{method}_{name}"]
    assert vis.shape == ref.shape
    if name == "all":
        assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6
    else:
        scale = np.abs(g["b_vis_CPUMatMul_all"]).max()
        np.testing.assert_allclose(vis, ref, rtol=0, atol=2e-6 * scale)


def test_antizenith_source_gives_zero(device):
    """tests/test_matvis_gpu.py:15-25: a source below the horizon contributes nothing."""
    lat = np.deg2rad(-30.72)
    ants = {0: (0.0, 0.0, 0.0), 1: (10.0, 5.0, 0.0), 2: (-3.0, 8.0, 0.0)}
    vis = mv.simulate_vis(ants, np.ones((1, 1)), np.array([np.pi]), np.array([-lat]), np.array([1e8]),
                          np.array([0.0]), [mv.GaussianBeam(0.3)], lat, precision=2)
    assert np.all(vis == 0)


def test_multibeam_invariances(device):
    """tests/test_matvis_gpu.py:28-110: replicated beams == one beam; permuted beam list + remapped idx."""
    cfg = wl.subset(wl.config1(), nsrc=300, nfreq=1, ntimes=2, nant=3)
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    kw = dict(fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], times=cfg["lsts"],
              telescope_loc=cfg["latitude"], precision=2)
    b = mv.GaussianBeam(0.2)
    v1 = mv.simulate_vis(ants, beams=[b] * 3, beam_idx=np.zeros(3, int), **kw)
    v2 = mv.simulate_vis(ants, beams=[b], **kw)
    np.testing.assert_array_equal(v1, v2)
    ba, bb = mv.GaussianBeam(0.2), mv.GaussianBeam(0.35)
    vab = mv.simulate_vis(ants, beams=[ba, bb], beam_idx=np.array([0, 1, 0]), **kw)
    vba = mv.simulate_vis(ants, beams=[bb, ba], beam_idx=np.array([1, 0, 1]), **kw)
    np.testing.assert_array_equal(vab, vba)
    v010 = mv.simulate_vis(ants, beams=[ba, bb], beam_idx=np.array([0, 1, 0]), **kw)
    v101 = mv.simulate_vis(ants, beams=[ba, bb], beam_idx=np.array([1, 0, 1]), **kw)
    assert not np.allclose(v010, v101, rtol=0, atol=1e-12)


def test_mixed_beams_rejected(device):
    cfg = wl.subset(wl.config1(), nsrc=50, nfreq=1, ntimes=1, nant=3)
    grid = wl.dipole_beams(np.random.default_rng(0), 1, dgrid_deg=5.0)[0]
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    with pytest.raises(ValueError, match="GPUBeamInterpolator only supports beam_lists with either"):
        mv.simulate_vis(ants, cfg["fluxes"], cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"],
                        [grid, mv.GaussianBeam(0.2), mv.GaussianBeam(0.2)], cfg["latitude"])


def test_single_vs_double_precision(device):
    """tests/test_matvis_gpu.py:127-139: precision 1 vs 2 within 1e-5 absolute."""
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=2000, nfreq=1, ntimes=1, nant=40, seed=3)
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    kw = dict(fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], times=cfg["lsts"],
              beams=cfg["beams"], telescope_loc=cfg["latitude"], polarized=True, beam_idx=cfg["beam_idx"])
    v1 = mv.simulate_vis(ants, precision=1, **kw)
    v2 = mv.simulate_vis(ants, precision=2, **kw)
    np.testing.assert_allclose(v1, v2, atol=1e-5 * max(1.0, np.abs(v2).max()), rtol=0)


def test_simulate_single_frequency_matches_simulate_vis(device):
    cfg = wl.subset(wl.config1(), nsrc=500, ntimes=2)
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    vall = mv.simulate_vis(ants, cfg["fluxes"], cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], cfg["beams"],
                           cfg["latitude"], precision=2)
    v0 = mv.simulate(antpos=cfg["antpos"], freq=cfg["freqs"][1], times=cfg["lsts"], skycoords=(cfg["ra"], cfg["dec"]),
                     telescope_loc=cfg["latitude"], I_sky=cfg["fluxes"][:, 1], beam_list=cfg["beams"], precision=2)
    np.testing.assert_array_equal(v0, vall[1])



def test_simulate_vis_frequency_batches(device, caplog):
    """Under a max_memory below the whole job, simulate_vis runs contiguous frequency
    batches into one host array; the result meets the parity bar like the one-job run."""
    import logging
    from dataclasses import replace

    from matvis_b200.engine import estimate_device_bytes, plan_job

    cfg = wl.subset(wl.config2(nfreq=5, ntimes=2), nsrc=3000, nant=24, seed=7)
    cfg["fluxes"] = cfg["fluxes"] * np.array([0.5, 1.0, 3.0, 9.0, 0.2])  # a different Z scale per batch
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    kw = dict(fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], times=cfg["lsts"],
              beams=cfg["beams"], telescope_loc=cfg["latitude"], polarized=True, beam_idx=cfg["beam_idx"],
              precision=2, freq_group=1)
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"],
                           freqs=cfg["freqs"], lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"],
                           beam_idx=cfg["beam_idx"], polarized=True, precision=2, freq_group=1)

    def size(n):
        return estimate_device_bytes(replace(spec, freqs=spec.freqs[:n], fluxes=spec.fluxes[:, :n]))

    max_memory = (size(2) + size(3)) / 2 / 0.9
    assert plan_job(spec, max_memory * 0.9) == (2, 1)
    whole = mv.simulate_vis(ants, **kw)
    with caplog.at_level(logging.INFO, logger="matvis_b200.wrapper"):
        batched = mv.simulate_vis(ants, max_memory=max_memory, **kw)
    assert "in batches of 2" in caplog.text
    assert batched.shape == whole.shape == (5, 2, 24 * 24, 2, 2)
    ref = _oracle_job(cfg)
    assert _cos(batched, ref, 2) <= 1e-6
    assert _cos(whole, ref, 2) <= 1e-6
    assert _cos(batched, whole, 2) <= 1e-6

def test_plugin_chain_matches_engine(device):
    """The reference call order (rotate, select_chunk, beam, tau, Z, matprod, sum_chunks)
    through the mirrored plugin classes gives the engine's result."""
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=3000, nfreq=1, ntimes=2, nant=20, seed=5)
    freq = float(cfg["freqs"][0])
    nant = len(cfg["antpos"])
    flux = np.sqrt(0.5 * cfg["fluxes"][:, 0])
    coords = mv.CoordinateRotationLST(flux=flux, times=cfg["lsts"], telescope_loc=cfg["latitude"],
                                      skycoords=(cfg["ra"], cfg["dec"]), source_buffer=1.0, precision=2)
    bm = mv.B200BeamInterpolator(beam_list=cfg["beams"], beam_idx=cfg["beam_idx"], polarized=True, nant=nant,
                                 freq=freq, nsrc=coords.nsrc_alloc, precision=2)
    tc = mv.TauCalculator(antpos=cfg["antpos"], freq=freq, nsrc=coords.nsrc_alloc, precision=2)
    zc = mv.ZMatrixCalc(nant=nant, nfeed=2, nax=2, nsrc=coords.nsrc_alloc)
    mp = mv.B200MatMul(nchunks=1, nfeed=2, nant=nant, antpairs=None, precision=2)
    for o in (coords, bm, tc, zc, mp):
        o.setup()
    vis = np.zeros((len(cfg["lsts"]), nant * nant, 2, 2), dtype=complex)
    for t in range(len(cfg["lsts"])):
        coords.rotate(t)
        crd, fl, n = coords.select_chunk(0, t)
        A = bm(crd[0], crd[1], check=t == 0)
        ext = tc(crd)
        z = zc(fl, A, ext, bm.beam_idx)
        mp(z, 0)
        mp.sum_chunks(vis[t])
    ref = _oracle_job(dict(cfg, freqs=cfg["freqs"][:1], fluxes=cfg["fluxes"][:, :1]))[0]
    assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6


@pytest.mark.parametrize("matprod", ["VectorDot", "MatMul"])
def test_redundant_pairs_through_products(device, matprod):
    """Redundant-baseline representatives of a 37-element hexagon (the
    hera_profile pair list, cli.py:316-319) through both products."""
    from matvis_b200.pairs import redundant_antpairs

    cfg = wl.config1()
    cfg["antpos"] = wl.hex_array(37, 14.6)
    cfg["antpairs"] = redundant_antpairs(cfg["antpos"])
    assert len(cfg["antpairs"]) == 63
    ref = _oracle_job(cfg, matprod="VectorDot")
    vis = _engine(cfg, precision=2, matprod=matprod).run().cpu().numpy()[..., 0, 0]
    assert vis.shape == ref.shape
    full = _oracle_job(dict(cfg, antpairs=None))
    scale = np.abs(full).max()
    np.testing.assert_allclose(vis, ref, rtol=0, atol=1e-6 * scale)


def test_run_to_host_matches_device_result(device):
    """The streamed device -> host path returns exactly the device visibilities."""
    cfg = wl.config1()
    eng = _engine(cfg, precision=1)
    dev_vis = eng.run().cpu().numpy()
    host = eng.run_to_host()
    np.testing.assert_array_equal(host, dev_vis)
    out = np.zeros_like(dev_vis)
    assert eng.run_to_host(out) is out
    np.testing.assert_array_equal(out, dev_vis)
    with pytest.raises(ValueError):
        eng.run_to_host(np.zeros(dev_vis.shape, dtype=np.complex128))


def test_beamfits_beam_through_simulate_vis(device, tmp_path):
    """A beamfits E-field beam (written and read back) interpolated to two
    frequencies inside its range, against the oracle driven with the same
    re-gridded grids."""
    from matvis_b200.beamfits import BeamFits, read_beamfits, write_beamfits

    rng = np.random.default_rng(12)
    naz, nza = 180, 46
    az = np.deg2rad(np.arange(naz) * (359.0 / (naz - 1)))
    za = np.deg2rad(np.linspace(0, 90, nza))
    A, Z = np.meshgrid(az, za)
    data = np.zeros((2, 2, 2, nza, naz), dtype=complex)
    for i in range(2):
        g = 1.0 + 0.05 * i
        data[0, 0, i], data[1, 0, i] = g * np.cos(Z) * np.cos(A), -g * np.sin(A)
        data[0, 1, i], data[1, 1, i] = g * np.cos(Z) * np.sin(A), g * np.cos(A)
    path = tmp_path / "beam.fits"
    write_beamfits(path, BeamFits("efield", data, az, za, np.array([100e6, 110e6]), ["x", "y"], [], "linear"))
    beam = read_beamfits(path)
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=3000, nfreq=2, ntimes=2, nant=12, seed=5)
    freqs = np.array([102e6, 107.5e6])
    fluxes = cfg["fluxes"][:, :2]
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    vis = mv.simulate_vis(ants, fluxes, cfg["ra"], cfg["dec"], freqs, cfg["lsts"], [beam], cfg["latitude"],
                          polarized=True, precision=2)
    ref = []
    for i, f in enumerate(freqs):
        g = beam.to_grid_beam(f)
        ob = [orc.GridBeam(data=g.data.astype(np.complex128), az=g.az, za=g.za)]
        ref.append(orc.simulate_vis(ants=ants, fluxes=fluxes[:, i : i + 1], ra=cfg["ra"], dec=cfg["dec"],
                                    freqs=freqs[i : i + 1], lsts=cfg["lsts"], latitude=cfg["latitude"], beams=ob,
                                    polarized=True)[0])
    ref = np.asarray(ref)
    assert vis.shape == ref.shape
    assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6


def test_one_beam_per_antenna(device):
    """nbeam == nant (beam_idx None -> beam a for antenna a, core/beams.py:64-68)
    with 10 polarised beams: nbeam * F * X = 40 reads the beams from L2 instead
    of staging them in shared memory."""
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=2500, nfreq=1, ntimes=2, nant=10, seed=9)
    rng = np.random.default_rng(4)
    base = cfg["beams"][0]
    cfg["beams"] = [mv.GridBeam(data=(base.data * (1 + 0.05 * rng.normal(size=base.data.shape))).astype(np.complex64),
                                az=base.az, za=base.za) for _ in range(10)]
    cfg["beam_idx"] = None
    ref = _oracle_job(cfg)
    for mode in ("fp16x3", "bf16x6"):
        vis = _engine(cfg, precision=2, gemm_mode=mode).run().cpu().numpy()
        assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6, mode


def test_allocate_then_run_uploads_inputs(device):
    """An engine allocated explicitly still uploads its inputs before the first run."""
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=2000, nfreq=1, ntimes=1, nant=10, seed=9)
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True, precision=2)
    e1 = VisEngine(spec)
    e1.allocate()
    v1 = e1.run().cpu().numpy()
    v2 = VisEngine(spec).run().cpu().numpy()
    assert np.abs(v1).max() > 0
    np.testing.assert_array_equal(v1, v2)

