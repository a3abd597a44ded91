"""Grouped launches: the frequencies of a time step in one tau/Z, one product
and one reduction launch, each frequency on its own Z panel.

* tau/Z: every panel of the grouped launch is bit-identical to the panel the
  per-frequency launch writes (same arithmetic, frequency read from a device
  array instead of a kernel argument);
* product: each panel's visibilities equal its own product's within the
  accumulation tolerance (the k-slice plan fills waves for all panels' units,
  so the slice boundaries, not the sums, may differ);
* a whole job with freq_group 1, 3 and 8 against the FP64 oracle (1e-6).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from matvis_b200 import _lib  # noqa: E402
from matvis_b200 import workloads as wl  # noqa: E402
from matvis_b200.engine import VisEngine, job_from_arrays  # noqa: E402
from matvis_b200.getz import ZPanel  # noqa: E402
from matvis_b200.matprod import B200MatMul  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu


def _spec(cfg, **kw):
    return job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True, **kw)


@pytest.mark.parametrize("sky", ["stokes", "pol"])
def test_grouped_tau_z_panels_equal_per_frequency_panels(device, sky):
    cfg = wl.subset(wl.config2(nfreq=8, ntimes=2), nsrc=5000, nfreq=5, ntimes=1, nant=70, seed=3)
    if sky == "pol":
        cfg["fluxes"] = wl.polarised_sky(cfg)
    eng = VisEngine(_spec(cfg, freq_group=5))
    eng.upload()
    eng.run()
    assert eng.fgroup == 5 and len(eng.panels) == 5
    grouped = [p.data.clone() for p in eng.panels]
    beam = eng.bmfunc.interpolated_beam
    one = ZPanel(eng.zcalc.mode, eng.nant, 2, 2, eng.cap, device)
    for f in range(5):
        one.data.zero_()
        if sky == "pol":
            _lib.check(_lib.lib.mvb_tau_z_pol(
                _lib.ptr(eng.antpos), eng.nant, float(eng.freqs[f]), _lib.ptr(eng.crd), eng.cap, _lib.ptr(eng.n_above),
                eng.cap, _lib.ptr(eng.coh[f]), _lib.ptr(eng.kept), _lib.ptr(eng.rot2), _lib.ptr(beam), beam.shape[-1],
                beam.shape[0], _lib.ptr(eng.bmfunc.beam_index_dev), eng.zcalc.mode, eng.zscale, _lib.ptr(one.data),
                one.Mpad, one.Kcap, _lib.stream_handle()))
        else:
            _lib.check(_lib.lib.mvb_tau_z(
                _lib.ptr(eng.antpos), eng.nant, float(eng.freqs[f]), _lib.ptr(eng.crd), eng.cap, _lib.ptr(eng.n_above),
                eng.cap, _lib.ptr(eng.sflux[f]), _lib.ptr(eng.kept), _lib.ptr(beam), beam.shape[-1], beam.shape[0],
                _lib.ptr(eng.bmfunc.beam_index_dev), 2, 2, eng.zcalc.mode, eng.zscale, _lib.ptr(one.data), one.Mpad,
                one.Kcap, _lib.stream_handle()))
        torch.cuda.synchronize()
        assert torch.equal(one.data, grouped[f]), f


@pytest.mark.parametrize("mode", ["fp16x3", "tf32x3"])
def test_grouped_product_matches_single_products(device, mode):
    rng = np.random.default_rng(9)
    nant, nfeed, K, G = 150, 2, 24000, 3
    mp = B200MatMul(1, nfeed, nant, None, precision=2, gemm_mode=mode, k_chunk=2048)
    mp.setup()
    panels = ZPanel.group(G, mp.mode, nant, nfeed, 1, K, device)
    zs = [rng.normal(size=(nant * nfeed, K)) + 1j * rng.normal(size=(nant * nfeed, K)) for _ in range(G)]
    # one scale for the group (the engine's panels share the job's power-of-two scale)
    scale = _lib.f16_scale(max(np.abs(z).max() for z in zs) * (1 + 2**-10)) if mode == "fp16x3" else 1.0
    singles = []
    for g in range(G):
        zt = torch.as_tensor(zs[g].astype(np.complex64), device=device)
        one = torch.zeros((nant * nant, nfeed, nfeed), dtype=torch.complex128, device=device)
        mp.compute(zt, one)
        singles.append(one.cpu().numpy())
        _lib.check(_lib.lib.mvb_z_pack(_lib.ptr(zt), 0, nant * nfeed, K, K, mp.mode, scale, _lib.ptr(panels[g].data),
                                       panels[g].Mpad, panels[g].Kcap, _lib.stream_handle()))
        panels[g].scale, panels[g].n_dev, panels[g].n_host = scale, None, K
    out = torch.zeros((G, nant * nant, nfeed, nfeed), dtype=torch.complex128, device=device)
    mp.enqueue_grouped(panels, out, k_chunk=2048)
    torch.cuda.synchronize()
    _lib.check_status_word(mp.status, "grouped product")
    got = out.cpu().numpy()
    for g in range(G):
        err = orc.cosine_error_metric(got[g], singles[g], nfeed)
        assert err <= 2e-7, (g, err)


@pytest.mark.parametrize("group", [1, 3, 8])
def test_job_with_frequency_groups_vs_oracle(device, group):
    cfg = wl.subset(wl.config2(nfreq=16, ntimes=3), nsrc=4000, nfreq=7, ntimes=2, nant=40, seed=12)
    eng = VisEngine(_spec(cfg, freq_group=group, precision=2))
    vis = eng.run().cpu().numpy()
    assert eng.fgroup == min(group, 7)
    # per time step: rotate, count, scatter, beam coordinates, beam planes, then tau/Z, product, reduce per group
    assert eng.launches_per_run() == 2 * (1 + 4 + 3 * -(-7 // eng.fgroup))
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in cfg["beams"]]
    ref = orc.simulate_vis(ants={i: tuple(p) for i, p in enumerate(cfg["antpos"])}, fluxes=cfg["fluxes"],
                           ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], lsts=cfg["lsts"],
                           latitude=cfg["latitude"], beams=beams, polarized=True, beam_idx=cfg["beam_idx"])
    err = orc.cosine_error_metric(vis, ref, 2)
    assert err <= 1e-6, err


def test_autotuner_reports_its_choice(device):
    """capture() times (k_chunk, drain interval) candidates on the job's panel and
    records the winner; the captured job still meets the parity bar."""
    from matvis_b200 import autotune

    cfg = wl.subset(wl.config2(nfreq=4, ntimes=2), nsrc=20000, nfreq=2, ntimes=1, seed=2)
    eng = VisEngine(_spec(cfg, precision=2))
    eng.upload()
    eng.run()
    autotune._cache.clear()
    eng.capture()
    t = eng.tuned
    assert t["k_chunk"] in autotune.KC_CANDIDATES and t["drain_ksteps"] in (1, 2)
    assert len(t["timed_ms"]) >= 2 and min(t["timed_ms"].values()) == t["ms"]
    vis = eng.run().cpu().numpy()
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in cfg["beams"]]
    ref = orc.simulate_vis(ants={i: tuple(p) for i, p in enumerate(cfg["antpos"])}, fluxes=cfg["fluxes"],
                           ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], lsts=cfg["lsts"],
                           latitude=cfg["latitude"], beams=beams, polarized=True, beam_idx=cfg["beam_idx"])
    assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6
    # a later, uncaptured job of the same shape (simulate_vis's path) takes the tuned choice
    again = VisEngine(_spec(cfg, precision=2))
    again.allocate()
    assert (again.k_chunk, again.matprod.drain_ksteps) == (t["k_chunk"], t["drain_ksteps"])
    assert again.tuned["cached"]
    out = again.run_to_host()
    assert orc.cosine_error_metric(out, ref, 2) <= 1e-6


def test_batched_products_of_different_shapes_equal_their_own_launches(device):
    """mvb_herk_batch over three panel groups of different shapes (rows, columns,
    panels per group) leaves in each group's workspace exactly the partial tiles
    of that group's own mvb_herk_grouped call, and the reductions agree bit for bit."""
    rng = np.random.default_rng(21)
    shapes = [(40, 2, 9000, 3), (150, 2, 24000, 1), (70, 1, 15000, 2)]  # (nant, nfeed, K, panels)
    items = []
    for nant, nfeed, K, G in shapes:
        mp = B200MatMul(1, nfeed, nant, None, precision=2, gemm_mode="fp16x3", k_chunk=2048)
        mp.setup()
        panels = ZPanel.group(G, mp.mode, nant, nfeed, 1, K, device)
        for p in panels:
            z = rng.normal(size=(nant * nfeed, K)) + 1j * rng.normal(size=(nant * nfeed, K))
            zt = torch.as_tensor(z.astype(np.complex64), device=device)
            _lib.check(_lib.lib.mvb_z_pack(_lib.ptr(zt), 0, nant * nfeed, K, K, mp.mode, 1.0, _lib.ptr(p.data),
                                           p.Mpad, p.Kcap, _lib.stream_handle()))
            p.scale, p.n_dev, p.n_host = 1.0, None, K
        items.append((mp, panels, G, nant, nfeed))
    # each group alone
    alone_ws, alone_out = [], []
    for mp, panels, G, nant, nfeed in items:
        out = torch.zeros((G, nant * nant, nfeed, nfeed), dtype=torch.complex128, device=device)
        mp.workspace(panels[0], 2048, G).zero_()
        mp.enqueue_grouped(panels, out, k_chunk=2048)
        torch.cuda.synchronize()
        alone_ws.append(mp.workspace(panels[0], 2048, G).clone())
        alone_out.append(out.cpu().numpy())
        mp.workspace(panels[0], 2048, G).zero_()
    # all three in one launch
    groups = (_lib.HerkGroup * 3)()
    for i, (mp, panels, G, _, _) in enumerate(items):
        groups[i] = mp.batch_group(panels, 2048)
    _lib.check(_lib.lib.mvb_herk_batch(_lib.c_void_p(_lib.ctypes.addressof(groups)), 3, _lib.GEMM_F16_3, 0,
                                       _lib.stream_handle()))
    for i, (mp, panels, G, nant, nfeed) in enumerate(items):
        out = torch.zeros((G, nant * nant, nfeed, nfeed), dtype=torch.complex128, device=device)
        mp.reduce_grouped(panels, out, k_chunk=2048)
        torch.cuda.synchronize()
        _lib.check_status_word(mp.status, f"batched group {i}")
        # the workspace (zeroed before either run) holds the same bytes, all but
        # its last 256: the launch's work-unit counter, which ends at a count that
        # depends on the launch (units plus CTAs)
        assert torch.equal(mp.workspace(panels[0], 2048, G)[:-256], alone_ws[i][:-256]), i
        np.testing.assert_array_equal(out.cpu().numpy(), alone_out[i])
