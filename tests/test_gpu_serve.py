"""Served form: continuous batching gives each job the same result alone and in a mix."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from matvis_b200 import workloads as wl  # noqa: E402
from matvis_b200.engine import VisEngine  # noqa: E402
from matvis_b200.serve import VisServer, latency_summary  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu


def _jobs():
    return [spec for _, spec in wl.config5_jobs(njobs=6, seed=11, nsrc_max=20000, nant_max=96)]


def test_served_results_equal_alone_and_in_mix(device):
    jobs = _jobs()
    alone = [VisEngine(s).run().cpu().numpy() for s in jobs]
    srv = VisServer(max_active=4)
    # staggered arrivals: later jobs arrive while earlier ones are on the GPU
    ids = srv.serve_stream([(0.002 * i, s) for i, s in enumerate(jobs)])
    assert srv.max_concurrent >= 2
    # the products of several jobs shared launches
    assert 0 < srv.batch_launches < srv.batched_groups
    for jid, a, s in zip(ids, alone, jobs):
        r = srv.result(jid)
        assert r.error is None
        expect = a if s.polarized else a[..., 0, 0]
        np.testing.assert_array_equal(r.vis, expect)
    summ = latency_summary(srv.results)
    assert summ["jobs"] == len(jobs) and summ["p99_s"] >= summ["p50_s"] > 0


def test_served_job_matches_oracle(device):
    spec = _jobs()[0]
    srv = VisServer()
    jid = srv.submit(spec)
    srv.run_until_idle()
    vis = srv.result(jid).vis
    ants = {i: tuple(p) for i, p in enumerate(spec.antpos)}
    ra = np.arctan2(spec.eci[1], spec.eci[0])
    dec = np.arcsin(np.clip(spec.eci[2], -1, 1))
    beams = [orc.GaussianPowerBeam(b.sigma) if hasattr(b, "sigma") else
             orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in spec.beams]
    ref = orc.simulate_vis(ants=ants, fluxes=spec.fluxes, ra=ra, dec=dec, freqs=spec.freqs, lsts=spec.lsts,
                           latitude=spec.latitude, beams=beams, polarized=spec.polarized)
    F = 2 if spec.polarized else 1
    v = vis if spec.polarized else vis[..., None, None]
    r = ref if spec.polarized else ref[..., None, None]
    assert orc.cosine_error_metric(v, r, F) <= 1e-6


def test_admission_respects_budget(device):
    jobs = _jobs()
    from matvis_b200.engine import estimate_device_bytes

    biggest = max(estimate_device_bytes(s) for s in jobs)
    srv = VisServer(hbm_budget=int(1.5 * biggest), max_active=8)
    srv.serve_stream([(0.0, s) for s in jobs])
    assert srv.peak_in_use <= srv.budget
    assert all(r.error is None for r in srv.results.values())
    with pytest.raises(ValueError, match="HBM"):
        VisServer(hbm_budget=16).submit(jobs[0])


def test_served_jobs_share_beam_and_named_sky_copies(device):
    """Polarised jobs with equal beam grids share one device copy; jobs naming the
    same sky (JobSpec.sky_key) share its directions and fluxes; results equal the
    unshared runs bit for bit."""
    from dataclasses import replace

    from matvis_b200 import devcache

    cfg = wl.subset(wl.config2(nfreq=3, ntimes=2), nsrc=4000, nfreq=3, ntimes=2, nant=30, seed=4)
    from matvis_b200.engine import job_from_arrays

    base = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True)
    plain = VisEngine(base).run().cpu().numpy()
    other_times = replace(base, lsts=base.lsts + 0.3)
    plain2 = VisEngine(other_times).run().cpu().numpy()
    e1 = VisEngine(replace(base, sky_key="sky-A"))
    e1.upload()
    e2 = VisEngine(replace(other_times, sky_key="sky-A"))
    e2.upload()
    assert e1.eci.data_ptr() == e2.eci.data_ptr() and e1.sflux.data_ptr() == e2.sflux.data_ptr()
    assert e1.bmfunc.grids.data_ptr() == e2.bmfunc.grids.data_ptr()
    np.testing.assert_array_equal(e1.run().cpu().numpy(), plain)
    np.testing.assert_array_equal(e2.run().cpu().numpy(), plain2)
    assert devcache.CACHE.hits >= 2


def test_served_results_equal_without_batched_products(device):
    """The same jobs with each job's products on its own stream (no shared
    launches) give the same visibilities bit for bit."""
    jobs = _jobs()[:4]
    a = VisServer(max_active=4)
    ia = a.serve_stream([(0.0, s) for s in jobs])
    b = VisServer(max_active=4, batch_products=False)
    ib = b.serve_stream([(0.0, s) for s in jobs])
    assert a.batch_launches > 0 and b.batch_launches == 0
    for x, y in zip(ia, ib):
        np.testing.assert_array_equal(a.result(x).vis, b.result(y).vis)


def test_served_stream_from_a_generator_without_kept_results(device):
    """A lazily built stream (config5_stream) serves every job; keep_results=False
    keeps latencies and term counts only."""
    srv = VisServer(max_active=4, keep_results=False)
    ids = srv.serve_stream(wl.config5_stream(njobs=8, seed=13, nsrc_max=20000, nant_max=96))
    assert len(ids) == 8 and srv.launches > 0
    summ = latency_summary(srv.results)
    assert summ["jobs"] == 8 and summ["terms"] > 0
    assert all(r.vis is None and r.error is None for r in srv.results.values())


def test_small_jobs_form_a_priority_class(device):
    """With one execution slot, a small job submitted after a large one is admitted
    first and runs on a high-priority stream; both results are correct."""
    from matvis_b200.serve import estimate_terms

    big, small = _jobs()[:2]
    if estimate_terms(big) < estimate_terms(small):
        big, small = small, big
    srv = VisServer(max_active=1, small_job_terms=estimate_terms(small))
    jb = srv.submit(big)
    js = srv.submit(small)
    srv.poll()
    assert [j.jid for j in srv._active + srv._finishing] == [js]
    srv.run_until_idle()
    assert srv.result(js).error is None and srv.result(jb).error is None
    assert srv.result(js).queue_s <= srv.result(jb).queue_s
    np.testing.assert_array_equal(srv.result(js).vis, (lambda a: a if small.polarized else a[..., 0, 0])(
        VisEngine(small).run().cpu().numpy()))


def test_turn_backlog_is_bounded(device):
    """With turns_ahead=1 the server never holds more than one enqueued,
    incomplete turn when it enqueues the next, and the results equal the
    unbounded server's bit for bit."""
    jobs = _jobs()[:4]
    srv = VisServer(max_active=4, turns_ahead=1)
    seen = []
    advance = srv._advance

    def watched():
        seen.append(len(srv._turns))
        advance()

    srv._advance = watched
    ia = srv.serve_stream([(0.0, s) for s in jobs])
    free = VisServer(max_active=4, turns_ahead=None)
    ib = free.serve_stream([(0.0, s) for s in jobs])
    assert seen and max(seen) <= 1
    for x, y in zip(ia, ib):
        np.testing.assert_array_equal(srv.result(x).vis, free.result(y).vis)


def test_admission_survives_out_of_memory(device, monkeypatch):
    """An allocation that runs out of device memory at admission keeps the job
    queued while others run (it is admitted once one retires), and fails only
    that job when nothing else holds memory; the server keeps serving."""
    import matvis_b200.serve as serve_mod

    jobs = _jobs()[:3]
    real = serve_mod.VisEngine.allocate
    fails = {"n": 1}  # the second job's first admission runs out

    def flaky(self):
        if getattr(self.spec, "_flaky", False) and fails["n"] > 0:
            fails["n"] -= 1
            raise torch.OutOfMemoryError("simulated")
        return real(self)

    monkeypatch.setattr(serve_mod.VisEngine, "allocate", flaky)
    jobs[1]._flaky = True
    srv = VisServer(max_active=4)
    ids = srv.serve_stream([(0.0, s) for s in jobs])
    assert srv.oom_retries == 1
    assert all(srv.result(i).error is None for i in ids)
    # alone on the device, a job that cannot be placed fails by itself
    fails["n"] = 1
    lone = VisServer(max_active=4)
    (jid,) = lone.serve_stream([(0.0, jobs[1])])
    assert lone.result(jid).error == "out of device memory at admission"
