"""Edge cases through simulate_vis / the engine against the oracle: an empty sky,
one antenna, times with every source below the horizon (zeros, as the CPU
driver gives them, cpu/cpu.py:249-253), and pair lists with i > j."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import matvis_b200 as mv  # noqa: E402
from matvis_b200 import workloads as wl  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu


def _sim(cfg, **kw):
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    return mv.simulate_vis(ants, cfg["fluxes"], cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], cfg["beams"],
                           cfg["latitude"], polarized=cfg["polarized"], precision=2, beam_idx=cfg.get("beam_idx"),
                           **kw)


def _ref(cfg, **kw):
    beams = []
    for b in cfg["beams"]:
        beams.append(orc.GaussianPowerBeam(sigma=b.sigma) if isinstance(b, mv.GaussianBeam)
                     else orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za))
    return orc.simulate_vis(ants={i: tuple(p) for i, p in enumerate(cfg["antpos"])}, fluxes=cfg["fluxes"],
                            ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], lsts=cfg["lsts"],
                            latitude=cfg["latitude"], beams=beams, polarized=cfg["polarized"],
                            beam_idx=cfg.get("beam_idx"), **kw)


@pytest.mark.parametrize("matprod", ["MatMul", "VectorDot"])
def test_empty_sky_gives_zeros(device, matprod):
    cfg = wl.config1()
    cfg.update(ra=np.zeros(0), dec=np.zeros(0), fluxes=np.zeros((0, len(cfg["freqs"]))))
    vis = _sim(cfg, matprod_method=matprod)
    assert vis.shape == (len(cfg["freqs"]), len(cfg["lsts"]), 16 * 16)
    assert np.all(vis == 0)


@pytest.mark.parametrize("matprod", ["MatMul", "VectorDot"])
def test_single_antenna(device, matprod):
    """One antenna: the autocorrelation, real as conj(z) z is in the reference."""
    cfg = wl.config1()
    cfg["antpos"] = cfg["antpos"][:1]
    vis = _sim(cfg, matprod_method=matprod)
    ref = _ref(cfg)
    assert vis.shape == ref.shape == (2, 4, 1)
    np.testing.assert_allclose(vis, ref, rtol=1e-6, atol=0)
    assert np.all(vis.imag == 0) and np.all(vis.real > 0)


def test_times_with_no_source_above_horizon(device):
    """Sources near the south celestial pole seen from +60 deg latitude: never up."""
    cfg = wl.config1()
    n = 500
    rng = np.random.default_rng(2)
    cfg.update(ra=rng.uniform(0, 2 * np.pi, n), dec=np.deg2rad(rng.uniform(-89, -45, n)),
               fluxes=np.ones((n, len(cfg["freqs"]))), latitude=np.deg2rad(60.0))
    for matprod in ("MatMul", "VectorDot"):
        assert np.all(_sim(cfg, matprod_method=matprod) == 0)


@pytest.mark.parametrize("matprod,kernel", [("MatMul", "auto"), ("VectorDot", "vecdot"), ("VectorDot", "herk")])
def test_pairs_in_both_orders(device, matprod, kernel):
    """antpairs with i < j, i > j and i == j (cpu/matprod.py:21-30 gathers [i, j] as given),
    a VectorDot request on either pair kernel."""
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=3000, nfreq=1, ntimes=2, nant=20, seed=21)
    pairs = np.array([(0, 5), (5, 0), (3, 3), (19, 2), (2, 19), (7, 12), (12, 7), (0, 19)])
    vis = _sim(cfg, antpairs=pairs, matprod_method=matprod, pair_product=kernel)
    ref = _ref(cfg, antpairs=pairs, matprod="VectorDot")
    scale = np.abs(_ref(cfg)).max()
    np.testing.assert_allclose(vis, ref, rtol=0, atol=1e-6 * scale)
    # V_ji = V_ij^H, and the one-feed autocorrelations of (3, 3) are real
    np.testing.assert_allclose(vis[:, :, 1], np.conj(np.swapaxes(vis[:, :, 0], -1, -2)), rtol=0, atol=1e-6 * scale)
    assert np.all(vis[:, :, 2, 0, 0].imag == 0) and np.all(vis[:, :, 2, 1, 1].imag == 0)


@pytest.mark.parametrize("polarized", [True, False])
def test_nonfinite_beam_raises_the_reference_error(device, polarized):
    """A NaN in a beam grid that the sources sample makes simulate_vis raise the
    reference's ValueError (core/beams.py:202-206), from the kernel's status word."""
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=2000, nfreq=1, ntimes=1, nant=8, seed=5)
    bad = cfg["beams"][0].data.copy()
    bad[:, :, :30, :] = np.nan  # zenith angles 0..29 deg: every beam axis and feed
    cfg["beams"] = [mv.GridBeam(data=bad, az=cfg["beams"][0].az, za=cfg["beams"][0].za)] + list(cfg["beams"][1:])
    cfg["beam_idx"] = np.zeros(8, dtype=int)
    cfg["polarized"] = polarized
    with pytest.raises(ValueError, match="Beam interpolation resulted in an invalid value"):
        _sim(cfg)
    # the same job on the intact beam still runs on this device afterwards
    cfg["beams"] = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=2000, nfreq=1, ntimes=1, nant=8, seed=5)["beams"]
    vis = _sim(cfg)
    assert np.all(np.isfinite(vis))
