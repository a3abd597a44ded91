"""Polarised sky on the GPU: the coherency frame rotation against the reference's
own ``calc_coherency_rotation`` / ``_rotate_frame_coherency`` outputs
(``tests/golden/coherency.npz``), and visibilities against the oracle's direct
sum V_ij = exptau_j conj(exptau_i) E_j C' E_i^H.

Tolerances: frame rotations 1e-12 absolute (FP64 trigonometry on both sides);
rotated coherencies 1e-12 relative to the largest entry; visibilities
max |dV| / sqrt(|V_ii| |V_jj|) <= 1e-6.
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
KEYS = ("eh", "em", "v", "bm1", "bpn", "eral", "xpl", "ypl", "sphi", "cphi")


def _astrom(g):
    return {k: (g[f"erfa_{k}"] if g[f"erfa_{k}"].ndim else float(g[f"erfa_{k}"])) for k in KEYS}


def _check_frame(rot, g, case, topo):
    kept = rot.kept_index[: len(g[f"{case}_above"])].cpu().numpy()
    n = int(rot.n_above.item())
    assert n == len(g[f"{case}_above"])
    np.testing.assert_array_equal(kept, g[f"{case}_above"])
    got = rot.frame_rotation[:n].cpu().numpy()  # (n, 2): cos X, sin X
    ref = g[f"{case}_rot"]
    finite = ~np.isnan(ref).any(axis=(0, 1))
    np.testing.assert_allclose(got[finite, 0], ref[0, 0, finite], rtol=0, atol=1e-12)
    np.testing.assert_allclose(got[finite, 1], ref[0, 1, finite], rtol=0, atol=1e-12)
    if (~finite).any():
        # the reference divides 0 by 0 where the two unit vectors coincide; the limit is no perturbation
        az, za = orc.enu_to_az_za(topo[0], topo[1], orientation="astropy")
        ab = g[f"{case}_above"][~finite]
        lim = orc.coherency_rotation(g["ra"][ab], g["dec"][ab], np.pi / 2 - za[ab], az[ab],
                                     orc.ENU_TO_ALTAZ @ g[f"{case}_rigid"])
        np.testing.assert_allclose(got[~finite, 0], lim[0, 0], rtol=0, atol=1e-12)
        np.testing.assert_allclose(got[~finite, 1], lim[0, 1], rtol=0, atol=1e-12)
    flux = rot.flux_above_horizon[:n].cpu().numpy()
    ref_c = g[f"{case}_rotated"]
    finite_c = ~np.isnan(ref_c).any(axis=(1, 2, 3))
    scale = np.abs(g["coherency"]).max()
    np.testing.assert_allclose(flux[finite_c], ref_c[finite_c], rtol=0, atol=1e-12 * scale)
    assert np.all(rot.flux_above_horizon[n:].cpu().numpy() == 0)


def test_frame_rotation_lst_matches_reference(device):
    g = golden("coherency")
    rot = mv.CoordinateRotationLST(flux=g["coherency"], times=np.array([float(g["lst_lst"])]),
                                   telescope_loc=float(g["lat"]), skycoords=(g["ra"], g["dec"]), source_buffer=1.0)
    rot.setup()
    rot.rotate(0)
    rot.select_chunk(0, 0)
    _check_frame(rot, g, "lst", rot.all_coords_topo.cpu().numpy())


def test_frame_rotation_erfa_matches_reference(device):
    g = golden("coherency")
    rot = mv.CoordinateRotationERFA(0.0, flux=g["coherency"], times=np.array([0.0]), telescope_loc=float(g["lat"]),
                                    skycoords=(g["ra"], g["dec"]), source_buffer=1.0, astrom=[_astrom(g)])
    rot.setup()
    rot.rotate(0)
    np.testing.assert_allclose(rot.all_coords_topo.cpu().numpy(), g["erfa_topo"], rtol=0, atol=4e-15)
    rot.select_chunk(0, 0)
    _check_frame(rot, g, "erfa", rot.all_coords_topo.cpu().numpy())


def _polarised_cfg(seed=8, nant=14, nsrc=3000):
    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=nsrc, nfreq=2, ntimes=2, nant=nant, seed=seed)
    rng = np.random.default_rng(seed)
    I = cfg["fluxes"]
    frac = rng.uniform(0, 0.8, I.shape)
    d = rng.normal(size=(3,) + I.shape)
    d /= np.linalg.norm(d, axis=0)
    q, u, v = I * frac * d
    return cfg, orc.stokes_to_coherency(I, q, u, v)


def _oracle(cfg, fluxes, **kw):
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in cfg["beams"]]
    return orc.simulate_vis(ants={i: tuple(p) for i, p in enumerate(cfg["antpos"])}, fluxes=fluxes, ra=cfg["ra"],
                            dec=cfg["dec"], freqs=cfg["freqs"], lsts=cfg["lsts"], latitude=cfg["latitude"],
                            beams=beams, polarized=True, beam_idx=cfg["beam_idx"], **kw)


def _engine(cfg, fluxes, **kw):
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=fluxes, ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True, **kw)
    return VisEngine(spec).run().cpu().numpy()


@pytest.mark.parametrize("mode", ["fp16x3", "bf16x6"])
def test_polarised_sky_vs_oracle(device, mode):
    cfg, coh = _polarised_cfg()
    ref = _oracle(cfg, coh)
    vis = _engine(cfg, coh, precision=2, gemm_mode=mode)
    assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6
    # the polarisation matters at this level
    unpol = _oracle(cfg, cfg["fluxes"])
    assert orc.cosine_error_metric(unpol, ref, 2) > 1e-3


def test_polarised_sky_erfa_frame_vs_oracle(device):
    g = golden("coherency")
    cfg, coh = _polarised_cfg(seed=11, nant=10, nsrc=2000)
    astrom = [_astrom(g), _astrom(g)]
    ref = _oracle(cfg, coh, astrom=astrom)
    vis = _engine(cfg, coh, precision=2, astrom=astrom)
    assert orc.cosine_error_metric(vis, ref, 2) <= 1e-6


def test_unpolarised_coherency_equals_scalar_flux(device):
    cfg, _ = _polarised_cfg(seed=13, nant=12, nsrc=2500)
    coh = orc.stokes_to_coherency(cfg["fluxes"], 0, 0, 0)
    a = _engine(cfg, coh, precision=2)
    b = _engine(cfg, cfg["fluxes"], precision=2)
    assert orc.cosine_error_metric(a, b, 2) <= 1e-6


def test_polarised_sky_through_simulate_vis(device):
    cfg, coh = _polarised_cfg(seed=17, nant=8, nsrc=1500)
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    vis = mv.simulate_vis(ants, coh, cfg["ra"], cfg["dec"], cfg["freqs"], cfg["lsts"], cfg["beams"], cfg["latitude"],
                          polarized=True, precision=2, beam_idx=cfg["beam_idx"])
    assert orc.cosine_error_metric(vis, _oracle(cfg, coh), 2) <= 1e-6
