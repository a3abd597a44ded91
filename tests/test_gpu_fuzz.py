"""Seeded randomized parity: many small jobs through ``simulate_vis`` against the
FP64 oracle, drawn across the shapes the kernels branch on -- antenna counts on
both sides of the 64- and 128-row block boundaries, one or two feeds, empty and
non-empty skies, every split mode, both products (MatMul, VectorDot with a
random pair list on either pair kernel), source chunking, complex64 and
complex128 output, gridded and Gaussian beams, Stokes-I and polarised
(coherency) skies, the LST rotation and the ERFA-style apparent place.

Tolerance: max |dV| / sqrt(|V_ii| |V_jj|) <= 1e-6 (3e-5 for the bf16x3 split,
which is not held to 1e-6 anywhere).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import matvis_b200 as mv  # noqa: E402
from matvis_b200 import workloads as wl  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = 48


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    nant = int(rng.choice([1, 2, 7, 32, 33, 63, 64, 65, 100, 128, 129, 140]))
    polarized = bool(rng.integers(0, 2))
    nsrc = int(rng.choice([0, 1, 50, 700, 3000]))
    nfreq, ntimes = int(rng.integers(1, 4)), int(rng.integers(1, 4))
    mode = str(rng.choice(["fp16x3", "bf16x6", "tf32x3", "bf16x3"]))
    matprod = str(rng.choice(["MatMul", "VectorDot"]))
    pair_kernel = str(rng.choice(["auto", "vecdot", "herk"]))
    use_pairs = matprod == "VectorDot" or bool(rng.integers(0, 2))
    nchunks = int(rng.integers(1, 4))
    precision = int(rng.integers(1, 3))
    antpos = np.column_stack([rng.uniform(-200, 200, nant), rng.uniform(-200, 200, nant), np.zeros(nant)])
    ra, dec = wl.isotropic(rng, nsrc)
    freqs = np.sort(rng.uniform(100e6, 200e6, nfreq))
    fluxes = wl.powerlaw_flux(rng, nsrc)[:, None] * (freqs / 150e6)[None, :] ** -0.8
    lsts = np.sort(rng.uniform(0, 2 * np.pi, ntimes))
    if polarized or rng.integers(0, 2):
        beams = wl.dipole_beams(rng, 2, dgrid_deg=2.0)
        beam_idx = rng.integers(0, 2, nant)
    else:
        beams, beam_idx = [mv.GaussianBeam(sigma=float(rng.uniform(0.15, 0.4)))], None
    if polarized and rng.integers(0, 2):
        fluxes = wl.polarised_sky({"fluxes": fluxes}, seed=seed)
    rotation = {}
    if rng.integers(0, 2):
        time_s = np.sort(rng.uniform(0, 3600, ntimes))
        rotation = dict(astrom=wl.synthetic_astrom(lsts, -0.536, seed=seed), time_s=time_s,
                        update_bcrs_every=float(rng.choice([0.0, 300.0])))
    pairs = None
    if use_pairs:
        npairs = int(rng.integers(1, max(2, nant * nant // 3)))
        pairs = np.column_stack([rng.integers(0, nant, npairs), rng.integers(0, nant, npairs)])
    return dict(antpos=antpos, ra=ra, dec=dec, freqs=freqs, fluxes=fluxes, lsts=lsts, beams=beams, beam_idx=beam_idx,
                polarized=polarized, mode=mode, matprod=matprod, pair_kernel=pair_kernel, pairs=pairs,
                nchunks=nchunks, precision=precision, rotation=rotation)


def _oracle_beams(beams):
    return [orc.GaussianPowerBeam(sigma=b.sigma) if isinstance(b, mv.GaussianBeam)
            else orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in beams]


@pytest.mark.parametrize("seed", range(CASES))
def test_random_job_vs_oracle(device, seed):
    c = _case(seed)
    ants = {i: tuple(p) for i, p in enumerate(c["antpos"])}
    latitude = -0.536
    rot_kw = {}
    if c["rotation"]:
        rot_kw = dict(coord_method="CoordinateRotationERFA", coord_method_params=c["rotation"])
    vis = mv.simulate_vis(ants, c["fluxes"], c["ra"], c["dec"], c["freqs"], c["lsts"], c["beams"], latitude,
                          polarized=c["polarized"], precision=c["precision"], beam_idx=c["beam_idx"],
                          antpairs=c["pairs"], matprod_method=c["matprod"], pair_product=c["pair_kernel"],
                          gemm_mode=c["mode"], min_chunks=c["nchunks"], **rot_kw)
    ref = orc.simulate_vis(ants=ants, fluxes=c["fluxes"], ra=c["ra"], dec=c["dec"], freqs=c["freqs"], lsts=c["lsts"],
                           latitude=latitude, beams=_oracle_beams(c["beams"]), polarized=c["polarized"],
                           beam_idx=c["beam_idx"], antpairs=c["pairs"], matprod="VectorDot" if c["pairs"] is not None
                           else "MatMul", **c["rotation"])
    assert vis.shape == ref.shape, (vis.shape, ref.shape)
    if len(c["ra"]) == 0:
        assert np.all(vis == 0)
        return
    # the metric normalises by the autocorrelations: take them from an all-pairs oracle run
    full = ref if c["pairs"] is None else orc.simulate_vis(
        ants=ants, fluxes=c["fluxes"], ra=c["ra"], dec=c["dec"], freqs=c["freqs"], lsts=c["lsts"], latitude=latitude,
        beams=_oracle_beams(c["beams"]), polarized=c["polarized"], beam_idx=c["beam_idx"], **c["rotation"])
    nfeed = 2 if c["polarized"] else 1
    nant = len(c["antpos"])
    v4 = vis if c["polarized"] else vis[..., None, None]
    r4 = ref if c["polarized"] else ref[..., None, None]
    f4 = full if c["polarized"] else full[..., None, None]
    autos = f4.reshape(f4.shape[:2] + (nant, nant, nfeed, nfeed))[:, :, np.arange(nant), np.arange(nant)]
    auto_mag = np.abs(np.diagonal(autos, axis1=-2, axis2=-1))  # (Nf, Nt, nant, nfeed)
    pairs = c["pairs"] if c["pairs"] is not None else np.array([(i, j) for i in range(nant) for j in range(nant)])
    ai, aj = pairs[:, 0], pairs[:, 1]
    # out[pair, p, q] pairs feed q of antenna ai with feed p of antenna aj
    norm = np.sqrt(auto_mag[:, :, ai, None, :] * auto_mag[:, :, aj, :, None])
    err = np.abs(v4 - r4)
    scale = np.where(norm > 0, norm, 1.0)
    worst = float(np.max(np.where(norm > 0, err / scale, err)))
    tol = 3e-5 if c["mode"] == "bf16x3" else 1e-6
    assert worst <= tol, (seed, worst, {k: v for k, v in c.items() if k in ("mode", "matprod", "pair_kernel",
                                                                            "nchunks", "precision", "polarized")},
                          "erfa" if c["rotation"] else "lst", np.ndim(c["fluxes"]))
