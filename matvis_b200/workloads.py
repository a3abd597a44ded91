"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is used: skies, arrays and beams are generated here from
seeded ``numpy.random.default_rng(20261203 + config_id)`` streams.

* config 1: 16 antennas uniform in [-50, 50]^2 m, 2,000 isotropic sources,
  log-uniform I(150 MHz) in [0.1, 10] Jy with spectral index N(-0.8, 0.2),
  100 and 150 MHz, 4 LSTs 10 min apart at latitude -30.72 deg, achromatic
  Gaussian beam sigma = 0.2 rad, unpolarised.
* config 2 (HERA-350-like): 320 antennas on a 14.6 m hexagonal grid (the 320
  sites nearest the centre of a centre-filled hexagon) plus 30 outriggers
  uniform in a 1 km disc; 196,608 sources at the centres of an equal-area
  nside = 128 pixelisation (HEALPix ring scheme, Gorski et al. 2005, written out
  below); lognormal (sigma = 1) Stokes I; 64 frequencies over 100-200 MHz;
  16 LSTs 10 min apart; 4 polarised dipole-like beams on a 1 deg grid
  (az 0..360 inclusive, za 0..90) with a seeded 1 % complex perturbation;
  per-antenna beam_idx uniform in {0..3}.
* config 3: config 2's array and beams, 1,000,000 isotropic sources with
  N(>S) ~ S^-1.5 on [0.05, 100] Jy; a 5,000-pair sparse list.
* config 4: config 2's array and beams, 500,000 sources (flux as config 3),
  256 frequencies over 100-200 MHz x 64 LSTs over 6 h.
"""

from __future__ import annotations

import numpy as np

from .beam_models import GaussianBeam, GridBeam

SIDEREAL_DAY_S = 86164.0905
HERA_LAT = np.deg2rad(-30.72)


def rng_for(config_id: int) -> np.random.Generator:
    return np.random.default_rng(20261203 + config_id)


def healpix_ring_centres(nside: int) -> tuple[np.ndarray, np.ndarray]:
    """(ra, dec) of the 12 nside^2 equal-area pixel centres, ring ordering.

    Ring i = 1 .. 4 nside - 1:
      polar caps (i < nside, mirrored for i > 3 nside): z = 1 - i^2 / (3 nside^2),
        phi_j = pi / (2 i) (j - 1/2), j = 1 .. 4 i;
      equatorial belt: z = 4/3 - 2 i / (3 nside),
        phi_j = pi / (2 nside) (j - s / 2), s = (i - nside + 1) mod 2, j = 1 .. 4 nside.
    """
    zs, phis = [], []
    for i in range(1, 4 * nside):
        if i < nside or i > 3 * nside:
            ii = i if i < nside else 4 * nside - i
            z = 1.0 - ii * ii / (3.0 * nside * nside)
            if i > 3 * nside:
                z = -z
            j = np.arange(1, 4 * ii + 1)
            phi = np.pi / (2.0 * ii) * (j - 0.5)
        else:
            z = 4.0 / 3.0 - 2.0 * i / (3.0 * nside)
            s = (i - nside + 1) % 2
            j = np.arange(1, 4 * nside + 1)
            phi = np.pi / (2.0 * nside) * (j - s / 2.0)
        zs.append(np.full(len(j), z))
        phis.append(phi)
    z = np.concatenate(zs)
    phi = np.concatenate(phis)
    return phi, np.arcsin(z)


def hex_array(n: int, spacing: float) -> np.ndarray:
    """The n sites nearest the centre of a centre-filled hexagonal grid (x, y, 0)."""
    r = 1
    while 3 * r * (r + 1) + 1 < n:
        r += 1
    pts = []
    for q in range(-r, r + 1):
        for s in range(max(-r, -q - r), min(r, -q + r) + 1):
            x = spacing * (q + s / 2.0)
            y = spacing * (s * np.sqrt(3) / 2.0)
            pts.append((x, y))
    pts = np.array(pts)
    d = np.hypot(pts[:, 0], pts[:, 1])
    ang = np.arctan2(pts[:, 1], pts[:, 0])
    order = np.lexsort((ang, np.round(d, 6)))
    sel = pts[order[:n]]
    return np.column_stack([sel, np.zeros(n)])


def uniform_disc(rng, n: int, radius: float) -> np.ndarray:
    r = radius * np.sqrt(rng.uniform(size=n))
    th = 2 * np.pi * rng.uniform(size=n)
    return np.column_stack([r * np.cos(th), r * np.sin(th), np.zeros(n)])


def isotropic(rng, n: int) -> tuple[np.ndarray, np.ndarray]:
    ra = rng.uniform(0, 2 * np.pi, n)
    dec = np.arcsin(rng.uniform(-1, 1, n))
    return ra, dec


def powerlaw_flux(rng, n: int, smin=0.05, smax=100.0, slope=1.5) -> np.ndarray:
    """Inverse CDF of N(>S) ~ S^-slope truncated to [smin, smax]."""
    u = rng.uniform(size=n)
    a, b = smin**-slope, smax**-slope
    return (a - u * (a - b)) ** (-1.0 / slope)


def dipole_beams(rng, nbeam=4, dgrid_deg=1.0, perturb=0.01) -> list[GridBeam]:
    """Polarised dipole-like E-field grids (nax=2, nfeed=2), az 0..360 incl., za 0..90."""
    az = np.deg2rad(np.arange(0, 360 + dgrid_deg / 2, dgrid_deg))
    za = np.deg2rad(np.arange(0, 90 + dgrid_deg / 2, dgrid_deg))
    AZ, ZA = np.meshgrid(az, za, indexing="xy")
    taper = np.cos(ZA)
    # axis 0: azimuthal component, axis 1: zenith-angle component
    ex = np.array(
        [
            [-np.sin(AZ) * taper, np.cos(AZ) * taper],  # ax 0: feeds x, y
            [np.cos(ZA) * np.cos(AZ) * taper, np.cos(ZA) * np.sin(AZ) * taper],  # ax 1: feeds x, y
        ]
    )
    beams = []
    for _ in range(nbeam):
        pert = 1 + perturb * (rng.normal(size=ex.shape) + 1j * rng.normal(size=ex.shape))
        pert[..., -1] = pert[..., 0]  # 360 deg column repeats 0 deg
        beams.append(GridBeam(data=(ex * pert).astype(np.complex64), az=az, za=za, beam_type="efield"))
    return beams


def lst_grid(ntimes: int, spacing_s: float, start: float = 0.7) -> np.ndarray:
    return start + np.arange(ntimes) * 2 * np.pi * spacing_s / SIDEREAL_DAY_S


def config1():
    rng = rng_for(1)
    nant, nsrc = 16, 2000
    antpos = np.column_stack([rng.uniform(-50, 50, nant), rng.uniform(-50, 50, nant), np.zeros(nant)])
    ra, dec = isotropic(rng, nsrc)
    freqs = np.array([100e6, 150e6])
    i150 = 10 ** rng.uniform(-1, 1, nsrc)
    alpha = rng.normal(-0.8, 0.2, nsrc)
    fluxes = i150[:, None] * (freqs[None, :] / 150e6) ** alpha[:, None]
    return dict(
        antpos=antpos, ra=ra, dec=dec, fluxes=fluxes, freqs=freqs, lsts=lst_grid(4, 600.0), latitude=HERA_LAT,
        beams=[GaussianBeam(sigma=0.2)], beam_idx=None, polarized=False, antpairs=None, precision=2,
    )


def hera350(rng) -> np.ndarray:
    core = hex_array(320, 14.6)
    out = uniform_disc(rng, 30, 1000.0)
    return np.vstack([core, out])


def config2(nfreq: int = 64, ntimes: int = 16, nside: int = 128):
    rng = rng_for(2)
    antpos = hera350(rng)
    ra, dec = healpix_ring_centres(nside)
    flux0 = rng.lognormal(0.0, 1.0, len(ra))
    freqs = np.linspace(100e6, 200e6, nfreq)
    fluxes = np.repeat(flux0[:, None], nfreq, axis=1)
    beams = dipole_beams(rng, 4)
    beam_idx = rng.integers(0, 4, len(antpos))
    return dict(
        antpos=antpos, ra=ra, dec=dec, fluxes=fluxes, freqs=freqs, lsts=lst_grid(ntimes, 600.0), latitude=HERA_LAT,
        beams=beams, beam_idx=beam_idx, polarized=True, antpairs=None, precision=1,
    )


def config3(nsrc: int = 1_000_000, nfreq: int = 1, ntimes: int = 1, npairs: int = 5000):
    rng = rng_for(3)
    antpos = hera350(rng_for(2))
    beams = dipole_beams(rng_for(2), 4)
    beam_idx = rng_for(2).integers(0, 4, len(antpos))
    ra, dec = isotropic(rng, nsrc)
    flux0 = powerlaw_flux(rng, nsrc)
    freqs = np.linspace(100e6, 200e6, max(nfreq, 1)) if nfreq > 1 else np.array([150e6])
    nant = len(antpos)
    iu, ju = np.triu_indices(nant, k=1)
    pick = rng.choice(len(iu), size=npairs, replace=False)
    pairs = np.column_stack([iu[pick], ju[pick]])
    return dict(
        antpos=antpos, ra=ra, dec=dec, fluxes=np.repeat(flux0[:, None], len(freqs), axis=1), freqs=freqs,
        lsts=lst_grid(ntimes, 600.0), latitude=HERA_LAT, beams=beams, beam_idx=beam_idx, polarized=True,
        antpairs=pairs, precision=1,
    )


def config4(nsrc: int = 500_000, nfreq: int = 256, ntimes: int = 64):
    rng = rng_for(4)
    antpos = hera350(rng_for(2))
    beams = dipole_beams(rng_for(2), 4)
    beam_idx = rng_for(2).integers(0, 4, len(antpos))
    ra, dec = isotropic(rng, nsrc)
    flux0 = powerlaw_flux(rng, nsrc)
    freqs = np.linspace(100e6, 200e6, nfreq)
    lsts = 0.7 + np.linspace(0, 2 * np.pi * 6 * 3600 / SIDEREAL_DAY_S, ntimes)
    return dict(
        antpos=antpos, ra=ra, dec=dec, fluxes=np.repeat(flux0[:, None], nfreq, axis=1), freqs=freqs, lsts=lsts,
        latitude=HERA_LAT, beams=beams, beam_idx=beam_idx, polarized=True, antpairs=None, precision=1,
    )


def polarised_sky(cfg: dict, seed: int = 2, max_frac: float = 0.8) -> np.ndarray:
    """A polarised version of a workload's sky: seeded Q, U, V of random direction
    and polarised fraction uniform in [0, max_frac) of Stokes I, returned as the
    (N, Nf, 2, 2) coherency 0.5 [[I + Q, U - iV], [U + iV, I - Q]] (the
    reference's coherency convention for a polarised sky)."""
    rng = np.random.default_rng(seed)
    i = np.asarray(cfg["fluxes"], dtype=np.float64)
    frac = rng.uniform(0, max_frac, i.shape)
    d = rng.normal(size=(3,) + i.shape)
    d /= np.linalg.norm(d, axis=0)
    q, u, v = i * frac * d
    c = np.empty(i.shape + (2, 2), dtype=np.complex128)
    c[..., 0, 0] = 0.5 * (i + q)
    c[..., 1, 1] = 0.5 * (i - q)
    c[..., 0, 1] = 0.5 * (u - 1j * v)
    c[..., 1, 0] = 0.5 * (u + 1j * v)
    return c


def synthetic_astrom(lsts, latitude: float, seed: int = 3) -> list[dict]:
    """Seeded astrometry parameters of the ERFA apparent-place step, one dict per
    time (the fields of ERFA's ASTROM structure that the rotation uses): Earth's
    heliocentric direction eh at 1 AU (em), its barycentric velocity v (|v| = 1e-4
    c, perpendicular to eh) with bm1 = sqrt(1 - v^2), a bias-precession-nutation
    matrix bpn 0.35 deg from the identity (about 25 years of precession), polar
    motion of 1 microradian, the Earth rotation angle eral = the LST, and the
    site latitude.  Stand-ins for the caller's astropy-derived values, for timing."""
    rng = np.random.default_rng(seed)
    lam, eps = rng.uniform(0, 2 * np.pi), np.deg2rad(23.44)
    eh = np.array([np.cos(lam), np.sin(lam) * np.cos(eps), np.sin(lam) * np.sin(eps)])
    v = 1e-4 * np.array([-np.sin(lam), np.cos(lam) * np.cos(eps), np.cos(lam) * np.sin(eps)])
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    ang = np.deg2rad(0.35)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    bpn = np.eye(3) + np.sin(ang) * k + (1 - np.cos(ang)) * (k @ k)
    base = dict(eh=eh, em=1.0, v=v, bm1=float(np.sqrt(1 - v @ v)), bpn=bpn, xpl=1e-6, ypl=-1e-6,
                sphi=float(np.sin(latitude)), cphi=float(np.cos(latitude)))
    return [dict(base, eral=float(l)) for l in np.asarray(lsts, dtype=np.float64)]


def subset(cfg: dict, nsrc: int | None = None, nfreq: int | None = None, ntimes: int | None = None,
           nant: int | None = None, seed: int = 0) -> dict:
    """A smaller seeded slice of a configuration (for oracle-checkable tests)."""
    c = dict(cfg)
    rng = np.random.default_rng(seed)
    if nsrc is not None and nsrc < len(c["ra"]):
        pick = np.sort(rng.choice(len(c["ra"]), size=nsrc, replace=False))
        c["ra"], c["dec"], c["fluxes"] = c["ra"][pick], c["dec"][pick], c["fluxes"][pick]
    if nfreq is not None and nfreq < len(c["freqs"]):
        fi = np.sort(rng.choice(len(c["freqs"]), size=nfreq, replace=False))
        c["freqs"], c["fluxes"] = c["freqs"][fi], c["fluxes"][:, fi]
    if ntimes is not None and ntimes < len(c["lsts"]):
        ti = np.sort(rng.choice(len(c["lsts"]), size=ntimes, replace=False))
        c["lsts"] = c["lsts"][ti]
    if nant is not None and nant < len(c["antpos"]):
        c["antpos"] = c["antpos"][:nant]
        if c.get("beam_idx") is not None:
            c["beam_idx"] = np.asarray(c["beam_idx"])[:nant]
        if c.get("antpairs") is not None:
            ap = np.asarray(c["antpairs"])
            c["antpairs"] = ap[(ap[:, 0] < nant) & (ap[:, 1] < nant)]
    return c


def config5_jobs(njobs: int = 2000, rate_hz: float = 20.0, seed: int = 5, nsrc_max: int = 500_000,
                 nant_max: int = 512):
    """The config-5 stream as a list (see ``config5_stream``)."""
    return list(config5_stream(njobs, rate_hz, seed, nsrc_max, nant_max))


def config5_stream(njobs: int = 2000, rate_hz: float = 20.0, seed: int = 5, nsrc_max: int = 500_000,
                   nant_max: int = 512):
    """Served-form stream: Poisson arrivals (rate_hz), per job Nant log-uniform in
    [16, nant_max] (positions uniform in a 300 m disc), Nsrc log-uniform in
    [1e3, nsrc_max] isotropic with N(>S) ~ S^-1.5 fluxes, Nfreq U{1..32},
    Ntimes U{1..16}, beam either the unpolarised Gaussian or config 2's polarised
    grid.  Yields (arrival_s, JobSpec) in arrival order, building each job only
    when it is asked for."""
    from .engine import JobSpec
    from .coordinates import point_source_crd_eq

    rng = rng_for(seed)
    grid_beams = dipole_beams(rng_for(2), 1)
    t = 0.0
    for _ in range(njobs):
        t += rng.exponential(1.0 / rate_hz)
        nant = int(round(np.exp(rng.uniform(np.log(16), np.log(nant_max)))))
        nsrc = int(round(np.exp(rng.uniform(np.log(1000), np.log(nsrc_max)))))
        nf = int(rng.integers(1, 33))
        nt = int(rng.integers(1, 17))
        pol = bool(rng.integers(0, 2))
        antpos = uniform_disc(rng, nant, 300.0)
        ra, dec = isotropic(rng, nsrc)
        flux = powerlaw_flux(rng, nsrc)
        freqs = np.sort(rng.uniform(100e6, 200e6, nf))
        lsts = rng.uniform(0, 2 * np.pi) + np.arange(nt) * 2 * np.pi * 600 / SIDEREAL_DAY_S
        spec = JobSpec(antpos=antpos, eci=point_source_crd_eq(ra, dec), fluxes=np.repeat(flux[:, None], nf, axis=1),
                       freqs=freqs, lsts=lsts, latitude=HERA_LAT,
                       beams=grid_beams if pol else [GaussianBeam(sigma=0.2)], polarized=pol, precision=1)
        yield t, spec
