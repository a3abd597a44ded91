"""Generate the golden fixtures in this directory from the reference's own code.

Run from the repository root with the reference tree present::

    python tests/golden/make_golden.py --reference-root <path to the matvis project>

(or set MATVIS_REFERENCE_ROOT).  ``NF_HERA_Dipole_small.fits`` beside the
fixtures is the reference's own beam file (``src/matvis/data``), copied as is
for the beamfits reader tests.

It loads the reference modules through ``refload`` (inert stand-ins replace the
absent astropy / pyuvdata / cupy) and records, for seeded inputs, what the
reference functions return:

* ``matprod.npz``   -- ``CPUMatMul`` / ``CPUVectorDot`` on the known-answer Z of
  ``tests/test_matprod.py:45-65`` and on a seeded random Z;
* ``bilinear.npz``  -- ``gpu_beam_interpolation`` (``gpu/beams.py:127-200``) on the
  grids of ``tests/test_beam_interp_gpu.py:12-64`` and on seeded random grids;
* ``coords.npz``    -- ``point_source_crd_eq``, ``eci_to_enu_matrix``,
  ``enu_to_az_za`` and ``CoordinateRotation.select_chunk``;
* ``tauz.npz``      -- ``TauCalculator`` and ``ZMatrixCalc``;
* ``chunks.npz``    -- ``get_required_chunks`` over a parameter grid;
* ``pipeline.npz``  -- end-to-end visibilities from the reference plugin classes
  driven in the loop order of ``cpu/cpu.py:247-272``;
* ``erfa.npz``      -- ``CoordinateRotationERFA._ld / _ab / _bpn / _atioq``
  (``cpu/coords.py:89-181``) on seeded unit vectors and astrom parameters;
* ``coherency.npz`` -- ``calc_coherency_rotation`` (``coordinates.py:288-330``,
  with ``vecs2rot``, ``axis_angle_rotation_matrix``,
  ``spherical_basis_vector_rotation_matrix``, ``theta_hat``, ``phi_hat``) and
  ``CoordinateRotation._rotate_frame_coherency`` (``core/coords.py:152-175``) on
  seeded sources, for the rigid LST frame and for the ERFA apparent-place frame;
  the astropy-derived average rotation ``_calc_average_rotation_matrix`` is
  replaced by the frame's rigid 3x3 (ICRS -> alt/az cartesian, x north, y east);
* ``redundancies.npz`` -- ``get_redundancies`` (``cli.py:273-290``) on hexagonal,
  jittered, random and co-located antenna layouts.  ``cli.py`` imports click,
  astropy, line_profiler and pyuvdata at module level, so only that function's
  source is compiled (it needs numpy alone).

The fixtures are small (< 1 MB) and committed; the tests never read the
reference tree.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import refload  # noqa: E402

if "--reference-root" in sys.argv:
    refload.set_reference_root(sys.argv[sys.argv.index("--reference-root") + 1])
ref = refload.load_reference()


def _save(name, **arrays):
    path = HERE / name
    np.savez_compressed(path, **arrays)
    print(f"wrote {path.name}: {sorted(arrays)}")


# ---------------------------------------------------------------------------
def make_matprod():
    out = {}
    for method in ("CPUMatMul", "CPUVectorDot"):
        cls = getattr(ref.cpu_matprod, method)
        for nfeed in (1, 2):
            for precision in (1, 2):
                for explicit in (True, False):
                    for nchunks in (1, 2):
                        nant, nsrc = 5, 15
                        antpairs = np.array([(i, j) for i in range(nant) for j in range(nant)]) if explicit else None
                        obj = cls(nchunks=nchunks, nfeed=nfeed, nant=nant, antpairs=antpairs, precision=precision)
                        obj.setup()
                        ctype = ref.utils.get_dtypes(precision)[1]
                        z = np.arange(nfeed * nant * nsrc, dtype=ctype).reshape((nfeed * nant, nsrc)) + 1j
                        res = np.zeros((obj.npairs, nfeed, nfeed), dtype=ctype)
                        obj(z, chunk=0)
                        obj.sum_chunks(res)
                        key = f"arange_{method}_f{nfeed}_p{precision}_e{int(explicit)}_c{nchunks}"
                        out[key] = res
    # seeded random Z with a sparse pair list, both methods, precision 2
    rng = np.random.default_rng(20261203)
    nant, nfeed, nax, nsrc = 7, 2, 2, 40
    z = rng.normal(size=(nant * nfeed, nax * nsrc)) + 1j * rng.normal(size=(nant * nfeed, nax * nsrc))
    pairs = np.array([(0, 1), (3, 2), (6, 6), (1, 0), (5, 4), (2, 6)])
    out["random_z"] = z
    out["random_pairs"] = pairs
    for method in ("CPUMatMul", "CPUVectorDot"):
        for name, ap in (("all", None), ("sparse", pairs)):
            obj = getattr(ref.cpu_matprod, method)(nchunks=1, nfeed=nfeed, nant=nant, antpairs=ap, precision=2)
            obj.setup()
            res = np.zeros((obj.npairs, nfeed, nfeed), dtype=complex)
            obj(z, chunk=0)
            obj.sum_chunks(res)
            out[f"random_{method}_{name}"] = res
    _save("matprod.npz", **out)


# ---------------------------------------------------------------------------
def make_bilinear():
    g = ref.gpu_beams.gpu_beam_interpolation
    out = {}
    # tests/test_beam_interp_gpu.py:12-35 (identity at nodes)
    za = np.linspace(0, 1, 3)
    az = np.linspace(0, 2 * np.pi, 6)
    AZ, ZA = np.meshgrid(az, za, indexing="xy")
    beam = np.array([1 - ZA**2, 2 - ZA**2 + np.sin(AZ)])[:, None, None]
    dza, daz = za[1] - za[0], az[1] - az[0]
    out["ident_beam"] = beam
    out["ident_params"] = np.array([[daz, dza, 0.0]] * 2)
    out["ident_az"] = AZ.flatten()
    out["ident_za"] = ZA.flatten()
    out["ident_out"] = np.asarray(g(beam, [daz] * 2, [dza] * 2, [0.0] * 2, AZ.flatten(), ZA.flatten()))
    # tests/test_beam_interp_gpu.py:38-64 (linear beam on a 2x-decimated grid)
    za = np.linspace(0, 1, 5)
    az = np.linspace(0, 1, 5)
    AZ, ZA = np.meshgrid(az, za, indexing="xy")
    beam = np.array([1 - ZA])[:, None, None]
    dec_beam = beam[:, :, :, ::2][..., ::2]
    dza, daz = za[1] - za[0], az[1] - az[0]
    out["lin_beam"] = dec_beam
    out["lin_params"] = np.array([[daz * 2, dza * 2, 0.0]])
    out["lin_az"] = AZ.flatten()
    out["lin_za"] = ZA.flatten()
    out["lin_out"] = np.asarray(g(dec_beam, [daz * 2], [dza * 2], [0.0], AZ.flatten(), ZA.flatten()))
    out["lin_truth"] = np.sqrt(beam[:, 0, 0].reshape(1, -1))
    # seeded complex polarised grids, points inside and outside the grid
    rng = np.random.default_rng(7)
    nbeam, nax, nfeed, nza, naz = 2, 2, 2, 10, 13
    cgrid = rng.normal(size=(nbeam, nax, nfeed, nza, naz)) + 1j * rng.normal(size=(nbeam, nax, nfeed, nza, naz))
    params = np.array([[0.5, 0.17, 0.0], [0.5, 0.17, 0.0]])
    paz = np.concatenate([rng.uniform(0, 0.5 * (naz - 1), 300), [0.0, 0.5 * (naz - 1), -1e-9, 0.5 * (naz - 1) + 1e-9, 1.0, 2.0]])
    pza = np.concatenate([rng.uniform(0, 0.17 * (nza - 1), 300), [0.0, 0.17 * (nza - 1), 0.3, 0.3, -1e-9, 0.17 * (nza - 1) + 1e-9]])
    out["cplx_beam"] = cgrid
    out["cplx_params"] = params
    out["cplx_az"] = paz
    out["cplx_za"] = pza
    out["cplx_out"] = np.asarray(g(cgrid, params[:, 0], params[:, 1], params[:, 2], paz, pza))
    # seeded real power grid with non-zero azmin
    pgrid = rng.uniform(0.1, 1.0, size=(1, 1, 1, 12, 20))
    pp = np.array([[0.3, 0.13, 0.2]])
    qaz = rng.uniform(0.1, 0.2 + 0.3 * 19 + 0.1, 200)
    qza = rng.uniform(0.0, 0.13 * 11 + 0.05, 200)
    out["pow_beam"] = pgrid
    out["pow_params"] = pp
    out["pow_az"] = qaz
    out["pow_za"] = qza
    out["pow_out"] = np.asarray(g(pgrid, pp[:, 0], pp[:, 1], pp[:, 2], qaz, qza))
    _save("bilinear.npz", **out)


# ---------------------------------------------------------------------------
class _LSTRotation(ref.core_coords.CoordinateRotation):
    """Reference horizon selection fed by the rigid LST rotation of the reference tests."""

    def __init__(self, lsts, lat, eci, **kw):
        super().__init__(**kw)
        self._lsts = lsts
        self._lat = lat
        self._eci = eci

    def rotate(self, t):
        m = ref.coordinates.eci_to_enu_matrix(self._lsts[t], self._lat)
        self.all_coords_topo[:] = np.dot(m, self._eci)


def make_coords():
    c = ref.coordinates
    out = {}
    rng = np.random.default_rng(11)
    ra = np.concatenate([np.array([0.0, 45.0, 90.0, 135.0, 180.0, 270.0, 360.0]) * np.pi / 180, rng.uniform(0, 2 * np.pi, 50)])
    dec = np.concatenate([np.array([90.0, -90.0, 0.0, 30.0, -30.0, 10.0, -89.0]) * np.pi / 180, np.arcsin(rng.uniform(-1, 1, 50))])
    out["crd_ra"] = ra
    out["crd_dec"] = dec
    out["crd_eq"] = np.asarray(c.point_source_crd_eq(ra, dec))
    hl = np.array([[0.0, -0.5361], [1.3, 0.2], [4.0, -1.2], [2 * np.pi, 0.0], [-0.7, 0.9]])
    out["mat_hl"] = hl
    out["mat_eci_to_enu"] = np.array([c.eci_to_enu_matrix(h, l) for h, l in hl])
    out["mat_enu_to_eci"] = np.array([c.enu_to_eci_matrix(h, l) for h, l in hl])
    e = np.concatenate([rng.uniform(-1, 1, 200) * 0.7, [1.0, 0.0, 0.0, 0.0, 0.6]])
    n = np.concatenate([rng.uniform(-1, 1, 200) * 0.7, [0.0, 1.0, 0.0, -1.0, 0.8]])
    out["azza_e"] = e
    out["azza_n"] = n
    for orient in ("astropy", "uvbeam"):
        az, za = c.enu_to_az_za(e, n, orientation=orient)
        out[f"azza_{orient}_az"] = az
        out[f"azza_{orient}_za"] = za
    az, za = c.enu_to_az_za(e, n, orientation="uvbeam", periodic_azimuth=False)
    out["azza_uvbeam_nonperiodic_az"] = az
    # select_chunk on a 3,000-source sky in 2 chunks (exercises the source_buffer rule)
    nsrc = 3000
    sra = rng.uniform(0, 2 * np.pi, nsrc)
    sdec = np.arcsin(rng.uniform(-1, 1, nsrc))
    eci = np.asarray(c.point_source_crd_eq(sra, sdec))
    flux = np.sqrt(0.5 * rng.uniform(0.1, 10, nsrc))
    lsts = np.array([0.1, 2.0, 4.5])
    lat = np.deg2rad(-30.72)
    rot = _LSTRotation(
        lsts, lat, eci, flux=flux, times=lsts, telescope_loc=None, skycoords=np.zeros(nsrc), chunk_size=1500, source_buffer=0.7, precision=2
    )
    rot.setup()
    out["sel_eci"] = eci
    out["sel_flux"] = flux
    out["sel_lsts"] = lsts
    out["sel_lat"] = np.array(lat)
    out["sel_chunk_size"] = np.array(1500)
    out["sel_alloc"] = np.array(rot.nsrc_alloc)
    for t in range(len(lsts)):
        rot.rotate(t)
        out[f"sel_topo_t{t}"] = rot.all_coords_topo.copy()
        for ch in range(2):
            crd, fl, nn = rot.select_chunk(ch, t)
            out[f"sel_n_t{t}_c{ch}"] = np.array(nn)
            out[f"sel_crd_t{t}_c{ch}"] = crd[:, :nn].copy()
            out[f"sel_flux_t{t}_c{ch}"] = fl.copy()
    _save("coords.npz", **out)


# ---------------------------------------------------------------------------
def make_tauz():
    out = {}
    rng = np.random.default_rng(5)
    nant, nsrc = 6, 25
    antpos = np.column_stack([rng.uniform(-500, 500, nant), rng.uniform(-500, 500, nant), rng.uniform(-2, 2, nant)])
    crd = rng.normal(size=(3, nsrc))
    crd /= np.linalg.norm(crd, axis=0)
    freq = 173.25e6
    tc = ref.core_tau.TauCalculator(antpos=antpos, freq=freq, nsrc=nsrc, precision=2)
    tc.setup()
    ext = tc(crd).copy()
    out["antpos"] = antpos
    out["crd"] = crd
    out["freq"] = np.array(freq)
    out["exptau"] = ext
    sqrt_flux = rng.uniform(0.1, 3.0, nsrc)
    nbeam, nfeed, nax = 3, 2, 2
    beam = rng.normal(size=(nbeam, nfeed, nax, nsrc)) + 1j * rng.normal(size=(nbeam, nfeed, nax, nsrc))
    beam_idx = np.array([2, 0, 1, 1, 0, 2])
    zc = ref.core_getz.ZMatrixCalc(nant=nant, nfeed=nfeed, nax=nax, nsrc=nsrc, ctype=np.complex128)
    zc.setup()
    out["sqrt_flux"] = sqrt_flux
    out["beam"] = beam
    out["beam_idx"] = beam_idx
    out["z"] = zc(sqrt_flux, beam, ext.copy(), beam_idx).copy()
    zc1 = ref.core_getz.ZMatrixCalc(nant=nant, nfeed=1, nax=1, nsrc=nsrc, ctype=np.complex128)
    zc1.setup()
    b1 = beam[:1, :1, :1]
    out["beam1"] = b1
    out["z1"] = zc1(sqrt_flux, b1, ext.copy(), None).copy()
    _save("tauz.npz", **out)


# ---------------------------------------------------------------------------
def make_chunks():
    rows = []
    for freemem in (2**20, 2**26, 2**30, 2**34):
        for nant in (16, 350):
            for nsrc in (2000, 196608, 1000000):
                for pol in (False, True):
                    nax = nfeed = 2 if pol else 1
                    for precision in (1, 2):
                        for sb in (1.0, 0.55):
                            ch = ref.utils.get_required_chunks(freemem, nax, nfeed, nant, nsrc, 4, 91 * 361 * 4, precision, sb, 0.9)
                            rows.append([freemem, nax, nfeed, nant, nsrc, 4, 91 * 361 * 4, precision, sb, 0.9, ch])
    _save("chunks.npz", table=np.array(rows, dtype=np.float64))


# ---------------------------------------------------------------------------
def _reference_pipeline(antpos, freq, lsts, lat, ra, dec, I_sky, grids, grid_params, beam_idx, polarized, antpairs, nchunks, method, gauss_sigma=None):
    """Reference plugin classes in the loop order of cpu/cpu.py:247-272."""
    c = ref.coordinates
    nant = len(antpos)
    nfeed = nax = 2 if polarized else 1
    nsrc = len(I_sky)
    eci = np.asarray(c.point_source_crd_eq(ra, dec))
    chunk_size = int(np.ceil(nsrc / nchunks))
    rot = _LSTRotation(
        lsts,
        lat,
        eci,
        flux=np.sqrt(0.5 * I_sky),
        times=np.asarray(lsts),
        telescope_loc=None,
        skycoords=np.zeros(nsrc),
        chunk_size=chunk_size,
        source_buffer=1.0,
        precision=2,
    )
    rot.setup()
    alloc = rot.nsrc_alloc
    nbeam = len(grids) if grids is not None else 1
    taucalc = ref.core_tau.TauCalculator(antpos=antpos, freq=freq, nsrc=alloc, precision=2)
    taucalc.setup()
    zcalc = ref.core_getz.ZMatrixCalc(nant=nant, nfeed=nfeed, nax=nax, nsrc=alloc, ctype=np.complex128)
    zcalc.setup()
    mp = getattr(ref.cpu_matprod, method)(nchunks, nfeed, nant, antpairs, precision=2)
    mp.setup()
    vis = np.zeros((len(lsts), mp.npairs, nfeed, nfeed), dtype=complex)
    for t in range(len(lsts)):
        rot.rotate(t)
        for ch in range(nchunks):
            crd, flux, nn = rot.select_chunk(ch, t)
            az, za = c.enu_to_az_za(crd[0], crd[1], orientation="uvbeam")
            if grids is None:
                beam = np.zeros((1, 1, 1, alloc), dtype=complex)
                beam[0, 0, 0] = np.exp(-(za**2) / (2 * gauss_sigma**2))
            else:
                beam = np.zeros((nbeam, nfeed, nax, alloc), dtype=complex)
                ref.gpu_beams.gpu_beam_interpolation(grids, grid_params[:, 0], grid_params[:, 1], grid_params[:, 2], az, za, beam_at_src=beam)
            ext = taucalc(crd)
            z = zcalc(flux, beam, ext, beam_idx)
            mp(z, ch)
        mp.sum_chunks(vis[t])
    return vis if polarized else vis[:, :, 0, 0]


def make_pipeline():
    out = {}
    rng = np.random.default_rng(20261204)
    # (a) unpolarised, analytic Gaussian (sigma 0.2 rad), 16 antennas, 300 sources
    nant, nsrc = 16, 300
    antpos = np.column_stack([rng.uniform(-50, 50, nant), rng.uniform(-50, 50, nant), np.zeros(nant)])
    ra = rng.uniform(0, 2 * np.pi, nsrc)
    dec = np.arcsin(rng.uniform(-1, 1, nsrc))
    freqs = np.array([100e6, 150e6])
    i150 = 10 ** rng.uniform(-1, 1, nsrc)
    alpha = rng.normal(-0.8, 0.2, nsrc)
    fluxes = i150[:, None] * (freqs[None, :] / 150e6) ** alpha[:, None]
    lsts = 0.7 + np.arange(4) * 2 * np.pi * 600 / 86164.0905
    lat = np.deg2rad(-30.72)
    out["a_antpos"] = antpos
    out["a_ra"] = ra
    out["a_dec"] = dec
    out["a_freqs"] = freqs
    out["a_fluxes"] = fluxes
    out["a_lsts"] = lsts
    out["a_lat"] = np.array(lat)
    out["a_sigma"] = np.array(0.2)
    out["a_vis"] = np.array(
        [
            _reference_pipeline(antpos, f, lsts, lat, ra, dec, fluxes[:, i], None, None, None, False, None, 1, "CPUMatMul", gauss_sigma=0.2)
            for i, f in enumerate(freqs)
        ]
    )
    # (b) polarised, two gridded complex beams with beam_idx, sparse pairs, 2 chunks
    nant, nsrc = 12, 2400
    antpos = np.column_stack([rng.uniform(-300, 300, nant), rng.uniform(-300, 300, nant), rng.uniform(-1, 1, nant)])
    ra = rng.uniform(0, 2 * np.pi, nsrc)
    dec = np.arcsin(rng.uniform(-1, 1, nsrc))
    freqs = np.array([110e6, 187.5e6])
    fluxes = rng.lognormal(0.0, 1.0, (nsrc, 1)) * np.ones((1, 2))
    lsts = np.array([0.2, 1.9, 5.1])
    naz, nza = 37, 10  # 10 deg steps, az 0..360 inclusive, za 0..90
    azg = np.deg2rad(np.arange(naz) * 10.0)
    zag = np.deg2rad(np.arange(nza) * 10.0)
    AZ, ZA = np.meshgrid(azg, zag, indexing="xy")
    grids = np.zeros((2, 2, 2, nza, naz), dtype=complex)
    for b in range(2):
        ex = np.array([[np.cos(ZA) * np.cos(AZ), -np.sin(AZ)], [np.cos(ZA) * np.sin(AZ), np.cos(AZ)]])  # (feed, ax)
        pert = 1 + 0.05 * (rng.normal(size=ex.shape) + 1j * rng.normal(size=ex.shape))
        pert[..., -1] = pert[..., 0]  # periodic azimuth column
        grids[b] = (ex * pert * np.cos(ZA) ** (1 + b)).transpose(1, 0, 2, 3)  # (ax, feed, za, az)
    params = np.array([[azg[1] - azg[0], zag[1] - zag[0], 0.0]] * 2)
    beam_idx = rng.integers(0, 2, nant)
    pairs = np.array([(i, j) for i in range(nant) for j in range(nant) if (i + 2 * j) % 3 == 0])
    out["b_antpos"] = antpos
    out["b_ra"] = ra
    out["b_dec"] = dec
    out["b_freqs"] = freqs
    out["b_fluxes"] = fluxes
    out["b_lsts"] = lsts
    out["b_lat"] = np.array(np.deg2rad(-30.72))
    out["b_grids"] = grids
    out["b_grid_params"] = params
    out["b_beam_idx"] = beam_idx
    out["b_pairs"] = pairs
    for method in ("CPUMatMul", "CPUVectorDot"):
        for name, ap in (("all", None), ("sparse", pairs)):
            if method == "CPUVectorDot" and ap is None:
                continue
            out[f"b_vis_{method}_{name}"] = np.array(
                [
                    _reference_pipeline(antpos, f, lsts, out["b_lat"], ra, dec, fluxes[:, i], grids, params, beam_idx, True, ap, 2, method)
                    for i, f in enumerate(freqs)
                ]
            )
    _save("pipeline.npz", **out)


def seeded_astrom(rng, lat):
    """Astrom-like parameters of realistic size (the pyerfa apco output is not available)."""
    eh = rng.normal(size=3)
    eh /= np.linalg.norm(eh)
    v = rng.normal(size=3)
    v *= 1.0e-4 / np.linalg.norm(v)  # ~30 km/s in units of c
    a, b, c = rng.normal(size=3) * 1e-3
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    rz = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rx = np.array([[1, 0, 0], [0, cc, -sc], [0, sc, cc]])
    return {
        "eh": eh, "em": 1.0 + 0.0167 * rng.uniform(-1, 1), "v": v, "bm1": float(np.sqrt(1 - v @ v)),
        "bpn": rz @ ry @ rx, "eral": rng.uniform(0, 2 * np.pi), "xpl": 1e-6 * rng.normal(), "ypl": 1e-6 * rng.normal(),
        "sphi": np.sin(lat), "cphi": np.cos(lat),
    }


def make_erfa():
    rot_cls = ref.cpu_coords.CoordinateRotationERFA

    class _Self:
        xp = np

    rng = np.random.default_rng(31)
    nsrc = 500
    ra = rng.uniform(0, 2 * np.pi, nsrc)
    dec = np.arcsin(rng.uniform(-1, 1, nsrc))
    eci = np.asarray(ref.coordinates.point_source_crd_eq(ra, dec))
    out = {"eci": eci}
    for t in range(3):
        astrom = seeded_astrom(rng, np.deg2rad(-30.72))
        for k, val in astrom.items():
            out[f"t{t}_{k}"] = np.asarray(val)
        p = eci.copy()
        rot_cls._ld(_Self(), p, astrom["eh"], astrom["em"], 1e-6)
        out[f"t{t}_after_ld"] = p.copy()
        rot_cls._ab(_Self(), p, astrom["v"], astrom["em"], astrom["bm1"])
        out[f"t{t}_after_ab"] = p.copy()
        rot_cls._bpn(_Self(), p, astrom)
        out[f"t{t}_bcrs"] = p.copy()
        top = p.copy()
        rot_cls._atioq(_Self(), top, astrom)
        out[f"t{t}_topo"] = top
    _save("erfa.npz", **out)


def reference_get_redundancies():
    import ast

    src = (refload.REF_ROOT / "src" / "matvis" / "cli.py").read_text()
    tree = ast.parse(src)
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "get_redundancies")
    mod = ast.Module(body=[fn], type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, "cli.py", "exec"), ns)
    return ns["get_redundancies"]


def make_redundancies():
    sys.path.insert(0, str(HERE.parents[1]))
    from matvis_b200 import workloads as wl

    get_red = reference_get_redundancies()
    rng = np.random.default_rng(41)
    layouts = {
        "hex37": wl.hex_array(37, 14.6),
        "hex127_jitter": wl.hex_array(127, 14.6) + np.column_stack([rng.normal(0, 2e-3, (127, 2)), np.zeros(127)]),
        "hera350": wl.hera350(np.random.default_rng(20261205)),
        "random40": np.column_stack([rng.uniform(-100, 100, (40, 2)), np.zeros(40)]),
        "colocated": np.array([[0, 0, 0], [0, 0, 0], [14.6, 0, 0], [14.6, 0, 0], [0, 14.6, 0], [-14.6, 0, 0.0]]),
        "line_half": np.column_stack([np.arange(12) * 0.005, np.zeros(12), np.zeros(12)]),
        "two": np.array([[0.0, 0, 0], [1.0, 2.0, 0]]),
        "one": np.zeros((1, 3)),
    }
    out = {}
    for name, pos in layouts.items():
        bls = pos[np.newaxis, :, :2] - pos[:, np.newaxis, :2]
        for nd in (2, 0, -1):
            pairs = np.asarray(get_red(bls, ndecimals=nd), dtype=np.int64).reshape(-1, 2)
            out[f"{name}_pos"] = pos
            out[f"{name}_nd{nd}"] = pairs
    _save("redundancies.npz", **out)


def make_coherency():
    coords = ref.coordinates
    rng = np.random.default_rng(51)
    lat = np.deg2rad(-30.72)
    nsrc, nfreq = 400, 3
    ra = rng.uniform(0, 2 * np.pi, nsrc)
    dec = np.arcsin(rng.uniform(-1, 1, nsrc))
    eci = np.asarray(coords.point_source_crd_eq(ra, dec))
    stokes_i = rng.uniform(0.5, 3.0, (nsrc, nfreq))
    frac = rng.uniform(0, 0.9, (nsrc, nfreq))
    direction = rng.normal(size=(3, nsrc, nfreq))
    direction /= np.linalg.norm(direction, axis=0)
    q, u, v = stokes_i * frac * direction
    coh = np.empty((nsrc, nfreq, 2, 2), dtype=complex)
    coh[..., 0, 0] = 0.5 * (stokes_i + q)
    coh[..., 1, 1] = 0.5 * (stokes_i - q)
    coh[..., 0, 1] = 0.5 * (u - 1j * v)
    coh[..., 1, 0] = 0.5 * (u + 1j * v)
    enu_to_altaz = np.array([[0.0, 1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    out = {"ra": ra, "dec": dec, "coherency": coh, "lat": lat}
    saved = coords._calc_average_rotation_matrix

    class _Self:
        xp = np
        telescope_loc = None

    try:
        for case in ("lst", "erfa"):
            if case == "lst":
                lst = 1.234
                rigid = np.asarray(coords.eci_to_enu_matrix(lst, lat))
                topo = rigid @ eci
                out["lst_lst"] = lst
            else:
                astrom = seeded_astrom(rng, lat)
                for k, val in astrom.items():
                    out[f"erfa_{k}"] = np.asarray(val)
                rot_cls = ref.cpu_coords.CoordinateRotationERFA
                p = eci.copy()
                rot_cls._ld(_Self(), p, astrom["eh"], astrom["em"], 1e-6)
                rot_cls._ab(_Self(), p, astrom["v"], astrom["em"], astrom["bm1"])
                rot_cls._bpn(_Self(), p, astrom)
                topo = p.copy()
                rot_cls._atioq(_Self(), topo, astrom)
                # rigid part of the apparent place: BPN then the CIRS -> ENU rotation
                probe = np.eye(3)
                rot_cls._atioq(_Self(), probe, astrom)
                rigid = probe @ np.asarray(astrom["bpn"])
            r_avg = enu_to_altaz @ rigid
            coords._calc_average_rotation_matrix = lambda time, location, _r=r_avg: _r
            az, za = coords.enu_to_az_za(topo[0], topo[1], orientation="astropy")
            above = np.flatnonzero(topo[2] > 0)
            alt = np.pi / 2 - za[above]
            rot = coords.calc_coherency_rotation(ra=ra[above], dec=dec[above], alt=alt, az=az[above], time=None,
                                                 location=None)
            rotated = ref.core_coords.CoordinateRotation._rotate_frame_coherency(
                _Self(), coh[above], ra[above], dec[above], alt, az[above], None)
            out[f"{case}_topo"] = topo
            out[f"{case}_rigid"] = rigid
            out[f"{case}_above"] = above
            out[f"{case}_rot"] = np.asarray(rot)
            out[f"{case}_rotated"] = np.asarray(rotated)
    finally:
        coords._calc_average_rotation_matrix = saved
    _save("coherency.npz", **out)


if __name__ == "__main__":
    make_matprod()
    make_bilinear()
    make_coords()
    make_tauz()
    make_chunks()
    make_pipeline()
    make_erfa()
    make_redundancies()
    make_coherency()
