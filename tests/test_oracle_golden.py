"""The FP64 oracle against fixtures frozen from the reference's own functions.

Fixtures: ``tests/golden/*.npz`` (made by ``tests/golden/make_golden.py``).
"""

import numpy as np
import pytest

from oracle import oracle as orc

from .conftest import golden


def test_matprod_arange_known_answer():
    """tests/test_matprod.py:45-65 (arange Z, feed transpose), both methods."""
    g = golden("matprod")
    for key in g.files:
        if not key.startswith("arange_"):
            continue
        _, method, f, p, e, c = key.split("_")
        nfeed, precision = int(f[1]), int(p[1])
        nant, nsrc = 5, 15
        z = np.arange(nfeed * nant * nsrc, dtype=complex).reshape(nfeed * nant, nsrc) + 1j
        pairs = orc.all_pairs(nant)
        if method == "CPUMatMul":
            res = orc.matmul_vis(z, nant, nfeed, pairs if e == "e1" else None)
        else:
            res = orc.vectordot_vis(z, nant, nfeed, pairs)
        np.testing.assert_allclose(res, g[key], rtol=1e-7 if precision == 2 else 1e-6)


def test_matprod_random_sparse():
    g = golden("matprod")
    z, pairs = g["random_z"], g["random_pairs"]
    np.testing.assert_allclose(orc.matmul_vis(z, 7, 2), g["random_CPUMatMul_all"], rtol=1e-12)
    np.testing.assert_allclose(orc.matmul_vis(z, 7, 2, pairs), g["random_CPUMatMul_sparse"], rtol=1e-12)
    np.testing.assert_allclose(orc.vectordot_vis(z, 7, 2, pairs), g["random_CPUVectorDot_sparse"], rtol=1e-12)
    np.testing.assert_allclose(orc.vectordot_vis(z, 7, 2, orc.all_pairs(7)), g["random_CPUVectorDot_all"], rtol=1e-12)


@pytest.mark.parametrize("case", ["ident", "lin", "cplx", "pow"])
def test_bilinear_matches_reference(case):
    """gpu/beams.py:127-200 on the grids of tests/test_beam_interp_gpu.py and seeded grids."""
    g = golden("bilinear")
    p = g[f"{case}_params"]
    out = orc.bilinear_beam(g[f"{case}_beam"], p[:, 0], p[:, 1], p[:, 2], g[f"{case}_az"], g[f"{case}_za"])
    np.testing.assert_allclose(out, g[f"{case}_out"], rtol=1e-12, atol=1e-14)


def test_bilinear_linear_exactness():
    """tests/test_beam_interp_gpu.py:38-64: a linear beam interpolates exactly."""
    g = golden("bilinear")
    np.testing.assert_allclose(g["lin_out"][:, 0, 0], g["lin_truth"], atol=1e-12)


def test_coordinates_match_reference():
    g = golden("coords")
    np.testing.assert_array_equal(orc.point_source_crd_eq(g["crd_ra"], g["crd_dec"]), g["crd_eq"])
    for (h, lat), m in zip(g["mat_hl"], g["mat_eci_to_enu"]):
        np.testing.assert_array_equal(orc.eci_to_enu_matrix(h, lat), m)
    for orient in ("astropy", "uvbeam"):
        az, za = orc.enu_to_az_za(g["azza_e"], g["azza_n"], orientation=orient)
        np.testing.assert_array_equal(az, g[f"azza_{orient}_az"])
        np.testing.assert_array_equal(za, g[f"azza_{orient}_za"])
    az, _ = orc.enu_to_az_za(g["azza_e"], g["azza_n"], orientation="uvbeam", periodic_azimuth=False)
    np.testing.assert_array_equal(az, g["azza_uvbeam_nonperiodic_az"])


def test_zenith_and_inverse():
    """tests/test_coordinates.py:71-160: RA=LST, Dec=lat lies at zenith."""
    lat = np.deg2rad(-30.7215)
    lsts = np.linspace(0, 2 * np.pi, 24)
    eci = orc.point_source_crd_eq(lsts, lat * np.ones(24))
    for i, lst in enumerate(lsts):
        top = orc.rotate_fixed_order(orc.eci_to_enu_matrix(lst, lat), eci)
        assert np.isclose(top[0, i], 0.0) and np.isclose(top[1, i], 0.0) and np.isclose(top[2, i], 1.0)
        az, za = orc.enu_to_az_za(top[0], top[1], orientation="uvbeam")
        assert np.isclose(za[i], 0.0)


def test_select_chunk_matches_reference():
    """core/coords.py:99-150 through the reference's own select_chunk."""
    g = golden("coords")
    eci, flux = g["sel_eci"], g["sel_flux"]
    cs, alloc = int(g["sel_chunk_size"]), int(g["sel_alloc"])
    assert alloc == orc.nsrc_alloc(cs, 0.7)
    for t, lst in enumerate(g["sel_lsts"]):
        rot = orc.eci_to_enu_matrix(lst, float(g["sel_lat"]))
        top = orc.rotate_fixed_order(rot, eci)
        # the reference fixture used np.dot; the fixed order agrees to rounding
        np.testing.assert_allclose(top, g[f"sel_topo_t{t}"], rtol=0, atol=1e-15)
        for ch in range(2):
            crd, fl, n, kept = orc.select_chunk(top, flux, ch, cs, alloc)
            assert n == int(g[f"sel_n_t{t}_c{ch}"])
            np.testing.assert_allclose(crd[:, :n], g[f"sel_crd_t{t}_c{ch}"], rtol=0, atol=1e-15)
            np.testing.assert_array_equal(fl, g[f"sel_flux_t{t}_c{ch}"])


def test_select_chunk_overflow():
    top = np.zeros((3, 10))
    top[2] = 1.0
    with pytest.raises(ValueError, match="nsrc_alloc"):
        orc.select_chunk(top, np.ones(10), 0, 10, 5)


def test_tau_and_z_match_reference():
    g = golden("tauz")
    ext = orc.exptau(g["antpos"], float(g["freq"]), g["crd"])
    np.testing.assert_allclose(ext, g["exptau"], rtol=1e-13)
    z = orc.zmatrix(g["sqrt_flux"], g["beam"], g["exptau"], g["beam_idx"], 2, 2)
    np.testing.assert_allclose(z, g["z"], rtol=1e-14)
    z1 = orc.zmatrix(g["sqrt_flux"], g["beam1"], g["exptau"], None, 1, 1)
    np.testing.assert_allclose(z1, g["z1"], rtol=1e-14)


def test_chunk_planning_matches_reference():
    t = golden("chunks")["table"]
    for row in t:
        fm, nax, nfeed, nant, nsrc, nbeam, npix, prec, sb, mb, ch = row
        got = orc.get_required_chunks(fm, int(nax), int(nfeed), int(nant), int(nsrc), int(nbeam), int(npix), int(prec), sb, mb)
        assert got == int(ch)


def test_pipeline_unpolarized_matches_reference():
    g = golden("pipeline")
    ants = {i: tuple(p) for i, p in enumerate(g["a_antpos"])}
    vis = orc.simulate_vis(
        ants=ants,
        fluxes=g["a_fluxes"],
        ra=g["a_ra"],
        dec=g["a_dec"],
        freqs=g["a_freqs"],
        lsts=g["a_lsts"],
        latitude=float(g["a_lat"]),
        beams=[orc.GaussianPowerBeam(sigma=float(g["a_sigma"]))],
    )
    np.testing.assert_allclose(vis, g["a_vis"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("method,name", [("CPUMatMul", "all"), ("CPUMatMul", "sparse"), ("CPUVectorDot", "sparse")])
def test_pipeline_polarized_matches_reference(method, name):
    g = golden("pipeline")
    grids = g["b_grids"]
    p = g["b_grid_params"]
    naz, nza = grids.shape[-1], grids.shape[-2]
    beams = [
        orc.GridBeam(data=grids[b], az=p[b, 2] + p[b, 0] * np.arange(naz), za=p[b, 1] * np.arange(nza)) for b in range(grids.shape[0])
    ]
    ants = {i: tuple(x) for i, x in enumerate(g["b_antpos"])}
    vis = orc.simulate_vis(
        ants=ants,
        fluxes=g["b_fluxes"],
        ra=g["b_ra"],
        dec=g["b_dec"],
        freqs=g["b_freqs"],
        lsts=g["b_lsts"],
        latitude=float(g["b_lat"]),
        beams=beams,
        polarized=True,
        beam_idx=g["b_beam_idx"],
        antpairs=None if name == "all" else g["b_pairs"],
        matprod="MatMul" if method == "CPUMatMul" else "VectorDot",
        nchunks=2,
    )
    np.testing.assert_allclose(vis, g[f"b_vis_{method}_{name}"], rtol=1e-9, atol=1e-11)


def _astrom(g, t):
    keys = ("eh", "em", "v", "bm1", "bpn", "eral", "xpl", "ypl", "sphi", "cphi")
    return {k: (g[f"t{t}_{k}"] if g[f"t{t}_{k}"].ndim else float(g[f"t{t}_{k}"])) for k in keys}


def test_erfa_steps_match_reference():
    """cpu/coords.py:89-181 (_ld, _ab, _bpn, _atioq) through the reference's own methods."""
    g = golden("erfa")
    for t in range(3):
        a = _astrom(g, t)
        p1 = orc.erfa_ld(g["eci"], a["eh"], a["em"], 1e-6)
        np.testing.assert_allclose(p1, g[f"t{t}_after_ld"], rtol=0, atol=1e-15)
        p2 = orc.erfa_ab(g[f"t{t}_after_ld"], a["v"], a["em"], a["bm1"])
        np.testing.assert_allclose(p2, g[f"t{t}_after_ab"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(orc.erfa_bcrs(g["eci"], a), g[f"t{t}_bcrs"], rtol=0, atol=2e-15)
        top = orc.erfa_atioq_matrix(a) @ g[f"t{t}_bcrs"]
        np.testing.assert_allclose(top, g[f"t{t}_topo"], rtol=0, atol=2e-15)


def test_coherency_rotation_matches_reference():
    """coordinates.py:288-580 and core/coords.py:152-175 through the reference's
    own functions; the restatement equals them wherever the reference is finite
    and is the unperturbed rotation where it divides 0 by 0."""
    g = golden("coherency")
    for case in ("lst", "erfa"):
        topo, ab = g[f"{case}_topo"], g[f"{case}_above"]
        az, za = orc.enu_to_az_za(topo[0], topo[1], orientation="astropy")
        rot = orc.coherency_rotation(g["ra"][ab], g["dec"][ab], np.pi / 2 - za[ab], az[ab],
                                     orc.ENU_TO_ALTAZ @ g[f"{case}_rigid"])
        ref = g[f"{case}_rot"]
        finite = ~np.isnan(ref).any(axis=(0, 1))
        np.testing.assert_allclose(rot[..., finite], ref[..., finite], rtol=0, atol=1e-15)
        assert np.isfinite(rot).all()
        np.testing.assert_allclose(rot[0, 0] ** 2 + rot[0, 1] ** 2, 1.0, rtol=0, atol=1e-14)
        c = orc.rotate_coherency(g["coherency"][ab], rot)
        fc = ~np.isnan(g[f"{case}_rotated"]).any(axis=(1, 2, 3))
        np.testing.assert_allclose(c[fc], g[f"{case}_rotated"][fc], rtol=0, atol=1e-15)


def test_oracle_unpolarised_coherency_equals_scalar():
    from matvis_b200 import workloads as wl

    cfg = wl.subset(wl.config2(nfreq=2, ntimes=2), nsrc=400, nfreq=1, ntimes=2, nant=5, seed=3)
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in cfg["beams"]]
    kw = dict(ants={i: tuple(p) for i, p in enumerate(cfg["antpos"])}, ra=cfg["ra"], dec=cfg["dec"],
              freqs=cfg["freqs"], lsts=cfg["lsts"], latitude=cfg["latitude"], beams=beams, polarized=True,
              beam_idx=cfg["beam_idx"])
    a = orc.simulate_vis(fluxes=cfg["fluxes"], **kw)
    b = orc.simulate_vis(fluxes=orc.stokes_to_coherency(cfg["fluxes"], 0, 0, 0), **kw)
    np.testing.assert_allclose(b, a, rtol=0, atol=1e-12 * np.abs(a).max())


@pytest.mark.parametrize("layout", ["hex37", "hex127_jitter", "hera350", "random40", "colocated", "line_half", "two",
                                    "one"])
@pytest.mark.parametrize("nd", [2, 0, -1])
def test_oracle_redundancies_match_reference(layout, nd):
    """The oracle's get_redundancies (the reference arm's pair list) against the
    reference's own function (cli.py:273-290)."""
    g = golden("redundancies")
    got = orc.redundant_antpairs(g[f"{layout}_pos"], ndecimals=nd)
    np.testing.assert_array_equal(got, g[f"{layout}_nd{nd}"].reshape(-1, 2))
