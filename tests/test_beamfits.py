"""Beamfits reader / writer, frequency interpolation and periodic re-gridding
(host logic; the grids then go through the same interpolation kernel as any
GridBeam)."""

import numpy as np
import pytest

from matvis_b200.beamfits import BeamFits, read_beamfits, read_fits, write_beamfits


def _dipole(nza=46, naz=180, freqs=(100e6, 101e6), closed=False, seed=3):
    rng = np.random.default_rng(seed)
    az = np.deg2rad(np.linspace(0, 360, naz) if closed else np.arange(naz) * (359.0 / (naz - 1)))
    za = np.deg2rad(np.linspace(0, 90, nza))
    A, Z = np.meshgrid(az, za)
    data = np.zeros((2, 2, len(freqs), nza, naz), dtype=complex)
    for i, f in enumerate(freqs):
        g = 1 + 0.01 * (f - freqs[0]) / 1e6
        data[0, 0, i] = g * np.cos(Z) * np.cos(A)
        data[1, 0, i] = -g * np.sin(A)
        data[0, 1, i] = g * np.cos(Z) * np.sin(A)
        data[1, 1, i] = g * np.cos(A)
    data *= 1 + 0.01 * (rng.normal(size=data.shape) + 1j * rng.normal(size=data.shape))
    return BeamFits("efield", data, az, za, np.asarray(freqs, dtype=float), ["x", "y"], [], "linear")


def test_roundtrip_efield(tmp_path):
    b = _dipole()
    p = tmp_path / "b.fits"
    write_beamfits(p, b)
    r = read_beamfits(p)
    assert r.beam_type == "efield" and r.feed_array == ["x", "y"] and r.freq_interp_kind == "linear"
    np.testing.assert_array_equal(r.data, b.data)
    np.testing.assert_allclose(r.az, b.az, rtol=0, atol=1e-13)
    np.testing.assert_allclose(r.za, b.za, rtol=0, atol=1e-13)
    np.testing.assert_array_equal(r.freq_array, b.freq_array)
    hdrs = read_fits(p)
    assert len(hdrs) == 1 and hdrs[0][0]["NAXIS"] == 7 and hdrs[0][0]["CTYPE1"] == "AZIMUTH"


def test_roundtrip_power(tmp_path):
    b = _dipole().efield_to_power()
    assert b.beam_type == "power" and b.polarization_array == ["xx", "yy"]
    np.testing.assert_allclose(b.data[0, 0].real, np.sum(np.abs(_dipole().data[:, 0]) ** 2, axis=0))
    p = tmp_path / "p.fits"
    write_beamfits(p, b)
    r = read_beamfits(p)
    assert r.beam_type == "power" and r.polarization_array == ["xx", "yy"]
    np.testing.assert_array_equal(r.data, b.data)


def test_frequency_interpolation_linear():
    b = _dipole()
    mid = b.at_frequency(100.25e6)
    np.testing.assert_allclose(mid.data[:, :, 0], 0.75 * b.data[:, :, 0] + 0.25 * b.data[:, :, 1], rtol=1e-14)
    np.testing.assert_array_equal(b.at_frequency(101e6).data[:, :, 0], b.data[:, :, 1])
    with pytest.raises(ValueError):
        b.at_frequency(99e6)
    with pytest.raises(ValueError):
        b.at_frequency(102e6)
    b.freq_interp_kind = "nearest"
    np.testing.assert_array_equal(b.at_frequency(100.7e6).data[:, :, 0], b.data[:, :, 1])


def test_periodic_regrid():
    b = _dipole(naz=180)  # 0 .. 359 degrees, one short step before the wrap
    g = b.to_grid_beam(100e6)
    assert len(g.az) == 181 and abs(g.az[-1] - 2 * np.pi) < 1e-12
    np.testing.assert_allclose(np.diff(g.az), np.deg2rad(2.0), rtol=1e-12)
    # the closing column repeats the 0-degree one, and on-grid samples survive
    np.testing.assert_allclose(g.data[..., -1], g.data[..., 0], rtol=0, atol=1e-15)
    np.testing.assert_allclose(g.data[..., 0], b.data[:, :, 0, :, 0], rtol=0, atol=1e-15)
    # a grid already closed at 360 degrees is kept as it is
    c = _dipole(naz=181, closed=True)
    gc = c.to_grid_beam(100e6)
    np.testing.assert_array_equal(gc.az, c.az)
    np.testing.assert_array_equal(gc.data, c.data[:, :, 0])


def test_regridded_values_are_linear_in_azimuth():
    b = _dipole(naz=180)
    az, d = b.periodic_grid()
    src_az = np.concatenate([b.az, [b.az[0] + 2 * np.pi]])
    src = np.concatenate([b.data, b.data[..., :1]], axis=-1)
    for j in (1, 57, 179, 180):
        i = np.searchsorted(src_az, az[j], side="right") - 1
        i = min(i, len(src_az) - 2)
        w = (az[j] - src_az[i]) / (src_az[i + 1] - src_az[i])
        np.testing.assert_allclose(d[..., j], (1 - w) * src[..., i] + w * src[..., i + 1], rtol=1e-13, atol=1e-15)


def test_rejects_non_fits(tmp_path):
    p = tmp_path / "x.fits"
    p.write_bytes(b"not a fits file" * 300)
    with pytest.raises(Exception):
        read_beamfits(p)


# ----------------------------------------------------------------------------
# The reference's own beam file (src/matvis/data/NF_HERA_Dipole_small.fits, read
# by the reference's test fixtures with UVBeam.read_beamfits, tests/conftest.py:9-24)
# ----------------------------------------------------------------------------
HERA_FITS = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "NF_HERA_Dipole_small.fits"
# primary image axes, NAXIS1 fastest: az 180, za 91, freq 2, feed 2, IF 1, vec 2, complex 2
HERA_SHAPE = (2, 2, 1, 2, 2, 91, 180)


def _hera_header_end(raw: bytes) -> int:
    """Byte offset of the primary data: the header's 80-byte cards up to END,
    rounded up to whole 2880-byte records."""
    i = 0
    while not raw[i:i + 80].startswith(b"END"):
        i += 80
    return -(-(i + 80) // 2880) * 2880


def test_hera_beamfits_axes_and_metadata():
    b = read_beamfits(HERA_FITS)
    assert b.beam_type == "efield" and b.feed_array == ["x", "y"] and b.freq_interp_kind == "linear"
    assert b.data.shape == (2, 2, 2, 91, 180)  # (vec, feed, freq, za, az)
    np.testing.assert_array_equal(b.freq_array, [100e6, 101e6])
    np.testing.assert_allclose(np.rad2deg(b.az), np.arange(180) * (359.0 / 179.0), rtol=0, atol=1e-9)
    np.testing.assert_allclose(np.rad2deg(b.za), np.arange(91) * 2.0, rtol=0, atol=1e-12)
    # NORMSTD = 'peak': the largest E-field component magnitude is 1
    assert np.abs(b.data).max() == pytest.approx(1.0, abs=1e-12)


def test_hera_beamfits_values_decoded_independently():
    """Every value against the big-endian float64 block read straight from the
    file, and spot values by explicit offset arithmetic."""
    import struct

    raw = HERA_FITS.read_bytes()
    off = _hera_header_end(raw)
    n = int(np.prod(HERA_SHAPE))
    block = np.frombuffer(raw[off:off + 8 * n], dtype=">f8").reshape(HERA_SHAPE)
    want = block[0, :, 0] + 1j * block[1, :, 0]  # (vec, feed, freq, za, az)
    b = read_beamfits(HERA_FITS)
    np.testing.assert_array_equal(b.data, want)
    rng = np.random.default_rng(17)
    for _ in range(64):
        v, fd, fr, z, a = (int(rng.integers(0, s)) for s in (2, 2, 2, 91, 180))
        idx = [(((((c * 2 + v) * 1 + 0) * 2 + fd) * 2 + fr) * 91 + z) * 180 + a for c in (0, 1)]
        re, im = (struct.unpack(">d", raw[off + 8 * i: off + 8 * i + 8])[0] for i in idx)
        assert b.data[v, fd, fr, z, a] == complex(re, im)


def test_hera_beamfits_frequency_interpolation_is_the_linear_blend():
    """FINTERP = linear (core/beams.py:82-93 interpolates to the simulation
    frequency): the beam at 100.4 MHz is 0.6 x (100 MHz) + 0.4 x (101 MHz)."""
    b = read_beamfits(HERA_FITS)
    got = b.at_frequency(100.4e6)
    assert got.data.shape == (2, 2, 1, 91, 180)
    np.testing.assert_allclose(got.data[:, :, 0], 0.6 * b.data[:, :, 0] + 0.4 * b.data[:, :, 1], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(b.at_frequency(101e6).data[:, :, 0], b.data[:, :, 1])
    with pytest.raises(ValueError):
        b.at_frequency(99e6)


def test_hera_beamfits_periodic_grid():
    """The 180-sample azimuth axis (359/179 degrees apart) is re-gridded onto 2-degree
    steps closing at 360 degrees: the 0- and 360-degree columns are the file's first
    column, and each new column is the linear blend of its two file neighbours."""
    b = read_beamfits(HERA_FITS)
    az, d = b.periodic_grid()
    assert len(az) == 181
    np.testing.assert_allclose(np.rad2deg(az), np.arange(181) * 2.0, rtol=0, atol=1e-9)
    np.testing.assert_array_equal(d[..., 0], b.data[..., 0])
    np.testing.assert_array_equal(d[..., -1], b.data[..., 0])
    step = 359.0 / 179.0
    for k in (1, 45, 90, 179):
        j = int(np.floor(2.0 * k / step))
        w = (2.0 * k - j * step) / step
        np.testing.assert_allclose(d[..., k], (1 - w) * b.data[..., j] + w * b.data[..., j + 1], rtol=0, atol=1e-12)
