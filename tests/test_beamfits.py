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
