"""Host-side beam checks on the CPU: the reference's beam-list errors
(core/beams.py:35-99, exercised by its tests/test_beams.py:60-90), the grid
validation, per-antenna beam indices and the frequency selection of beamfits
beams."""

import numpy as np
import pytest

from matvis_b200.beamfits import BeamFits
from matvis_b200.beams import (GaussianBeam, GridBeam, _wrangle_beams, beams_at_frequency, is_chromatic,
                               resolve_beam_idx)


def _grid(beam_type="efield", nax=2, nfeed=2, nza=10, naz=37):
    za = np.linspace(0, np.pi / 2, nza)
    az = np.linspace(0, 2 * np.pi, naz)
    data = np.ones((nax, nfeed, nza, naz), dtype=np.complex128)
    return GridBeam(data=data, az=az, za=za, beam_type=beam_type)


def test_beam_list_errors_match_the_reference():
    b = _grid()
    with pytest.raises(ValueError, match="beam_idx must be provided"):
        _wrangle_beams(None, [b, b], polarized=True, nant=3, freq=1e8)
    with pytest.raises(ValueError, match="beam_idx must be length nant"):
        _wrangle_beams(np.array([0, 1]), [b, b], polarized=True, nant=3, freq=1e8)
    with pytest.raises(ValueError, match="beam_idx contains indices greater than the number of beams"):
        _wrangle_beams(np.array([0, 1, 2]), [b, b], polarized=True, nant=3, freq=1e8)
    with pytest.raises(ValueError, match="beam type must be efield if using polarized=True"):
        _wrangle_beams(None, [_grid("power", nax=1, nfeed=1)], polarized=True, nant=3, freq=1e8)
    with pytest.raises(ValueError, match="beam type must be efield if using polarized=True"):
        _wrangle_beams(None, [GaussianBeam(sigma=0.2)], polarized=True, nant=3, freq=1e8)
    beams, nbeam, idx = _wrangle_beams(None, [b, b, b], polarized=True, nant=3, freq=1e8)
    assert nbeam == 3 and idx is None and len(beams) == 3
    _wrangle_beams(None, [GaussianBeam(sigma=0.2)], polarized=False, nant=5, freq=1e8)


def test_grid_beam_validation():
    b = _grid()
    assert b.Nfeeds == 2 and b.azmin == 0.0
    assert b.daz == pytest.approx(2 * np.pi / 36) and b.dza == pytest.approx(np.pi / 18)
    with pytest.raises(ValueError, match="shape"):
        GridBeam(data=np.ones((2, 10, 37)), az=b.az, za=b.za)
    with pytest.raises(ValueError, match="does not match"):
        GridBeam(data=np.ones((2, 2, 10, 36)), az=b.az, za=b.za)
    with pytest.raises(ValueError, match="beam_type"):
        GridBeam(data=b.data, az=b.az, za=b.za, beam_type="voltage")
    with pytest.raises(ValueError, match="start at 0"):
        GridBeam(data=b.data, az=b.az, za=b.za + 0.1)


def test_power_grid():
    b = _grid()
    b.data[0, 1] *= 2.0
    p = b.power_grid(feed=1)
    assert p.shape == (1, 1, 10, 37) and np.allclose(p, 4.0 + 1.0)
    pw = _grid("power", nax=1, nfeed=1)
    assert np.allclose(pw.power_grid(), 1.0)


def test_resolve_beam_idx():
    assert resolve_beam_idx(None, 1, 4).tolist() == [0, 0, 0, 0]
    assert resolve_beam_idx(None, 4, 4).tolist() == [0, 1, 2, 3]
    got = resolve_beam_idx([1, 0, 1], 2, 3)
    assert got.dtype == np.int32 and got.tolist() == [1, 0, 1]


def test_beamfits_beams_are_taken_per_frequency():
    nza, naz = 10, 37
    za = np.linspace(0, np.pi / 2, nza)
    az = np.linspace(0, 2 * np.pi, naz)
    data = np.stack([np.full((nza, naz), 1.0), np.full((nza, naz), 3.0)])  # (Nfreqs, nza, naz)
    data = np.broadcast_to(data, (2, 2, 2, nza, naz)).astype(np.complex128)
    fits = BeamFits("efield", data, az, za, np.array([100e6, 200e6]), ["x", "y"], [], "linear")
    grid, gauss = _grid(), GaussianBeam(sigma=0.2)
    assert is_chromatic([grid, fits]) and not is_chromatic([grid, gauss])
    at = beams_at_frequency([grid, fits, gauss], 150e6)
    assert at[0] is grid and at[2] is gauss and isinstance(at[1], GridBeam)
    assert np.allclose(at[1].data, 2.0)  # linear in frequency, halfway between 1 and 3
