"""Beam files in the beamfits layout (the FITS form of a UVBeam) without pyuvdata.

Covers the beam ingest the reference does through pyuvdata: reading a beamfits
file (``UVBeam.read_beamfits``, tests/conftest.py:10-15), interpolating it to a
simulation frequency (``UVBeam.interp(freq_array=...)`` in ``_wrangle_beams``,
core/beams.py:82-93; the file's ``FINTERP`` kind, linear for the HERA dipole
file) and handing the az/za grid to the interpolation kernel (what
``prepare_for_map_coords`` takes from ``UVBeam._prepare_coordinate_data``,
gpu/beams.py:15-19).

The FITS reading is a small self-contained parser of the primary image and
IMAGE / BINTABLE extension headers (2880-byte records of 80-character cards,
big-endian data).  Axes are found by their ``CTYPE``: ``AZIMUTH``,
``ZENANGLE``, ``FREQ``, ``FEEDIND`` (E-field) or ``STOKES`` (power),
``IF``, ``VECIND``, ``COMPLEX``; coordinates are ``CRVAL + (i + 1 - CRPIX) CDELT``.

Azimuth grids that cover the circle but stop one step short of 360 degrees
(the HERA file: 180 samples 359/179 degrees apart) are resampled onto a uniform
grid that ends at 360 degrees, by linear interpolation between azimuth
neighbours with the 0-degree samples repeated at 360 degrees, so that the
kernel's in-grid bilinear interpolation is periodic.  The reference's own GPU
comparison test re-grids the same file onto such a grid for the same reason
(src/matvis/_test_utils.py:60-75); pyuvdata's re-gridding itself cannot run
here, so values at the wrap are this module's linear rule.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .beam_models import GridBeam

_BLOCK = 2880
_CARD = 80
_DTYPES = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}
# AIPS polarisation codes used by beamfits power beams
_POLS = {-5: "xx", -6: "yy", -7: "xy", -8: "yx", 1: "pI", 2: "pQ", 3: "pU", 4: "pV"}


def _parse_value(text: str):
    text = text.strip()
    if text.startswith("'"):
        end = text.find("'", 1)
        while end != -1 and end + 1 < len(text) and text[end + 1] == "'":
            end = text.find("'", end + 2)
        return text[1:end].replace("''", "'").rstrip()
    body = text.split("/", 1)[0].strip()
    if body in ("T", "F"):
        return body == "T"
    if not body:
        return None
    try:
        return int(body)
    except ValueError:
        return float(body.replace("D", "E"))


def _read_header(buf: memoryview, off: int) -> tuple[dict, int]:
    hdr: dict = {}
    while True:
        if off + _BLOCK > len(buf):
            raise ValueError("truncated FITS header")
        block = bytes(buf[off : off + _BLOCK]).decode("ascii")
        off += _BLOCK
        for i in range(0, _BLOCK, _CARD):
            card = block[i : i + _CARD]
            key = card[:8].strip()
            if key == "END":
                return hdr, off
            if card[8:10] == "= ":
                hdr[key] = _parse_value(card[10:])


def _data_bytes(hdr: dict) -> int:
    naxis = int(hdr.get("NAXIS", 0))
    if naxis == 0:
        return 0
    n = 1
    for a in range(1, naxis + 1):
        n *= int(hdr[f"NAXIS{a}"])
    n = n * abs(int(hdr["BITPIX"])) // 8
    return n + int(hdr.get("PCOUNT", 0)) * int(hdr.get("GCOUNT", 1))


def read_fits(path) -> list[tuple[dict, np.ndarray | bytes | None]]:
    """All HDUs of a FITS file: (header, data) with image data as arrays in numpy
    axis order (NAXISn first, NAXIS1 last), BSCALE / BZERO applied."""
    raw = Path(path).read_bytes()
    buf = memoryview(raw)
    off, out = 0, []
    while off + _BLOCK <= len(buf):
        hdr, off = _read_header(buf, off)
        nbytes = _data_bytes(hdr)
        data = None
        if nbytes:
            chunk = raw[off : off + nbytes]
            if hdr.get("XTENSION", "IMAGE") in ("IMAGE",) or "SIMPLE" in hdr:
                shape = tuple(int(hdr[f"NAXIS{a}"]) for a in range(int(hdr["NAXIS"]), 0, -1))
                data = np.frombuffer(chunk, dtype=_DTYPES[int(hdr["BITPIX"])]).reshape(shape).astype(np.float64)
                if "BSCALE" in hdr or "BZERO" in hdr:
                    data = data * float(hdr.get("BSCALE", 1.0)) + float(hdr.get("BZERO", 0.0))
            else:
                data = chunk
        out.append((hdr, data))
        off += math.ceil(nbytes / _BLOCK) * _BLOCK
    if not out:
        raise ValueError(f"{path}: not a FITS file")
    return out


def _axis(hdr: dict, name: str) -> int | None:
    for a in range(1, int(hdr.get("NAXIS", 0)) + 1):
        if str(hdr.get(f"CTYPE{a}", "")).strip().upper() == name:
            return a
    return None


def _coords(hdr: dict, a: int) -> np.ndarray:
    n = int(hdr[f"NAXIS{a}"])
    return float(hdr.get(f"CRVAL{a}", 0.0)) + (np.arange(n) + 1 - float(hdr.get(f"CRPIX{a}", 1.0))) * float(
        hdr.get(f"CDELT{a}", 1.0))


@dataclass
class BeamFits:
    """A beam read from a beamfits file.

    ``data``: (Naxes_vec, Nfeeds or Npols, Nfreqs, Nza, Naz) complex128;
    ``az`` / ``za`` in radians, ``freq_array`` in Hz.
    """

    beam_type: str
    data: np.ndarray
    az: np.ndarray
    za: np.ndarray
    freq_array: np.ndarray
    feed_array: list = field(default_factory=list)
    polarization_array: list = field(default_factory=list)
    freq_interp_kind: str = "linear"
    header: dict = field(default_factory=dict, repr=False)

    # ------------------------------------------------------------ frequency
    def at_frequency(self, freq: float) -> "BeamFits":
        """The beam at one frequency (the file's FINTERP kind: linear or nearest)."""
        f = np.asarray(self.freq_array, dtype=np.float64)
        freq = float(freq)
        hit = np.flatnonzero(np.isclose(f, freq, rtol=0, atol=1e-3))
        if hit.size:
            d = self.data[:, :, hit[:1]]
        else:
            if len(f) < 2 or not f.min() < freq < f.max():
                raise ValueError(f"frequency {freq} Hz is outside the beam's range [{f.min()}, {f.max()}] Hz")
            order = np.argsort(f)
            fs = f[order]
            j = int(np.searchsorted(fs, freq))
            lo, hi = order[j - 1], order[j]
            if self.freq_interp_kind == "nearest":
                d = self.data[:, :, [lo if freq - fs[j - 1] <= fs[j] - freq else hi]]
            elif self.freq_interp_kind == "linear":
                w = (freq - f[lo]) / (f[hi] - f[lo])
                d = ((1.0 - w) * self.data[:, :, lo] + w * self.data[:, :, hi])[:, :, None]
            else:
                raise ValueError(f"frequency interpolation kind {self.freq_interp_kind!r} is not supported")
        return BeamFits(self.beam_type, d, self.az, self.za, np.array([freq]), list(self.feed_array),
                        list(self.polarization_array), self.freq_interp_kind, self.header)

    # ------------------------------------------------------------ power
    def efield_to_power(self) -> "BeamFits":
        """Auto-polarisation power beams P_ff = sum_vec |E[vec, f]|^2 (cross
        polarisations not computed), as a 1-vector power beam."""
        if self.beam_type == "power":
            return self
        p = np.sum(np.abs(self.data) ** 2, axis=0, keepdims=True).astype(np.complex128)
        pols = [f"{fd}{fd}" for fd in self.feed_array]
        return BeamFits("power", p, self.az, self.za, self.freq_array, list(self.feed_array), pols,
                        self.freq_interp_kind, self.header)

    # ------------------------------------------------------------ grid
    def periodic_grid(self) -> tuple[np.ndarray, np.ndarray]:
        """(az, data) on a uniform azimuth grid that ends at az[0] + 2 pi.

        A grid already closed at 360 degrees is returned unchanged; one that
        covers the circle but stops short of it is resampled linearly (with the
        first column repeated at az[0] + 2 pi); a partial-circle grid is left
        as it is (sources outside it get zero response)."""
        az = np.asarray(self.az, dtype=np.float64)
        d = self.data
        if len(az) < 2:
            return az, d
        daz = float(az[1] - az[0])
        span = float(az[-1] - az[0])
        if abs(span - 2 * np.pi) <= 1e-9 * 2 * np.pi or span + daz < 2 * np.pi - abs(daz) * 0.5:
            return az, d
        nout = int(math.ceil(2 * np.pi / daz - 1e-9)) + 1  # spacing no coarser than the file's
        new = az[0] + np.linspace(0.0, 2 * np.pi, nout)
        ext_az = np.concatenate([az, [az[0] + 2 * np.pi]])
        ext = np.concatenate([d, d[..., :1]], axis=-1)
        j = np.clip(np.searchsorted(ext_az, new, side="right") - 1, 0, len(ext_az) - 2)
        w = (new - ext_az[j]) / (ext_az[j + 1] - ext_az[j])
        out = ext[..., j] * (1.0 - w) + ext[..., j + 1] * w
        return new, out

    def to_grid_beam(self, freq: float | None = None, periodic: bool = True) -> GridBeam:
        """GridBeam (nax, nfeed, nza, naz) at ``freq`` (the single stored
        frequency when None), for ``mvb_beam_interp``."""
        b = self if freq is None else self.at_frequency(freq)
        if b.data.shape[2] != 1:
            raise ValueError("the beam holds several frequencies: give freq")
        az, d = b.periodic_grid() if periodic else (b.az, b.data)
        d = np.ascontiguousarray(d[:, :, 0])
        if b.beam_type == "power":
            d = d.real
        return GridBeam(data=d, az=az, za=np.asarray(b.za, dtype=np.float64), beam_type=b.beam_type)


def read_beamfits(path) -> BeamFits:
    """Read a beamfits file (E-field or power beam on an az/za grid)."""
    hdus = read_fits(path)
    hdr, arr = hdus[0]
    if arr is None:
        raise ValueError(f"{path}: no primary image")
    if str(hdr.get("COORDSYS", "az_za")).strip() != "az_za":
        raise ValueError("only az_za pixel coordinate systems are supported")
    a_az, a_za, a_f = _axis(hdr, "AZIMUTH"), _axis(hdr, "ZENANGLE"), _axis(hdr, "FREQ")
    if None in (a_az, a_za, a_f):
        raise ValueError("beamfits primary image needs AZIMUTH, ZENANGLE and FREQ axes")
    naxis = int(hdr["NAXIS"])

    def npaxis(a):  # FITS axis number -> numpy axis index
        return naxis - a

    a_feed, a_pol = _axis(hdr, "FEEDIND"), _axis(hdr, "STOKES")
    a_vec, a_cplx, a_if = _axis(hdr, "VECIND"), _axis(hdr, "COMPLEX"), _axis(hdr, "IF")
    beam_type = str(hdr.get("BTYPE", "efield" if a_feed else "power")).strip().lower()
    if beam_type == "intensity":
        beam_type = "power"
    x = arr
    if a_cplx is not None and int(hdr[f"NAXIS{a_cplx}"]) == 2:
        ax = npaxis(a_cplx)
        x = np.take(x, 0, axis=ax) + 1j * np.take(x, 1, axis=ax)
        removed = [a_cplx]
    else:
        x = x.astype(np.complex128)
        if a_cplx is not None:
            x = np.take(x, 0, axis=npaxis(a_cplx))
        removed = [a_cplx] if a_cplx is not None else []
    if a_if is not None:
        if int(hdr[f"NAXIS{a_if}"]) != 1:
            raise ValueError("only single-spectral-window beams are supported")
        x = np.take(x, 0, axis=npaxis(a_if) - sum(r > a_if for r in removed))
        removed.append(a_if)

    def cur(a):  # numpy axis of FITS axis a after the removals
        return npaxis(a) - sum(r > a for r in removed)

    a_pf = a_feed if a_feed is not None else a_pol
    order = [a_vec, a_pf, a_f, a_za, a_az]
    present = [a for a in order if a is not None]
    x = np.transpose(x, [cur(a) for a in present])
    if a_vec is None:
        x = x[None]
    if a_pf is None:
        x = x[:, None]
    az = np.deg2rad(_coords(hdr, a_az)) if str(hdr.get(f"CUNIT{a_az}", "deg")).strip() == "deg" else _coords(hdr, a_az)
    za = np.deg2rad(_coords(hdr, a_za)) if str(hdr.get(f"CUNIT{a_za}", "deg")).strip() == "deg" else _coords(hdr, a_za)
    freqs = _coords(hdr, a_f)
    feeds, pols = [], []
    if a_feed is not None:
        fl = str(hdr.get("FEEDLIST", "")).strip().strip("[]")
        feeds = [s.strip().strip("'\"") for s in fl.split(",") if s.strip()] or ["x", "y"][: x.shape[1]]
    if a_pol is not None:
        pols = [_POLS.get(int(round(v)), str(v)) for v in _coords(hdr, a_pol)]
    return BeamFits(beam_type=beam_type, data=np.ascontiguousarray(x), az=az, za=za, freq_array=freqs,
                    feed_array=feeds, polarization_array=pols,
                    freq_interp_kind=str(hdr.get("FINTERP", "linear")).strip().lower(), header=dict(hdr))


def _card(key: str, value, comment: str = "") -> str:
    if isinstance(value, bool):
        v = f"{'T' if value else 'F':>20}"
    elif isinstance(value, (int, np.integer)):
        v = f"{int(value):>20}"
    elif isinstance(value, (float, np.floating)):
        v = f"{float(value):>20.17G}"
    else:
        v = "'" + str(value).replace("'", "''").ljust(8) + "'"
    c = f"{key:<8}= {v}"
    if comment:
        c += f" / {comment}"
    return c[:_CARD].ljust(_CARD)


def write_beamfits(path, beam: BeamFits) -> None:
    """Write ``beam`` in the beamfits primary-image layout read by :func:`read_beamfits`
    (E-field: AZIMUTH, ZENANGLE, FREQ, FEEDIND, IF, VECIND, COMPLEX; power:
    STOKES in place of FEEDIND)."""
    d = np.asarray(beam.data)
    nvec, npf, nf, nza, naz = d.shape
    arr = np.stack([d.real, d.imag])[:, :, None]  # complex, vec, if, pf, f, za, az
    az_deg, za_deg = np.rad2deg(beam.az), np.rad2deg(beam.za)
    cards = [_card("SIMPLE", True), _card("BITPIX", -64), _card("NAXIS", 7)]
    for a, n in enumerate(reversed(arr.shape), start=1):
        cards.append(_card(f"NAXIS{a}", n))
    cards += [_card("EXTEND", True), _card("BTYPE", beam.beam_type), _card("COORDSYS", "az_za"),
              _card("FINTERP", beam.freq_interp_kind)]
    if beam.beam_type == "efield":
        cards.append(_card("FEEDLIST", "[" + ", ".join(beam.feed_array) + "]"))

    def axis(a, ctype, crval, cdelt, unit=None):
        out = [_card(f"CTYPE{a}", ctype), _card(f"CRVAL{a}", float(crval)), _card(f"CRPIX{a}", 1),
               _card(f"CDELT{a}", float(cdelt))]
        if unit:
            out.append(_card(f"CUNIT{a}", unit))
        return out

    step = lambda v: float(v[1] - v[0]) if len(v) > 1 else 1.0  # noqa: E731
    cards += axis(1, "AZIMUTH", az_deg[0], step(az_deg), "deg")
    cards += axis(2, "ZENANGLE", za_deg[0], step(za_deg), "deg")
    cards += axis(3, "FREQ", beam.freq_array[0], step(beam.freq_array), "Hz")
    if beam.beam_type == "efield":
        cards += axis(4, "FEEDIND", 1, 1)
    else:
        codes = {v: k for k, v in _POLS.items()}
        p = [codes[s] for s in beam.polarization_array]
        cards += axis(4, "STOKES", p[0], (p[1] - p[0]) if len(p) > 1 else -1)
    cards += axis(5, "IF", 1, 1) + axis(6, "VECIND", 1, 1) + axis(7, "COMPLEX", 1, 1)
    cards.append("END".ljust(_CARD))
    head = "".join(cards)
    head += " " * (-len(head) % _BLOCK)
    body = np.ascontiguousarray(arr, dtype=">f8").tobytes()
    body += b"\0" * (-len(body) % _BLOCK)
    Path(path).write_bytes(head.encode("ascii") + body)
