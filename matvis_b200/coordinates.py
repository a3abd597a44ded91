"""Host-side coordinate helpers (input preparation, FP64 numpy).

Same functions and conventions as the reference's ``coordinates.py``; they build
the per-job inputs (source unit vectors, the per-time 3x3 rotation) that the CUDA
kernels consume.  Per-source work per time step runs on the GPU.
"""

from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

#: below this many sources one numpy pass beats handing the work to threads
_PAR_MIN = 1 << 17
#: chunk granule (elements): a multiple of every SIMD width, so each chunk is
#: split into vector body and tail exactly as the whole array would be
_PAR_GRANULE = 8192


def point_source_crd_eq(ra, dec):
    """ECI unit vectors, shape (3, N); coordinates.py:174-200.

    Large skies are cut into granule-aligned chunks evaluated by the same numpy
    ufuncs on host threads (numpy releases the GIL inside them), so every
    element is bit-identical to the single-pass result; the kernels' horizon
    selection depends on that.
    """
    ra = np.asarray(ra, dtype=np.float64)
    dec = np.asarray(dec, dtype=np.float64)
    nthreads = min(os.cpu_count() or 1, 16)
    if ra.shape != dec.shape or ra.size < _PAR_MIN or nthreads < 2:
        return np.asarray([np.cos(ra) * np.cos(dec), np.cos(dec) * np.sin(ra), np.sin(dec)])
    r, d = ra.reshape(-1), dec.reshape(-1)
    n = r.size
    out = np.empty((3, n), dtype=np.float64)
    step = -(-n // nthreads)
    step = -(-step // _PAR_GRANULE) * _PAR_GRANULE

    def work(lo):
        sl = slice(lo, min(lo + step, n))
        cd = np.cos(d[sl])
        np.multiply(np.cos(r[sl]), cd, out=out[0, sl])
        np.multiply(cd, np.sin(r[sl]), out=out[1, sl])
        np.sin(d[sl], out=out[2, sl])

    with ThreadPoolExecutor(nthreads) as ex:
        list(ex.map(work, range(0, n, step)))
    return out.reshape((3,) + ra.shape)


def eci_to_enu_matrix(ha, lat):
    """3x3 ECI -> ENU rotation for hour angle (here: LST) and latitude; coordinates.py:91-125."""
    return np.array(
        [
            [-np.sin(ha), np.cos(ha), 0.0 * ha],
            [-np.sin(lat) * np.cos(ha), -np.sin(lat) * np.sin(ha), np.cos(lat)],
            [np.cos(lat) * np.cos(ha), np.cos(lat) * np.sin(ha), np.sin(lat)],
        ],
        dtype=np.float64,
    )


def enu_to_eci_matrix(ha, lat):
    """Inverse of :func:`eci_to_enu_matrix`; coordinates.py:128-160."""
    return np.array(
        [
            [-np.sin(ha), -np.cos(ha) * np.sin(lat), np.cos(ha) * np.cos(lat)],
            [np.cos(ha), -np.sin(ha) * np.sin(lat), np.sin(ha) * np.cos(lat)],
            [0.0 * ha, np.cos(lat), np.sin(lat)],
        ],
        dtype=np.float64,
    )


def enu_to_az_za(enu_e, enu_n, orientation="astropy", periodic_azimuth=True):
    """Azimuth / zenith angle of ENU direction cosines; coordinates.py:31-88."""
    assert orientation in ("astropy", "uvbeam"), "orientation must be either 'astropy' or 'uvbeam'"
    enu_e = np.asarray(enu_e, dtype=np.float64)
    enu_n = np.asarray(enu_n, dtype=np.float64)
    lsqr = enu_n**2.0 + enu_e**2.0
    mask = lsqr < 1
    zeta = np.zeros_like(lsqr)
    zeta[mask] = np.sqrt(1 - lsqr[mask])
    az = np.arctan2(enu_e, enu_n)
    za = 0.5 * np.pi - np.arcsin(zeta)
    if orientation == "uvbeam":
        az = 0.5 * np.pi - az
    if periodic_azimuth:
        az = np.mod(az, 2 * np.pi)
    return az, za


def latitude_of(telescope_loc) -> float:
    """Latitude in radians from a float or an object with a ``lat`` attribute."""
    lat = getattr(telescope_loc, "lat", telescope_loc)
    lat = getattr(lat, "rad", lat)
    return float(lat)


def lsts_of(times) -> np.ndarray:
    """Local sidereal times (radians) for the time axis.

    The rotation here is the rigid LST rotation, so ``times`` are LSTs in
    radians (a 1-D array); an object with ``.rad`` is unwrapped.
    """
    t = getattr(times, "rad", times)
    t = np.atleast_1d(np.asarray(t, dtype=np.float64))
    if t.ndim != 1:
        raise ValueError("times must be a 1-D array of LSTs (radians)")
    return t


def radec_of(skycoords) -> tuple[np.ndarray, np.ndarray]:
    """(ra, dec) in radians from a (ra, dec) pair or an object with ra / dec."""
    if hasattr(skycoords, "ra") and hasattr(skycoords, "dec"):
        ra, dec = skycoords.ra, skycoords.dec
        ra = getattr(ra, "rad", ra)
        dec = getattr(dec, "rad", dec)
    else:
        ra, dec = skycoords
    return np.asarray(ra, dtype=np.float64), np.asarray(dec, dtype=np.float64)


class SkyCoords:
    """Minimal (ra, dec) container in radians, the sky input of the plugins."""

    def __init__(self, ra, dec):
        self.ra = np.asarray(ra, dtype=np.float64)
        self.dec = np.asarray(dec, dtype=np.float64)
        if self.ra.shape != self.dec.shape:
            raise ValueError("ra and dec must have the same shape")

    def __len__(self):
        return len(self.ra)


#: ENU (east, north, up) -> the alt/az cartesian frame (x north, y east, z up)
#: that coordinates.point_source_crd_eq(az, alt) uses in the reference
ENU_TO_ALTAZ = np.array([[0.0, 1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])

ASTROM_KEYS = ("eh", "em", "v", "bm1", "bpn", "eral", "xpl", "ypl", "sphi", "cphi")


def atioq_matrix(astrom) -> np.ndarray:
    """CIRS -> ENU rotation of the apparent-place step (the reference's
    CoordinateRotationERFA._atioq, cpu/coords.py:89-116): Earth rotation angle,
    polar motion, then hour-angle/declination -> ENU at the observer latitude."""
    ce, se = np.cos(astrom["eral"]), np.sin(astrom["eral"])
    c2h = np.array([[ce, se, 0], [-se, ce, 0], [0, 0, 1]], dtype=np.float64)
    sx, cx = np.sin(astrom["xpl"]), np.cos(astrom["xpl"])
    sy, cy = np.sin(astrom["ypl"]), np.cos(astrom["ypl"])
    pm = np.array([[cx, 0, sx], [sx * sy, cy, -cx * sy], [-sx * cy, sy, cx * cy]], dtype=np.float64)
    enu = np.array([[0, 1, 0], [-astrom["sphi"], 0, astrom["cphi"]], [astrom["cphi"], 0, astrom["sphi"]]],
                   dtype=np.float64)
    return enu.dot(pm.dot(c2h))


def pack_astrom(astrom, dlim: float = 1e-6) -> np.ndarray:
    """The 18 doubles mvb_bcrs takes: eh[3], em, dlim, v[3], bm1, bpn[9]."""
    return np.ascontiguousarray(np.concatenate([
        np.asarray(astrom["eh"], dtype=np.float64).reshape(3), [float(astrom["em"]), dlim],
        np.asarray(astrom["v"], dtype=np.float64).reshape(3), [float(astrom["bm1"])],
        np.asarray(astrom["bpn"], dtype=np.float64).reshape(9)]))


def bcrs_refresh_plan(time_s, update_every: float) -> list[bool]:
    """Which time steps recompute the apparent-place directions: the first, and
    any step more than update_every seconds after the last refresh
    (cpu/coords.py:194-199)."""
    plan, last = [], None
    for t, ts in enumerate(np.asarray(time_s, dtype=np.float64)):
        if last is None or ts - time_s[last] > update_every:
            plan.append(True)
            last = t
        else:
            plan.append(False)
    return plan
