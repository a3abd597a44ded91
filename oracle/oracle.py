"""FP64 CPU oracle for the matvis per-(time, frequency) visibility path.

TEST INFRASTRUCTURE ONLY.  This module is the checker: ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  The product (``matvis_b200``) never does; the product
runs only on the CUDA library and fails loudly without it.

It restates, in plain numpy at complex128 / float64 (the reference's precision=2),
the reference CPU path ``matvis.cpu.simulate`` with ``CPUMatMul`` / ``CPUVectorDot``.
Each function names the reference lines it follows (paths relative to the
reference project root).

Parity pinning: ``tests/golden/make_golden.py`` runs the reference's own functions
(loaded with inert stand-ins for astropy / pyuvdata / cupy, which are absent) and
freezes their outputs in ``tests/golden/*.npz``; ``tests/test_oracle_golden.py``
checks every function below against those fixtures.  Two pieces of the reference
cannot be executed here at all and are therefore restated, not pinned:

* the astropy / ERFA sky rotation (``cpu/coords.py``): replaced by the rigid
  LST rotation ``eci_to_enu_matrix(lst, lat) @ point_source_crd_eq(ra, dec)`` that
  the reference's own coordinate tests use (``tests/test_coordinates.py:71-160``);
* pyuvdata's ``UVBeam`` / analytic beams: replaced by the reference GPU bilinear
  scheme (``gpu/beams.py:127-200``, pinned) on in-memory grids, plus an achromatic
  Gaussian power beam defined in this file.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy import ndimage

#: Speed of light in m/s (the SI-defined value astropy's ``constants.c`` carries).
SPEED_OF_LIGHT = 299792458.0


# ---------------------------------------------------------------------------
# Coordinates (src/matvis/coordinates.py)
# ---------------------------------------------------------------------------
def point_source_crd_eq(ra, dec):
    """ECI unit vectors of sources; ``coordinates.py:174-200``. Shape (3, N)."""
    ra = np.asarray(ra, dtype=np.float64)
    dec = np.asarray(dec, dtype=np.float64)
    return np.asarray([np.cos(ra) * np.cos(dec), np.cos(dec) * np.sin(ra), np.sin(dec)])


def eci_to_enu_matrix(ha, lat):
    """3x3 ECI->ENU rotation; ``coordinates.py:91-125``."""
    return np.array(
        [
            [-np.sin(ha), np.cos(ha), 0.0 * ha],
            [-np.sin(lat) * np.cos(ha), -np.sin(lat) * np.sin(ha), np.cos(lat)],
            [np.cos(lat) * np.cos(ha), np.cos(lat) * np.sin(ha), np.sin(lat)],
        ],
        dtype=np.float64,
    )


def rotate_fixed_order(rot, eci):
    """Topocentric ENU coordinates ``rot @ eci`` in one fixed operation order.

    Row r is ``(R[r,0]*x + R[r,1]*y) + R[r,2]*z`` with each multiply and add
    rounded separately (numpy elementwise operations never fuse).  The CUDA
    rotation kernel evaluates exactly this sequence with ``__dmul_rn`` /
    ``__dadd_rn``, so the horizon test ``z > 0`` selects bit-identical sources.
    """
    rot = np.asarray(rot, dtype=np.float64)
    x, y, z = (np.asarray(eci[i], dtype=np.float64) for i in range(3))
    out = np.empty((3, x.size), dtype=np.float64)
    for r in range(3):
        out[r] = (rot[r, 0] * x + rot[r, 1] * y) + rot[r, 2] * z
    return out


def enu_to_az_za(enu_e, enu_n, orientation="astropy", periodic_azimuth=True):
    """Azimuth / zenith angle from ENU direction cosines; ``coordinates.py:31-88``."""
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


# ---------------------------------------------------------------------------
# Horizon selection (src/matvis/core/coords.py:77-150)
# ---------------------------------------------------------------------------
def nsrc_alloc(chunk_size: int, source_buffer: float) -> int:
    """Capacity of the above-horizon buffers; ``core/coords.py:77-82``."""
    if chunk_size > 1000:
        return int(chunk_size * source_buffer)
    return chunk_size


def select_chunk(topo, flux, chunk: int, chunk_size: int, alloc: int):
    """Strict ``z > 0`` selection of one source chunk; ``core/coords.py:99-150``.

    Returns (coords (3, alloc), flux (alloc,), n, kept_indices).  Slots past ``n``
    hold zero coordinates here (the reference keeps stale values there, which only
    ever meet zero flux).
    """
    slc = slice(chunk * chunk_size, (chunk + 1) * chunk_size)
    t = topo[:, slc]
    f = flux[slc]
    kept = np.where(t[2] > 0)[0]
    n = len(kept)
    if n > alloc:
        raise ValueError(
            f"nsrc_alloc ({alloc}) is too small for the number of sources above "
            f"horizon ({n}). Try increasing source_buffer."
        )
    coords = np.zeros((3, alloc), dtype=np.float64)
    fl = np.zeros(alloc, dtype=f.dtype)
    coords[:, :n] = t[:, kept]
    fl[:n] = f[kept]
    return coords, fl, n, kept + chunk * chunk_size


# ---------------------------------------------------------------------------
# Beams
# ---------------------------------------------------------------------------
@dataclass
class GridBeam:
    """A beam tabulated on a regular (za, az) grid.

    ``data`` has shape (nax, nfeed, nza, naz): complex E-field components when
    ``beam_type == "efield"``, a real power pattern (1, 1, nza, naz) when
    ``beam_type == "power"``.  ``za[0]`` must be 0 (the reference maps
    ``za / dza`` to the row coordinate, ``gpu/beams.py:184``).
    """

    data: np.ndarray
    az: np.ndarray
    za: np.ndarray
    beam_type: str = "efield"

    @property
    def daz(self):
        return float(np.diff(self.az)[0])

    @property
    def dza(self):
        return float(np.diff(self.za)[0])

    @property
    def azmin(self):
        return float(np.min(self.az))


@dataclass
class GaussianPowerBeam:
    """Achromatic Gaussian beam in zenith angle, unpolarised.

    E-field amplitude ``exp(-za^2 / (2 sigma^2))``; the power pattern is its
    square, and the simulation takes ``sqrt`` of the power as ``cpu/beams.py:46``.
    """

    sigma: float
    beam_type: str = "power"

    def power(self, za):
        return np.exp(-(za**2) / (self.sigma**2))


def bilinear_beam(grids, daz, dza, azmin, az, za):
    """Order-1 ``map_coordinates`` per (beam, feed, axis); ``gpu/beams.py:127-200``.

    ``grids`` has shape (nbeam, nax, nfeed, nza, naz); the output is
    (nbeam, nfeed, nax, nsrc) complex128, with ``sqrt`` applied for power grids.
    Points outside ``[0, n-1]`` on either grid axis give 0 (scipy's
    ``mode='constant'``, which cupyx mirrors).
    """
    grids = np.asarray(grids)
    nbeam, nax, nfeed = grids.shape[:3]
    out = np.zeros((nbeam, nfeed, nax, len(az)), dtype=np.complex128)
    for bm in range(nbeam):
        coords = np.asarray([za / dza[bm], (az - azmin[bm]) / daz[bm]])
        for fd in range(nfeed):
            for ax in range(nax):
                g = grids[bm, ax, fd]
                if np.iscomplexobj(g):
                    v = ndimage.map_coordinates(g.real.astype(np.float64), coords, order=1) + 1j * ndimage.map_coordinates(
                        g.imag.astype(np.float64), coords, order=1
                    )
                else:
                    v = ndimage.map_coordinates(g.astype(np.float64), coords, order=1)
                out[bm, fd, ax] = v
    if not np.iscomplexobj(grids):
        out = np.sqrt(out)
    return out


def beam_response(beams, polarized: bool, crd_e, crd_n):
    """Interpolated beam (nbeam, nfeed, nax, nsrc) at ENU direction cosines.

    Follows ``GPUBeamInterpolator._interp`` (``gpu/beams.py:103-124``): uvbeam
    azimuth orientation, then :func:`bilinear_beam`; analytic Gaussian power beams
    are evaluated directly (``sqrt`` of power, ``cpu/beams.py:43-46``).
    """
    az, za = enu_to_az_za(crd_e, crd_n, orientation="uvbeam")
    nfeed = nax = 2 if polarized else 1
    out = np.zeros((len(beams), nfeed, nax, len(az)), dtype=np.complex128)
    for i, bm in enumerate(beams):
        if isinstance(bm, GaussianPowerBeam):
            if polarized:
                raise ValueError("beam type must be efield if using polarized=True")
            out[i, 0, 0] = np.sqrt(bm.power(za))
        else:
            if polarized and bm.beam_type != "efield":
                raise ValueError("beam type must be efield if using polarized=True")
            data = bm.data
            if not polarized and bm.beam_type == "efield":
                # Unpolarised use of an E-field grid: power of feed 0 summed over
                # the vector axes (the single-feed power pattern), as prepared by
                # prepare_beam_unpolarized (core/beams.py:15-32) for feed "x".
                data = np.sum(np.abs(data[:, :1]) ** 2, axis=0, keepdims=True)
            out[i] = bilinear_beam(data[None], [bm.daz], [bm.dza], [bm.azmin], az, za)[0]
    return out


# ---------------------------------------------------------------------------
# tau, Z, products (src/matvis/core/tau.py, core/getz.py, cpu/matprod.py)
# ---------------------------------------------------------------------------
def exptau(antpos, freq, crd):
    """``exp(+i 2 pi nu / c * D . X)``; ``core/tau.py:30-31, 65-66`` (code sign)."""
    ap = np.asarray(antpos, dtype=np.float64) * (2.0 * np.pi * freq) * 1j / SPEED_OF_LIGHT
    return np.exp(ap @ np.asarray(crd, dtype=np.float64))


def zmatrix(sqrt_flux, beam, ext, beam_idx, nfeed, nax):
    """Z (nant*nfeed, nax*nsrc); ``core/getz.py:80-100``."""
    nant, nsrc = ext.shape
    e = ext * sqrt_flux
    z = np.empty((nant, nfeed, nax, nsrc), dtype=np.complex128)
    for fd in range(nfeed):
        for ax in range(nax):
            z[:, fd, ax, :] = e
    if beam_idx is None:
        z *= beam
    else:
        for ant, bmidx in enumerate(beam_idx):
            z[ant] *= beam[bmidx]
    return z.reshape(nant * nfeed, nax * nsrc)


def matmul_vis(z, nant, nfeed, antpairs=None):
    """``CPUMatMul.compute``; ``cpu/matprod.py:11-32``. Returns (npairs, nfeed, nfeed)."""
    v = z.conj().dot(z.T)
    v = v.reshape(nant, nfeed, nant, nfeed).transpose((0, 2, 3, 1))
    if antpairs is None:
        return v.reshape(nant * nant, nfeed, nfeed)
    ap = np.asarray(antpairs)
    return v[ap[:, 0], ap[:, 1]]


def vectordot_vis(z, nant, nfeed, antpairs):
    """``CPUVectorDot.compute``; ``cpu/matprod.py:35-53``."""
    z = z.reshape((nant, nfeed, -1))
    ap = np.asarray(antpairs)
    out = np.empty((len(ap), nfeed, nfeed), dtype=np.complex128)
    for i, (ai, aj) in enumerate(ap):
        out[i] = z[aj].dot(z[ai].conj().T)
    return out


def all_pairs(nant):
    """Default pair list, ``i`` slow; ``core/matprod.py:37-40``."""
    return np.array([(i, j) for i in range(nant) for j in range(nant)])


# ---------------------------------------------------------------------------
# Driver (src/matvis/cpu/cpu.py:163-277) and wrapper (src/matvis/wrapper.py)
# ---------------------------------------------------------------------------
def simulate(
    *,
    antpos,
    freq,
    lsts,
    latitude,
    ra,
    dec,
    I_sky,
    beam_list,
    polarized=False,
    beam_idx=None,
    antpairs=None,
    nchunks=1,
    source_buffer=1.0,
    matprod="MatMul",
    eci=None,
    astrom=None,
    time_s=None,
    update_bcrs_every=0.0,
    coherency=None,
):
    """One frequency, all times; ``cpu/cpu.py:163-277`` at precision=2.

    ``coherency`` (N, 2, 2) complex (polarised only): a polarised sky.  Each
    time its frame is rotated to alt/az (``coherency_rotation`` with the time's
    rigid ICRS -> alt/az rotation) and the visibilities are summed directly as
    V_ij = exptau_j conj(exptau_i) E_j C' E_i^H.

    With ``astrom`` (one apco parameter dict per time) the rotation is the
    ERFA-style apparent place of ``CoordinateRotationERFA`` (cpu/coords.py:186-230),
    refreshing the deflected/aberrated directions when more than
    ``update_bcrs_every`` seconds of ``time_s`` have passed (every step when
    ``time_s`` is None); otherwise the LST rotation.

    Returns (ntimes, npairs, nfeed, nfeed) complex128 when polarized, else
    (ntimes, npairs).
    """
    antpos = np.asarray(antpos, dtype=np.float64)
    nant = antpos.shape[0]
    nfeed = nax = 2 if polarized else 1
    nsrc = len(I_sky)
    nbeam = len(beam_list)
    if beam_idx is None and nbeam not in (1, nant):
        raise ValueError("If number of beams provided is not 1 or nant, beam_idx must be provided.")
    if beam_idx is None and nbeam == nant:
        beam_idx = np.arange(nant)
    if beam_idx is None:
        beam_idx = np.zeros(nant, dtype=int)
    flux = np.sqrt(0.5 * np.asarray(I_sky, dtype=np.float64))  # cpu/cpu.py:188
    if eci is None:
        eci = point_source_crd_eq(ra, dec)
    chunk_size = int(np.ceil(nsrc / nchunks))
    alloc = nsrc_alloc(chunk_size, source_buffer)
    pairs = all_pairs(nant) if antpairs is None else np.asarray(antpairs)
    vis = np.zeros((len(lsts), len(pairs), nfeed, nfeed), dtype=np.complex128)
    last, bcrs = None, None
    for t, lst in enumerate(lsts):
        if astrom is None:
            topo = rotate_fixed_order(eci_to_enu_matrix(lst, latitude), eci)
        else:
            if last is None or time_s is None or time_s[t] - time_s[last] > update_bcrs_every:
                bcrs, last = erfa_bcrs(eci, astrom[t]), t
            topo = rotate_fixed_order(erfa_atioq_matrix(astrom[t]), bcrs)
        if coherency is not None:
            rigid = (eci_to_enu_matrix(lst, latitude) if astrom is None
                     else erfa_atioq_matrix(astrom[t]) @ np.asarray(astrom[t]["bpn"], dtype=np.float64))
            vis[t] += _polsky_vis_time(topo, eci, coherency, rigid, antpos, freq, beam_list, beam_idx, nchunks,
                                       chunk_size, alloc, pairs if antpairs is not None else None, nant, ra, dec)
            continue
        for c in range(nchunks):
            crd, fl, n, _ = select_chunk(topo, flux, c, chunk_size, alloc)
            if n == 0:
                continue  # contributes exact zeros (CPU-driver semantics)
            crd = crd[:, :n]
            fl = fl[:n]
            beam = beam_response(beam_list, polarized, crd[0], crd[1])
            ext = exptau(antpos, freq, crd)
            z = zmatrix(fl, beam, ext, beam_idx, nfeed, nax)
            if matprod in ("MatMul", "CPUMatMul"):
                vis[t] += matmul_vis(z, nant, nfeed, antpairs)
            else:
                vis[t] += vectordot_vis(z, nant, nfeed, pairs)
    return vis if polarized else vis[:, :, 0, 0]


def _polsky_vis_time(topo, eci, coherency, rigid, antpos, freq, beam_list, beam_idx, nchunks, chunk_size, alloc,
                     pairs, nant, ra, dec):
    """One time of the polarised-sky sum (chunks as in cpu/cpu.py:247-272)."""
    nf = 2
    out = np.zeros((nant * nant if pairs is None else len(pairs), nf, nf), dtype=np.complex128)
    r_avg = ENU_TO_ALTAZ @ rigid
    for c in range(nchunks):
        c0 = c * chunk_size
        sel = np.flatnonzero(topo[2, c0 : c0 + chunk_size] > 0) + c0
        if len(sel) == 0:
            continue
        if len(sel) > alloc:
            raise ValueError("nsrc_alloc too small")
        crd = topo[:, sel]
        az, za = enu_to_az_za(crd[0], crd[1], orientation="astropy")
        rot = coherency_rotation(ra[sel], dec[sel], np.pi / 2 - za, az, r_avg)
        cp = rotate_coherency(coherency[sel][:, None], rot)[:, 0]
        beam = beam_response(beam_list, True, crd[0], crd[1])  # (B, F, X, n)
        ext = exptau(antpos, freq, crd)  # (A, n)
        y = ext[:, None, None, :] * beam[beam_idx]  # (A, F, X, n)
        w = np.einsum("apxs,sxy->apys", y, cp)
        v = np.einsum("jpys,iqys->ijpq", w, np.conj(y))
        out += v.reshape(nant * nant, nf, nf) if pairs is None else v[pairs[:, 0], pairs[:, 1]]
    return out


def simulate_vis(
    *,
    ants,
    fluxes,
    ra,
    dec,
    freqs,
    lsts,
    latitude,
    beams,
    polarized=False,
    beam_idx=None,
    antpairs=None,
    matprod="MatMul",
    nchunks=1,
    source_buffer=1.0,
    **rotation,
):
    """Frequency loop of ``wrapper.simulate_vis``; ``wrapper.py:150-199``.
    ``rotation`` holds the ERFA keywords of :func:`simulate` (astrom, time_s,
    update_bcrs_every)."""
    antpos = np.array([ants[k] for k in ants.keys()], dtype=np.float64)
    fluxes = np.asarray(fluxes)
    assert fluxes.shape[:2] == (len(ra), len(freqs)), "The `fluxes` array must have shape (NSRCS, NFREQS[, 2, 2])."
    pol_sky = fluxes.ndim == 4
    eci = point_source_crd_eq(ra, dec)
    out = []
    for i, freq in enumerate(freqs):
        out.append(
            simulate(
                antpos=antpos,
                freq=freq,
                lsts=lsts,
                latitude=latitude,
                ra=ra,
                dec=dec,
                I_sky=np.real(np.trace(fluxes[:, i], axis1=-2, axis2=-1)) if pol_sky else fluxes[:, i],
                coherency=fluxes[:, i] if pol_sky else None,
                beam_list=beams,
                polarized=polarized,
                beam_idx=beam_idx,
                antpairs=antpairs,
                nchunks=nchunks,
                source_buffer=source_buffer,
                matprod=matprod,
                eci=eci,
                **rotation,
            )
        )
    return np.asarray(out)


# ---------------------------------------------------------------------------
# Redundant-baseline pair selection (src/matvis/cli.py:273-290, :316)
# ---------------------------------------------------------------------------
def get_redundancies(bls, ndecimals: int = 2):
    """One (i, j), i < j, per class of equal rounded (u, v) up to sign, in the
    order the reference's double loop meets them; ``cli.py:273-290``."""
    bls = np.round(np.asarray(bls, dtype=np.float64), decimals=ndecimals)
    seen = set()
    pairs = []
    nant = bls.shape[0]
    for i in range(nant):
        for j in range(i + 1, nant):
            u, v = bls[i, j]
            if (u, v) not in seen and (-u, -v) not in seen:
                seen.add((u, v))
                pairs.append([i, j])
    return pairs


def redundant_antpairs(antpos, ndecimals: int = 2):
    """(npairs, 2) representatives for the east/north baselines ``pos[j] - pos[i]``
    (``cli.py:316``)."""
    antpos = np.asarray(antpos, dtype=np.float64)
    bls = antpos[np.newaxis, :, :2] - antpos[:, np.newaxis, :2]
    return np.asarray(get_redundancies(bls, ndecimals), dtype=np.int64).reshape(-1, 2)


# ---------------------------------------------------------------------------
# Chunk planning (src/matvis/_utils.py:124-319)
# ---------------------------------------------------------------------------
def get_required_chunks(freemem, nax, nfeed, nant, nsrc, nbeam, nbeampix, precision, source_buffer=1.0, memory_buffer=0.9):
    """Byte-model chunk count; ``_utils.py:124-209``."""
    if not (0 < memory_buffer <= 1.0):
        raise ValueError("memory_buffer must be in the range (0, 1]")
    rsize = 4 * precision
    csize = 2 * rsize
    total = freemem
    ch = 0
    while total >= freemem * memory_buffer and ch < 100:
        ch += 1
        nchunk = int(nsrc // ch * source_buffer)
        total = (
            nant * 3 * rsize
            + nsrc * rsize
            + nbeampix * nfeed * nax * csize
            + 3 * nsrc * rsize
            + 3 * 3 * rsize
            + 3 * nsrc * rsize
            + 3 * nchunk * rsize
            + nchunk * rsize
            + nant * nchunk * csize
            + nbeam * nfeed * nax * nchunk * csize
            + nchunk * nfeed * nant * nax * csize
            + ch * nfeed * nant * nfeed * nant * csize
        )
    return max(ch, 1)


def cosine_error_metric(v, ref, nfeed):
    """Max over outputs of ``|V - V_ref| / sqrt(|V_ii^pp| |V_jj^qq|)`` (all-pairs layout).

    ``v`` / ``ref``: (..., nant*nant, nfeed, nfeed).  The denominator uses the
    oracle's autocorrelations, bounding each cross term by Cauchy-Schwarz.
    """
    ref = np.asarray(ref)
    v = np.asarray(v)
    nant = int(round(np.sqrt(ref.shape[-3])))
    r = ref.reshape(ref.shape[:-3] + (nant, nant, nfeed, nfeed))
    d = (v - ref).reshape(r.shape)
    auto = np.abs(np.einsum("...iipp->...ip", r))  # (..., nant, nfeed)
    # out[i, j, p, q] pairs feed q of antenna i with feed p of antenna j.
    den = np.sqrt(auto[..., :, None, None, :] * auto[..., None, :, :, None])
    den = np.where(den > 0, den, np.inf)
    return float(np.max(np.abs(d) / den)) if d.size else 0.0


# ---------------------------------------------------------------------------
# ERFA-style apparent place (src/matvis/cpu/coords.py:89-215)
# ---------------------------------------------------------------------------
#: Schwarzschild radius of the Sun in au (cpu/coords.py:11).
ERFA_SRS = 1.97412574336e-8


def erfa_ld(p, e, em, dlim):
    """Light deflection by the Sun; ``CoordinateRotationERFA._ld`` (cpu/coords.py:118-148)."""
    p = np.array(p, dtype=np.float64)
    e = np.asarray(e, dtype=np.float64)
    qpe = (p.T + e).T
    qdqpe = np.sum(p * qpe, axis=0)
    qdqpe = np.clip(qdqpe, dlim, None)
    w = ERFA_SRS / em / qdqpe
    eq = np.cross(e.T, p.T)
    peq = np.cross(p.T, eq).T
    return p + w[None] * peq


def erfa_ab(pnat, v, s, bm1):
    """Aberration; ``CoordinateRotationERFA._ab`` (cpu/coords.py:150-174), including its
    use of the already-scaled direction in the w2 term."""
    pnat = np.array(pnat, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    pdv = np.dot(v, pnat)
    w1 = 1.0 + pdv / (1.0 + bm1)
    w2 = ERFA_SRS / s
    pnat = pnat * bm1
    pnat = pnat + np.outer(v, w1) + w2 * (v - (pdv * pnat).T).T
    return pnat / np.linalg.norm(pnat, axis=0)


def erfa_atioq_matrix(astrom):
    """CIRS -> ENU 3x3 of ``CoordinateRotationERFA._atioq`` (cpu/coords.py:89-116)."""
    ce, se = np.cos(astrom["eral"]), np.sin(astrom["eral"])
    c2h = np.array([[ce, se, 0], [-se, ce, 0], [0, 0, 1]])
    sx, cx = np.sin(astrom["xpl"]), np.cos(astrom["xpl"])
    sy, cy = np.sin(astrom["ypl"]), np.cos(astrom["ypl"])
    pm = np.array([[cx, 0, sx], [sx * sy, cy, -cx * sy], [-sx * cy, sy, cx * cy]])
    enu = np.array([[0, 1, 0], [-astrom["sphi"], 0, astrom["cphi"]], [astrom["cphi"], 0, astrom["sphi"]]])
    return enu.dot(pm.dot(c2h))


def erfa_bcrs(eci, astrom, dlim=1e-6):
    """_set_bcrs (cpu/coords.py:186-215): deflection, aberration, bias-precession-nutation."""
    p = erfa_ld(eci, astrom["eh"], astrom["em"], dlim)
    p = erfa_ab(p, astrom["v"], astrom["em"], astrom["bm1"])
    return np.asarray(astrom["bpn"], dtype=np.float64) @ p


# ---------------------------------------------------------------------------
# Polarised sky: frame rotation of the source coherency
# (coordinates.py:288-580, core/coords.py:152-175)
# ---------------------------------------------------------------------------
ENU_TO_ALTAZ = np.array([[0.0, 1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])


def _theta_hat(theta, phi):
    """coordinates.py:537-556."""
    return np.stack([np.cos(phi) * np.cos(theta), np.sin(phi) * np.cos(theta), -np.sin(theta)])


def _phi_hat(theta, phi):
    """coordinates.py:559-576."""
    return np.stack([-np.sin(phi), np.cos(phi), np.zeros_like(phi)])


def coherency_rotation(ra, dec, alt, az, r_avg):
    """2x2 (cos X, sin X; -sin X, cos X) per source, shape (2, 2, N):
    calc_coherency_rotation (coordinates.py:288-330) with the average
    ICRS -> alt/az rotation ``r_avg`` supplied.  The perturbation rotation
    carrying r_avg . frame_vec onto the alt/az vector (vecs2rot,
    coordinates.py:387-452) is the identity where the two vectors coincide
    exactly (the reference divides 0 by 0 there)."""
    ra, dec, alt, az = (np.asarray(x, dtype=np.float64) for x in (ra, dec, alt, az))
    frame = point_source_crd_eq(ra, dec)
    altaz = point_source_crd_eq(az, alt)
    r1 = r_avg @ frame
    axis = np.cross(r1, altaz, axis=0)
    sin_psi = np.linalg.norm(axis, axis=0)
    cos_psi = np.sum(r1 * altaz, axis=0)
    psi = np.arctan2(sin_psi, cos_psi)
    with np.errstate(invalid="ignore", divide="ignore"):
        n = np.where(sin_psi > 0, axis / np.where(sin_psi > 0, sin_psi, 1.0), 0.0)
    zero = np.zeros_like(ra)
    k = np.array([[zero, -n[2], n[1]], [n[2], zero, -n[0]], [-n[1], n[0], zero]])
    k2 = np.einsum("abn,bcn->acn", k, k)
    perturb = np.eye(3)[..., None] + np.sin(psi) * k + (1.0 - np.cos(psi)) * k2
    exact = np.einsum("abn,bc->acn", perturb, r_avg)
    th = _theta_hat(np.pi / 2 - dec, ra)
    ph = _phi_hat(np.pi / 2 - dec, ra)
    bh = np.einsum("ban,bn->an", exact, _theta_hat(np.pi / 2 - alt, az))
    cos_x = np.sum(bh * th, axis=0)
    sin_x = np.sum(bh * ph, axis=0)
    return np.array([[cos_x, sin_x], [-sin_x, cos_x]])


def rotate_coherency(coh, rot):
    """C' = R^T C R per source and frequency; core/coords.py:170-173.
    coh (N, Nf, 2, 2), rot (2, 2, N)."""
    return np.einsum("ban,nfbc,cdn->nfad", rot, coh, rot)


def stokes_to_coherency(i, q, u, v):
    """0.5 [[I + Q, U - iV], [U + iV, I - Q]] with shape (..., 2, 2)."""
    i, q, u, v = np.broadcast_arrays(*(np.asarray(x, dtype=np.float64) for x in (i, q, u, v)))
    c = np.empty(i.shape + (2, 2), dtype=np.complex128)
    c[..., 0, 0] = 0.5 * (i + q)
    c[..., 1, 1] = 0.5 * (i - q)
    c[..., 0, 1] = 0.5 * (u - 1j * v)
    c[..., 1, 0] = 0.5 * (u + 1j * v)
    return c
