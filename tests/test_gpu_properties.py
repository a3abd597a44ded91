"""Size-independent properties at the larger configurations (config 3 / config 4
shapes), where the FP64 oracle would take minutes per slice:

* Hermitian symmetry of the all-pairs output: V[i, j, p, q] = conj(V[j, i, q, p]);
* autocorrelations real and non-negative;
* linearity in the source flux (I -> 4 I gives V -> 4 V);
* MatMul (tensor cores) and VectorDot (pair loop) agree on a sparse pair list;
* splitting the sources into chunks gives the same visibilities;
* a seeded source subset checked against the oracle at full antenna count.

Tolerances are the path's: 1e-6 of the autocorrelation scale.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from matvis_b200 import workloads as wl  # noqa: E402
from matvis_b200.engine import VisEngine, job_from_arrays  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(cfg, **kw):
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=cfg["polarized"], **{"antpairs": cfg.get("antpairs"), **kw})
    return VisEngine(spec).run().cpu().numpy()


@pytest.fixture(scope="module")
def c4_small():
    # config 4 shape per slice (350 antennas, 500,000 sources), 2 freqs x 3 times spanning 6 h
    c = wl.config4(nfreq=256, ntimes=64)
    return wl.subset(c, nfreq=2, ntimes=3, seed=4)


def test_config4_hermitian_and_autos(device, c4_small):
    v = _run(dict(c4_small, antpairs=None))  # (Nf, Nt, A*A, 2, 2)
    A = len(c4_small["antpos"])
    v = v.reshape(v.shape[0], v.shape[1], A, A, 2, 2)
    vt = np.conj(np.swapaxes(np.swapaxes(v, 2, 3), 4, 5))
    scale = np.abs(np.einsum("ftiipp->ftip", v)).max()
    assert np.abs(v - vt).max() <= 1e-6 * scale
    autos = np.einsum("ftiipp->ftip", v)
    assert np.abs(autos.imag).max() <= 1e-6 * scale
    assert autos.real.min() >= 0


def test_config4_linear_in_flux(device, c4_small):
    v1 = _run(dict(c4_small, antpairs=None))
    v4 = _run(dict(c4_small, antpairs=None, fluxes=4.0 * c4_small["fluxes"]))
    scale = np.abs(v1).max()
    assert np.abs(v4 - 4.0 * v1).max() <= 4e-6 * scale


def test_config4_chunking_invariant(device, c4_small):
    v1 = _run(dict(c4_small, antpairs=None))
    v3 = _run(dict(c4_small, antpairs=None), nchunks=3)
    scale = np.abs(v1).max()
    assert np.abs(v3 - v1).max() <= 1e-6 * scale


def test_config3_sparse_matmul_vs_vectordot(device):
    """The per-pair kernel (pinned: the cost model sends 5,000 pairs to the
    Hermitian product) against the tensor-core product's pair gather."""
    c = wl.config3(nsrc=1_000_000, npairs=5000)
    vm = _run(c, matprod="MatMul")
    vd = _run(c, matprod="VectorDot", pair_product="vecdot")
    full = _run(dict(c, antpairs=np.array([(i, i) for i in range(len(c["antpos"]))])))
    scale = np.abs(full).max()
    assert vm.shape == vd.shape == (1, 1, 5000, 2, 2)
    assert np.abs(vm - vd).max() <= 2e-6 * scale


def test_config3_subset_vs_oracle(device):
    """All 350 antennas, 5,000 pairs, a 30,000-source seeded subset of config 3."""
    c = wl.subset(wl.config3(nsrc=1_000_000, npairs=5000), nsrc=30000, seed=3)
    vm = _run(c, matprod="MatMul")
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in c["beams"]]
    ants = {i: tuple(p) for i, p in enumerate(c["antpos"])}
    ref = orc.simulate_vis(ants=ants, fluxes=c["fluxes"], ra=c["ra"], dec=c["dec"], freqs=c["freqs"], lsts=c["lsts"],
                           latitude=c["latitude"], beams=beams, polarized=True, beam_idx=c["beam_idx"],
                           antpairs=c["antpairs"])
    autos = _run(dict(c, antpairs=np.array([(i, i) for i in range(len(c["antpos"]))])))
    scale = np.abs(autos).max()
    assert np.abs(vm - ref).max() <= 1e-6 * scale


@pytest.fixture(scope="module")
def c3_dense_ref():
    """A 30,000-source seeded subset of config 3, all 350 antennas and pairs, and its FP64 oracle."""
    c = wl.subset(wl.config3(nsrc=1_000_000, npairs=5000), nsrc=30000, seed=5)
    c["antpairs"] = None
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in c["beams"]]
    ants = {i: tuple(p) for i, p in enumerate(c["antpos"])}
    ref = orc.simulate_vis(ants=ants, fluxes=c["fluxes"], ra=c["ra"], dec=c["dec"], freqs=c["freqs"], lsts=c["lsts"],
                           latitude=c["latitude"], beams=beams, polarized=True, beam_idx=c["beam_idx"])
    return c, ref


@pytest.mark.parametrize("mode,tol", [("fp16x3", 1e-6), ("bf16x6", 1e-6), ("tf32x3", 1e-6), ("bf16x3", 3e-5)])
def test_config3_split_modes_vs_oracle(device, c3_dense_ref, mode, tol):
    """Per split mode, max |dV| / sqrt(|V_ii| |V_jj|) over every output of the
    config-3 subset (complex128 output, so the product's error is what is seen)."""
    c, ref = c3_dense_ref
    vis = _run(c, precision=2, gemm_mode=mode)
    err = orc.cosine_error_metric(vis, ref, 2)
    print(f"config3 subset {mode}: max normalised error {err:.3e}")
    assert err <= tol, err


def test_config4_subset_vs_oracle(device):
    """Config 4 (6 h of LSTs, so the above-horizon count varies per time):
    complex64 output against the FP64 oracle on a seeded 4-frequency x 4-time
    subset, all 350 antennas, a 20,000-source subset of the sky."""
    c = wl.subset(wl.config4(nfreq=256, ntimes=64), nsrc=20000, nfreq=4, ntimes=4, seed=44)
    vis = _run(dict(c, antpairs=None), precision=1)
    assert vis.dtype == np.complex64
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in c["beams"]]
    ants = {i: tuple(p) for i, p in enumerate(c["antpos"])}
    ref = orc.simulate_vis(ants=ants, fluxes=c["fluxes"], ra=c["ra"], dec=c["dec"], freqs=c["freqs"], lsts=c["lsts"],
                           latitude=c["latitude"], beams=beams, polarized=True, beam_idx=c["beam_idx"])
    eci = orc.point_source_crd_eq(c["ra"], c["dec"])
    counts = [int(((orc.eci_to_enu_matrix(l, c["latitude"]) @ eci)[2] > 0).sum()) for l in c["lsts"]]
    assert len(set(counts)) == len(counts)  # the above-horizon count differs at every time
    err = orc.cosine_error_metric(vis, ref, 2)
    print(f"config4 subset complex64: max normalised error {err:.3e}")
    assert err <= 1e-6, err
