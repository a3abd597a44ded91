"""Parity at the headline sizes: whole (f, t) slices, every source, antenna and
pair, against the FP64 oracle.

* config 2 (the benchmark's workload): 350 antennas x 196,608 sources, K = 196,608
  columns of Z per slice;
* config 3: 350 antennas x 1,000,000 sources, K ~ 1e6 columns per slice, where the
  product's partial sums are longest.

The split modes the product offers at the 1e-6 bar (fp16x3, the default, and
tf32x3) are checked with complex128 output, so that the product's own error is
what is measured; the default configuration is also checked with the complex64
output the benchmark times.  Metric: max over outputs of |V - V_oracle| /
sqrt(|V_ii| |V_jj|) (autocorrelation-normalised; Cauchy-Schwarz bounds it).
The oracle sums config 3 in source chunks (cpu/cpu.py:247-272) to bound host
memory; the chunk sum is the same sum.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from matvis_b200 import workloads as wl  # noqa: E402
from matvis_b200.engine import VisEngine, job_from_arrays  # noqa: E402
from oracle import oracle as orc  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _run(cfg, **kw):
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=cfg["lsts"], latitude=cfg["latitude"], beams=cfg["beams"], beam_idx=cfg["beam_idx"],
                           polarized=True, antpairs=None, **kw)
    eng = VisEngine(spec)
    out = eng.run().cpu().numpy()
    del eng
    torch.cuda.empty_cache()
    return out


def _oracle(cfg, nchunks=1):
    beams = [orc.GridBeam(data=b.data.astype(np.complex128), az=b.az, za=b.za) for b in cfg["beams"]]
    v = orc.simulate(antpos=np.asarray(cfg["antpos"]), freq=float(cfg["freqs"][0]), lsts=cfg["lsts"],
                     latitude=cfg["latitude"], ra=cfg["ra"], dec=cfg["dec"], I_sky=cfg["fluxes"][:, 0],
                     beam_list=beams, polarized=True, beam_idx=cfg["beam_idx"], nchunks=nchunks)
    return v[None]  # (1, Nt, A*A, 2, 2)


def _slice(cfg, f, t):
    c = dict(cfg)
    c["freqs"] = np.asarray(cfg["freqs"])[f:f + 1]
    c["fluxes"] = np.asarray(cfg["fluxes"])[:, f:f + 1]
    c["lsts"] = np.asarray(cfg["lsts"])[t:t + 1]
    return c


@pytest.fixture(scope="module")
def c2_slice():
    """Config 2's middle frequency at its last time step, whole sky."""
    cfg = wl.config2()
    c = _slice(cfg, 32, 15)
    return c, _oracle(c)


@pytest.fixture(scope="module")
def c3_slice():
    """Config 3's one slice, 1,000,000 sources."""
    c = wl.config3(nsrc=1_000_000)
    c["antpairs"] = None
    return c, _oracle(c, nchunks=8)


@pytest.mark.parametrize("mode", ["fp16x3", "tf32x3"])
def test_config2_full_slice_vs_oracle(device, c2_slice, mode):
    c, ref = c2_slice
    vis = _run(c, precision=2, gemm_mode=mode)
    err = orc.cosine_error_metric(vis, ref, 2)
    print(f"config2 full slice ({len(c['ra'])} sources) {mode}: max normalised error {err:.3e}")
    assert err <= TOL, err


def test_config2_full_slice_complex64_vs_oracle(device, c2_slice):
    """The benchmark's own configuration: fp16x3, complex64 output."""
    c, ref = c2_slice
    vis = _run(c, precision=1, gemm_mode="fp16x3")
    assert vis.dtype == np.complex64
    err = orc.cosine_error_metric(vis, ref, 2)
    print(f"config2 full slice complex64 fp16x3: max normalised error {err:.3e}")
    assert err <= TOL, err


@pytest.mark.parametrize("mode", ["fp16x3", "tf32x3"])
def test_config3_full_slice_vs_oracle(device, c3_slice, mode):
    c, ref = c3_slice
    vis = _run(c, precision=2, gemm_mode=mode)
    err = orc.cosine_error_metric(vis, ref, 2)
    print(f"config3 full slice ({len(c['ra'])} sources) {mode}: max normalised error {err:.3e}")
    assert err <= TOL, err
