"""ERFA-style apparent place on the GPU (``mvb_bcrs`` + ``mvb_rotate``) against the
reference's own ``CoordinateRotationERFA`` steps (``tests/golden/erfa.npz``) and
the oracle.

Tolerances: apparent directions and topocentric vectors within 4e-15 absolute of
the reference (FP64 throughout; the kernel and numpy differ in operation order
only); visibilities through the ERFA rotation within the pipeline bound
max |dV| / sqrt(|V_ii| |V_jj|) <= 1e-6.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import matvis_b200 as mv  # noqa: E402
from matvis_b200 import _lib  # noqa: E402
from matvis_b200 import workloads as wl  # noqa: E402
from matvis_b200.coordinates import pack_astrom  # noqa: E402
from matvis_b200.engine import VisEngine, job_from_arrays  # noqa: E402
from oracle import oracle as orc  # noqa: E402

from .conftest import golden  # noqa: E402

pytestmark = pytest.mark.gpu
KEYS = ("eh", "em", "v", "bm1", "bpn", "eral", "xpl", "ypl", "sphi", "cphi")


def _astrom(t):
    g = golden("erfa")
    return {k: (g[f"t{t}_{k}"] if g[f"t{t}_{k}"].ndim else float(g[f"t{t}_{k}"])) for k in KEYS}


def _plugin(times, update_bcrs_every=0.0):
    g = golden("erfa")
    eci = g["eci"]
    ra, dec = np.arctan2(eci[1], eci[0]), np.arcsin(eci[2])
    rot = mv.CoordinateRotationERFA(update_bcrs_every, flux=np.ones(eci.shape[1]), times=np.asarray(times),
                                    telescope_loc=wl.HERA_LAT, skycoords=(ra, dec), source_buffer=1.0,
                                    astrom=[_astrom(t) for t in range(3)])
    rot.setup()
    rot.eci.copy_(torch.as_tensor(eci))  # the fixture's exact unit vectors
    return rot


def test_bcrs_kernel_matches_reference_steps(device):
    g = golden("erfa")
    rot = _plugin([0.0, 1.0, 2.0])
    for t in range(3):
        rot.rotate(t)
        np.testing.assert_allclose(rot._bcrs.cpu().numpy(), g[f"t{t}_bcrs"], rtol=0, atol=4e-15)
        np.testing.assert_allclose(rot.all_coords_topo.cpu().numpy(), g[f"t{t}_topo"], rtol=0, atol=4e-15)


def test_bcrs_refreshes_after_interval(device):
    """times 0, 60, 400 s with a 100 s interval: the second step reuses the
    first step's apparent directions, the third recomputes them."""
    g = golden("erfa")
    rot = _plugin([0.0, 60.0, 400.0], update_bcrs_every=100.0)
    b0 = g["t0_bcrs"]
    rot.rotate(0)
    rot.rotate(1)
    stale = orc.erfa_atioq_matrix(_astrom(1)) @ b0
    np.testing.assert_allclose(rot.all_coords_topo.cpu().numpy(), stale, rtol=0, atol=4e-15)
    assert np.abs(stale - g["t1_topo"]).max() > 1e-6  # the refresh is observable
    rot.rotate(2)
    np.testing.assert_allclose(rot.all_coords_topo.cpu().numpy(), g["t2_topo"], rtol=0, atol=4e-15)


def test_bcrs_rejects_bad_parameters(device):
    eci = torch.zeros((3, 4), dtype=torch.float64, device="cuda")
    out = torch.zeros_like(eci)
    a = pack_astrom(_astrom(0))
    a[3] = 0.0  # em
    rc = _lib.lib.mvb_bcrs(_lib.ptr(eci), 4, a.ctypes.data_as(_lib.c_void_p), _lib.ptr(out), None)
    assert rc == _lib.MVB_ERR_ARG


@pytest.mark.parametrize("update,time_s", [(0.0, None), (100.0, np.array([0.0, 60.0, 400.0]))])
def test_erfa_engine_vs_oracle(device, update, time_s):
    cfg = wl.config1()
    astrom = [_astrom(t) for t in range(3)]
    lsts = np.zeros(3)  # unused by the ERFA rotation beyond the time count
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    ref = orc.simulate_vis(ants=ants, fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=lsts, latitude=cfg["latitude"], beams=[orc.GaussianPowerBeam(sigma=0.2)],
                           astrom=astrom, time_s=time_s, update_bcrs_every=update)
    spec = job_from_arrays(ants=cfg["antpos"], fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=lsts, latitude=cfg["latitude"], beams=cfg["beams"], precision=2, gemm_mode="bf16x6",
                           astrom=astrom, time_s=time_s, update_bcrs_every=update)
    vis = VisEngine(spec).run().cpu().numpy()[..., 0, 0]
    err = orc.cosine_error_metric(vis[..., None, None], ref[..., None, None], 1)
    assert err <= 1e-6, err


def test_simulate_vis_erfa_keywords(device):
    cfg = wl.config1()
    astrom = [_astrom(t) for t in range(3)]
    ants = {i: tuple(p) for i, p in enumerate(cfg["antpos"])}
    kw = dict(ants=ants, fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"], times=np.zeros(3),
              beams=cfg["beams"], telescope_loc=cfg["latitude"], precision=2)
    vis = mv.simulate_vis(**kw, coord_method="GPUCoordinateRotationERFA",
                          coord_method_params={"astrom": astrom, "time_s": [0.0, 60.0, 400.0],
                                               "update_bcrs_every": 100.0})
    ref = orc.simulate_vis(ants=ants, fluxes=cfg["fluxes"], ra=cfg["ra"], dec=cfg["dec"], freqs=cfg["freqs"],
                           lsts=np.zeros(3), latitude=cfg["latitude"], beams=[orc.GaussianPowerBeam(sigma=0.2)],
                           astrom=astrom, time_s=np.array([0.0, 60.0, 400.0]), update_bcrs_every=100.0)
    err = orc.cosine_error_metric(vis[..., None, None], ref[..., None, None], 1)
    assert err <= 1e-6, err
