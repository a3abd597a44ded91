"""matvis_b200: the matvis per-(time, frequency) visibility path on NVIDIA B200 (sm_100a).

Drop-in for ``matvis.simulate_vis`` / ``simulate`` and the backend plugin classes
(``CoordinateRotation``, ``BeamInterpolator``, ``TauCalculator``, ``ZMatrixCalc``,
``MatProd``), computing on hand-written CUDA kernels behind the C ABI of
``include/matvis_b200.h``.  There is no CPU fallback: importing the package
without the built library raises ImportError.
"""

from . import _lib  # noqa: F401  (loads libmatvis_b200.so, fails loudly if absent)
from ._lib import GEMM_MODES, MatvisB200Error
from ._utils import get_desired_chunks, get_dtypes, get_required_chunks
from .beamfits import BeamFits, read_beamfits, write_beamfits
from .beams import B200BeamInterpolator, BeamInterpolator, GaussianBeam, GridBeam
from .coordinates import SkyCoords, eci_to_enu_matrix, enu_to_az_za, enu_to_eci_matrix, point_source_crd_eq
from .coords import CoordinateRotation, CoordinateRotationERFA, CoordinateRotationLST
from .engine import JobSpec, VisEngine
from .getz import ZMatrixCalc, ZPanel
from .matprod import B200MatMul, B200VectorDot, MatProd
from .simulate import simulate, simulate_vis
from .tau import TauCalculator

HAVE_GPU = True

__all__ = [
    "B200BeamInterpolator",
    "BeamFits",
    "B200MatMul",
    "B200VectorDot",
    "BeamInterpolator",
    "CoordinateRotation",
    "CoordinateRotationERFA",
    "CoordinateRotationLST",
    "GEMM_MODES",
    "GaussianBeam",
    "GridBeam",
    "JobSpec",
    "MatProd",
    "MatvisB200Error",
    "SkyCoords",
    "TauCalculator",
    "VisEngine",
    "ZMatrixCalc",
    "ZPanel",
    "eci_to_enu_matrix",
    "enu_to_az_za",
    "enu_to_eci_matrix",
    "get_desired_chunks",
    "get_dtypes",
    "get_required_chunks",
    "point_source_crd_eq",
    "read_beamfits",
    "simulate",
    "simulate_vis",
    "write_beamfits",
]
