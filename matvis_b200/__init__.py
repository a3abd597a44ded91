"""matvis_b200: the matvis per-(time, frequency) visibility path on NVIDIA B200 (sm_100a).

Drop-in for ``matvis.simulate_vis`` / ``simulate`` and the backend plugin classes
(``CoordinateRotation``, ``BeamInterpolator``, ``TauCalculator``, ``ZMatrixCalc``,
``MatProd``), computing on hand-written CUDA kernels behind the C ABI of
``include/matvis_b200.h``.  There is no CPU fallback.

The names below are resolved on first use: the host-only modules
(``beam_models``, ``coordinates``, ``workloads``, ``_utils``, ``beamfits``,
``sharding``) import without the GPU library, and the first access to anything
that computes (``simulate_vis``, the plugin classes, ``VisEngine`` ...) loads
``libmatvis_b200.so`` and raises ImportError if it is not built.
"""

from __future__ import annotations

import importlib

#: public name -> submodule that defines it
_EXPORTS = {
    "GEMM_MODES": "_lib",
    "MatvisB200Error": "_lib",
    "get_desired_chunks": "_utils",
    "get_dtypes": "_utils",
    "get_required_chunks": "_utils",
    "BeamFits": "beamfits",
    "read_beamfits": "beamfits",
    "write_beamfits": "beamfits",
    "GaussianBeam": "beam_models",
    "GridBeam": "beam_models",
    "B200BeamInterpolator": "beams",
    "BeamInterpolator": "beams",
    "SkyCoords": "coordinates",
    "eci_to_enu_matrix": "coordinates",
    "enu_to_az_za": "coordinates",
    "enu_to_eci_matrix": "coordinates",
    "point_source_crd_eq": "coordinates",
    "CoordinateRotation": "coords",
    "CoordinateRotationERFA": "coords",
    "CoordinateRotationLST": "coords",
    "JobSpec": "engine",
    "VisEngine": "engine",
    "ZMatrixCalc": "getz",
    "ZPanel": "getz",
    "B200MatMul": "matprod",
    "B200VectorDot": "matprod",
    "MatProd": "matprod",
    "simulate": "wrapper",
    "simulate_vis": "wrapper",
    "TauCalculator": "tau",
}

HAVE_GPU = True

__all__ = sorted(_EXPORTS)


def __getattr__(name: str):
    mod = _EXPORTS.get(name)
    if mod is None:
        raise AttributeError(f"module 'matvis_b200' has no attribute {name!r}")
    value = getattr(importlib.import_module(f".{mod}", __name__), name)
    globals()[name] = value
    return value


def __dir__():
    return sorted(set(globals()) | set(_EXPORTS))
