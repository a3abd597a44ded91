"""Load the reference matvis modules in a container that lacks their third-party deps.

Test infrastructure only: used by ``make_golden.py`` to run the reference's own
arithmetic (matprod, bilinear beam interpolation, coordinate helpers, horizon
selection, tau, Z, chunk planning) and freeze its outputs as fixtures.

The reference imports astropy, pyuvdata and cupy at module level, none of which
are installed.  The arithmetic on the hot path does not use them (it is numpy /
scipy / cupy array code), so they are replaced by small stand-in modules:

* ``astropy.constants.c`` is the exact SI speed of light (299792458 m/s), the
  value astropy defines;
* ``cupy`` / ``cupyx.scipy.ndimage`` are numpy / scipy.ndimage (the reference's
  GPU beam routine is written against the scipy-compatible cupyx API);
* every other imported name is an inert placeholder class.

Nothing here is imported by the product or by the tests at run time; only the
fixture generator uses it, and only where the reference tree is present.
"""

from __future__ import annotations

import importlib
import os
import sys
import types
from pathlib import Path

import numpy as np

#: Root of the reference (matvis) project tree: the MATVIS_REFERENCE_ROOT
#: environment variable, or ``make_golden.py --reference-root``.
REF_ROOT = Path(os.environ.get("MATVIS_REFERENCE_ROOT", "reference"))
REF_PKG = REF_ROOT / "src" / "matvis"


def set_reference_root(path) -> None:
    """Point the loader at the reference project tree (before ``load_reference``)."""
    global REF_ROOT, REF_PKG
    REF_ROOT = Path(path)
    REF_PKG = REF_ROOT / "src" / "matvis"


class _Placeholder:
    """Inert stand-in for a third-party class only used in type hints / isinstance."""

    def __init__(self, *a, **k):
        raise RuntimeError("placeholder class from a missing dependency was used")


def _module(name: str, **attrs) -> types.ModuleType:
    mod = types.ModuleType(name)
    mod.__dict__.update(attrs)
    sys.modules[name] = mod
    return mod


def _install_stubs() -> None:
    # --- astropy -----------------------------------------------------------
    class _C:
        value = 299792458.0

    _module("astropy")
    _module("astropy.units", rad=1.0, s=1.0, deg=1.0)
    sys.modules["astropy"].units = sys.modules["astropy.units"]
    _module("astropy.constants", c=_C())
    _module(
        "astropy.coordinates",
        EarthLocation=_Placeholder,
        SkyCoord=_Placeholder,
        AltAz=_Placeholder,
        Latitude=_Placeholder,
        Longitude=_Placeholder,
    )
    _module("astropy.coordinates.builtin_frames", AltAz=_Placeholder)
    _module("astropy.coordinates.erfa_astrom", erfa_astrom=None)
    _module("astropy.time", Time=_Placeholder)

    # --- pyuvdata ------------------------------------------------------------
    _module("pyuvdata", UVBeam=_Placeholder, BeamInterface=_Placeholder)
    _module("pyuvdata.analytic_beam", AnalyticBeam=_Placeholder, GaussianBeam=_Placeholder)
    _module("pyuvdata.beam_interface", BeamInterface=_Placeholder)
    _module("pyuvdata.uvbeam", UVBeam=_Placeholder)
    _module("pyuvdata.utils")
    _module("pyuvdata.utils.pol", polstr2num=lambda *a, **k: None)
    _module("pyuvdata.telescopes", Telescope=_Placeholder)

    # --- cupy -> numpy / scipy shim -------------------------------------------
    from scipy import ndimage as sp_ndimage

    class _Device:
        def synchronize(self):
            return None

    cuda = types.SimpleNamespace(Device=_Device)
    cp = _module("cupy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(cp, name, getattr(np, name))
    cp.cuda = cuda
    cp.asnumpy = np.asarray
    cp.get_array_module = lambda *a: np
    _module("cupyx")
    _module("cupyx.scipy")
    _module("cupyx.scipy.ndimage", map_coordinates=sp_ndimage.map_coordinates)
    sys.modules["cupyx"].scipy = sys.modules["cupyx.scipy"]
    sys.modules["cupyx.scipy"].ndimage = sys.modules["cupyx.scipy.ndimage"]

    for name in ("line_profiler", "docstring_parser"):
        _module(name, combine_docstrings=lambda *a, **k: (lambda f: f))


def load_reference():
    """Return a namespace with the reference modules the fixtures are made from."""
    if not REF_PKG.exists():
        raise FileNotFoundError(f"reference tree not found at {REF_PKG}")
    _install_stubs()
    # Package shells: set __path__ without executing the package __init__ files,
    # which import the astropy-based wrapper.
    pkg = _module("matvis", HAVE_GPU=False, DATA_PATH=REF_PKG / "data")
    pkg.__path__ = [str(REF_PKG)]
    for sub in ("core", "cpu", "gpu"):
        m = _module(f"matvis.{sub}")
        m.__path__ = [str(REF_PKG / sub)]
        setattr(pkg, sub, m)
    ns = types.SimpleNamespace()
    ns.utils = importlib.import_module("matvis._utils")
    ns.coordinates = importlib.import_module("matvis.coordinates")
    ns.core_coords = importlib.import_module("matvis.core.coords")
    ns.core_tau = importlib.import_module("matvis.core.tau")
    ns.core_getz = importlib.import_module("matvis.core.getz")
    ns.core_matprod = importlib.import_module("matvis.core.matprod")
    ns.cpu_matprod = importlib.import_module("matvis.cpu.matprod")
    ns.gpu_beams = importlib.import_module("matvis.gpu.beams")
    ns.cpu_coords = importlib.import_module("matvis.cpu.coords")
    return ns
