"""Import EMerge's hot-path modules from a read-only checkout without gmsh or emsutil.

Used only by ``make_golden.py`` in a container that has the reference checkout; nothing on the
GPU path imports this.  ``gmsh`` and ``emsutil`` are replaced by empty stand-ins, and ``emerge``
is registered as a bare package so ``src/emerge/__init__.py`` (which imports gmsh at line 63 and
emsutil at lines 80-84) never runs.  The hot-path modules themselves import unchanged.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

def _reference_src() -> str:
    src = os.environ.get("EMERGE_REFERENCE_SRC")
    if not src:
        raise RuntimeError("set EMERGE_REFERENCE_SRC to the src/emerge folder of an EMerge checkout")
    if not os.path.isdir(src):
        raise RuntimeError(f"EMERGE_REFERENCE_SRC={src!r} is not a folder")
    return src


def load():
    reference_src = _reference_src()
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/emerge_b200_numba_cache")
    if "emerge" in sys.modules and getattr(sys.modules["emerge"], "_stubbed", False):
        return _modules()
    sys.modules["gmsh"] = types.ModuleType("gmsh")
    ems = types.ModuleType("emsutil")

    class Material:  # only the name is needed at import time
        pass

    ems.Material = Material
    ems.AIR = Material(); ems.PEC = Material(); ems.COPPER = Material()
    ems.CoordDependent = object
    lib = types.ModuleType("emsutil.lib"); lib.AIR = ems.AIR; ems.lib = lib
    emd = types.ModuleType("emsutil.emdata"); emd.EHField = object; emd.EHFieldFF = object
    sys.modules.update({"emsutil": ems, "emsutil.lib": lib, "emsutil.emdata": emd})
    pkg = types.ModuleType("emerge")
    pkg.__path__ = [reference_src]
    pkg._stubbed = True
    sys.modules["emerge"] = pkg
    return _modules()


def _modules():
    m = types.SimpleNamespace()
    m.curlcurl = importlib.import_module("emerge._emerge.physics.microwave.assembly.curlcurl")
    m.robinbc = importlib.import_module("emerge._emerge.physics.microwave.assembly.robinbc")
    m.nedelec2 = importlib.import_module("emerge._emerge.elements.nedelec2")
    m.optimized = importlib.import_module("emerge._emerge.mth.optimized")
    m.solver = importlib.import_module("emerge._emerge.solver")
    m.bc = importlib.import_module("emerge._emerge.physics.microwave.microwave_bc")
    m.cs = importlib.import_module("emerge._emerge.cs")
    m.sparam = importlib.import_module("emerge._emerge.physics.microwave.sparam")
    return m
