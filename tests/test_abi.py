"""CPU: the C-ABI library loads and exports every entry point include/*.h declares."""
import ctypes
import glob
import os
import re

import pytest

import vecgeom_b200
from vecgeom_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(vgb_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_built():
    assert os.path.exists(_lib.LIB_PATH), "libvgb.so missing: run make -C vecgeom_b200/csrc"


def test_every_declared_symbol_exported():
    names = declared_functions()
    assert "vgb_batch" in names and "vgb_geometry_close" in names
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_signatures_cover_header():
    names = set(declared_functions())
    missing = [n for n in names if n not in _lib.SIGNATURES]
    assert not missing, f"no ctypes signature for {missing}"


def test_errors_are_statuses_not_aborts():
    L = vecgeom_b200.lib()
    assert L.vgb_geometry_create(None) == _lib.EINVAL
    assert b"NULL" in L.vgb_last_error()
    g = vecgeom_b200.Geometry()
    with pytest.raises(vecgeom_b200.VgbError):
        g.UnplacedBox(-1., 1., 1.)
    with pytest.raises(vecgeom_b200.VgbError):
        g.LogicalVolume("x", 42)
    b = g.UnplacedBox(1., 2., 3.)
    lv = g.LogicalVolume("b", b)
    pv = lv.Place(g.Transformation3D())
    import numpy as np
    pts = vecgeom_b200.SOA3D(np.zeros(4), np.zeros(4), np.zeros(4))
    with pytest.raises(vecgeom_b200.VgbError, match="not closed"):
        pv.Inside(pts, np.zeros(4, np.int32))
