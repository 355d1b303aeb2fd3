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


def declared_arity():
    """Number of parameters of every vgb_* function declared in include/*.h."""
    out = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"\b(vgb_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
            args = m.group(2).strip()
            out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_python_signatures_match_header_arity():
    bad = {n: (k, len(_lib.SIGNATURES[n][1])) for n, k in declared_arity().items()
           if n in _lib.SIGNATURES and len(_lib.SIGNATURES[n][1]) != k}
    assert not bad, f"argument counts (header, ctypes) differ: {bad}"


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


def test_cpp_facade_compiles_and_links(tmp_path):
    """include/vecgeom_b200.hpp (the VPlacedVolume/SOA3D facade) compiles with the
    reference's call shapes and links against libvgb.so."""
    import subprocess
    src = tmp_path / "facade.cpp"
    src.write_text(r'''
#include "vecgeom_b200.hpp"
#include <cstdio>
using namespace vecgeom_b200;
int main(int argc, char **) {
  static_assert(sizeof(SOA3D<double>) == 48, "SOA3D member layout");
  if (argc > 5) {  // never taken: the calls only have to compile and link
    Geometry g;
    VPlacedVolume pv = g.Place(g.LogicalVolume("b", g.UnplacedBox(1, 2, 3)), g.Transformation3D());
    double corners[24] = {0};
    int shapes[] = {g.UnplacedOrb(1), g.UnplacedParallelepiped(1, 2, 3, 10, 20, 30),
                    g.UnplacedParaboloid(1, 2, 3),
                    g.UnplacedTrapezoid(4, 0.1, 0.2, 3, 2, 2, 0, 3, 2, 2, 0),
                    g.UnplacedTrapezoid(corners)};
    (void)shapes;
    double x[1] = {0}, out[1];
    SOA3D<double> p(x, x, x, 1);
    bool c[1];
    int in[1], ids[1];
    pv.Contains(p, c);
    pv.Inside(p, in);
    pv.DistanceToIn(p, p, x, out);
    pv.DistanceToInMinimize(p, p, 3, out, ids);
    pv.DistanceToOut(p, p, x, out);
    pv.DistanceToOut(p, p, x, out, ids);
    pv.SafetyToIn(p, out);
    pv.SafetyToInMinimize(p, out);
    pv.SafetyToOut(p, out);
    pv.SafetyToOutMinimize(p, out);
  }
  std::puts("ok");
  return 0;
}
''')
    exe = tmp_path / "facade"
    lib = os.path.join(ROOT, "vecgeom_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", lib, "-lvgb", f"-Wl,-rpath,{lib}",
                    "-Wl,--unresolved-symbols=ignore-in-shared-libs"], check=True)
