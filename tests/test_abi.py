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


FACADE_VS_REFERENCE = r'''
// The facade (include/vecgeom_b200.hpp) and the reference (oracle/_ref, linked
// into the same process through its C shim) run the VPlacedVolume SOA3D
// virtuals on the same SOA3D arrays; the program compares them with the parity
// bar and prints "ok" when every shape and op agrees.
#include "vecgeom_b200.hpp"
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>
using namespace vecgeom_b200;
extern "C" {
void *vgref_box(double, double, double);
void *vgref_tube(double, double, double, double, double);
void *vgref_cone(double, double, double, double, double, double, double);
void *vgref_trd(double, double, double, double, double);
void *vgref_transform_euler(double, double, double, double, double, double);
void *vgref_logical(const char *, void *);
void *vgref_place(void *, void *);
int vgref_batch(void *, int, int64_t, double *, double *, double *, double *, double *, double *,
                double *, void *, int *, int, int);
}
static bool close_enough(double a, double b) {
  if (std::isnan(a) && std::isnan(b)) return true;
  if (std::isinf(a) || std::isinf(b)) return a == b;
  const double d = std::fabs(a - b);
  return d <= 1e-9 || d <= 1e-12 * std::fabs(b);
}
int main() {
  const int n = 20000;
  std::mt19937_64 rng(0x5EED);
  std::uniform_real_distribution<double> u(-45., 45.);
  std::normal_distribution<double> g(0., 1.);
  std::vector<double> x(n), y(n), z(n), dx(n), dy(n), dz(n), st(n, 1e30);
  for (int i = 0; i < n; ++i) {
    x[i] = u(rng); y[i] = u(rng); z[i] = u(rng);
    double a = g(rng), b = g(rng), c = g(rng), r = std::sqrt(a * a + b * b + c * c);
    dx[i] = a / r; dy[i] = b / r; dz[i] = c / r;
  }
  SOA3D<double> p(x.data(), y.data(), z.data(), n), d(dx.data(), dy.data(), dz.data(), n);
  const double place[6] = {-4., 6., 2.5, 30., 45., 60.};
  Geometry geo;
  struct Case { const char *name; int ours; void *ref; };
  Case cases[] = {
      {"box", geo.UnplacedBox(10, 20, 30), vgref_box(10, 20, 30)},
      {"tube", geo.UnplacedTube(5, 20, 30, 0, 4.71238898038469),
       vgref_tube(5, 20, 30, 0, 4.71238898038469)},
      {"cone", geo.UnplacedCone(0, 10, 5, 20, 25, 0, 6.283185307179586),
       vgref_cone(0, 10, 5, 20, 25, 0, 6.283185307179586)},
      {"trd", geo.UnplacedTrd(10, 20, 15, 25, 30), vgref_trd(10, 20, 15, 25, 30)}};
  std::vector<VPlacedVolume> pvs;
  std::vector<void *> rpvs;
  for (auto &c : cases) {
    pvs.push_back(geo.Place(geo.LogicalVolume(c.name, c.ours),
                            geo.Transformation3D(place[0], place[1], place[2], place[3], place[4],
                                                 place[5])));
    rpvs.push_back(vgref_place(vgref_logical(c.name, c.ref),
                               vgref_transform_euler(place[0], place[1], place[2], place[3],
                                                     place[4], place[5])));
  }
  geo.CloseGeometry();
  int bad = 0;
  for (size_t k = 0; k < pvs.size(); ++k) {
    const VPlacedVolume &pv = pvs[k];
    void *rp = rpvs[k];
    std::vector<double> a(n), b(n), cur(n), cur_ref(n);
    std::vector<int> ia(n), ib(n), ids(n, -7), ids_ref(n, -7);
    std::vector<unsigned char> ca(n), cb(n);
    pv.Contains(p, reinterpret_cast<bool *>(ca.data()));
    vgref_batch(rp, 0, n, x.data(), y.data(), z.data(), 0, 0, 0, 0, cb.data(), 0, 0, 1);
    for (int i = 0; i < n; ++i) bad += ca[i] != cb[i];
    pv.Inside(p, ia.data());
    vgref_batch(rp, 1, n, x.data(), y.data(), z.data(), 0, 0, 0, 0, ib.data(), 0, 0, 1);
    for (int i = 0; i < n; ++i) bad += ia[i] != ib[i];
    struct Op { int code; bool dir; };
    for (Op op : {Op{2, true}, Op{3, true}, Op{4, false}, Op{5, false}}) {
      if (op.code == 2) pv.DistanceToIn(p, d, st.data(), a.data());
      if (op.code == 3) pv.DistanceToOut(p, d, st.data(), a.data());
      if (op.code == 4) pv.SafetyToIn(p, a.data());
      if (op.code == 5) pv.SafetyToOut(p, a.data());
      vgref_batch(rp, op.code, n, x.data(), y.data(), z.data(), op.dir ? dx.data() : 0,
                  op.dir ? dy.data() : 0, op.dir ? dz.data() : 0, op.dir ? st.data() : 0,
                  b.data(), 0, 0, 1);
      for (int i = 0; i < n; ++i) bad += !close_enough(a[i], b[i]);
    }
    // the Minimize forms against their definitions over the reference's values
    std::vector<double> dti_ref(n), sti_ref(n), sto_ref(n);
    vgref_batch(rp, 4, n, x.data(), y.data(), z.data(), 0, 0, 0, 0, sti_ref.data(), 0, 0, 1);
    vgref_batch(rp, 5, n, x.data(), y.data(), z.data(), 0, 0, 0, 0, sto_ref.data(), 0, 0, 1);
    for (int i = 0; i < n; ++i) cur[i] = cur_ref[i] = 5. + (i % 40);
    vgref_batch(rp, 2, n, x.data(), y.data(), z.data(), dx.data(), dy.data(), dz.data(),
                cur_ref.data(), dti_ref.data(), 0, 0, 1);
    pv.DistanceToInMinimize(p, d, 3, cur.data(), ids.data());
    for (int i = 0; i < n; ++i) {
      const double c0 = 5. + (i % 40);
      const bool upd = dti_ref[i] < c0;
      bad += !close_enough(cur[i], upd ? dti_ref[i] : c0) || ids[i] != (upd ? 3 : -7);
    }
    for (int i = 0; i < n; ++i) cur[i] = 5. + (i % 40);
    pv.SafetyToInMinimize(p, cur.data());
    for (int i = 0; i < n; ++i) bad += !close_enough(cur[i], std::fmin(sti_ref[i], 5. + (i % 40)));
    for (int i = 0; i < n; ++i) cur[i] = 5. + (i % 40);
    pv.SafetyToOutMinimize(p, cur.data());
    for (int i = 0; i < n; ++i) bad += !close_enough(cur[i], std::fmin(sto_ref[i], 5. + (i % 40)));
    std::vector<int> node(n);
    pv.DistanceToOut(p, d, st.data(), a.data(), node.data());
    vgref_batch(rp, 3, n, x.data(), y.data(), z.data(), dx.data(), dy.data(), dz.data(), st.data(),
                b.data(), 0, 0, 1);
    for (int i = 0; i < n; ++i) bad += !close_enough(a[i], b[i]) || node[i] != (b[i] < st[i] ? -1 : -2);
    std::printf("%s: %d mismatches so far\n", cases[k].name, bad);
  }
  std::puts(bad ? "FAILED" : "ok");
  return bad ? 1 : 0;
}
'''


@pytest.mark.gpu
def test_cpp_facade_runs_beside_the_reference(tmp_path):
    """The C++ facade runs every VPlacedVolume SOA3D batch virtual on the GPU,
    and the reference runs the same calls on the same SOA3D arrays in the same
    process (host buffers, so the library stages them); results agree with the
    parity bar."""
    import subprocess
    import oracle
    if not oracle.RefLib.available():
        pytest.skip("oracle/_ref not built")
    src = tmp_path / "facade_vs_ref.cpp"
    src.write_text(FACADE_VS_REFERENCE)
    exe = tmp_path / "facade_vs_ref"
    lib = os.path.join(ROOT, "vecgeom_b200", "lib")
    ref = os.path.dirname(oracle.REF_SO)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", lib, "-lvgb", f"-Wl,-rpath,{lib}", "-L", ref, "-lvgref",
                    f"-Wl,-rpath,{ref}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
