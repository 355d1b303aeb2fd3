"""Geometry ingestion and export formats (vgb_geometry_serialize / _deserialize /
_save / _load, vgb_geometry_export_cpp).

  * flat image: a geometry rebuilt from its image writes the same image again
    and navigates bit for bit like the original (host build of the navigators);
    corrupted, truncated and foreign images are refused;
  * C++ export (GeomCppExporter::DumpGeometry's layout, source/CppExporter.cpp):
    the source compiles against the reference's own headers, the reference
    builds the geometry from it, and the reference's SimpleNavigator traces it
    exactly as this library traces the original.
"""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from make_nav_golden import MAX_STEPS, PSTEP, isolated, zoo_inputs
from navhelpers import build, load_hostcheck
from vecgeom_b200._lib import VgbError
from vecgeom_b200.geometry import Geometry

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HAVE_REF_TREE = oracle.reference_tree() is not None
GEOMETRIES = ["detector", "zoo", "zoo2"]
# the exported source also rebuilds the torus (the CPU reference and the host
# build agree there)
EXPORT_GEOMETRIES = GEOMETRIES + ["zoo_torus"]


@pytest.fixture(scope="module")
def hc():
    return load_hostcheck()


def raw_trace(L, g, pts, dirs, ms=MAX_STEPS):
    """hc_nav_trace over an existing geometry: (placed ids, steps, safeties, nsteps)."""
    n = len(pts[0])
    ids = np.full(n * ms, -7, np.int32)
    steps = np.zeros(n * ms)
    saf = np.zeros(n * ms)
    nst = np.zeros(n, np.int32)
    a = lambda v: np.ascontiguousarray(v).ctypes.data  # noqa: E731
    rc = L.hc_nav_trace(g.handle, n, *(a(v) for v in pts), *(a(v) for v in dirs), PSTEP, ms,
                        a(ids), a(steps), a(saf), a(nst), 0)
    assert rc == 0
    return ids, steps, saf, nst


def assert_same_trace(a, b, ms, what):
    ia, sa, fa, na = a
    ib, sb, fb, nb = b
    assert np.array_equal(na, nb), f"{what}: step counts differ"
    m = (np.arange(ms)[None, :] < na[:, None]).ravel()
    assert np.array_equal(ia[m], ib[m]), f"{what}: next ids differ"
    for x, y, k in ((sa, sb, "steps"), (fa, fb, "safeties")):
        x, y = x[m], y[m]
        assert np.all((x == y) | (np.isnan(x) & np.isnan(y))), f"{what}: {k} differ"


def tracks():
    return zoo_inputs()


# ---------------------------------------------------------------------------
# flat image
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("geometry", GEOMETRIES)
def test_image_round_trip_navigates_identically(hc, geometry):
    g, _ = build(hc, geometry, close=False)
    image = g.Serialize()
    g2 = Geometry.FromImage(image, library=hc)
    assert g2.Serialize() == image
    pts, dirs = tracks()
    assert_same_trace(raw_trace(hc, g2, pts, dirs), raw_trace(hc, g, pts, dirs), MAX_STEPS,
                      f"{geometry} image")


def test_image_file_round_trip(hc, tmp_path):
    g, _ = build(hc, "zoo2", close=False)
    path = str(tmp_path / "zoo2.vgbgeom")
    g.Save(path)
    with open(path, "rb") as f:
        assert f.read() == g.Serialize()
    assert Geometry.Load(path, library=hc).Serialize() == g.Serialize()


def test_image_refuses_damage(hc):
    g, _ = build(hc, "zoo2", close=False)
    image = bytearray(g.Serialize())
    cases = {"truncated": bytes(image[:-9]), "empty": b"", "short": bytes(image[:20])}
    flipped = bytearray(image)
    flipped[len(image) // 2] ^= 0x40
    cases["bit flip"] = bytes(flipped)
    foreign = bytearray(image)
    foreign[0:8] = b"NOTVGBGM"
    cases["foreign"] = bytes(foreign)
    for what, data in cases.items():
        with pytest.raises(VgbError) as e:
            Geometry.FromImage(data, library=hc)
        assert e.value.status == 1, what  # VGB_EINVAL


def test_image_buffer_too_small(hc):
    g, _ = build(hc, "detector", close=False)
    n = ctypes.c_size_t()
    assert hc.vgb_geometry_serialize(g.handle, None, 0, ctypes.byref(n)) == 0
    buf = ctypes.create_string_buffer(n.value)
    assert hc.vgb_geometry_serialize(g.handle, buf, n.value - 1, ctypes.byref(n)) == 7  # ENOSPC


# ---------------------------------------------------------------------------
# C++ export, rebuilt by the reference
# ---------------------------------------------------------------------------
def compile_export(source: str, workdir: str) -> str:
    """The exported source plus a C entry point, compiled against the reference's
    headers with oracle/Makefile's flags (at -O0 for speed: SSE2 arithmetic
    rounds the same at any level), linked to oracle/_ref."""
    src = os.path.join(workdir, "detector.cpp")
    with open(src, "w") as f:
        f.write(source)
        f.write('\nextern "C" void *vgx_generate() { return (void *)generateDetector(); }\n')
    so = os.path.join(workdir, "libdetector.so")
    ref_so = os.path.abspath(oracle.REF_SO)
    cmd = (["g++"] + oracle.reference_cxxflags() + ["-O0", "-shared", src, "-o", so, ref_so,
                                                     f"-Wl,-rpath,{os.path.dirname(ref_so)}"])
    subprocess.run(cmd, check=True, capture_output=True)
    return so


def _trace_exported(so, order, pts, dirs, ms):
    ref = oracle.RefLib()
    lib = ctypes.CDLL(so)
    lib.vgx_generate.restype = ctypes.c_void_p
    world = lib.vgx_generate()
    ref.L.vgref_set_world(ctypes.c_void_p(world))
    ref.L.vgref_close_geometry()
    ids, steps, saf, nst = oracle.ref_nav_trace(ref, pts, dirs, PSTEP, ms, 1)
    # the function creates the placements in `order`; the reference numbers
    # placed volumes consecutively, the world last
    base = ref.L.vgref_placed_id(ctypes.c_void_p(world)) - (len(order) - 1)
    ours = np.array([order[i - base] if i >= 0 else i for i in ids], np.int32)
    return ours, steps, saf, nst


@pytest.mark.skipif(not (HAVE_REF_TREE and oracle.RefLib.available()),
                    reason="needs the reference's headers and oracle/_ref")
@pytest.mark.parametrize("geometry", EXPORT_GEOMETRIES)
def test_exported_cpp_rebuilt_by_reference_navigates_identically(hc, geometry, tmp_path):
    g, _ = build(hc, geometry, close=False)
    src = g.ExportCpp()
    order = [int(v) for v in re.search(r"creates the placements:([ 0-9]*)", src).group(1).split()]
    so = compile_export(src, str(tmp_path))
    pts, dirs = tracks()
    want = raw_trace(hc, g, pts, dirs)
    got = isolated(_trace_exported, so, order, pts, dirs, MAX_STEPS)
    assert_same_trace(got, want, MAX_STEPS, f"{geometry} exported")


def test_export_layout(hc):
    """The reference exporter's statements: transformations, logical volumes
    over new Unplaced*, PlaceDaughter, the world placement; every shape kind of
    the mixed geometries is written, numbers with 17 significant digits."""
    g, _ = build(hc, "zoo2", close=False)
    src = g.ExportCpp()
    assert "VPlacedVolume const * generateDetector() {" in src
    for cls in ("UnplacedOrb", "UnplacedParallelepiped", "UnplacedParaboloid",
                "UnplacedTrapezoid", "UnplacedBooleanVolume", "UnplacedBox", "UnplacedTrd"):
        assert f"new {cls}(" in src, cls
    assert "->PlaceDaughter( lvol" in src and "return world;" in src
    g1, _ = build(hc, "zoo_all", close=False)
    src1 = g1.ExportCpp()
    for cls in ("UnplacedTube", "UnplacedCone", "UnplacedSphere", "UnplacedPolycone",
                "UnplacedPolyhedron", "UnplacedBooleanVolume"):
        assert f"new {cls}(" in src1, cls


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["zoo2", "zoo2_abbox"])
def test_gpu_geometry_from_image_matches_fixture(name):
    """A geometry loaded from its flat image, closed and navigated on the GPU,
    reproduces the reference's traces (tests/golden/nav fixtures)."""
    from navhelpers import assert_traces_equal, gpu_trace, load_fixture
    d, pts, dirs = load_fixture(name)
    ms = int(d["max_steps"])
    g0, placed = build(None, str(d["geometry"]), close=False)
    g = Geometry.FromImage(g0.Serialize())
    g.CloseGeometry()
    got = gpu_trace(g, placed, pts, dirs, ms, navigator=str(d["navigator"]))
    want = (d["next_ids"], d["steps"], d["safeties"], d["nsteps"])
    assert_traces_equal(got, want, ms, f"gpu {name} from image")
