"""ABBoxNavigator (navigation/ABBoxNavigator.h, source/ABBoxManager.cpp)
against the reference, and SimpleNavigator on the mixed-shape geometry.

Fixtures (tests/golden/make_nav_golden.py, written by the reference):
detector_abbox / zoo_abbox / row_abbox (ABBoxNavigator traces), zoo
(SimpleNavigator on the mixed-shape geometry), zoo2 / zoo2_abbox (both
navigators on the second mixed geometry: orb, parallelepiped, paraboloid,
trapezoids, union, intersection), zoo_boxes (ComputeABBox of all nine shape
types under random placements).  Records must match bit for bit:
  * CPU: the navigators of navigation.cuh / abbox.cuh built for the host, with
    the shared hit list large (sorted walk) and tiny (one-by-one walk);
  * GPU: vgb_abbox_nav_trace / vgb_abbox_nav_find_next_boundary_and_step and
    vgb_nav_trace through the C ABI.
The live reference (oracle/_ref) adds longer traces and the torus, each
geometry built in a fresh process.
"""
import numpy as np
import pytest

import oracle
from navhelpers import (NAV_GOLDEN, assert_traces_equal, build, dev, gpu_trace, host_trace,
                        load_fixture, load_hostcheck)
from make_nav_golden import (reference_boxes_isolated, reference_trace_isolated, row_inputs,
                             zoo_inputs)
from vecgeom_b200 import workloads as W
from vecgeom_b200.geometry import ComputeABBox

HAVE_REF = oracle.RefLib.available()
FIXTURES = ["detector_abbox", "zoo_abbox", "row_abbox", "zoo", "zoo2", "zoo2_abbox"]


def want_of(d):
    return d["next_ids"], d["steps"], d["safeties"], d["nsteps"]


@pytest.fixture(scope="module")
def hc():
    return load_hostcheck()


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
def test_abbox_boxes_match_fixture(hc):
    """ComputeABBox for box, tube, cone, sphere, torus, polycone, polyhedron,
    box-tube and trd under random rotations, in and out of containers."""
    d = np.load(NAV_GOLDEN + "/zoo_boxes.npz")
    g, placed = build(hc, "zoo_all", close=False)
    got = np.array([ComputeABBox(g, p) for p in placed])
    assert got.shape == d["boxes"].shape
    assert np.array_equal(got, d["boxes"])


def test_trd_extent_keeps_the_reference_typo(hc):
    """UnplacedTrd::Extent's upper x bound reads fDY1 (volumes/UnplacedTrd.h:147-150)."""
    from vecgeom_b200.geometry import Geometry
    g = Geometry(library=hc)
    world = g.LogicalVolume("w", g.UnplacedBox(100., 100., 100.))
    trd = g.LogicalVolume("t", g.UnplacedTrd(30., 10., 5., 6., 20.))
    pv = world.PlaceDaughter(trd, g.Transformation3D())
    g.SetWorld(world.Place(g.Transformation3D()))
    lo_hi = ComputeABBox(g, pv)
    assert lo_hi[0] == -30. - 1e-3 and lo_hi[3] == 10. + 1e-3  # max(dy1=5, dx2=10), not 30


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_abbox_boxes_match_reference_zoo2(hc):
    """ComputeABBox of orb, paraboloid, trapezoids (their Extents), union and
    intersection under random rotations."""
    g, placed = build(hc, "zoo2_abbox", close=False)
    got = np.array([ComputeABBox(g, p) for p in placed])
    want = reference_boxes_isolated("zoo2_abbox")
    assert np.array_equal(got, want)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_abbox_boxes_match_reference_detector(hc):
    g, placed = build(hc, "detector", close=False)
    got = np.array([ComputeABBox(g, p) for p in placed])
    want = reference_boxes_isolated("detector")
    assert np.array_equal(got, want)


# cap 2: the one-by-one walk of lists longer than the buffer, which matches
# the reference wherever such a list holds no equal box distances (true of
# these fixtures)
@pytest.mark.parametrize("cap", [512, 2], ids=["sorted_walk", "one_by_one"])
@pytest.mark.parametrize("name", FIXTURES)
def test_host_navigators_match_fixtures(hc, name, cap):
    d, pts, dirs = load_fixture(name)
    ms = int(d["max_steps"])
    nav = str(d["navigator"])
    if nav == "simple" and cap != 512:
        pytest.skip("the hit list only exists in ABBoxNavigator")
    got = host_trace(hc, str(d["geometry"]), pts, dirs, ms, navigator=nav, cap=cap)
    assert_traces_equal(got, want_of(d), ms, f"host {name}")


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_host_abbox_matches_reference_long_traces(hc):
    (x, y, z), (dx, dy, dz) = W.isotropic_tracks(1000, W.SEED_BASE + 57)
    rng = np.random.default_rng(8)
    pts = (np.concatenate([x, rng.uniform(-1050, 1050, 1000)]),
           np.concatenate([y, rng.uniform(-1050, 1050, 1000)]),
           np.concatenate([z, rng.uniform(-1250, 1250, 1000)]))
    _, dirs2 = W.isotropic_tracks(1000, W.SEED_BASE + 58)
    dirs = tuple(np.concatenate([a, b]) for a, b in zip((dx, dy, dz), dirs2))
    ms = 300
    want = reference_trace_isolated(pts, dirs, ms, 1, "detector", "abbox")
    got = host_trace(hc, "detector", pts, dirs, ms, navigator="abbox", cap=512)
    assert_traces_equal(got, want, ms, "host detector abbox")


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("geometry,navigator", [("zoo_torus", "simple"),
                                                ("zoo_abbox_torus", "abbox")])
def test_host_zoo_with_torus_matches_reference(hc, geometry, navigator):
    """With a torus in the geometry the trace is compared with the reference
    build whose torus takes correctly rounded atan2/sin/cos/cbrt, as libvgb's
    does; the C-library build differs from it on a few tracks by itself."""
    pts, dirs = W.zoo_tracks(2000, W.SEED_BASE + 59)
    ms = 100
    want = reference_trace_isolated(pts, dirs, ms, 8, geometry, navigator, crlibm=True)
    got = host_trace(hc, geometry, pts, dirs, ms, navigator=navigator)
    assert_traces_equal(got, want, ms, f"host {geometry} {navigator}")


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_host_row_matches_reference_full_crossing(hc):
    """Tracks that cross all 300 boxes (600+ steps), lists shrinking from 300."""
    pts, dirs = row_inputs(16)
    ms = 700
    want = reference_trace_isolated(pts, dirs, ms, 1, "row", "abbox")
    assert (want[3] > 600).all()
    got = host_trace(hc, "row", pts, dirs, ms, navigator="abbox", cap=512)
    assert_traces_equal(got, want, ms, "host row")


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", FIXTURES)
def test_gpu_navigators_match_fixtures(name):
    d, pts, dirs = load_fixture(name)
    ms = int(d["max_steps"])
    g, placed = build(None, str(d["geometry"]), close=True)
    got = gpu_trace(g, placed, pts, dirs, ms, navigator=str(d["navigator"]))
    assert_traces_equal(got, want_of(d), ms, f"gpu {name}")


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_gpu_abbox_matches_reference_many_tracks():
    pts, dirs = W.isotropic_tracks(4096, W.SEED_BASE + 78)
    ms = 128
    want = reference_trace_isolated(pts, dirs, ms, 1, "detector", "abbox")
    g, placed = build(None, "detector", close=True)
    got = gpu_trace(g, placed, pts, dirs, ms, navigator="abbox")
    assert_traces_equal(got, want, ms, "gpu detector abbox vs reference")


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("geometry,navigator", [("zoo_torus", "simple"),
                                                ("zoo_abbox_torus", "abbox")])
def test_gpu_zoo_with_torus_matches_reference(geometry, navigator):
    """The torus on the GPU: traces through the mixed-shape geometry with the
    torus against the reference build whose torus takes correctly rounded
    atan2/sin/cos/cbrt (libvgb evaluates them correctly rounded on the GPU)."""
    pts, dirs = W.zoo_tracks(2000, W.SEED_BASE + 59)
    ms = 100
    want = reference_trace_isolated(pts, dirs, ms, 8 if navigator == "simple" else 1, geometry,
                                    navigator, crlibm=True)
    g, placed = build(None, geometry, close=True)
    got = gpu_trace(g, placed, pts, dirs, ms, navigator=navigator)
    assert_traces_equal(got, want, ms, f"gpu {geometry} {navigator} vs reference")


@pytest.mark.gpu
def test_gpu_row_full_crossing_matches_host(hc):
    """Hit lists of up to 300 boxes on the GPU (introsort order) against the
    host build, over the full crossing."""
    pts, dirs = row_inputs(64)
    ms = 700
    g, placed = build(None, "row", close=True)
    got = gpu_trace(g, placed, pts, dirs, ms, navigator="abbox")
    want = host_trace(hc, "row", pts, dirs, ms, navigator="abbox", cap=1024)
    assert (want[3] > 600).all()
    assert_traces_equal(got, want, ms, "gpu row vs host")


@pytest.mark.gpu
def test_gpu_one_by_one_walk_matches_host(hc):
    """A mother with 6,500 daughters (more than the GPU's shared list holds):
    the kernel walks the hits one by one; the host build's sorted walk over the
    whole list gives the same records (no equal box distances here)."""
    pts, dirs = row_inputs(32)
    ms = 48
    g, placed = build(None, "row_long", close=True)
    got = gpu_trace(g, placed, pts, dirs, ms, navigator="abbox")
    want = host_trace(hc, "row_long", pts, dirs, ms, navigator="abbox", cap=8192)
    assert (want[3] == ms).all()
    assert_traces_equal(got, want, ms, "gpu long row vs host")


@pytest.mark.gpu
def test_gpu_abbox_single_steps_match_trace():
    """vgb_nav_locate + vgb_abbox_nav_find_next_boundary_and_step, step by step,
    reproduce the first records of the ABBoxNavigator fixture."""
    import torch
    import vecgeom_b200 as V
    d, pts, dirs = load_fixture("detector_abbox")
    ms = int(d["max_steps"])
    n = len(pts[0])
    g, placed = build(None, "detector", close=True)
    nav = V.ABBoxNavigator(g)
    a = V.NavStatePool(g, n)
    b = V.NavStatePool(g, n)
    P = [dev(v) for v in pts]
    D = V.SOA3D(*(dev(v) for v in dirs))
    nav.LocatePoint(V.SOA3D(*P), a)
    pstep = torch.full((n,), 1e30, dtype=torch.float64, device="cuda")
    step = torch.zeros(n, dtype=torch.float64, device="cuda")
    saf = torch.zeros(n, dtype=torch.float64, device="cuda")
    want_ids = d["next_ids"].reshape(n, ms)
    want_steps = d["steps"].reshape(n, ms)
    want_saf = d["safeties"].reshape(n, ms)
    nst = d["nsteps"]
    cur, nxt = a, b
    for k in range(3):
        nav.FindNextBoundaryAndStep(V.SOA3D(*P), D, cur, nxt, pstep, step, saf)
        torch.cuda.synchronize()
        live = nst > k
        assert np.array_equal(step.cpu().numpy()[live], want_steps[live, k])
        assert np.array_equal(saf.cpu().numpy()[live], want_saf[live, k])
        assert np.array_equal(nxt.tops()[live], want_ids[live, k])
        P = [P[j] + D_j * step for j, D_j in enumerate((D.x, D.y, D.z))]
        cur, nxt = nxt, cur
    assert nav.error_flags() == 0


@pytest.mark.gpu
def test_gpu_abbox_bad_arguments():
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import _lib
    g, _ = build(None, "detector", close=True)
    nav = V.ABBoxNavigator(g)
    pool = V.NavStatePool(g, 4)
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.VgbError):
        nav.FindNextBoundaryAndStep(V.SOA3D(x, x, x), V.SOA3D(x, x, x), pool, pool, x, x)
    nst = torch.zeros(4, dtype=torch.int32, device="cuda")
    with pytest.raises(_lib.VgbError):
        nav.Trace(V.SOA3D(x, x, x), V.SOA3D(x, x, x), 1e30, -1, nst)
