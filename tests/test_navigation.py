"""Navigation: SimpleNavigator over the layered detector, against the reference.

The reference's SimpleNavigator (navigation/SimpleNavigator.h:204-596) traced
the tracks of tests/golden/nav/detector.npz (tests/golden/make_nav_golden.py);
the next-volume ids, steps and safeties must match bit for bit:
  * CPU: the navigator of navigation.cuh built for the host (single lane);
  * GPU: vgb_nav_trace / vgb_nav_locate / vgb_nav_find_next_boundary_and_step
    through the C ABI (one warp per track).
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from vecgeom_b200 import _lib
from vecgeom_b200 import workloads as W
from vecgeom_b200.geometry import Geometry

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden", "nav", "detector.npz")
HC_SO = os.path.join(ROOT, "_build", "hostcheck", "libvgb_hostcheck.so")


def load_golden():
    d = np.load(GOLDEN)
    pts = (d["x"], d["y"], d["z"])
    dirs = (d["dx"], d["dy"], d["dz"])
    return d, pts, dirs


def assert_traces_equal(got, want, max_steps, what=""):
    """got/want = (ids, steps, safeties, nsteps) with records at i*max_steps."""
    gi, gs, gf, gn = got
    wi, ws, wf, wn = want
    bad = np.flatnonzero(gn != wn)
    assert len(bad) == 0, f"{what}: step counts differ for tracks {bad[:8].tolist()}"
    mask = (np.arange(max_steps)[None, :] < wn[:, None]).ravel()
    for name, a, b in (("next ids", gi, wi), ("steps", gs, ws), ("safeties", gf, wf)):
        a = np.asarray(a)[mask]
        b = np.asarray(b)[mask]
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
        k = np.flatnonzero(~same)
        assert len(k) == 0, f"{what}: {name} differ at {len(k)} records, first {k[:5].tolist()}"


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def hc():
    subprocess.run(["make", "-C", os.path.join(HERE, "hostcheck")], check=True,
                   stdout=subprocess.DEVNULL)
    L = ctypes.CDLL(HC_SO)
    for name, (res, args) in _lib.SIGNATURES.items():
        f = getattr(L, name, None)
        if f is not None:
            f.restype = res
            f.argtypes = args
    vp = ctypes.c_void_p
    L.hc_nav_trace.restype = ctypes.c_int
    L.hc_nav_trace.argtypes = ([vp, ctypes.c_int64] + [vp] * 6 + [ctypes.c_double, ctypes.c_int32]
                               + [vp] * 4 + [ctypes.c_int32])
    return L


def host_trace(L, pts, dirs, max_steps, pstep=1e30, screen=0):
    g = Geometry(library=L)
    placed = W.build_detector(W.VgbBuilder(g, close=False))
    assert [p.id for p in placed] == list(range(len(placed)))
    n = len(pts[0])
    ids = np.full(n * max_steps, -7, np.int32)
    steps = np.zeros(n * max_steps)
    saf = np.zeros(n * max_steps)
    nst = np.zeros(n, np.int32)
    a = lambda v: np.ascontiguousarray(v).ctypes.data  # noqa: E731
    rc = L.hc_nav_trace(g.handle, n, *(a(v) for v in pts), *(a(v) for v in dirs), pstep,
                        max_steps, a(ids), a(steps), a(saf), a(nst), screen)
    assert rc == 0
    return ids, steps, saf, nst, g


def test_detector_layout(hc):
    g = Geometry(library=hc)
    placed = W.build_detector(W.VgbBuilder(g, close=False))
    assert len(placed) == W.DetectorSpec().placed_count() == 14011


@pytest.mark.parametrize("screen", [0, 1], ids=["fp64", "fp32_screen"])
def test_host_navigator_matches_golden(hc, screen):
    """Both forms: the float screen of FP32+refine must not change a record."""
    d, pts, dirs = load_golden()
    ms = int(d["max_steps"])
    ids, steps, saf, nst, _ = host_trace(hc, pts, dirs, ms, screen=screen)
    assert_traces_equal((ids, steps, saf, nst),
                        (d["next_ids"], d["steps"], d["safeties"], d["nsteps"]), ms, "host")


@pytest.mark.skipif(not oracle.RefLib.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("screen", [0, 1], ids=["fp64", "fp32_screen"])
def test_host_navigator_matches_reference_long_traces(hc, screen):
    """More tracks and longer traces than the fixture, against the live reference."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_nav_golden import reference_trace
    (x, y, z), (dx, dy, dz) = W.isotropic_tracks(1000, W.SEED_BASE + 55)
    rng = np.random.default_rng(7)
    pts = (np.concatenate([x, rng.uniform(-1050, 1050, 1000)]),
           np.concatenate([y, rng.uniform(-1050, 1050, 1000)]),
           np.concatenate([z, rng.uniform(-1250, 1250, 1000)]))
    _, dirs2 = W.isotropic_tracks(1000, W.SEED_BASE + 56)
    dirs = tuple(np.concatenate([a, b]) for a, b in zip((dx, dy, dz), dirs2))
    ms = 300
    ids, steps, saf, nst, _ = host_trace(hc, pts, dirs, ms, screen=screen)
    want = reference_trace(oracle.RefLib(), pts, dirs, ms, nthreads=os.cpu_count() or 1)
    assert_traces_equal((ids, steps, saf, nst), want, ms, "host long")


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


def gpu_detector():
    import vecgeom_b200 as V
    g = V.Geometry()
    placed = W.build_detector(W.VgbBuilder(g))
    return g, placed


def gpu_trace(g, pts, dirs, ms, pstep=1e30, precision=0):
    import torch
    import vecgeom_b200 as V
    n = len(pts[0])
    nav = V.SimpleNavigator(g)
    ids = torch.full((n * ms,), -7, dtype=torch.int32, device="cuda")
    steps = torch.zeros(n * ms, dtype=torch.float64, device="cuda")
    saf = torch.zeros(n * ms, dtype=torch.float64, device="cuda")
    nst = torch.zeros(n, dtype=torch.int32, device="cuda")
    nav.Trace(V.SOA3D(*(dev(a) for a in pts)), V.SOA3D(*(dev(a) for a in dirs)), pstep, ms, nst,
              ids, steps, saf, precision=precision)
    torch.cuda.synchronize()
    assert nav.error_flags() == 0
    return ids.cpu().numpy(), steps.cpu().numpy(), saf.cpu().numpy(), nst.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32_refine"])
def test_gpu_trace_matches_golden(precision):
    d, pts, dirs = load_golden()
    ms = int(d["max_steps"])
    g, _ = gpu_detector()
    got = gpu_trace(g, pts, dirs, ms, precision=precision)
    assert_traces_equal(got, (d["next_ids"], d["steps"], d["safeties"], d["nsteps"]), ms, "gpu")


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.RefLib.available(), reason="oracle/_ref not built")
def test_gpu_trace_matches_reference_many_tracks():
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_nav_golden import reference_trace
    pts, dirs = W.isotropic_tracks(4096, W.SEED_BASE + 77)
    ms = 128
    g, _ = gpu_detector()
    want = reference_trace(oracle.RefLib(), pts, dirs, ms, nthreads=os.cpu_count() or 1)
    for precision in (0, 1):
        got = gpu_trace(g, pts, dirs, ms, precision=precision)
        assert_traces_equal(got, want, ms, f"gpu (precision {precision}) vs reference")


@pytest.mark.gpu
def test_gpu_locate_and_single_steps_match_trace():
    """vgb_nav_locate + two vgb_nav_find_next_boundary_and_step calls reproduce
    the first two records of the trace, and the pool keeps the reference layout."""
    import torch
    import vecgeom_b200 as V
    d, pts, dirs = load_golden()
    ms = int(d["max_steps"])
    n = len(pts[0])
    g, placed = gpu_detector()
    nav = V.SimpleNavigator(g)
    a = V.NavStatePool(g, n)
    b = V.NavStatePool(g, n)
    assert a.stride == 16 + 8 * (g.getMaxDepth() + 1) == 56
    P = [dev(v) for v in pts]
    D = V.SOA3D(*(dev(v) for v in dirs))
    nav.LocatePoint(V.SOA3D(*P), a)
    st = a.to_numpy()
    assert (st["header"] >> 1 == g.getMaxDepth() + 1).all()
    pstep = torch.full((n,), 1e30, dtype=torch.float64, device="cuda")
    step = torch.zeros(n, dtype=torch.float64, device="cuda")
    saf = torch.zeros(n, dtype=torch.float64, device="cuda")
    want_ids = d["next_ids"].reshape(n, ms)
    want_steps = d["steps"].reshape(n, ms)
    want_saf = d["safeties"].reshape(n, ms)
    nst = d["nsteps"]
    cur, nxt = a, b
    for k in range(2):
        nav.FindNextBoundaryAndStep(V.SOA3D(*P), D, cur, nxt, pstep, step, saf,
                                    precision=k % 2)
        torch.cuda.synchronize()
        live = nst > k
        s = step.cpu().numpy()
        assert np.array_equal(s[live], want_steps[live, k])
        assert np.array_equal(saf.cpu().numpy()[live], want_saf[live, k])
        assert np.array_equal(nxt.tops()[live], want_ids[live, k])
        # advance like the trace client: p += d * step
        P = [P[j] + D_j * step for j, D_j in enumerate((D.x, D.y, D.z))]
        cur, nxt = nxt, cur
    assert nav.error_flags() == 0


@pytest.mark.gpu
def test_navpool_round_trip_and_bad_arguments():
    import vecgeom_b200 as V
    g, _ = gpu_detector()
    pool = V.NavStatePool(g, 8)
    st = np.zeros(8, pool.dtype())
    st["level"] = np.arange(8) % 5
    st["path"][:, 0] = 0
    pool.from_numpy(st)
    back = pool.to_numpy()
    assert np.array_equal(back["level"], st["level"])
    with pytest.raises(_lib.VgbError):
        V.NavStatePool(g, -1)
