"""Navigation test helpers: the host build of the navigators (hostcheck
library), the GPU traces through libvgb, and trace comparison.

Traces are (next ids, steps, safeties, nsteps) with the records of track i at
i * max_steps; next ids are positions in the list the geometry builder returns
(-1 once outside the world)."""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

from vecgeom_b200 import _lib
from vecgeom_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HC_SO = os.path.join(ROOT, "_build", "hostcheck", "libvgb_hostcheck.so")
NAV_GOLDEN = os.path.join(HERE, "golden", "nav")
if os.path.join(HERE, "golden") not in sys.path:
    sys.path.insert(0, os.path.join(HERE, "golden"))


def load_hostcheck():
    subprocess.run(["make", "-C", os.path.join(HERE, "hostcheck")], check=True,
                   stdout=subprocess.DEVNULL)
    L = ctypes.CDLL(HC_SO)
    for name, (res, args) in _lib.SIGNATURES.items():
        f = getattr(L, name, None)
        if f is not None:
            f.restype = res
            f.argtypes = args
    vp = ctypes.c_void_p
    L.hc_nav_basket.restype = ctypes.c_int
    L.hc_nav_basket.argtypes = [vp, ctypes.c_int64] + [vp] * 7 + [ctypes.c_int32] + [vp] * 8
    for fn in ("hc_nav_trace", "hc_abbox_trace"):
        getattr(L, fn).restype = ctypes.c_int
        getattr(L, fn).argtypes = ([vp, ctypes.c_int64] + [vp] * 6 + [ctypes.c_double,
                                   ctypes.c_int32] + [vp] * 4 + [ctypes.c_int32])
    return L


def load_fixture(name: str):
    d = np.load(os.path.join(NAV_GOLDEN, name + ".npz"))
    return d, (d["x"], d["y"], d["z"]), (d["dx"], d["dy"], d["dz"])


def build(geom_lib_or_geometry, geometry: str, close: bool):
    """Builds the named geometry (make_nav_golden.build_geometry) in a
    vecgeom_b200 Geometry; returns (geometry, placed list)."""
    from make_nav_golden import build_geometry
    from vecgeom_b200.geometry import Geometry
    g = geom_lib_or_geometry
    if not isinstance(g, Geometry):
        g = Geometry(library=g) if g is not None else Geometry()
    placed = build_geometry(W.VgbBuilder(g, close=close), geometry)
    return g, placed


def to_positions(ids: np.ndarray, placed) -> np.ndarray:
    pos = {int(p.id): k for k, p in enumerate(placed)}
    return np.array([pos[int(i)] if i >= 0 else int(i) for i in ids], np.int32)


def host_trace(L, geometry: str, pts, dirs, max_steps, navigator="simple", pstep=1e30, cap=128,
               screen=0):
    g, placed = build(L, geometry, close=False)
    n = len(pts[0])
    ids = np.full(n * max_steps, -7, np.int32)
    steps = np.zeros(n * max_steps)
    saf = np.zeros(n * max_steps)
    nst = np.zeros(n, np.int32)
    a = lambda v: np.ascontiguousarray(v).ctypes.data  # noqa: E731
    args = [g.handle, n, *(a(v) for v in pts), *(a(v) for v in dirs), pstep, max_steps, a(ids),
            a(steps), a(saf), a(nst)]
    rc = (L.hc_nav_trace(*args, screen) if navigator == "simple" else L.hc_abbox_trace(*args, cap))
    assert rc == 0
    return to_positions(ids, placed), steps, saf, nst


def dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    return (t if dtype is None else t.to(dtype)).cuda()


def gpu_trace(g, placed, pts, dirs, ms, navigator="simple", pstep=1e30, precision=0):
    import torch
    import vecgeom_b200 as V
    n = len(pts[0])
    ids = torch.full((n * ms,), -7, dtype=torch.int32, device="cuda")
    steps = torch.zeros(n * ms, dtype=torch.float64, device="cuda")
    saf = torch.zeros(n * ms, dtype=torch.float64, device="cuda")
    nst = torch.zeros(n, dtype=torch.int32, device="cuda")
    P = V.SOA3D(*(dev(a) for a in pts))
    D = V.SOA3D(*(dev(a) for a in dirs))
    if navigator == "simple":
        nav = V.SimpleNavigator(g)
        nav.Trace(P, D, pstep, ms, nst, ids, steps, saf, precision=precision)
    else:
        nav = V.ABBoxNavigator(g)
        nav.Trace(P, D, pstep, ms, nst, ids, steps, saf)
    torch.cuda.synchronize()
    assert nav.error_flags() == 0
    return (to_positions(ids.cpu().numpy(), placed), steps.cpu().numpy(), saf.cpu().numpy(),
            nst.cpu().numpy())


def assert_traces_equal(got, want, max_steps, what=""):
    """got/want = (ids, steps, safeties, nsteps); every record bit for bit."""
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


BASKET_KEYS = ("px", "py", "pz", "distance", "safety", "nextnode", "newtop", "boundary")


def host_basket(L, geometry: str, pts, dirs, pstep, prior: int) -> dict:
    """hc_nav_basket: the basket step after `prior` single steps (host build)."""
    g, placed = build(L, geometry, close=False)
    n = len(pts[0])
    out = {k: np.zeros(n) for k in BASKET_KEYS[:5]}
    out.update({k: np.zeros(n, np.int32) for k in BASKET_KEYS[5:]})
    a = lambda v: np.ascontiguousarray(v).ctypes.data  # noqa: E731
    rc = L.hc_nav_basket(g.handle, n, *(a(v) for v in pts), *(a(v) for v in dirs),
                         a(np.ascontiguousarray(pstep, np.float64)), prior,
                         *(a(out[k]) for k in BASKET_KEYS))
    assert rc == 0
    pos = {int(p.id): k for k, p in enumerate(placed)}
    out["newtop"] = np.array([pos[int(i)] if i >= 0 else int(i) for i in out["newtop"]],
                             np.int32)
    return out


def assert_basket_equal(got: dict, want: dict, what=""):
    """Every field bit for bit (NaN marks tracks outside before the step)."""
    for k in BASKET_KEYS:
        a, b = np.asarray(got[k]), np.asarray(want[k])
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
        bad = np.flatnonzero(~same)
        assert len(bad) == 0, f"{what}: {k} differs for tracks {bad[:6].tolist()}"
