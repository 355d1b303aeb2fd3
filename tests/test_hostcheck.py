"""CPU: libvgb's shape arithmetic, compiled for the host, against the reference.

The kernels' per-point functions are __host__ __device__; tests/hostcheck builds
them for the host (test-only library, never loaded by the product).  These
tests run the golden cases (reference Scalar outputs) through that build, so
every shape's math is pinned to the reference before it runs on a GPU.  The
GPU tests then check the same functions as device code through libvgb.so.
"""
import ctypes
import glob
import os
import subprocess

import numpy as np
import pytest

from helpers import PLACEMENTS, assert_distances, assert_exact
from test_oracle_golden import load_case, spec_from_meta
from vecgeom_b200 import _lib
from vecgeom_b200 import workloads as W
from vecgeom_b200.geometry import Geometry

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO = os.path.join(ROOT, "_build", "hostcheck", "libvgb_hostcheck.so")
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
HOST_SHAPES = {"box", "tube", "cone", "sphere", "trd", "torus", "polycone", "polyhedron", "orb",
               "parallelepiped", "paraboloid", "trapezoid", "trapezoidcorners",
               "boolsub", "boolunion", "boolinter"}


@pytest.fixture(scope="module")
def hc():
    subprocess.run(["make", "-C", os.path.join(HERE, "hostcheck")], check=True,
                   stdout=subprocess.DEVNULL)
    L = ctypes.CDLL(SO)
    for name, (res, args) in _lib.SIGNATURES.items():
        f = getattr(L, name, None)
        if f is not None:
            f.restype = res
            f.argtypes = args
    vp = ctypes.c_void_p
    L.hc_batch.restype = ctypes.c_int
    L.hc_batch.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64] + [vp] * 8
    return L


def host_run(L, geom, pv, op, pts, dirs=None, step=None):
    n = len(pts[0])
    out = np.zeros(n, {0: np.uint8, 1: np.int32}.get(op, np.float64))
    p = [np.ascontiguousarray(a) for a in pts]
    d = [np.ascontiguousarray(a) for a in dirs] if dirs is not None else [None] * 3
    addr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    rc = L.hc_batch(geom.handle, pv.id, op, n, *(addr(a) for a in p), *(addr(a) for a in d),
                    addr(step), out.ctypes.data)
    assert rc == 0, f"hc_batch rc={rc}"
    return out


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_host_build_matches_reference(hc, path):
    d, meta = load_case(path)
    if meta["kind"] not in HOST_SHAPES:
        pytest.skip(f"{meta['kind']} not in this build")
    spec = spec_from_meta(meta)
    g = Geometry(library=hc)
    lv = g.LogicalVolume(spec.kind, W.build_unplaced(g, spec))
    pv = lv.Place(g.Transformation3D(*PLACEMENTS[str(d["placement"])]))
    pm = (d["mx"], d["my"], d["mz"])
    dm = (d["mdx"], d["mdy"], d["mdz"])
    pl = (d["lx"], d["ly"], d["lz"])
    dl = (d["ldx"], d["ldy"], d["ldz"])
    step = np.ascontiguousarray(d["step"])
    assert_exact(host_run(hc, g, pv, 0, pm), d["contains"], "Contains")
    assert_exact(host_run(hc, g, pv, 1, pm), d["inside"], "Inside")
    assert_distances(host_run(hc, g, pv, 4, pm), d["safety_to_in"], "SafetyToIn")
    assert_distances(host_run(hc, g, pv, 5, pl), d["safety_to_out"], "SafetyToOut")
    # the torus takes correctly rounded atan2/sin/cos/cbrt: its distances are
    # pinned to the reference built with those (the *_crlibm outputs)
    sfx = "_crlibm" if spec.kind == "torus" else ""
    assert_distances(host_run(hc, g, pv, 2, pm, dm, step), d["distance_to_in" + sfx],
                     "DistanceToIn")
    assert_distances(host_run(hc, g, pv, 3, pl, dl, step), d["distance_to_out" + sfx],
                     "DistanceToOut")


def test_host_build_matches_reference_on_mixed_baskets(hc):
    """256 baskets of the mixed workload (jittered shapes of the eight kinds at
    random Euler placements and translations), every op, host build against the
    reference; the GPU runs the same comparison through the basket kernel."""
    import oracle
    from helpers import assert_distances, assert_exact
    from test_baskets import _reference_baskets
    if not oracle.RefLib.available():
        pytest.skip("oracle/_ref not built")
    bs = W.config4_baskets(256, seed=W.SEED_BASE + 49)
    for b in bs:
        b.n = min(b.n, 512)
    g = Geometry(library=hc)
    placed, offsets, pts, dirs, step = W.build_baskets(g, bs)
    want, keep = _reference_baskets(bs, offsets, pts, dirs, step, 0x3f)
    for pv, off, b in zip(placed, offsets, bs):
        sl = slice(off, off + b.n)
        k = keep[sl]
        p = tuple(a[sl] for a in pts)
        d = tuple(a[sl] for a in dirs)
        what = f"basket at {off} ({b.spec.kind}, placement {b.place})"
        for op in range(6):
            got = host_run(hc, g, pv, op, p, d if op in (2, 3) else None,
                           np.ascontiguousarray(step[sl]) if op in (2, 3) else None)
            w = want[("crlibm", op)] if b.spec.kind == "torus" and op in (2, 3) else want[op]
            if op < 2:
                assert_exact(got[k], w[sl][k], f"{what} op {op}")
            else:
                assert_distances(got[k], w[sl][k], f"{what} op {op}")


def test_host_fp32_refine_sphere_distance_to_in_equals_fp64(hc):
    """The FP32+refine DistanceToIn of the sphere (refine.cuh: float selection
    with certified decisions, FP64 value of the winning root, FP64 kernel for
    uncertain points) equals the FP64 form bit for bit; on the benchmark's
    tube/cone/sphere mix the float selection settles most points."""
    from helpers import shape_specs
    vp = ctypes.c_void_p
    hc.hc_refine_dti.restype = ctypes.c_int
    hc.hc_refine_dti.argtypes = [vp, ctypes.c_int32, ctypes.c_int64] + [vp] * 9
    cases = [("bench", W.config2_shapes()["sphere"], "identity", 1 << 18)]
    cases += [(k, s, pl, 1 << 15) for k, s in shape_specs().items() if s.kind == "sphere"
              for pl in ("identity", "generic")]
    for name, spec, pl, n in cases:
        g = Geometry(library=hc)
        pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(
            g.Transformation3D(*PLACEMENTS[pl]))
        wl = W.make_workload(spec, n, W.SEED_BASE + 2)
        a = [np.ascontiguousarray(v) for v in (wl.x, wl.y, wl.z, wl.dx, wl.dy, wl.dz, wl.step)]
        want = host_run(hc, g, pv, 2, a[:3], a[3:6], a[6])
        got = np.zeros(n)
        win = np.zeros(n, np.int32)
        assert hc.hc_refine_dti(g.handle, pv.id, n, *(v.ctypes.data for v in a), got.ctypes.data,
                                win.ctypes.data) == 0
        same = (got == want) | (np.isnan(got) & np.isnan(want))
        assert same.all(), f"{name} {pl}: {np.flatnonzero(~same)[:5]}"
        if name == "bench":
            assert (win > 0).mean() > 0.6, (win > 0).mean()
