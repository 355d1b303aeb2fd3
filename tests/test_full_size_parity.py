"""Parity at the benchmark sizes: the exact batches bench.py times, compared
with the reference itself.

For every shape of the three shape workloads (the box with 2^20 uniform
points; tube, cone and sphere with 2^22 mixed points; torus, polycone,
polyhedron and box minus tube with 2^22 mixed points) the same seeded arrays
the benchmark draws run through libvgb on the GPU, and the reference Scalar
backend (oracle/_ref, the reference compiled from its own sources) runs them on
every host core.  Ops as the benchmark runs them: Contains, Inside, SafetyToIn
and DistanceToIn on all points, SafetyToOut and DistanceToOut on the points
Contains() accepts.  The bar is the parity bar of helpers.py: Contains/Inside
bit-exact, distances and safeties within 1e-9 mm or 1e-12 relative (the torus
distances: against the reference built with correctly rounded atan2/sin/cos/
cbrt, as documented there).  Points on which the reference's
own result is undefined (helpers.reference_defined) are left out.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import (assert_distances, assert_exact, assert_torus_distances, ref_unplaced,
                     reference_defined)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.RefLib.available(), reason="oracle/_ref not built")]

CASES = [("box", "box"), ("shapes", "tube"), ("shapes", "cone"), ("shapes", "sphere"),
         ("heavy", "torus"), ("heavy", "polycone"), ("heavy", "polyhedron"),
         ("heavy", "boolsub")]
THREADS = os.cpu_count() or 1


def gpu_ops(spec, wl, sel):
    """The six ops through libvgb, the local ops on the points `sel` selects."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    g = V.Geometry()
    lv = g.LogicalVolume(spec.kind, W.build_unplaced(g, spec))
    pv = lv.Place(g.Transformation3D())
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    n = wl.n
    P = V.SOA3D(dev(wl.x), dev(wl.y), dev(wl.z))
    D = V.SOA3D(dev(wl.dx), dev(wl.dy), dev(wl.dz))
    S = dev(wl.step)
    PS = V.SOA3D(dev(wl.x[sel]), dev(wl.y[sel]), dev(wl.z[sel]))
    DS = V.SOA3D(dev(wl.dx[sel]), dev(wl.dy[sel]), dev(wl.dz[sel]))
    SS = dev(wl.step[sel])
    m = int(sel.sum())
    f8 = lambda k: torch.empty(k, dtype=torch.float64, device="cuda")  # noqa: E731
    out = {"contains": torch.empty(n, dtype=torch.uint8, device="cuda"),
           "inside": torch.empty(n, dtype=torch.int32, device="cuda"),
           "safety_to_in": f8(n), "distance_to_in": f8(n),
           "safety_to_out": f8(m), "distance_to_out": f8(m)}
    pv.Contains(P, out["contains"])
    pv.Inside(P, out["inside"])
    pv.SafetyToIn(P, out["safety_to_in"])
    pv.DistanceToIn(P, D, S, out["distance_to_in"])
    pv.SafetyToOut(PS, out["safety_to_out"])
    pv.DistanceToOut(PS, DS, SS, out["distance_to_out"])
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("config,shape", CASES, ids=[f"{c}-{s}" for c, s in CASES])
def test_bench_batch_matches_reference_at_full_size(config, shape):
    from vecgeom_b200 import workloads as W
    shapes, n, mix = W.bench_config(config)
    spec = shapes[shape]
    wl = W.make_workload(spec, n, W.bench_seed(list(shapes).index(shape)), mix=mix)
    keep = reference_defined(spec, wl.z)   # identity placement: local z = z
    if not keep.all():
        wl = W.ShapeWorkload(spec, *(np.ascontiguousarray(getattr(wl, k)[keep])
                                     for k in ("x", "y", "z", "dx", "dy", "dz", "step")))
        assert (~keep).sum() < 1e-3 * n
    ref = oracle.RefLib()
    rpv = ref.placed(ref_unplaced(ref, spec))
    pts, dirs = (wl.x, wl.y, wl.z), (wl.dx, wl.dy, wl.dz)
    want = {"contains": ref.batch(rpv, oracle.CONTAINS, pts, nthreads=THREADS),
            "inside": ref.batch(rpv, oracle.INSIDE, pts, nthreads=THREADS),
            "safety_to_in": ref.batch(rpv, oracle.SAFETY_TO_IN, pts, nthreads=THREADS)}
    if spec.kind == "sphere":
        want["distance_to_in"] = ref.usphere_distance_to_in(spec.params, ref.last_transform, pts,
                                                            dirs, nthreads=THREADS)
    else:
        want["distance_to_in"] = ref.batch(rpv, oracle.DISTANCE_TO_IN, pts, dirs, wl.step,
                                           nthreads=THREADS)
    sel = want["contains"].astype(bool)
    spts = tuple(np.ascontiguousarray(a[sel]) for a in pts)
    sdirs = tuple(np.ascontiguousarray(a[sel]) for a in dirs)
    want["safety_to_out"] = ref.batch(rpv, oracle.SAFETY_TO_OUT, spts, nthreads=THREADS)
    want["distance_to_out"] = ref.batch(rpv, oracle.DISTANCE_TO_OUT, spts, sdirs,
                                        np.ascontiguousarray(wl.step[sel]), nthreads=THREADS)
    if spec.kind == "torus":
        cr = oracle.RefLib(crlibm=True)
        cpv = cr.placed(ref_unplaced(cr, spec))
        want["distance_to_in_crlibm"] = cr.batch(cpv, oracle.DISTANCE_TO_IN, pts, dirs, wl.step,
                                                 nthreads=THREADS)
        want["distance_to_out_crlibm"] = cr.batch(cpv, oracle.DISTANCE_TO_OUT, spts, sdirs,
                                                  np.ascontiguousarray(wl.step[sel]),
                                                  nthreads=THREADS)
    got = gpu_ops(spec, wl, sel)
    what = f"{config}/{shape} ({wl.n} of {n} points)"
    assert_exact(got["contains"], want["contains"], f"{what} Contains")
    assert_exact(got["inside"], want["inside"], f"{what} Inside")
    for k in ("safety_to_in", "safety_to_out"):
        assert_distances(got[k], want[k], f"{what} {k}")
    if spec.kind == "torus":
        for k in ("distance_to_in", "distance_to_out"):
            stats = assert_torus_distances(got[k], want[k + "_crlibm"], want[k], f"{what} {k}")
            print(f"{what} {k}: {stats}")
    else:
        for k in ("distance_to_in", "distance_to_out"):
            assert_distances(got[k], want[k], f"{what} {k}")


def test_fp32_refine_at_full_size_equals_fp64():
    """The FP32+refine form on the benchmark's tube/cone/sphere batches (2^22
    mixed points each): every op bit-identical to the FP64 form, and the
    sphere's float selection really settles most of its DistanceToIn points
    (vgb_refine_counts)."""
    import ctypes
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    shapes, n, mix = W.bench_config("shapes")
    L = V.lib()
    for si, (name, spec) in enumerate(shapes.items()):
        wl = W.make_workload(spec, n, W.bench_seed(si), mix=mix)
        g = V.Geometry()
        pv = g.LogicalVolume(name, W.build_unplaced(g, spec)).Place(g.Transformation3D())
        g.CloseGeometry()
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
        P = V.SOA3D(dev(wl.x), dev(wl.y), dev(wl.z))
        D = V.SOA3D(dev(wl.dx), dev(wl.dy), dev(wl.dz))
        S = dev(wl.step)
        c = torch.empty(n, dtype=torch.uint8, device="cuda")
        pv.Contains(P, c)
        sel = c.bool()
        PS = V.SOA3D(P.x[sel].contiguous(), P.y[sel].contiguous(), P.z[sel].contiguous())
        DS = V.SOA3D(D.x[sel].contiguous(), D.y[sel].contiguous(), D.z[sel].contiguous())
        SS = S[sel].contiguous()
        V.check(L.vgb_refine_counts(None, None, 1))
        for meth, args, pts in (("Contains", (), P), ("Inside", (), P), ("SafetyToIn", (), P),
                                ("DistanceToIn", (D, S), P), ("SafetyToOut", (), PS),
                                ("DistanceToOut", (DS, SS), PS)):
            m = pts.size()
            dt = {"Contains": torch.uint8, "Inside": torch.int32}.get(meth, torch.float64)
            a = torch.full((m,), 7, dtype=dt, device="cuda")
            b = torch.full((m,), 9, dtype=dt, device="cuda")
            getattr(pv, meth)(pts, *args, a, precision=V.PREC_FP64)
            getattr(pv, meth)(pts, *args, b, precision=V.PREC_FP32_REFINE)
            torch.cuda.synchronize()
            same = (a == b) | (torch.isnan(a) & torch.isnan(b)) if dt == torch.float64 else a == b
            assert bool(same.all()), f"{name} {meth}: {int((~same).sum())} differ"
        cert, fb = ctypes.c_int64(), ctypes.c_int64()
        V.check(L.vgb_refine_counts(ctypes.byref(cert), ctypes.byref(fb), 1))
        if name == "sphere":
            assert cert.value + fb.value == n and cert.value > 0.6 * n, (cert.value, fb.value)
