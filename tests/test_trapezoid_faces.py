"""Trapezoid faces: points on each of the six faces and 1e-12 to 1e-6 off them
along the outward normal (both sides of the half tolerance, 5e-10), rays from
outside aimed at face points, rays from inside points through face points, and
rays with a zero z component (the DistanceToIn / DistanceToOut branch that
divides by v.z = 0), compared bit for bit with the reference's Scalar backend:

  * CPU: the host build of the shape arithmetic, every op;
  * GPU: libvgb through the placed-volume API, every op.
"""
import numpy as np
import pytest

import oracle
from helpers import assert_distances, assert_exact, shape_specs
from test_hostcheck import hc, host_run  # noqa: F401
from vecgeom_b200 import workloads as W
from vecgeom_b200.geometry import Geometry

HAVE_REF = oracle.RefLib.available()
NAMES = ["trapezoid", "trapezoidneg", "trapezoidtrd"]
OFFSETS = np.array([0., 1e-12, -1e-12, 3e-10, -3e-10, 5e-10, -5e-10, 7e-10, -7e-10, 1e-9, -1e-9,
                    1e-6, -1e-6])
# corner indices of the faces (source/UnplacedTrapezoid.cpp:215-262 for the
# sides; the z faces close the solid)
FACES = [(0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5), (0, 1, 3, 2), (4, 5, 7, 6)]
OPS = {"contains": oracle.CONTAINS, "inside": oracle.INSIDE,
       "distance_to_in": oracle.DISTANCE_TO_IN, "distance_to_out": oracle.DISTANCE_TO_OUT,
       "safety_to_in": oracle.SAFETY_TO_IN, "safety_to_out": oracle.SAFETY_TO_OUT}


def corners(spec):
    p = spec.params
    if spec.kind == "trapezoidcorners":
        return np.asarray(p["corners"], np.float64).reshape(8, 3)
    return W.trapezoid_corners(p["dz"], p["theta"], p["phi"], p["dy1"], p["dx1"], p["dx2"],
                               p["tan_alpha1"], p["dy2"], p["dx3"], p["dx4"], p["tan_alpha2"])


def face_cases(spec, seed, per_face=6):
    """(points, out_rays, in_rays, flat_in_rays, flat_out_rays) as SOA tuples."""
    rng = np.random.default_rng(seed)
    pt = corners(spec)
    centre = pt.mean(axis=0)
    dz = pt[7, 2]
    pts, tgt = [], []
    for fi, (a, b, c, d) in enumerate(FACES):
        if fi < 4:
            n = np.cross(pt[c] - pt[a], pt[d] - pt[b])
            n /= np.linalg.norm(n)
        else:
            n = np.array([0., 0., -1. if fi == 4 else 1.])
        for _ in range(per_face):
            u, v = rng.uniform(0.05, 0.95, 2)
            # on the quadrilateral a-b-c-d (bilinear in u, v; exact for a planar face
            # up to rounding)
            q = ((1 - u) * (1 - v) * pt[a] + u * (1 - v) * pt[b] + u * v * pt[c]
                 + (1 - u) * v * pt[d])
            tgt.append(q)
            for off in OFFSETS:
                pts.append(q + off * n)
    pts, tgt = np.array(pts), np.array(tgt)
    m = len(tgt)
    # rays from outside (beyond the bounding box) towards each face point
    dirs_out = rng.normal(size=(m, 3))
    dirs_out /= np.linalg.norm(dirs_out, axis=1)[:, None]
    start_out = tgt + 3. * np.abs(pt).max() * dirs_out
    v_out = -dirs_out
    # rays from points near the centre through each face point
    start_in = centre + rng.uniform(-1., 1., (m, 3))
    v_in = tgt - start_in
    v_in /= np.linalg.norm(v_in, axis=1)[:, None]
    # v.z = 0: starts at z levels at and near the z faces, and inside
    zs = np.array([dz, -dz, dz - 1e-10, -dz + 1e-10, dz - 6e-10, -dz + 6e-10, dz - 1e-9,
                   -dz + 1e-9, dz + 1e-10, 0., 0.3 * dz, -0.7 * dz])
    k = len(zs) * 8
    ang = rng.uniform(0., 2 * np.pi, k)
    vf = np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], axis=1)
    zrep = np.repeat(zs, 8)
    # (the starts sit near the axis of the solid at each z level)
    slope = (pt[4:, :2].mean(axis=0) - pt[:4, :2].mean(axis=0)) / 2
    axis_xy = centre[:2] + (zrep / dz)[:, None] * slope
    flat_in = np.column_stack([axis_xy + rng.uniform(-1., 1., (k, 2)), zrep])
    span = np.abs(pt[:, :2]).max() * 3.
    flat_out = flat_in - span * vf
    soa = lambda a: tuple(np.ascontiguousarray(a[:, j]) for j in range(3))  # noqa: E731
    return (soa(pts), (soa(start_out), soa(v_out)), (soa(start_in), soa(v_in)),
            (soa(flat_in), soa(vf)), (soa(flat_out), soa(vf)))


def all_cases(spec, seed):
    """Per op: (points, directions) -- DistanceToIn takes the outside and flat
    outside rays plus the face points moving inward; DistanceToOut the inside
    rays, the flat inside rays and the face points moving outward."""
    pts, out_r, in_r, flat_in, flat_out = face_cases(spec, seed)
    cat = lambda *t: tuple(np.concatenate(a) for a in zip(*t))  # noqa: E731
    rng = np.random.default_rng(seed + 1)
    n = len(pts[0])
    vr = rng.normal(size=(n, 3))
    vr /= np.linalg.norm(vr, axis=1)[:, None]
    vr = tuple(np.ascontiguousarray(vr[:, j]) for j in range(3))
    dti = (cat(out_r[0], flat_out[0], pts), cat(out_r[1], flat_out[1], vr))
    dto = (cat(in_r[0], flat_in[0], pts), cat(in_r[1], flat_in[1], vr))
    return pts, dti, dto


def reference(spec, pts, dti, dto):
    ref = oracle.RefLib()
    pv = ref.placed(oracle.ref_unplaced(ref, spec))
    out = {}
    for k, op in OPS.items():
        if k == "distance_to_in":
            out[k] = ref.batch(pv, op, dti[0], dti[1], np.full(len(dti[0][0]), 1e30))
        elif k == "distance_to_out":
            out[k] = ref.batch(pv, op, dto[0], dto[1], np.full(len(dto[0][0]), 1e30))
        else:
            out[k] = ref.batch(pv, op, pts)
    return out


def check(got, want, what):
    for k in ("contains", "inside"):
        assert_exact(got[k], want[k], f"{what} {k}")
    for k in ("distance_to_in", "distance_to_out", "safety_to_in", "safety_to_out"):
        assert_distances(got[k], want[k], f"{what} {k}")


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", NAMES)
def test_host_faces_match_reference(hc, name):  # noqa: F811
    spec = shape_specs()[name]
    pts, dti, dto = all_cases(spec, 21)
    want = reference(spec, pts, dti, dto)
    g = Geometry(library=hc)
    pv = g.LogicalVolume("t", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    got = {}
    for k, op in OPS.items():
        if k == "distance_to_in":
            got[k] = host_run(hc, g, pv, op, *dti, np.full(len(dti[0][0]), 1e30))
        elif k == "distance_to_out":
            got[k] = host_run(hc, g, pv, op, *dto, np.full(len(dto[0][0]), 1e30))
        else:
            got[k] = host_run(hc, g, pv, op, pts)
    check(got, want, name)
    # the cases reach every branch: surface points, flat rays that enter and
    # that miss, rays from inside that leave through a side face
    assert (want["inside"] == 1).sum() > 0 and (want["inside"] == 0).sum() > 0
    assert np.isfinite(want["distance_to_in"]).any() and np.isinf(want["distance_to_in"]).any()


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", NAMES)
def test_gpu_faces_match_reference(name):
    import torch
    import vecgeom_b200 as V
    spec = shape_specs()[name]
    pts, dti, dto = all_cases(spec, 21)
    want = reference(spec, pts, dti, dto)
    g = V.Geometry()
    pv = g.LogicalVolume("t", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    g.SetWorld(pv)
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    soa = lambda t: V.SOA3D(*(dev(a) for a in t))  # noqa: E731
    n, ni, no = len(pts[0]), len(dti[0][0]), len(dto[0][0])
    got = {"contains": torch.zeros(n, dtype=torch.uint8, device="cuda"),
           "inside": torch.zeros(n, dtype=torch.int32, device="cuda"),
           "safety_to_in": torch.zeros(n, dtype=torch.float64, device="cuda"),
           "safety_to_out": torch.zeros(n, dtype=torch.float64, device="cuda"),
           "distance_to_in": torch.zeros(ni, dtype=torch.float64, device="cuda"),
           "distance_to_out": torch.zeros(no, dtype=torch.float64, device="cuda")}
    P = soa(pts)
    pv.Contains(P, got["contains"])
    pv.Inside(P, got["inside"])
    pv.SafetyToIn(P, got["safety_to_in"])
    pv.SafetyToOut(P, got["safety_to_out"])
    pv.DistanceToIn(soa(dti[0]), soa(dti[1]), dev(np.full(ni, 1e30)), got["distance_to_in"])
    pv.DistanceToOut(soa(dto[0]), soa(dto[1]), dev(np.full(no, 1e30)), got["distance_to_out"])
    torch.cuda.synchronize()
    check({k: v.cpu().numpy() for k, v in got.items()}, want, name)
