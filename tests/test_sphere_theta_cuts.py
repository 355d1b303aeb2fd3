"""Sphere angle cuts: points and rays placed 0 to 1e-11 rad from every
theta cut the kernels compare with (stheta -/+ the half angular tolerance,
eTheta -/+ it).  The kernels decide such comparisons from z sin c - rho cos c
and evaluate atan2 only within ~3e-15 rad of a cut; these cases sit on both
sides of that margin.  Points near phi = 0 check the phi test, which a
full-phi sphere with a theta cut decides without atan2 away from that seam.

  * CPU: the host build of the shape arithmetic against the reference (Inside,
    Contains) and against USolids' USphere::DistanceToIn (the in-tree sphere
    DistanceToIn), every case;
  * GPU: libvgb against the same, for offsets of 1e-14 rad and more (closer
    to a cut the GPU's atan2 and the C library's may round to different
    sides, as for any transcendental; the decided comparisons do not).
"""
import math

import numpy as np
import pytest

import oracle
from helpers import assert_distances, assert_exact
from test_hostcheck import hc, host_run  # noqa: F401
from vecgeom_b200 import workloads as W
from vecgeom_b200.geometry import Geometry

HAVE_REF = oracle.RefLib.available()
HALF_ANG_TOL = 0.5e-9
OFFSETS = np.array([0., 1e-16, -1e-16, 3e-16, -3e-16, 1e-15, -1e-15, 3e-15, -3e-15, 6e-15, -6e-15,
                    1e-14, -1e-14, 1e-13, -1e-13, 1e-11, -1e-11])
SPECS = {
    "hemisphere": W.sphere_spec(10., 30., 0., 2 * math.pi, 0., math.pi / 2),
    "band": W.sphere_spec(5., 30., 0., 2 * math.pi, math.radians(30.), math.radians(60.)),
    "band_sector": W.sphere_spec(5., 30., 0.3, 4.0, 0.4, 1.9),
}


def cut_cases(spec, seed):
    """(points, rays, offsets): points at the cut angles + offsets inside the
    radial shell, and rays from outside aimed at points of the outer sphere at
    those angles."""
    p = spec.params
    rng = np.random.default_rng(seed)
    st, et = p["stheta"], p["stheta"] + p["dtheta"]
    cuts = [c for c in (st - HALF_ANG_TOL, st + HALF_ANG_TOL, et - HALF_ANG_TOL,
                        et + HALF_ANG_TOL) if 0. <= c <= math.pi]
    th = np.concatenate([c + OFFSETS for c in cuts] * 8)
    off = np.concatenate([OFFSETS for _ in cuts] * 8)
    n = len(th)
    phi = rng.uniform(0., 2 * math.pi, n)
    r = rng.uniform(p["rmin"] + 1., p["rmax"] - 1., n)
    pts = (r * np.sin(th) * np.cos(phi), r * np.sin(th) * np.sin(phi), r * np.cos(th))
    # rays: a target on the outer sphere at the cut angle, reached from 50 mm
    # outside along a direction pointing into the sphere
    t = np.stack([p["rmax"] * np.sin(th) * np.cos(phi), p["rmax"] * np.sin(th) * np.sin(phi),
                  p["rmax"] * np.cos(th)])
    v = np.stack(W.isotropic(rng, n))
    flip = (v * t).sum(axis=0) > 0
    v[:, flip] *= -1
    start = t - 50. * v
    rays = (tuple(np.ascontiguousarray(a) for a in start), tuple(np.ascontiguousarray(a) for a in v))
    return pts, rays, off


def seam_points(spec, seed):
    """Points of the radial shell at phi = 0 + offsets (the phi test of a
    full-phi sphere with a theta cut only matters within its half tolerance,
    5e-10 rad, of phi = 0), on both sides of x = 0, and on the z axis."""
    p = spec.params
    rng = np.random.default_rng(seed)
    dphi = np.array([0., 1e-12, -1e-12, 1e-10, -1e-10, 4e-10, -4e-10, 6e-10, -6e-10, 1e-9, -1e-9,
                     9e-9, -9e-9, 1.1e-8, -1.1e-8, 2e-8, -2e-8, math.pi / 2, math.pi, -math.pi])
    st, et = p["stheta"], p["stheta"] + p["dtheta"]
    th = np.repeat(np.linspace(st + 0.05, et - 0.05, 4), len(dphi))
    ph = np.tile(dphi, 4)
    r = rng.uniform(p["rmin"] + 1., p["rmax"] - 1., len(th))
    x, y, z = r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)
    axis = np.array([p["rmin"] + 2., p["rmax"] - 2., -(p["rmin"] + 2.)])
    return (np.concatenate([x, np.zeros(3), -np.zeros(3)]),
            np.concatenate([y, np.zeros(3), np.zeros(3)]),
            np.concatenate([z, axis, axis]))


def reference(spec, pts, rays):
    ref = oracle.RefLib()
    pv = ref.placed(oracle.ref_unplaced(ref, spec))
    return {"contains": ref.batch(pv, 0, pts), "inside": ref.batch(pv, 1, pts),
            "dti": ref.usphere_distance_to_in(spec.params, ref.last_transform, *rays)}


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(SPECS))
def test_host_theta_cuts_match_reference(hc, name):  # noqa: F811
    spec = SPECS[name]
    pts, rays, _ = cut_cases(spec, 11)
    want = reference(spec, pts, rays)
    g = Geometry(library=hc)
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    step = np.full(len(rays[0][0]), 1e30)
    assert_exact(host_run(hc, g, pv, 0, pts), want["contains"], "Contains")
    assert_exact(host_run(hc, g, pv, 1, pts), want["inside"], "Inside")
    assert_distances(host_run(hc, g, pv, 2, *rays, step), want["dti"], "DistanceToIn")


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(SPECS))
def test_host_phi_seam_matches_reference(hc, name):  # noqa: F811
    spec = SPECS[name]
    pts = seam_points(spec, 12)
    ref = oracle.RefLib()
    rpv = ref.placed(oracle.ref_unplaced(ref, spec))
    g = Geometry(library=hc)
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    assert_exact(host_run(hc, g, pv, 0, pts), ref.batch(rpv, 0, pts), "Contains")
    assert_exact(host_run(hc, g, pv, 1, pts), ref.batch(rpv, 1, pts), "Inside")


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(SPECS))
def test_gpu_phi_seam_matches_reference(name):
    import torch
    import vecgeom_b200 as V
    spec = SPECS[name]
    pts = seam_points(spec, 12)
    ref = oracle.RefLib()
    rpv = ref.placed(oracle.ref_unplaced(ref, spec))
    g = V.Geometry()
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    g.SetWorld(pv)
    g.CloseGeometry()
    n = len(pts[0])
    P = V.SOA3D(*(torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pts))
    c = torch.zeros(n, dtype=torch.uint8, device="cuda")
    i = torch.zeros(n, dtype=torch.int32, device="cuda")
    pv.Contains(P, c)
    pv.Inside(P, i)
    torch.cuda.synchronize()
    assert_exact(c.cpu().numpy(), ref.batch(rpv, 0, pts), "Contains")
    assert_exact(i.cpu().numpy(), ref.batch(rpv, 1, pts), "Inside")


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(SPECS))
def test_gpu_theta_cuts_match_reference(name):
    import torch
    import vecgeom_b200 as V
    spec = SPECS[name]
    pts, rays, off = cut_cases(spec, 11)
    want = reference(spec, pts, rays)
    keep = np.abs(off) >= 1e-14
    g = V.Geometry()
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    g.SetWorld(pv)
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    n = len(off)
    P = V.SOA3D(*(dev(a) for a in pts))
    c = torch.zeros(n, dtype=torch.uint8, device="cuda")
    i = torch.zeros(n, dtype=torch.int32, device="cuda")
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    pv.Contains(P, c)
    pv.Inside(P, i)
    pv.DistanceToIn(V.SOA3D(*(dev(a) for a in rays[0])), V.SOA3D(*(dev(a) for a in rays[1])),
                    dev(np.full(n, 1e30)), d)
    torch.cuda.synchronize()
    assert_exact(c.cpu().numpy()[keep], want["contains"][keep], "Contains")
    assert_exact(i.cpu().numpy()[keep], want["inside"][keep], "Inside")
    assert_distances(d.cpu().numpy()[keep], want["dti"][keep], "DistanceToIn")


def far_rays(spec, seed, n=4096):
    """Rays from 100 to 1000 rmax away (beyond the 100 rmax at which USolids'
    DistanceToIn splits an outer-sphere distance and re-enters from the split
    point, USphere.cc:685-689), aimed at random points of the radial shell;
    a quarter start on the z axis and a quarter in the z = 0 plane."""
    p = spec.params
    rng = np.random.default_rng(seed)
    tgt = np.stack(W.isotropic(rng, n)) * rng.uniform(0., p["rmax"], n)
    u = np.stack(W.isotropic(rng, n))
    u[:, : n // 4] = np.array([[0.], [0.], [1.]])
    u[2, n // 4: n // 2] = 0.
    u /= np.linalg.norm(u, axis=0)
    start = u * rng.uniform(100. * p["rmax"], 1000. * p["rmax"], n)
    v = tgt - start
    v /= np.linalg.norm(v, axis=0)
    return (tuple(np.ascontiguousarray(a) for a in start), tuple(np.ascontiguousarray(a) for a in v))


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(SPECS))
def test_host_far_rays_match_reference(hc, name):  # noqa: F811
    spec = SPECS[name]
    rays = far_rays(spec, 13)
    ref = oracle.RefLib()
    ref.placed(oracle.ref_unplaced(ref, spec))
    want = ref.usphere_distance_to_in(spec.params, ref.last_transform, *rays)
    assert np.isfinite(want).mean() > 0.3
    g = Geometry(library=hc)
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    step = np.full(len(rays[0][0]), 1e30)
    assert_distances(host_run(hc, g, pv, 2, *rays, step), want, "DistanceToIn (far rays)")


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(SPECS))
def test_gpu_far_rays_match_reference(name):
    import torch
    import vecgeom_b200 as V
    spec = SPECS[name]
    rays = far_rays(spec, 13)
    ref = oracle.RefLib()
    ref.placed(oracle.ref_unplaced(ref, spec))
    want = ref.usphere_distance_to_in(spec.params, ref.last_transform, *rays)
    g = V.Geometry()
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D())
    g.SetWorld(pv)
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    n = len(rays[0][0])
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    pv.DistanceToIn(V.SOA3D(*(dev(a) for a in rays[0])), V.SOA3D(*(dev(a) for a in rays[1])),
                    dev(np.full(n, 1e30)), d)
    torch.cuda.synchronize()
    assert_distances(d.cpu().numpy(), want, "DistanceToIn (far rays)")
