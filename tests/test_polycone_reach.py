"""Polycone DistanceToIn skips the sections a ray cannot reach: a ray that stays
farther from the z axis than a section's outer radius while it crosses the
section's z slab (both widened by 1e-3 mm + 1e-6 relative) gets kInfinity from
that section without the cone arithmetic.  These rays are built to pass each
section at its outer radius scaled by 1 +- 1e-3 ... 1e-12 and offset by about
the margin, at heights across the slab and just beyond its ends, some parallel
to the slabs: the results must equal the reference's bit for bit.

  * CPU: the host build of the shape arithmetic against the reference;
  * GPU: libvgb against the reference.
"""
import numpy as np
import pytest

import oracle
from helpers import PLACEMENTS, shape_specs
from test_hostcheck import hc, host_run  # noqa: F401
from vecgeom_b200 import workloads as W
from vecgeom_b200.geometry import Geometry

HAVE_REF = oracle.RefLib.available()
SPECS = {k: s for k, s in shape_specs().items() if s.kind == "polycone"}
SPECS["heavy"] = W.config3_shapes()["polycone"]


def grazing_rays(spec, n, seed):
    p = spec.params
    rng = np.random.default_rng(seed)
    zs = np.asarray(p["z"], float)
    rmax = np.asarray(p["rmax"], float)
    k = rng.integers(0, len(zs) - 1, n)
    zlo, zhi = zs[k], zs[k + 1]
    R = np.maximum(rmax[k], rmax[k + 1])
    zc = rng.uniform(zlo - 3e-3, zhi + 3e-3)
    delta = rng.choice([-1e-3, -1e-6, -1e-9, -1e-12, 0., 1e-12, 1e-9, 1e-6, 1e-3, 2e-3], n)
    rr = R * (1 + delta) + rng.choice([0., 1e-3, -1e-3, 1.1e-3, 0.9e-3], n)
    phi = rng.uniform(0, 2 * np.pi, n)
    vz = rng.choice([0., 1e-9, -1e-9, 0.01, -0.01, 0.3, -0.3, 1.0], n)
    d = np.stack([-np.sin(phi), np.cos(phi), vz])
    d /= np.linalg.norm(d, axis=0)
    start = np.stack([rr * np.cos(phi), rr * np.sin(phi), zc]) - rng.uniform(5., 300., n) * d
    return (tuple(np.ascontiguousarray(a) for a in start), tuple(np.ascontiguousarray(a) for a in d))


def reference(spec, placement, pts, dirs, step):
    ref = oracle.RefLib()
    rpv = ref.placed(oracle.ref_unplaced(ref, spec), *PLACEMENTS[placement])
    return ref.batch(rpv, oracle.DISTANCE_TO_IN, pts, dirs, step, nthreads=8)


def exact(got, want, what):
    same = (got == want) | (np.isnan(got) & np.isnan(want))
    assert same.all(), f"{what}: {int((~same).sum())} differ, first {np.flatnonzero(~same)[:5]}"


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", sorted(SPECS))
@pytest.mark.parametrize("placement", ["identity", "generic", "quirk16a"])
def test_host_grazing_rays_match_reference(hc, name, placement):  # noqa: F811
    spec = SPECS[name]
    pts, dirs = grazing_rays(spec, 1 << 15, 21)
    step = np.full(len(pts[0]), 1e30)
    g = Geometry(library=hc)
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D(*PLACEMENTS[placement]))
    exact(host_run(hc, g, pv, 2, pts, dirs, step), reference(spec, placement, pts, dirs, step),
          f"{name} {placement} DistanceToIn")


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("name", sorted(SPECS))
@pytest.mark.parametrize("placement", ["identity", "generic", "quirk16a"])
def test_gpu_grazing_rays_match_reference(name, placement):
    import torch
    import vecgeom_b200 as V
    spec = SPECS[name]
    pts, dirs = grazing_rays(spec, 1 << 15, 21)
    n = len(pts[0])
    step = np.full(n, 1e30)
    g = V.Geometry()
    pv = g.LogicalVolume("s", W.build_unplaced(g, spec)).Place(g.Transformation3D(*PLACEMENTS[placement]))
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    pv.DistanceToIn(V.SOA3D(*map(dev, pts)), V.SOA3D(*map(dev, dirs)), dev(step), out)
    torch.cuda.synchronize()
    exact(out.cpu().numpy(), reference(spec, placement, pts, dirs, step),
          f"{name} {placement} DistanceToIn")
