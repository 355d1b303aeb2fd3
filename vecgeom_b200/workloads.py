"""Seeded synthetic workloads for the shape and navigation benchmarks.

Plays the role of the reference's point/direction generators
(volumes/utilities/VolumeUtilities.h:67-452) with our own, seed-stable
sampling:
  * directions are isotropic unit vectors (normalised 3-D Gaussians);
  * "mixed" point sets are 1/3 uniform inside the shape, 1/3 uniform outside it
    within a bounding box 1.5x the shape's extent, and 1/3 within +-1e-6 mm of
    the surface (a boundary crossing between an inside and an outside sample,
    found by bisection, then moved by U(-1e-6, 1e-6) mm along the segment).
Each ShapeSpec carries an exact (tolerance-free) numpy containment test used
only to draw inputs; results are always computed by libvgb.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

SEED_BASE = 0x5EED


def isotropic(rng: np.random.Generator, n: int):
    v = rng.standard_normal((3, n))
    v /= np.sqrt((v * v).sum(axis=0))
    return v[0].copy(), v[1].copy(), v[2].copy()


@dataclass
class ShapeSpec:
    """One unplaced shape: constructor arguments plus sampling helpers."""
    kind: str                       # box, tube, cone, sphere, torus, polycone, polyhedron, boolsub,
                                    # trd, orb, parallelepiped, paraboloid, trapezoid,
                                    # trapezoidcorners
    params: dict
    half: tuple                     # half extents of the axis-aligned bounding box
    center: tuple = (0., 0., 0.)
    contains: Callable = field(default=None, repr=False)

    def bbox_sample(self, rng, n, scale=1.0):
        h = np.asarray(self.half) * scale
        c = np.asarray(self.center)
        u = rng.uniform(-1.0, 1.0, (3, n))
        return (c[0] + u[0] * h[0], c[1] + u[1] * h[1], c[2] + u[2] * h[2])


def _phi_in(phi, sphi, dphi):
    """phi in [sphi, sphi+dphi] (radians), wrap-aware."""
    if dphi >= 2 * math.pi - 1e-15:
        return np.ones_like(phi, dtype=bool)
    d = np.mod(phi - sphi, 2 * math.pi)
    return d <= dphi


def box_spec(dx, dy, dz) -> ShapeSpec:
    def contains(x, y, z):
        return (np.abs(x) <= dx) & (np.abs(y) <= dy) & (np.abs(z) <= dz)
    return ShapeSpec("box", dict(dx=dx, dy=dy, dz=dz), (dx, dy, dz), contains=contains)


def tube_spec(rmin, rmax, dz, sphi, dphi) -> ShapeSpec:
    def contains(x, y, z):
        r2 = x * x + y * y
        ok = (np.abs(z) <= dz) & (r2 <= rmax * rmax) & (r2 >= rmin * rmin)
        return ok & _phi_in(np.arctan2(y, x), sphi, dphi)
    return ShapeSpec("tube", dict(rmin=rmin, rmax=rmax, dz=dz, sphi=sphi, dphi=dphi),
                     (rmax, rmax, dz), contains=contains)


def cone_spec(rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi) -> ShapeSpec:
    def contains(x, y, z):
        t = (z + dz) / (2 * dz)
        rlo = rmin1 + (rmin2 - rmin1) * t
        rhi = rmax1 + (rmax2 - rmax1) * t
        r = np.sqrt(x * x + y * y)
        ok = (np.abs(z) <= dz) & (r <= rhi) & (r >= rlo)
        return ok & _phi_in(np.arctan2(y, x), sphi, dphi)
    R = max(rmax1, rmax2)
    return ShapeSpec("cone", dict(rmin1=rmin1, rmax1=rmax1, rmin2=rmin2, rmax2=rmax2, dz=dz,
                                  sphi=sphi, dphi=dphi), (R, R, dz), contains=contains)


def sphere_spec(rmin, rmax, sphi, dphi, stheta, dtheta) -> ShapeSpec:
    def contains(x, y, z):
        r2 = x * x + y * y + z * z
        ok = (r2 <= rmax * rmax) & (r2 >= rmin * rmin)
        th = np.arctan2(np.sqrt(x * x + y * y), z)
        ok &= (th >= stheta) & (th <= stheta + dtheta)
        return ok & _phi_in(np.arctan2(y, x), sphi, dphi)
    return ShapeSpec("sphere", dict(rmin=rmin, rmax=rmax, sphi=sphi, dphi=dphi, stheta=stheta,
                                    dtheta=dtheta), (rmax, rmax, rmax), contains=contains)


def torus_spec(rmin, rmax, rtor, sphi, dphi) -> ShapeSpec:
    def contains(x, y, z):
        rho = np.sqrt(x * x + y * y) - rtor
        d2 = rho * rho + z * z
        ok = (d2 <= rmax * rmax) & (d2 >= rmin * rmin)
        return ok & _phi_in(np.arctan2(y, x), sphi, dphi)
    R = rtor + rmax
    return ShapeSpec("torus", dict(rmin=rmin, rmax=rmax, rtor=rtor, sphi=sphi, dphi=dphi),
                     (R, R, rmax), contains=contains)


def orb_spec(r) -> ShapeSpec:
    def contains(x, y, z):
        return x * x + y * y + z * z <= r * r
    return ShapeSpec("orb", dict(r=r), (r, r, r), contains=contains)


def parallelepiped_spec(x, y, z, alpha, theta, phi) -> ShapeSpec:
    """Half-lengths x, y, z; alpha, theta, phi in degrees (the reference's
    UnplacedParallelepiped arguments)."""
    ta = math.tan(math.radians(alpha))
    tt = math.tan(math.radians(theta))
    tcp, tsp = tt * math.cos(math.radians(phi)), tt * math.sin(math.radians(phi))

    def contains(px, py, pz):
        ly = py - tsp * pz
        lx = px - (tcp * pz + ta * ly)
        return (np.abs(lx) <= x) & (np.abs(ly) <= y) & (np.abs(pz) <= z)
    hy = y + abs(tsp) * z
    hx = x + abs(tcp) * z + abs(ta) * hy
    return ShapeSpec("parallelepiped", dict(x=x, y=y, z=z, alpha=alpha, theta=theta, phi=phi),
                     (hx, hy, z), contains=contains)


def paraboloid_spec(rlo, rhi, dz) -> ShapeSpec:
    a = 2. * dz / (rhi * rhi - rlo * rlo)
    b = -dz * (rlo * rlo + rhi * rhi) / (rhi * rhi - rlo * rlo)

    def contains(x, y, z):
        return (np.abs(z) <= dz) & (z >= a * (x * x + y * y) + b)
    h = max(rlo, rhi)
    return ShapeSpec("paraboloid", dict(rlo=rlo, rhi=rhi, dz=dz), (h, h, dz), contains=contains)


def _trapezoid_shape(kind, params, corners) -> ShapeSpec:
    """ShapeSpec of a trapezoid given its 8 corners (0-3 at -dz, 4-7 at +dz):
    the bounding box of the corners and the four side planes' test."""
    pt = np.asarray(corners, np.float64).reshape(8, 3)
    dz = pt[7, 2]
    quads = ((0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5))
    planes = []
    for i1, i2, i3, i4 in quads:
        n = np.cross(pt[i3] - pt[i1], pt[i4] - pt[i2])
        n = n / np.linalg.norm(n)
        planes.append((n, -n.dot(pt[i1])))

    def contains(x, y, z):
        ok = np.abs(z) <= dz
        for n, d in planes:
            ok &= n[0] * x + n[1] * y + n[2] * z + d <= 0
        return ok
    lo, hi = pt.min(axis=0), pt.max(axis=0)
    return ShapeSpec(kind, params, tuple((hi - lo) / 2), center=tuple((hi + lo) / 2),
                     contains=contains)


def trapezoid_corners(dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4, tan_alpha2):
    """The 8 corners of UnplacedTrapezoid's parameters
    (source/UnplacedTrapezoid.cpp:673-685)."""
    tc, ts = math.tan(theta) * math.cos(phi), math.tan(theta) * math.sin(phi)
    out = []
    for z, dy, dxa, dxb, ta in ((-dz, dy1, dx1, dx2, tan_alpha1), (dz, dy2, dx3, dx4, tan_alpha2)):
        for sy, dx in ((-1, dxa), (1, dxb)):
            for sx in (-1, 1):
                out.append((z * tc + sy * dy * ta + sx * dx, z * ts + sy * dy, z))
    return np.array(out)


def trapezoid_spec(dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4,
                   tan_alpha2) -> ShapeSpec:
    """General trapezoid (UnplacedTrapezoid's 11 parameters, angles in radians)."""
    args = (dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4, tan_alpha2)
    names = ("dz", "theta", "phi", "dy1", "dx1", "dx2", "tan_alpha1", "dy2", "dx3", "dx4",
             "tan_alpha2")
    return _trapezoid_shape("trapezoid", dict(zip(names, args)), trapezoid_corners(*args))


def trapezoid_corners_spec(corners) -> ShapeSpec:
    """Trapezoid built from its 8 corners (UnplacedTrapezoid(TrapCorners_t))."""
    c = np.asarray(corners, np.float64).reshape(8, 3)
    return _trapezoid_shape("trapezoidcorners", dict(corners=c.ravel().tolist()), c)


def trd_spec(dx1, dx2, dy1, dy2, dz) -> ShapeSpec:
    def contains(x, y, z):
        t = (z + dz) / (2 * dz)
        hx = dx1 + (dx2 - dx1) * t
        hy = dy1 + (dy2 - dy1) * t
        return (np.abs(z) <= dz) & (np.abs(x) <= hx) & (np.abs(y) <= hy)
    return ShapeSpec("trd", dict(dx1=dx1, dx2=dx2, dy1=dy1, dy2=dy2, dz=dz),
                     (max(dx1, dx2), max(dy1, dy2), dz), contains=contains)


def polycone_spec(sphi, dphi, z, rmin, rmax) -> ShapeSpec:
    z = np.asarray(z, float)
    rmin = np.asarray(rmin, float)
    rmax = np.asarray(rmax, float)

    def contains(x, y, zz):
        r = np.sqrt(x * x + y * y)
        ok = np.zeros(x.shape, bool)
        for k in range(len(z) - 1):
            if z[k + 1] == z[k]:
                continue
            t = (zz - z[k]) / (z[k + 1] - z[k])
            insec = (zz >= z[k]) & (zz <= z[k + 1])
            lo = rmin[k] + (rmin[k + 1] - rmin[k]) * t
            hi = rmax[k] + (rmax[k + 1] - rmax[k]) * t
            ok |= insec & (r >= lo) & (r <= hi)
        return ok & _phi_in(np.arctan2(y, x), sphi, dphi)
    R = float(rmax.max())
    zc = 0.5 * (z[0] + z[-1])
    return ShapeSpec("polycone", dict(sphi=sphi, dphi=dphi, z=z, rmin=rmin, rmax=rmax),
                     (R, R, 0.5 * (z[-1] - z[0])), center=(0., 0., zc), contains=contains)


def polyhedron_spec(phi_start_deg, phi_delta_deg, sides, z, rmin, rmax) -> ShapeSpec:
    """Polyhedron with rmin/rmax as inner/outer apothems (distance to the side
    planes), as volumes/UnplacedPolyhedron.h takes them."""
    z = np.asarray(z, float)
    rmin = np.asarray(rmin, float)
    rmax = np.asarray(rmax, float)
    s0 = math.radians(phi_start_deg)
    dphi = math.radians(phi_delta_deg if phi_delta_deg > 0 else 360.0)
    sw = dphi / sides

    def contains(x, y, zz):
        phi = np.arctan2(y, x)
        rel = np.mod(phi - s0, 2 * math.pi)
        inphi = rel <= dphi if dphi < 2 * math.pi - 1e-12 else np.ones_like(rel, bool)
        k = np.minimum(np.floor(rel / sw), sides - 1)
        mid = s0 + (k + 0.5) * sw
        a = x * np.cos(mid) + y * np.sin(mid)   # distance along the side normal
        ok = np.zeros(x.shape, bool)
        for j in range(len(z) - 1):
            if z[j + 1] == z[j]:
                continue
            t = (zz - z[j]) / (z[j + 1] - z[j])
            inseg = (zz >= z[j]) & (zz <= z[j + 1])
            lo = rmin[j] + (rmin[j + 1] - rmin[j]) * t
            hi = rmax[j] + (rmax[j + 1] - rmax[j]) * t
            ok |= inseg & (a >= lo) & (a <= hi)
        return ok & inphi
    R = float(rmax.max()) / math.cos(math.pi / sides)
    zc = 0.5 * (z[0] + z[-1])
    return ShapeSpec("polyhedron", dict(phi_start_deg=phi_start_deg, phi_delta_deg=phi_delta_deg,
                                        sides=sides, z=z, rmin=rmin, rmax=rmax),
                     (R, R, 0.5 * (z[-1] - z[0])), center=(0., 0., zc), contains=contains)


def euler_rotation(phi, theta, psi) -> np.ndarray:
    """Row-major rotation of Transformation3D(tx,ty,tz, phi,theta,psi), angles in
    degrees (source/Transformation3D.cpp:93-114).  The master-to-local transform
    is local = R^T (master - t)."""
    d = math.pi / 180.
    sf, cf = math.sin(d * phi), math.cos(d * phi)
    st, ct = math.sin(d * theta), math.cos(d * theta)
    sp, cp = math.sin(d * psi), math.cos(d * psi)
    return np.array([[cp * cf - ct * sf * sp, -sp * cf - ct * sf * cp, st * sf],
                     [cp * sf + ct * cf * sp, -sp * sf + ct * cf * cp, -st * cf],
                     [sp * st, cp * st, ct]])


def to_local(place, x, y, z):
    """Mother-frame points in the frame of a placement (tx,ty,tz,phi,theta,psi)."""
    R = euler_rotation(*place[3:])
    a = np.stack([np.asarray(x) - place[0], np.asarray(y) - place[1], np.asarray(z) - place[2]])
    loc = R.T @ a.reshape(3, -1)
    return (loc[0].reshape(np.shape(x)), loc[1].reshape(np.shape(x)), loc[2].reshape(np.shape(x)))


IDENTITY_PLACE = (0., 0., 0., 0., 0., 0.)


def boolsub_spec(box_half, tube_rmax, tube_dz, left_place=IDENTITY_PLACE,
                 right_place=IDENTITY_PLACE) -> ShapeSpec:
    """Box minus a full solid tube, each component at its own placement
    (tx,ty,tz, Euler phi,theta,psi in degrees) in the boolean's frame."""
    bx, by, bz = box_half

    def contains(x, y, z):
        lx, ly, lz = to_local(left_place, x, y, z)
        inbox = (np.abs(lx) <= bx) & (np.abs(ly) <= by) & (np.abs(lz) <= bz)
        rx, ry, rz = to_local(right_place, x, y, z)
        intube = (rx * rx + ry * ry <= tube_rmax * tube_rmax) & (np.abs(rz) <= tube_dz)
        return inbox & ~intube
    params = dict(box_half=box_half, tube_rmax=tube_rmax, tube_dz=tube_dz)
    extent = (bx, by, bz)
    if tuple(left_place) != IDENTITY_PLACE or tuple(right_place) != IDENTITY_PLACE:
        params.update(left_place=list(left_place), right_place=list(right_place))
        e = float(np.linalg.norm(box_half)) + float(np.linalg.norm(left_place[:3]))
        extent = (e, e, e)
    return ShapeSpec("boolsub", params, extent, contains=contains)


# operation codes of UnplacedBooleanVolume (volumes/UnplacedBooleanVolume.h:10-14)
BOOL_OPS = {"boolunion": 0, "boolinter": 1, "boolsub": 2}


def boolean_spec(kind, box_half, tube_rmax, tube_dz, left_place=IDENTITY_PLACE,
                 right_place=IDENTITY_PLACE) -> ShapeSpec:
    """Box union / intersection with a full solid tube (kind "boolunion" or
    "boolinter"), each component at its own placement."""
    bx, by, bz = box_half

    def contains(x, y, z):
        lx, ly, lz = to_local(left_place, x, y, z)
        inbox = (np.abs(lx) <= bx) & (np.abs(ly) <= by) & (np.abs(lz) <= bz)
        rx, ry, rz = to_local(right_place, x, y, z)
        intube = (rx * rx + ry * ry <= tube_rmax * tube_rmax) & (np.abs(rz) <= tube_dz)
        return (inbox | intube) if kind == "boolunion" else (inbox & intube)
    params = dict(box_half=box_half, tube_rmax=tube_rmax, tube_dz=tube_dz,
                  left_place=list(left_place), right_place=list(right_place))
    e = max(float(np.linalg.norm(box_half)) + float(np.linalg.norm(left_place[:3])),
            float(np.hypot(tube_rmax, tube_dz)) + float(np.linalg.norm(right_place[:3])))
    return ShapeSpec(kind, params, (e, e, e), contains=contains)


# ---------------------------------------------------------------------------
# point sets
# ---------------------------------------------------------------------------

def _rejection(spec: ShapeSpec, rng, n: int, want_inside: bool, scale: float):
    if n <= 0:
        e = np.zeros(0)
        return e, e.copy(), e.copy()
    xs, ys, zs = [], [], []
    got = 0
    while got < n:
        m = max(1024, 2 * (n - got))
        x, y, z = spec.bbox_sample(rng, m, scale)
        c = spec.contains(x, y, z)
        sel = c if want_inside else ~c
        xs.append(x[sel]); ys.append(y[sel]); zs.append(z[sel])
        got += int(sel.sum())
    return (np.concatenate(xs)[:n], np.concatenate(ys)[:n], np.concatenate(zs)[:n])


def _near_surface(spec: ShapeSpec, rng, n: int, eps: float = 1e-6):
    a = np.stack(_rejection(spec, rng, n, True, 1.0))
    b = np.stack(_rejection(spec, rng, n, False, 1.5))
    lo, hi = a.copy(), b.copy()            # contains(lo) True, contains(hi) False
    for _ in range(64):
        mid = 0.5 * (lo + hi)
        c = spec.contains(mid[0], mid[1], mid[2])
        lo = np.where(c, mid, lo)
        hi = np.where(c, hi, mid)
    d = b - a
    d /= np.sqrt((d * d).sum(axis=0))
    off = rng.uniform(-eps, eps, n)
    p = 0.5 * (lo + hi) + d * off
    return p[0].copy(), p[1].copy(), p[2].copy()


def mixed_points(spec: ShapeSpec, n: int, seed: int):
    """1/3 inside, 1/3 outside in the 1.5x box, 1/3 within 1e-6 mm of the surface,
    interleaved in a seeded random order."""
    rng = np.random.default_rng(seed)
    n1 = n // 3
    n2 = n // 3
    n3 = n - n1 - n2
    parts = [_rejection(spec, rng, n1, True, 1.0), _rejection(spec, rng, n2, False, 1.5),
             _near_surface(spec, rng, n3)]
    x = np.concatenate([p[0] for p in parts])
    y = np.concatenate([p[1] for p in parts])
    z = np.concatenate([p[2] for p in parts])
    perm = rng.permutation(n)
    return x[perm].copy(), y[perm].copy(), z[perm].copy()


def uniform_points(spec: ShapeSpec, n: int, seed: int, scale: float = 1.5):
    rng = np.random.default_rng(seed)
    return spec.bbox_sample(rng, n, scale)


@dataclass
class ShapeWorkload:
    spec: ShapeSpec
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    dx: np.ndarray
    dy: np.ndarray
    dz: np.ndarray
    step: np.ndarray

    @property
    def n(self) -> int:
        return len(self.x)


def make_workload(spec: ShapeSpec, n: int, seed: int, mix: str = "mixed",
                  step_max: float = 1e30) -> ShapeWorkload:
    if mix == "mixed":
        x, y, z = mixed_points(spec, n, seed)
    else:
        x, y, z = uniform_points(spec, n, seed)
    dx, dy, dz = isotropic(np.random.default_rng(seed + 7919), n)
    return ShapeWorkload(spec, x, y, z, dx, dy, dz, np.full(n, step_max))


def _bench_workload_arrays(job):
    config, shape, n, seed, mix = job
    wl = make_workload(bench_config(config)[0][shape], n, seed, mix=mix)
    return wl.x, wl.y, wl.z, wl.dx, wl.dy, wl.dz, wl.step


def bench_workloads(jobs: list, processes: int | None = None) -> list:
    """The workloads of (benchmark config, shape name, n, seed, mix) jobs,
    drawn in spawned worker processes (numpy sampling of a 2^22-point mix takes
    seconds per shape).  Spawned, never forked, so it is safe after CUDA has
    started in the caller; the arrays equal those of sequential make_workload
    calls."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    if len(jobs) <= 1:
        arrays = [_bench_workload_arrays(j) for j in jobs]
    else:
        workers = min(len(jobs), processes or (os.cpu_count() or 1))
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            arrays = list(ex.map(_bench_workload_arrays, jobs))
    return [ShapeWorkload(bench_config(j[0])[0][j[1]], *a) for j, a in zip(jobs, arrays)]


# ---------------------------------------------------------------------------
# the named benchmark shapes
# ---------------------------------------------------------------------------

def config1_box() -> ShapeSpec:
    """Plain FP64 box, half-lengths (10, 20, 30) mm, unrotated at the origin."""
    return box_spec(10., 20., 30.)


def config2_shapes() -> dict:
    """Tube, cone, sphere of the FP32+refine vs FP64 comparison."""
    return {
        "tube": tube_spec(5., 20., 30., 0., 1.5 * math.pi),
        "cone": cone_spec(0., 10., 5., 20., 25., 0., 2 * math.pi),
        "sphere": sphere_spec(10., 30., 0., 2 * math.pi, 0., 0.5 * math.pi),
    }


def config3_shapes(seed: int = SEED_BASE + 3) -> dict:
    """Torus, polycone, polyhedron and box-minus-tube (compute-heavy shapes).
    Polycone: 10 z-planes from -100 to 100 mm, rmin ~ U(0,20), rmax ~ U(30,60),
    phi 0-300 deg.  Polyhedron: 8 sides, 6 z-planes evenly spaced in [-100, 100],
    rmin 10, rmax 40."""
    rng = np.random.default_rng(seed)
    zc = np.linspace(-100., 100., 10)
    return {
        "torus": torus_spec(0., 5., 50., 0., 2 * math.pi),
        "polycone": polycone_spec(0., math.radians(300.), zc, rng.uniform(0., 20., 10),
                                  rng.uniform(30., 60., 10)),
        "polyhedron": polyhedron_spec(0., 360., 8, np.linspace(-100., 100., 6),
                                      np.full(6, 10.), np.full(6, 40.)),
        "boolsub": boolsub_spec((30., 30., 30.), 15., 40.),
    }


def bench_config(name: str):
    """(shapes, points per shape, point mix) of a benchmark workload: "box"
    (the box, 2^20 points uniform in 1.5x its box), "shapes" (tube, cone,
    sphere, 2^22 mixed points each) or "heavy" (torus, polycone, polyhedron,
    box minus tube, 2^22 mixed points each)."""
    if name == "box":
        return {"box": config1_box()}, 1 << 20, "uniform"
    if name == "heavy":
        return config3_shapes(), 1 << 22, "mixed"
    if name == "shapes":
        return config2_shapes(), 1 << 22, "mixed"
    raise ValueError(name)


def bench_seed(shape_index: int, rank: int = 0) -> int:
    """Seed of the points of the shape_index-th shape of a benchmark workload
    on one rank (every rank draws its own batch)."""
    return SEED_BASE + 1000 * rank + shape_index


def build_unplaced(geom, spec: ShapeSpec) -> int:
    """Create spec's unplaced shape in a vecgeom_b200.Geometry; returns its id."""
    p = spec.params
    k = spec.kind
    if k == "box":
        return geom.UnplacedBox(p["dx"], p["dy"], p["dz"])
    if k == "tube":
        return geom.UnplacedTube(p["rmin"], p["rmax"], p["dz"], p["sphi"], p["dphi"])
    if k == "cone":
        return geom.UnplacedCone(p["rmin1"], p["rmax1"], p["rmin2"], p["rmax2"], p["dz"],
                                 p["sphi"], p["dphi"])
    if k == "sphere":
        return geom.UnplacedSphere(p["rmin"], p["rmax"], p["sphi"], p["dphi"], p["stheta"],
                                   p["dtheta"])
    if k == "torus":
        return geom.UnplacedTorus(p["rmin"], p["rmax"], p["rtor"], p["sphi"], p["dphi"])
    if k == "trd":
        return geom.UnplacedTrd(p["dx1"], p["dx2"], p["dy1"], p["dy2"], p["dz"])
    if k == "orb":
        return geom.UnplacedOrb(p["r"])
    if k == "paraboloid":
        return geom.UnplacedParaboloid(p["rlo"], p["rhi"], p["dz"])
    if k == "trapezoid":
        return geom.UnplacedTrapezoid(p["dz"], p["theta"], p["phi"], p["dy1"], p["dx1"], p["dx2"],
                                      p["tan_alpha1"], p["dy2"], p["dx3"], p["dx4"],
                                      p["tan_alpha2"])
    if k == "trapezoidcorners":
        return geom.UnplacedTrapezoidFromCorners(p["corners"])
    if k == "parallelepiped":
        return geom.UnplacedParallelepiped(p["x"], p["y"], p["z"], p["alpha"], p["theta"],
                                           p["phi"])
    if k == "polycone":
        return geom.UnplacedPolycone(p["sphi"], p["dphi"], p["rmin"], p["rmax"], p["z"])
    if k == "polyhedron":
        return geom.UnplacedPolyhedron(p["phi_start_deg"], p["phi_delta_deg"], p["sides"],
                                       p["z"], p["rmin"], p["rmax"])
    if k in BOOL_OPS:
        bx, by, bz = p["box_half"]
        lb = geom.LogicalVolume("sub_box", geom.UnplacedBox(bx, by, bz))
        lt = geom.LogicalVolume("sub_tube", geom.UnplacedTube(0., p["tube_rmax"], p["tube_dz"],
                                                              0., 2 * math.pi))
        left = lb.Place(geom.Transformation3D(*p.get("left_place", IDENTITY_PLACE)))
        right = lt.Place(geom.Transformation3D(*p.get("right_place", IDENTITY_PLACE)))
        return geom.UnplacedBooleanVolume(BOOL_OPS[k], left, right)
    raise ValueError(k)


# ---------------------------------------------------------------------------
# Layered cylindrical detector of the navigation benchmark
# ---------------------------------------------------------------------------
@dataclass
class DetectorSpec:
    """World box (half 2000 mm) with 10 concentric tube layers (inner radius
    100 + 100 k mm, 20 mm thick, dz 1200 mm).  Layer k holds 64 + 48 k box
    modules of half-lengths (10, 40, 600) mm at radius r_k + 10, each rotated
    about z to face the axis (Euler phi = 360 j / N_k degrees).  Every module
    holds 4 Trd sensors (dx 8 -> 6, dy 30 -> 25, dz 140 mm) at z = -450, -150,
    150, 450 mm.  Every module has its own logical volume (all share one
    unplaced box), so 1 + 10 + 2800 + 11200 = 14011 placed volumes, 4 levels.
    (The modules overlap their neighbours and stick out of their layer at the
    corners; navigation stays deterministic under the reference's rules.)"""
    world_half: float = 2000.
    n_layers: int = 10
    r0: float = 100.
    dr: float = 100.
    thickness: float = 20.
    layer_dz: float = 1200.
    module_half: tuple = (10., 40., 600.)
    modules0: int = 64
    modules_step: int = 48
    sensor_trd: tuple = (8., 6., 30., 25., 140.)
    sensor_z: tuple = (-450., -150., 150., 450.)

    def modules_in_layer(self, k: int) -> int:
        return self.modules0 + self.modules_step * k

    def placed_count(self) -> int:
        nm = sum(self.modules_in_layer(k) for k in range(self.n_layers))
        return 1 + self.n_layers + nm + nm * len(self.sensor_z)


class VgbBuilder:
    """Detector-builder adapter over this library's Geometry (close=False leaves
    the geometry open, for host-only use of its tables)."""

    def __init__(self, geom, close: bool = True):
        self.g = geom
        self._close = close

    def box(self, dx, dy, dz):
        return self.g.UnplacedBox(dx, dy, dz)

    def tube(self, rmin, rmax, dz, sphi, dphi):
        return self.g.UnplacedTube(rmin, rmax, dz, sphi, dphi)

    def trd(self, dx1, dx2, dy1, dy2, dz):
        return self.g.UnplacedTrd(dx1, dx2, dy1, dy2, dz)

    def shape(self, spec: ShapeSpec):
        return build_unplaced(self.g, spec)

    def transform(self, tx=0., ty=0., tz=0., phi=0., theta=0., psi=0.):
        return self.g.Transformation3D(tx, ty, tz, phi, theta, psi)

    def logical(self, label, unplaced):
        return self.g.LogicalVolume(label, unplaced)

    def place(self, logical, transform):
        return logical.Place(transform)

    def place_daughter(self, mother, daughter, transform):
        return mother.PlaceDaughter(daughter, transform)

    def set_world(self, placed):
        self.g.SetWorld(placed)

    def close(self):
        if self._close:
            self.g.CloseGeometry()


def build_detector(b, spec: DetectorSpec | None = None) -> list:
    """Builds the detector through a builder adapter (this library's or the
    reference's) in one fixed order; returns the placed volumes in creation
    order, which is also the order of their ids."""
    spec = spec or DetectorSpec()
    placed = []
    world_lv = b.logical("world", b.box(spec.world_half, spec.world_half, spec.world_half))
    world = b.place(world_lv, b.transform())
    placed.append(world)
    module_box = b.box(*spec.module_half)
    sensor_lv = b.logical("sensor", b.trd(*spec.sensor_trd))
    sensor_t = [b.transform(0., 0., z) for z in spec.sensor_z]
    for k in range(spec.n_layers):
        rin = spec.r0 + spec.dr * k
        layer_lv = b.logical(f"layer{k}", b.tube(rin, rin + spec.thickness, spec.layer_dz, 0.,
                                                 2 * math.pi))
        nk = spec.modules_in_layer(k)
        rc = rin + 0.5 * spec.thickness
        for j in range(nk):
            module_lv = b.logical(f"module{k}_{j}", module_box)
            for t in sensor_t:
                placed.append(b.place_daughter(module_lv, sensor_lv, t))
            phi = 360. * j / nk
            a = math.radians(phi)
            placed.append(b.place_daughter(layer_lv, module_lv,
                                           b.transform(rc * math.cos(a), rc * math.sin(a), 0.,
                                                       phi, 0., 0.)))
        placed.append(b.place_daughter(world_lv, layer_lv, b.transform()))
    b.set_world(world)
    b.close()
    return placed


def zoo_specs(exclude=()) -> list:
    """The shapes of the mixed navigation geometry: the box, tube/cone/sphere,
    torus/polycone/polyhedron/box-tube workloads and a trd, less the kinds in
    `exclude`."""
    specs = ([config1_box()] + list(config2_shapes().values()) + list(config3_shapes().values())
             + [trd_spec(20., 10., 25., 15., 30.)])
    return [s for s in specs if s.kind not in exclude]


def zoo2_specs(exclude=()) -> list:
    """The second mixed navigation geometry's shapes: orb, parallelepiped,
    paraboloid, two trapezoids (one from corners), a box-tube union and a
    box-tube intersection, less the kinds in `exclude` (every one reaches less
    than 135 mm from its centre)."""
    specs = [orb_spec(25.), parallelepiped_spec(20., 30., 40., 30., 20., 40.),
             paraboloid_spec(10., 30., 40.),
             trapezoid_spec(40., 0.3, 0.7, 20., 10., 15., 0.2, 30., 20., 27.5, 0.2),
             trapezoid_corners_spec([(-10., -20., -40.), (10., -20., -40.), (-10., 20., -40.),
                                     (10., 20., -40.), (-30., -40., 40.), (30., -40., 40.),
                                     (-30., 40., 40.), (30., 40., 40.)]),
             boolean_spec("boolunion", (20., 20., 20.), 12., 35.,
                          right_place=(8., 0., 0., 0., 0., 0.)),
             boolean_spec("boolinter", (25., 20., 15.), 18., 40.,
                          left_place=(2., -1., 3., 0., 0., 15.),
                          right_place=(0., 2., 0., 0., 90., 30.))]
    return [s for s in specs if s.kind not in exclude]


def build_zoo(b, specs: list, seed: int = SEED_BASE + 9) -> list:
    """Mixed-shape navigation geometry: a world box (half 1000 mm) with a 3x3x3
    grid of cells 600 mm apart.  Cell c holds specs[c % len(specs)] placed with
    a random Euler rotation (degrees) and an offset of up to 20 mm; every third
    cell instead holds a box container (half 160 mm, its own rotation) with the
    shape inside it (offset up to 5 mm) and a small trd in a corner, so paths
    are up to three levels deep.  Every shape reaches less than 135 mm from its
    centre, so nothing overlaps.  Returns the placed volumes in creation (= id)
    order."""
    rng = np.random.default_rng(seed)
    placed = []
    world_lv = b.logical("world", b.box(1000., 1000., 1000.))
    world = b.place(world_lv, b.transform())
    placed.append(world)
    lvs = [b.logical(f"zoo{k}", b.shape(sp)) for k, sp in enumerate(specs)]
    small_lv = b.logical("zoo_trd", b.trd(6., 4., 8., 5., 10.))
    box_u = b.box(160., 160., 160.)

    def rot():
        return tuple(float(a) for a in rng.uniform(0., 360., 3))

    c = 0
    for i in (-600., 0., 600.):
        for j in (-600., 0., 600.):
            for k in (-600., 0., 600.):
                off = rng.uniform(-20., 20., 3)
                lv = lvs[c % len(lvs)]
                if c % 3 == 2:
                    cont = b.logical(f"cont{c}", box_u)
                    placed.append(b.place_daughter(cont, lv, b.transform(*(off / 4.), *rot())))
                    placed.append(b.place_daughter(cont, small_lv,
                                                   b.transform(140., 140., -140., *rot())))
                    placed.append(b.place_daughter(world_lv, cont,
                                                   b.transform(i, j, k, *rot())))
                else:
                    placed.append(b.place_daughter(world_lv, lv,
                                                   b.transform(i + off[0], j + off[1], k + off[2],
                                                               *rot())))
                c += 1
    b.set_world(world)
    b.close()
    return placed


def zoo_tracks(n: int, seed: int):
    """n tracks: a third from near the cell centres (inside or near the shapes),
    the rest from uniform points of the world's inner 900 mm; isotropic
    directions."""
    rng = np.random.default_rng(seed)
    n0 = n // 3
    cells = np.array([(i, j, k) for i in (-600., 0., 600.) for j in (-600., 0., 600.)
                      for k in (-600., 0., 600.)])
    pick = cells[rng.integers(0, len(cells), n0)] + rng.uniform(-30., 30., (n0, 3))
    rest = rng.uniform(-900., 900., (n - n0, 3))
    p = np.concatenate([pick, rest])
    d = isotropic(rng, n)
    return tuple(np.ascontiguousarray(p[:, a]) for a in range(3)), d


def isotropic_tracks(n: int, seed: int):
    """n tracks from the origin with isotropic unit directions (normalised 3-D
    Gaussians)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(3, n))
    v /= np.linalg.norm(v, axis=0)
    z = np.zeros(n)
    return (z.copy(), z.copy(), z.copy()), (v[0].copy(), v[1].copy(), v[2].copy())


# ---------------------------------------------------------------------------
# Mixed baskets: many jittered shape instances with their own point batches
# ---------------------------------------------------------------------------
BASKET_KINDS = ("box", "tube", "cone", "sphere", "torus", "polycone", "polyhedron", "boolsub")


def basket_base_specs() -> dict:
    """The eight benchmark shapes the baskets draw from (box, tube/cone/sphere,
    torus/polycone/polyhedron/boolean subtraction)."""
    return {"box": config1_box(), **config2_shapes(), **config3_shapes()}


def jitter_spec(spec: ShapeSpec, rng) -> ShapeSpec:
    """The shape with its lengths scaled by independent factors U(0.8, 1.2)
    (angles and plane counts unchanged; radius ordering kept)."""
    u = lambda: float(rng.uniform(0.8, 1.2))  # noqa: E731
    p = spec.params
    k = spec.kind
    if k == "box":
        return box_spec(p["dx"] * u(), p["dy"] * u(), p["dz"] * u())
    if k == "tube":
        return tube_spec(p["rmin"] * u(), p["rmax"] * u(), p["dz"] * u(), p["sphi"], p["dphi"])
    if k == "cone":
        return cone_spec(p["rmin1"] * u(), p["rmax1"] * u(), p["rmin2"] * u(), p["rmax2"] * u(),
                         p["dz"] * u(), p["sphi"], p["dphi"])
    if k == "sphere":
        return sphere_spec(p["rmin"] * u(), p["rmax"] * u(), p["sphi"], p["dphi"], p["stheta"],
                           p["dtheta"])
    if k == "torus":
        return torus_spec(p["rmin"] * u(), p["rmax"] * u(), p["rtor"] * u(), p["sphi"], p["dphi"])
    if k == "polycone":
        z = np.asarray(p["z"]) * u()
        rmin = np.asarray(p["rmin"]) * u()
        rmax = np.maximum(np.asarray(p["rmax"]) * u(), rmin + 1.)
        return polycone_spec(p["sphi"], p["dphi"], z, rmin, rmax)
    if k == "polyhedron":
        z = np.asarray(p["z"]) * u()
        return polyhedron_spec(p["phi_start_deg"], p["phi_delta_deg"], p["sides"], z,
                               np.asarray(p["rmin"]) * u(), np.asarray(p["rmax"]) * u())
    if k == "boolsub":
        bx, by, bz = p["box_half"]
        return boolsub_spec((bx * u(), by * u(), bz * u()), p["tube_rmax"] * u(),
                            p["tube_dz"] * u())
    raise ValueError(k)


@dataclass
class Basket:
    spec: ShapeSpec
    place: tuple          # (tx, ty, tz, phi, theta, psi), degrees
    n: int
    seed: int


def config4_baskets(n_baskets: int = 4096, seed: int = SEED_BASE + 4, median: int = 1024,
                    sigma: float = 1.0, lo: int = 16, hi: int = 65536) -> list:
    """Baskets of the mixed workload: sizes clip(round(lognormal(ln median,
    sigma)), lo, hi) (sigma is our choice; only the median is given), shape kind
    uniform over the eight kinds, lengths jittered +-20%, Euler angles U(0, 360)
    degrees, translation U(-100, 100) mm."""
    rng = np.random.default_rng(seed)
    base = basket_base_specs()
    sizes = np.clip(np.round(rng.lognormal(math.log(median), sigma, n_baskets)), lo, hi)
    kinds = rng.integers(0, len(BASKET_KINDS), n_baskets)
    out = []
    for b in range(n_baskets):
        spec = jitter_spec(base[BASKET_KINDS[kinds[b]]], rng)
        t = rng.uniform(-100., 100., 3)
        a = rng.uniform(0., 360., 3)
        out.append(Basket(spec, (float(t[0]), float(t[1]), float(t[2]), float(a[0]),
                                 float(a[1]), float(a[2])), int(sizes[b]), seed + 17 * (b + 1)))
    return out


def basket_points(b: Basket):
    """The basket's points (mixed in the shape's frame, then moved to the
    mother frame of its placement), isotropic directions and step_max."""
    wl = make_workload(b.spec, b.n, b.seed)
    R = euler_rotation(*b.place[3:])
    loc = np.stack([wl.x, wl.y, wl.z])
    mst = R @ loc + np.asarray(b.place[:3])[:, None]
    d = R @ np.stack([wl.dx, wl.dy, wl.dz])
    return (mst[0], mst[1], mst[2]), (d[0], d[1], d[2]), wl.step


def build_baskets(geom, baskets: list):
    """Places every basket's shape instance in `geom` (one logical volume each)
    and concatenates the baskets' points.  Returns (placed volumes, offsets,
    (x, y, z), (dx, dy, dz), step_max)."""
    placed, offsets = [], []
    xs, ds, steps = [], [], []
    off = 0
    for k, b in enumerate(baskets):
        lv = geom.LogicalVolume(f"basket{k}", build_unplaced(geom, b.spec))
        placed.append(lv.Place(geom.Transformation3D(*b.place)))
        p, d, s = basket_points(b)
        xs.append(p)
        ds.append(d)
        steps.append(s)
        offsets.append(off)
        off += b.n
    cat = lambda parts, j: np.ascontiguousarray(np.concatenate([q[j] for q in parts]))  # noqa: E731
    pts = tuple(cat(xs, j) for j in range(3))
    dirs = tuple(cat(ds, j) for j in range(3))
    return placed, offsets, pts, dirs, np.ascontiguousarray(np.concatenate(steps))
