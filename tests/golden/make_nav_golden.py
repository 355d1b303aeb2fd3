"""Write the navigation fixtures of tests/golden/nav/ from the reference itself.

Builds a geometry in the reference (oracle/_ref/libvgref.so, built from the
reference sources by ``make -C oracle ref``) with the same builder code this
library's tests use (vecgeom_b200.workloads) and traces tracks with the
reference's navigators: LocatePoint, then GetSafety + FindNextBoundaryAndStep
per step (oracle/ref_driver.cpp vgref_nav_trace / vgref_abbox_nav_trace).

    detector.npz        layered detector, SimpleNavigator
    detector_abbox.npz  layered detector, ABBoxNavigator
    zoo.npz             mixed-shape geometry without the sphere and the torus,
                        SimpleNavigator
    zoo_abbox.npz       the same without the polyhedron too, ABBoxNavigator
    basket.npz          layered detector, SimpleNavigator's basket step and
                        GetSafeties after 0-3 single steps
    row_abbox.npz       300 boxes on a line, ABBoxNavigator (hit lists longer
                        than the GPU kernel's shared list)
    zoo_boxes.npz       ABBoxManager::ComputeABBox of every placed volume of the
                        mixed-shape geometry with all nine shapes

Next-volume ids are positions in the list the geometry builder returns
(for the detector that is also this library's placed-volume id).

Why shapes are left out: the reference's SphereImplementation::DistanceToIn is
a stub that returns kInfinity (volumes/kernel/SphereImplementation.h:84-93), so
its navigators never enter a sphere, while this library runs USolids'
USphere::DistanceToIn there; and the reference's polyhedron Contains reads past
its z-segment array for points within kTolerance above the last z-plane
(volumes/kernel/PolyhedronImplementation.h:745-780, FindZSegment returns the
segment count), which ABBoxNavigator's Contains check of a box the point is in
reaches when a track leaves a polyhedron through that plane.

Every geometry is built in a fresh process: the reference keeps one world.

    python tests/golden/make_nav_golden.py [fixture names]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from vecgeom_b200 import workloads as W  # noqa: E402

N_ORIGIN = 256
N_RANDOM = 256
N_ZOO = 384
MAX_STEPS = 64
PSTEP = 1e30
SEED = W.SEED_BASE + 5

# the fixtures leave the torus out too: its GPU distances can differ from the
# reference in the last bits (CUDA's and glibc's transcendentals), which a
# trace would carry on; the CPU tests cover it against the live reference
ZOO_EXCLUDE = {"zoo": ("sphere", "torus"), "zoo_abbox": ("sphere", "torus", "polyhedron"),
               "zoo_torus": ("sphere",), "zoo_abbox_torus": ("sphere", "polyhedron"),
               "zoo_all": ()}
# the second zoo (orb, parallelepiped, paraboloid, trapezoids, union,
# intersection); ABBoxNavigator needs every shape's Extent, which the
# reference's parallelepiped lacks
ZOO2_EXCLUDE = {"zoo2": (), "zoo2_abbox": ("parallelepiped",)}


def nav_inputs():
    """Tracks from the origin, then tracks from random points in the detector."""
    (x0, y0, z0), (dx0, dy0, dz0) = W.isotropic_tracks(N_ORIGIN, SEED)
    rng = np.random.default_rng(SEED + 1)
    x1 = rng.uniform(-1100., 1100., N_RANDOM)
    y1 = rng.uniform(-1100., 1100., N_RANDOM)
    z1 = rng.uniform(-1300., 1300., N_RANDOM)
    _, (dx1, dy1, dz1) = W.isotropic_tracks(N_RANDOM, SEED + 2)
    cat = lambda a, b: np.ascontiguousarray(np.concatenate([a, b]))  # noqa: E731
    return (cat(x0, x1), cat(y0, y1), cat(z0, z1)), (cat(dx0, dx1), cat(dy0, dy1), cat(dz0, dz1))


def zoo_inputs():
    return W.zoo_tracks(N_ZOO, SEED + 3)


def build_row(b, n: int = 300, pitch: float = 8.) -> list:
    """A world box (half 2000 mm, or more for long rows) with n small boxes
    (half 2 mm) on the x axis, `pitch` mm apart from x = -1200 mm: a ray along
    x has every one of them in its hit list."""
    last = -1200. + pitch * (n - 1) + 2.
    half = 2000. if last < 1900. else last + 100.
    world_lv = b.logical("world", b.box(half, 2000., 2000.))
    world = b.place(world_lv, b.transform())
    placed = [world]
    cell = b.logical("cell", b.box(2., 2., 2.))
    for i in range(n):
        placed.append(b.place_daughter(world_lv, cell, b.transform(-1200. + pitch * i, 0., 0.)))
    b.set_world(world)
    b.close()
    return placed


def row_inputs(n: int = 128):
    """Tracks from x = -1900 mm towards +x, within 1 mm of the axis and 1e-3 rad."""
    rng = np.random.default_rng(SEED + 4)
    x = np.full(n, -1900.)
    y, z = rng.uniform(-1., 1., n), rng.uniform(-1., 1., n)
    d = np.stack([np.ones(n), rng.uniform(-1e-3, 1e-3, n), rng.uniform(-1e-3, 1e-3, n)])
    d /= np.sqrt((d * d).sum(axis=0))
    return (x, y, z), (d[0].copy(), d[1].copy(), d[2].copy())


def build_geometry(b, geometry: str) -> list:
    """The named geometry through a builder adapter; the placed volumes in
    creation order."""
    if geometry == "detector":
        return W.build_detector(b)
    if geometry == "row":
        return build_row(b)
    if geometry == "row_long":
        return build_row(b, 6500, 5.)
    if geometry in ZOO2_EXCLUDE:
        return W.build_zoo(b, W.zoo2_specs(exclude=ZOO2_EXCLUDE[geometry]))
    return W.build_zoo(b, W.zoo_specs(exclude=ZOO_EXCLUDE[geometry]))


def reference_trace(ref, pts, dirs, max_steps=MAX_STEPS, nthreads=1, geometry="detector",
                    navigator="simple"):
    """Builds the geometry in the reference and traces; ids mapped to list
    positions.  ABBoxNavigator traces run on one thread (the reference's
    ABBoxManager shares one hit list)."""
    rb = oracle.RefBuilder(ref)
    placed = build_geometry(rb, geometry)
    to_ours = {int(r): k for k, r in enumerate(rb.ids(placed))}
    if navigator == "simple":
        ids, steps, saf, nst = oracle.ref_nav_trace(ref, pts, dirs, PSTEP, max_steps, nthreads)
    else:
        ids, steps, saf, nst = oracle.ref_abbox_nav_trace(ref, pts, dirs, PSTEP, max_steps)
    mapped = np.array([to_ours[int(i)] if i >= 0 else int(i) for i in ids], np.int32)
    return mapped, steps, saf, nst


def reference_boxes(ref, geometry: str) -> np.ndarray:
    """ABBoxManager::ComputeABBox of every placed volume, in list order."""
    rb = oracle.RefBuilder(ref)
    placed = build_geometry(rb, geometry)
    return np.array([oracle.ref_abbox(ref, p) for p in placed])


def basket_inputs(n: int = 512):
    """Points spread over the detector with isotropic directions; half the
    tracks propose a physical step U(0, 50) mm, the rest 1e30."""
    rng = np.random.default_rng(SEED + 6)
    pts = (rng.uniform(-1100., 1100., n), rng.uniform(-1100., 1100., n),
           rng.uniform(-1300., 1300., n))
    _, dirs = W.isotropic_tracks(n, SEED + 7)
    pstep = np.where(np.arange(n) % 2 == 0, rng.uniform(0., 50., n), 1e30)
    return pts, dirs, pstep


BASKET_PRIORS = (0, 1, 2, 3)


def reference_basket(ref, pts, dirs, pstep, priors=BASKET_PRIORS, geometry="detector"):
    """The reference's basket step after each number of prior steps; new top
    ids mapped to list positions."""
    rb = oracle.RefBuilder(ref)
    placed = build_geometry(rb, geometry)
    to_ours = {int(r): k for k, r in enumerate(rb.ids(placed))}
    out = {}
    for prior in priors:
        r = oracle.ref_nav_basket_step(ref, pts, dirs, pstep, prior)
        r["newtop"] = np.array([to_ours[int(i)] if i >= 0 else int(i) for i in r["newtop"]],
                               np.int32)
        for k, v in r.items():
            out[f"{k}_{prior}"] = v
    return out


def _basket(pts, dirs, pstep, priors, geometry):
    return reference_basket(oracle.RefLib(), pts, dirs, pstep, priors, geometry)


def reference_basket_isolated(pts, dirs, pstep, priors=BASKET_PRIORS, geometry="detector"):
    return isolated(_basket, pts, dirs, pstep, priors, geometry)


def _traced(pts, dirs, max_steps, nthreads, geometry, navigator, crlibm=False):
    return reference_trace(oracle.RefLib(crlibm=crlibm), pts, dirs, max_steps, nthreads, geometry,
                           navigator)


def _boxes(geometry):
    return reference_boxes(oracle.RefLib(), geometry)


def isolated(fn, *args):
    """fn(*args) in a fresh spawned process (a new reference world)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    with ProcessPoolExecutor(max_workers=1, mp_context=mp.get_context("spawn")) as ex:
        return ex.submit(fn, *args).result()


def reference_trace_isolated(pts, dirs, max_steps=MAX_STEPS, nthreads=1, geometry="detector",
                             navigator="simple", crlibm=False):
    """The trace in a fresh process; crlibm=True traces with the reference build
    whose torus takes correctly rounded atan2/sin/cos/cbrt."""
    return isolated(_traced, pts, dirs, max_steps, nthreads, geometry, navigator, crlibm)


def reference_boxes_isolated(geometry: str) -> np.ndarray:
    return isolated(_boxes, geometry)


TRACE_FIXTURES = (("detector", "detector", "simple", nav_inputs),
                  ("detector_abbox", "detector", "abbox", nav_inputs),
                  ("zoo", "zoo", "simple", zoo_inputs),
                  ("zoo_abbox", "zoo_abbox", "abbox", zoo_inputs),
                  ("row_abbox", "row", "abbox", row_inputs),
                  ("zoo2", "zoo2", "simple", zoo_inputs),
                  ("zoo2_abbox", "zoo2_abbox", "abbox", zoo_inputs))


def main(names=()) -> None:
    """Writes the fixtures named (all without names)."""
    out = os.path.join(HERE, "nav")
    for name, geometry, navigator, inputs in TRACE_FIXTURES:
        if names and name not in names:
            continue
        pts, dirs = inputs()
        ids, steps, saf, nst = reference_trace_isolated(pts, dirs, MAX_STEPS, 1, geometry,
                                                        navigator)
        path = os.path.join(out, name + ".npz")
        np.savez_compressed(path, x=pts[0], y=pts[1], z=pts[2], dx=dirs[0], dy=dirs[1],
                            dz=dirs[2], max_steps=MAX_STEPS, pstep=PSTEP, next_ids=ids,
                            steps=steps, safeties=saf, nsteps=nst, geometry=geometry,
                            navigator=navigator)
        print("wrote", os.path.relpath(path, ROOT), "mean steps", float(nst.mean()))
    if names and "basket" not in names:
        return
    pts, dirs, pstep = basket_inputs()
    rec = reference_basket_isolated(pts, dirs, pstep)
    path = os.path.join(out, "basket.npz")
    np.savez_compressed(path, x=pts[0], y=pts[1], z=pts[2], dx=dirs[0], dy=dirs[1], dz=dirs[2],
                        pstep=pstep, priors=np.array(BASKET_PRIORS), **rec)
    print("wrote", os.path.relpath(path, ROOT))
    boxes = reference_boxes_isolated("zoo_all")
    path = os.path.join(out, "zoo_boxes.npz")
    np.savez_compressed(path, boxes=boxes)
    print("wrote", os.path.relpath(path, ROOT), boxes.shape)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
