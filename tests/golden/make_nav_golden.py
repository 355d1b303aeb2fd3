"""Write tests/golden/nav/detector.npz from the reference itself.

Builds the layered detector (vecgeom_b200.workloads.build_detector) in the
reference (oracle/_ref/libvgref.so, built from the reference sources by
``make -C oracle ref``) and traces tracks with its SimpleNavigator
(LocatePoint, then GetSafety + FindNextBoundaryAndStep per step; see
oracle/ref_driver.cpp vgref_nav_trace).  Next-volume ids are stored in this
library's numbering (creation order of the placed volumes).

    python tests/golden/make_nav_golden.py
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
MAX_STEPS = 64
PSTEP = 1e30
SEED = W.SEED_BASE + 5


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


def reference_trace(ref, pts, dirs, max_steps=MAX_STEPS, nthreads=1):
    """Builds the detector in the reference and traces; ids mapped to ours."""
    rb = oracle.RefBuilder(ref)
    placed = W.build_detector(rb)
    to_ours = {int(r): k for k, r in enumerate(rb.ids(placed))}
    ids, steps, saf, nst = oracle.ref_nav_trace(ref, pts, dirs, PSTEP, max_steps, nthreads)
    mapped = np.array([to_ours[int(i)] if i >= 0 else int(i) for i in ids], np.int32)
    return mapped, steps, saf, nst


def main() -> None:
    ref = oracle.RefLib()
    pts, dirs = nav_inputs()
    ids, steps, saf, nst = reference_trace(ref, pts, dirs)
    path = os.path.join(HERE, "nav", "detector.npz")
    np.savez_compressed(path, x=pts[0], y=pts[1], z=pts[2], dx=dirs[0], dy=dirs[1], dz=dirs[2],
                        max_steps=MAX_STEPS, pstep=PSTEP, next_ids=ids, steps=steps,
                        safeties=saf, nsteps=nst)
    print("wrote", os.path.relpath(path, ROOT), "mean steps", float(nst.mean()))


if __name__ == "__main__":
    main()
