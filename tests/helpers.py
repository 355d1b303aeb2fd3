"""Shared test helpers: build the same shape in libvgb, the C oracle and the
reference (oracle/_ref), and compare results with the parity bar.

Parity bar (the FP64 form against the reference Scalar backend):
  * Contains / Inside / node indices: bit-exact;
  * distances and safeties: |a-b| <= 1e-9 mm or |a-b| <= 1e-12 |b|; both
    infinite with the same sign, or both NaN, also match.
"""
from __future__ import annotations

import math

import numpy as np

ABS_TOL = 1e-9
REL_TOL = 1e-12

# placements exercised by the parity tests: (tx, ty, tz, phi, theta, psi), degrees
PLACEMENTS = {
    "identity": (0., 0., 0., 0., 0., 0.),
    "translated": (5., -3., 7., 0., 0., 0.),
    "rotz90": (1., 2., 3., 90., 0., 0.),     # drops the 6e-17 entries (code 0x10a-like)
    "generic": (-4., 6., 2.5, 30., 45., 60.),
}


def distances_match(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    same_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    finite = np.isfinite(a) & np.isfinite(b)
    with np.errstate(invalid="ignore"):
        d = np.abs(a - b)
        ok = finite & ((d <= ABS_TOL) | (d <= REL_TOL * np.abs(b)))
    return ok | both_nan | same_inf


def assert_distances(a, b, what: str = "") -> None:
    ok = distances_match(a, b)
    if not ok.all():
        i = np.flatnonzero(~ok)[:8]
        raise AssertionError(f"{what}: {int((~ok).sum())} of {len(ok)} differ; first {i.tolist()}: "
                             f"got {np.asarray(a)[i].tolist()} want {np.asarray(b)[i].tolist()}")


def assert_exact(a, b, what: str = "") -> None:
    a = np.asarray(a)
    b = np.asarray(b)
    ok = a == b
    if not ok.all():
        i = np.flatnonzero(~ok)[:8]
        raise AssertionError(f"{what}: {int((~ok).sum())} of {len(ok)} differ; first {i.tolist()}: "
                             f"got {a[i].tolist()} want {b[i].tolist()}")


# ---------------------------------------------------------------------------
# building one ShapeSpec in each implementation
# ---------------------------------------------------------------------------
from oracle import oracle_generic_xform, oracle_unplaced, ref_unplaced  # noqa: E402,F401
from vecgeom_b200.workloads import build_unplaced as vgb_unplaced  # noqa: E402,F401


def shape_specs() -> dict:
    """The shapes of the parity tests: the benchmark shapes plus a trd."""
    from vecgeom_b200 import workloads as W
    s = {"box": W.box_spec(10., 20., 30.)}
    s.update(W.config2_shapes())
    s.update(W.config3_shapes())
    s["trd"] = W.trd_spec(10., 20., 15., 25., 30.)
    # variants that reach the phi-section and rmin branches
    s["tubesector"] = W.tube_spec(0., 20., 30., 0.3, 1.0)
    s["conesector"] = W.cone_spec(2., 10., 5., 20., 25., 0.5, 4.0)
    s["conesmall"] = W.cone_spec(0., 10., 0., 20., 25., -0.5, 1.2)
    s["spheresector"] = W.sphere_spec(5., 30., 0.3, 4.0, 0.4, 1.9)
    s["spherefull"] = W.sphere_spec(0., 25., 0., 2 * math.pi, 0., math.pi)
    s["trd1"] = W.trd_spec(10., 20., 15., 15., 30.)
    s["torussector"] = W.torus_spec(2., 6., 40., 0.4, 4.5)
    s["polyhedroncut"] = W.polyhedron_spec(30., 270., 6, [-40., -10., 20., 45.],
                                           [0., 8., 12., 5.], [25., 30., 35., 28.])
    s["polyhedronlarge"] = W.polyhedron_spec(-20., 120., 3, [-30., 30.], [5., 10.], [20., 30.])
    s["polyconefull"] = W.polycone_spec(0., 2 * math.pi, [-50., -20., -20., 10., 40.],
                                        [0., 5., 8., 0., 12.], [20., 25., 30., 18., 30.])
    return s
