"""Shared test helpers: build the same shape in libvgb, the C oracle and the
reference (oracle/_ref), and compare results with the parity bar.

Parity bar (the FP64 form against the reference Scalar backend):
  * Contains / Inside / node indices: bit-exact;
  * distances and safeties: |a-b| <= 1e-9 mm or |a-b| <= 1e-12 |b|; both
    infinite with the same sign, or both NaN, also match.

Torus distances are held to the same bar against the reference built with
correctly rounded atan2/sin/cos/cbrt (oracle/_ref/libvgref_crlibm.so).  The
reference solves the torus quartic with complex cube roots built from those C
library functions (volumes/kernel/TorusImplementation.h:283-316) and its
unpolished roots move with their last bits: on a few rays per hundred its own
DistanceToIn changes by up to ~3e-7 mm between glibc (whose cbrt is not
correctly rounded) and a correctly rounding library.  libvgb evaluates those
functions correctly rounded on the host and the GPU (crmath.cuh), so it matches
the correctly rounded build; against the glibc build it differs exactly on the
rays where the two reference builds differ from each other.
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
    # nonzero entries r1, r3, r5, r6, r8 only: rotation code 0x16A, whose
    # specialised transform carries the reference's typo (third row
    # m2*R5 + m2*R8, base/Transformation3D.h:388-392)
    "quirk16a": (2., -1., 3., 0., 30., 90.),
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


def assert_torus_distances(got, want_crlibm, want_glibc=None, what: str = "") -> dict:
    """The torus bar (module docstring): the parity bar against the reference
    built with correctly rounded functions; returns the number of rays on which
    the two reference builds themselves differ beyond the bar (where the glibc
    build's value depends on its library's rounding)."""
    assert_distances(got, want_crlibm, f"{what} (vs the reference with correctly rounded libm)")
    stats = {"n": len(np.asarray(got))}
    if want_glibc is not None:
        stats["libm_dependent"] = int((~distances_match(want_glibc, want_crlibm)).sum())
        stats["differ_from_glibc_build"] = int((~distances_match(got, want_glibc)).sum())
    return stats


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
from oracle import (oracle_generic_xform, oracle_unplaced, ref_unplaced,  # noqa: E402,F401
                    reference_defined)
from vecgeom_b200.workloads import build_unplaced as vgb_unplaced  # noqa: E402,F401


def shape_specs() -> dict:
    """The shapes of the parity tests: the benchmark shapes plus a trd, an orb
    and parallelepipeds."""
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
    # components with their own placements (the right one with 6e-17 entries the
    # specialised transform drops and the generic one keeps)
    s["orb"] = W.orb_spec(25.)
    s["orbsmall"] = W.orb_spec(0.7)
    s["parallelepiped"] = W.parallelepiped_spec(20., 30., 40., 30., 20., 40.)
    s["parallelepipedneg"] = W.parallelepiped_spec(15., 10., 25., -45., 35., 200.)
    s["parallelepipedbox"] = W.parallelepiped_spec(12., 8., 5., 0., 0., 0.)
    s["paraboloid"] = W.paraboloid_spec(10., 30., 40.)
    s["paraboloidinv"] = W.paraboloid_spec(25., 5., 20.)
    s["paraboloidtip"] = W.paraboloid_spec(0., 15., 30.)
    # trapezoids: slanted (theta, phi, alpha; planar faces need equal alphas and
    # (dx1 - dx2) / dy1 = (dx3 - dx4) / dy2), with negative angles, box-like
    # (test/unit_tests/TestTrap.cpp:59 "Test Boxlike #1"), and from the corners
    # of TestTrap.cpp:51-58 ("Test Trdlike #2")
    s["trapezoid"] = W.trapezoid_spec(40., 0.3, 0.7, 20., 10., 15., 0.2, 30., 20., 27.5, 0.2)
    s["trapezoidneg"] = W.trapezoid_spec(25., -0.4, 2.5, 10., 8., 6., -0.3, 15., 12., 9., -0.3)
    s["trapezoidbox"] = W.trapezoid_spec(40., 0., 0., 30., 20., 20., 0., 30., 20., 20., 0.)
    s["trapezoidtrd"] = W.trapezoid_corners_spec(
        [(-10., -20., -40.), (10., -20., -40.), (-10., 20., -40.), (10., 20., -40.),
         (-30., -40., 40.), (30., -40., 40.), (-30., 40., 40.), (30., 40., 40.)])
    s["boolunion"] = W.boolean_spec("boolunion", (20., 20., 20.), 12., 35.,
                                    right_place=(8., 0., 0., 0., 0., 0.))
    # (a union's left component stays at identity: the reference's union
    # DistanceToOut hands the left component the boolean-frame point, and with
    # a placed left component its walk does not end)
    s["boolunionxf"] = W.boolean_spec("boolunion", (15., 25., 10.), 10., 30.,
                                      right_place=(-5., 0., 2., 20., 90., 30.))
    s["boolinter"] = W.boolean_spec("boolinter", (20., 20., 20.), 15., 30.,
                                    right_place=(6., 0., 0., 0., 0., 0.))
    s["boolinterxf"] = W.boolean_spec("boolinter", (25., 20., 15.), 18., 40.,
                                      left_place=(2., -1., 3., 0., 0., 15.),
                                      right_place=(0., 2., 0., 0., 90., 30.))
    s["boolsubxf"] = W.boolsub_spec((30., 30., 30.), 15., 40., left_place=(2., -1., 3., 0., 0., 15.),
                                    right_place=(5., 0., -4., 0., 90., 0.))
    return s
