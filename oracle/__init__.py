"""CPU checkers for libvgb -- test infrastructure, NOT product code.

Two checkers, loaded with ctypes:
  * ``Oracle`` -- liboracle.so, the plain-C restatement of the reference
    algorithms in vgb_oracle.c (always built; travels with the repository).
  * ``RefLib`` -- _ref/libvgref.so, the reference VecGeom Scalar backend itself,
    compiled from the reference's own sources by oracle/Makefile.  Present
    wherever it was built; tests that need it skip when it is absent.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package.  The product (vecgeom_b200/) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvgref.so")
# the same reference build with its torus's atan2/sincos/cbrt correctly rounded
# (ref_crlibm.cpp); every other object keeps the C library's functions
REF_CR_SO = os.path.join(HERE, "_ref", "libvgref_crlibm.so")

# or_op / or_shape (vgb_oracle.h)
CONTAINS, INSIDE, DISTANCE_TO_IN, DISTANCE_TO_OUT, SAFETY_TO_IN, SAFETY_TO_OUT = range(6)
_vp, _d, _i, _i64 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int64


def build(with_ref: bool = True) -> None:
    """Compile the C restatement (and the reference shim when the tree is here)."""
    targets = ["oracle"] + (["ref"] if with_ref else [])
    subprocess.run(["make", "-C", HERE, "-j8"] + targets, check=True,
                   stdout=subprocess.DEVNULL)


def _make_print(target: str) -> str:
    return subprocess.run(["make", "-s", "-C", HERE, target], check=True, capture_output=True,
                          text=True).stdout.strip()


def reference_tree():
    """The reference source tree oracle/Makefile builds from, or None when it is
    absent (its base/Global.h missing)."""
    ref = _make_print("print-ref")
    return ref if os.path.exists(os.path.join(ref, "base", "Global.h")) else None


def reference_cxxflags() -> list:
    """The flags oracle/Makefile compiles the reference's sources with."""
    return _make_print("print-ref-cxxflags").split()


def reference_defined(spec, z_local) -> np.ndarray:
    """Points on which the reference's result is defined.  Its polyhedron
    Contains/Inside index the z-segment array with the number of z-planes below
    the point (volumes/kernel/PolyhedronImplementation.h:350-370, :763, :809),
    but its bounding tube reaches kTolerance beyond the end planes
    (source/UnplacedPolyhedron.cpp:120-130): a point within that band above the
    last plane reads one segment past the array, one at or just below the first
    plane (Inside) reads segment -1.  That is undefined behaviour (it crashed the
    reference on 2^22 near-surface points); libvgb clamps to the end segment.
    Comparisons with the reference, and timings of it, leave such points out."""
    z = np.asarray(z_local, np.float64)
    ok = np.ones(len(z), bool)
    if spec.kind == "polyhedron":
        zp = np.asarray(spec.params["z"], np.float64)
        band = 4e-9
        ok &= ~((np.abs(z - zp[0]) <= band) | (np.abs(z - zp[-1]) <= band))
    return ok


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def out_array(op: int, n: int) -> np.ndarray:
    if op == CONTAINS:
        return np.zeros(n, np.uint8)
    if op == INSIDE:
        return np.zeros(n, np.int32)
    return np.zeros(n, np.float64)


class Xform(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double * 3), ("r", ctypes.c_double * 9),
                ("trans_code", ctypes.c_int), ("rot_code", ctypes.c_int)]


class Oracle:
    """The C restatement (vgb_oracle.c)."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        for name, argn in (("or_box", 3), ("or_tube", 5)):
            f = getattr(L, name)
            f.restype = _vp
            f.argtypes = [_d] * argn
        L.or_shape_free.argtypes = [_vp]
        L.or_xform_euler.argtypes = [ctypes.POINTER(Xform)] + [_d] * 6
        L.or_xform_matrix.argtypes = [ctypes.POINTER(Xform), _d, _d, _d, _vp]
        L.or_xform_set_generic.argtypes = [ctypes.POINTER(Xform)]
        L.or_batch.restype = _i
        L.or_batch.argtypes = [_vp, ctypes.POINTER(Xform), _i, _i64] + [_vp] * 8
        self.L = L

    def shape(self, kind: str, *params):
        fn = getattr(self.L, "or_" + kind)
        return fn(*params)

    def xform(self, tx=0., ty=0., tz=0., phi=0., theta=0., psi=0., generic=False) -> Xform:
        x = Xform()
        self.L.or_xform_euler(ctypes.byref(x), tx, ty, tz, phi, theta, psi)
        if generic:
            self.L.or_xform_set_generic(ctypes.byref(x))
        return x

    def batch(self, shape, xf: Xform, op: int, pts, dirs=None, step=None) -> np.ndarray:
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
        n = len(x)
        if dirs is not None:
            dx, dy, dz = (np.ascontiguousarray(a, np.float64) for a in dirs)
        else:
            dx = dy = dz = None
        out = out_array(op, n)
        rc = self.L.or_batch(shape, ctypes.byref(xf), op, n, _p(x), _p(y), _p(z), _p(dx),
                             _p(dy), _p(dz), _p(step), _p(out))
        if rc != 0:
            raise RuntimeError(f"or_batch failed for op {op}")
        return out


class RefLib:
    """The reference VecGeom Scalar backend (oracle/_ref/libvgref.so); with
    crlibm=True the build whose torus uses correctly rounded atan2/sin/cos/cbrt
    (oracle/_ref/libvgref_crlibm.so)."""

    @staticmethod
    def available(crlibm: bool = False) -> bool:
        return os.path.exists(REF_CR_SO if crlibm else REF_SO)

    def __init__(self, crlibm: bool = False):
        L = ctypes.CDLL(REF_CR_SO if crlibm else REF_SO)
        for name, argn in (("vgref_box", 3), ("vgref_tube", 5), ("vgref_cone", 7),
                           ("vgref_sphere", 6), ("vgref_torus", 5), ("vgref_trd", 5)):
            f = getattr(L, name)
            f.restype = _vp
            f.argtypes = [_d] * argn
        L.vgref_orb.restype = _vp
        L.vgref_orb.argtypes = [_d]
        L.vgref_parallelepiped.restype = _vp
        L.vgref_parallelepiped.argtypes = [_d] * 6
        L.vgref_paraboloid.restype = _vp
        L.vgref_paraboloid.argtypes = [_d] * 3
        L.vgref_trapezoid.restype = _vp
        L.vgref_trapezoid.argtypes = [_d] * 11
        L.vgref_trapezoid_corners.restype = _vp
        L.vgref_trapezoid_corners.argtypes = [_vp]
        L.vgref_polycone.restype = _vp
        L.vgref_polycone.argtypes = [_d, _d, _i, _vp, _vp, _vp]
        L.vgref_polyhedron.restype = _vp
        L.vgref_polyhedron.argtypes = [_d, _d, _i, _i, _vp, _vp, _vp]
        L.vgref_boolean.restype = _vp
        L.vgref_boolean.argtypes = [_i, _vp, _vp]
        L.vgref_transform_euler.restype = _vp
        L.vgref_transform_euler.argtypes = [_d] * 6
        L.vgref_transform_matrix.restype = _vp
        L.vgref_transform_matrix.argtypes = [_d, _d, _d, _vp]
        L.vgref_transform_get.argtypes = [_vp, _vp, _vp]
        L.vgref_logical.restype = _vp
        L.vgref_logical.argtypes = [ctypes.c_char_p, _vp]
        L.vgref_place.restype = _vp
        L.vgref_place.argtypes = [_vp, _vp]
        L.vgref_place_daughter.restype = _vp
        L.vgref_place_daughter.argtypes = [_vp, _vp, _vp]
        L.vgref_batch.restype = _i
        L.vgref_batch.argtypes = [_vp, _i, _i64] + [_vp] * 9 + [_i, _i]
        L.vgref_set_world.argtypes = [_vp]
        L.vgref_close_geometry.restype = _i
        L.vgref_placed_id.restype = _i
        L.vgref_placed_id.argtypes = [_vp]
        L.vgref_nav_trace.restype = _i
        L.vgref_nav_trace.argtypes = [_i64] + [_vp] * 6 + [_d, _i] + [_vp] * 4 + [_i]
        L.vgref_nav_basket_step.restype = _i
        L.vgref_nav_basket_step.argtypes = [_i64] + [_vp] * 7 + [_i] + [_vp] * 8
        L.vgref_abbox_compute.restype = None
        L.vgref_abbox_compute.argtypes = [_vp, _vp]
        L.vgref_abbox_nav_trace.restype = _i
        L.vgref_abbox_nav_trace.argtypes = [_i64] + [_vp] * 6 + [_d, _i] + [_vp] * 4
        L.vgref_locate.restype = _i
        L.vgref_locate.argtypes = [_d, _d, _d, _vp]
        L.vgref_usphere_distance_to_in.restype = _i
        L.vgref_usphere_distance_to_in.argtypes = [_d] * 6 + [_vp, _i64] + [_vp] * 7
        self.L = L
        self._keep = []
        self.last_transform = None

    def placed(self, unplaced, tx=0., ty=0., tz=0., phi=0., theta=0., psi=0., label="v"):
        t = self.L.vgref_transform_euler(tx, ty, tz, phi, theta, psi)
        self.last_transform = t
        lv = self.L.vgref_logical(label.encode(), unplaced)
        return self.L.vgref_place(lv, t)

    def usphere_distance_to_in(self, p: dict, transform, pts, dirs, nthreads: int = 1):
        """USolids USphere::DistanceToIn (USolids/src/USphere.cc:630), the
        in-tree definition of the sphere DistanceToIn the reference stubs out."""
        import threading
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
        dx, dy, dz = (np.ascontiguousarray(a, np.float64) for a in dirs)
        n = len(x)
        out = np.zeros(n, np.float64)
        args = (p["rmin"], p["rmax"], p["sphi"], p["dphi"], p["stheta"], p["dtheta"], transform)

        def run(b, e):
            self.L.vgref_usphere_distance_to_in(*args, e - b, x[b:].ctypes.data, y[b:].ctypes.data,
                                                z[b:].ctypes.data, dx[b:].ctypes.data,
                                                dy[b:].ctypes.data, dz[b:].ctypes.data,
                                                out[b:].ctypes.data)
        if nthreads <= 1 or n < 4096:
            run(0, n)
        else:
            ch = (n + nthreads - 1) // nthreads
            ts = [threading.Thread(target=run, args=(b, min(n, b + ch))) for b in range(0, n, ch)]
            for t in ts:
                t.start()
            for t in ts:
                t.join()
        return out

    def batch(self, placed, op: int, pts, dirs=None, step=None, nthreads: int = 1,
              out=None, aux=None, daughter: int = 0) -> np.ndarray:
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
        n = len(x)
        if dirs is not None:
            dx, dy, dz = (np.ascontiguousarray(a, np.float64) for a in dirs)
        else:
            dx = dy = dz = None
        if out is None:
            out = np.zeros(n, np.bool_) if op == CONTAINS else out_array(op, n)
        self.L.vgref_batch(placed, op, n, _p(x), _p(y), _p(z), _p(dx), _p(dy), _p(dz),
                           _p(step), _p(out), _p(aux), daughter, nthreads)
        return out.view(np.uint8) if op == CONTAINS else out


class RefBuilder:
    """Detector-builder adapter over the reference (same methods as
    vecgeom_b200.workloads.VgbBuilder), for building one geometry in both."""

    def __init__(self, ref: RefLib):
        self.ref = ref
        self.L = ref.L

    def box(self, dx, dy, dz):
        return self.L.vgref_box(dx, dy, dz)

    def tube(self, rmin, rmax, dz, sphi, dphi):
        return self.L.vgref_tube(rmin, rmax, dz, sphi, dphi)

    def trd(self, dx1, dx2, dy1, dy2, dz):
        return self.L.vgref_trd(dx1, dx2, dy1, dy2, dz)

    def shape(self, spec):
        return ref_unplaced(self.ref, spec)

    def transform(self, tx=0., ty=0., tz=0., phi=0., theta=0., psi=0.):
        return self.L.vgref_transform_euler(tx, ty, tz, phi, theta, psi)

    def logical(self, label, unplaced):
        return self.L.vgref_logical(label.encode(), unplaced)

    def place(self, logical, transform):
        return self.L.vgref_place(logical, transform)

    def place_daughter(self, mother, daughter, transform):
        return self.L.vgref_place_daughter(mother, daughter, transform)

    def set_world(self, placed):
        self.L.vgref_set_world(placed)

    def close(self):
        self.L.vgref_close_geometry()

    def ids(self, placed) -> np.ndarray:
        return np.array([self.L.vgref_placed_id(p) for p in placed], np.int64)


def ref_nav_trace(ref: RefLib, pts, dirs, pstep: float, max_steps: int, nthreads: int = 1):
    """SimpleNavigator trace of the current reference world (see ref_driver.cpp):
    returns (next reference ids, steps, safeties, nsteps), records per track
    at i * max_steps."""
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
    dx, dy, dz = (np.ascontiguousarray(a, np.float64) for a in dirs)
    n = len(x)
    ids = np.full(n * max_steps, -7, np.int32)
    steps = np.zeros(n * max_steps)
    saf = np.zeros(n * max_steps)
    nst = np.zeros(n, np.int32)
    ref.L.vgref_nav_trace(n, _p(x), _p(y), _p(z), _p(dx), _p(dy), _p(dz), pstep, max_steps,
                          _p(ids), _p(steps), _p(saf), _p(nst), nthreads)
    return ids, steps, saf, nst


def ref_abbox_nav_trace(ref: RefLib, pts, dirs, pstep: float, max_steps: int):
    """ABBoxNavigator trace of the current reference world (single-threaded,
    see ref_driver.cpp vgref_abbox_nav_trace); same records as ref_nav_trace."""
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
    dx, dy, dz = (np.ascontiguousarray(a, np.float64) for a in dirs)
    n = len(x)
    ids = np.full(n * max_steps, -7, np.int32)
    steps = np.zeros(n * max_steps)
    saf = np.zeros(n * max_steps)
    nst = np.zeros(n, np.int32)
    ref.L.vgref_abbox_nav_trace(n, _p(x), _p(y), _p(z), _p(dx), _p(dy), _p(dz), pstep, max_steps,
                                _p(ids), _p(steps), _p(saf), _p(nst))
    return ids, steps, saf, nst


def ref_nav_basket_step(ref: RefLib, pts, dirs, pstep, prior: int) -> dict:
    """SimpleNavigator's basket step over the current reference world (see
    ref_driver.cpp vgref_nav_basket_step): start points after `prior` single
    steps, then per track distance, safety, next node, new top id, boundary."""
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
    dx, dy, dz = (np.ascontiguousarray(a, np.float64) for a in dirs)
    ps = np.ascontiguousarray(pstep, np.float64)
    n = len(x)
    out = {k: np.zeros(n) for k in ("px", "py", "pz", "distance", "safety")}
    out.update({k: np.zeros(n, np.int32) for k in ("nextnode", "newtop", "boundary")})
    ref.L.vgref_nav_basket_step(n, _p(x), _p(y), _p(z), _p(dx), _p(dy), _p(dz), _p(ps), prior,
                                *(_p(out[k]) for k in ("px", "py", "pz", "distance", "safety",
                                                       "nextnode", "newtop", "boundary")))
    return out


def ref_abbox(ref: RefLib, placed) -> np.ndarray:
    """ABBoxManager::ComputeABBox of a reference placed volume (lower, upper)."""
    out = np.zeros(6)
    ref.L.vgref_abbox_compute(placed, _p(out))
    return out


def ref_unplaced(ref: RefLib, spec):
    """Create spec's unplaced shape with the reference's own constructors."""
    import math
    L = ref.L
    p = spec.params
    k = spec.kind
    if k == "box":
        return L.vgref_box(p["dx"], p["dy"], p["dz"])
    if k == "tube":
        return L.vgref_tube(p["rmin"], p["rmax"], p["dz"], p["sphi"], p["dphi"])
    if k == "cone":
        return L.vgref_cone(p["rmin1"], p["rmax1"], p["rmin2"], p["rmax2"], p["dz"], p["sphi"],
                            p["dphi"])
    if k == "sphere":
        return L.vgref_sphere(p["rmin"], p["rmax"], p["sphi"], p["dphi"], p["stheta"],
                              p["dtheta"])
    if k == "torus":
        return L.vgref_torus(p["rmin"], p["rmax"], p["rtor"], p["sphi"], p["dphi"])
    if k == "trd":
        return L.vgref_trd(p["dx1"], p["dx2"], p["dy1"], p["dy2"], p["dz"])
    if k == "orb":
        return L.vgref_orb(p["r"])
    if k == "paraboloid":
        return L.vgref_paraboloid(p["rlo"], p["rhi"], p["dz"])
    if k == "trapezoid":
        return L.vgref_trapezoid(p["dz"], p["theta"], p["phi"], p["dy1"], p["dx1"], p["dx2"],
                                 p["tan_alpha1"], p["dy2"], p["dx3"], p["dx4"], p["tan_alpha2"])
    if k == "trapezoidcorners":
        c = np.ascontiguousarray(p["corners"], np.float64)
        return L.vgref_trapezoid_corners(c.ctypes.data)
    if k == "parallelepiped":
        return L.vgref_parallelepiped(p["x"], p["y"], p["z"], p["alpha"], p["theta"], p["phi"])
    if k in ("polycone", "polyhedron"):
        z, rmin, rmax = (np.ascontiguousarray(p[a], np.float64) for a in ("z", "rmin", "rmax"))
        ref._keep += [z, rmin, rmax]
        if k == "polycone":
            return L.vgref_polycone(p["sphi"], p["dphi"], len(z), z.ctypes.data,
                                    rmin.ctypes.data, rmax.ctypes.data)
        return L.vgref_polyhedron(p["phi_start_deg"], p["phi_delta_deg"], p["sides"], len(z),
                                  z.ctypes.data, rmin.ctypes.data, rmax.ctypes.data)
    if k in ("boolsub", "boolunion", "boolinter"):
        bx, by, bz = p["box_half"]
        ident = (0., 0., 0., 0., 0., 0.)
        left = ref.placed(L.vgref_box(bx, by, bz), *p.get("left_place", ident), label="sub_box")
        right = ref.placed(L.vgref_tube(0., p["tube_rmax"], p["tube_dz"], 0., 2 * math.pi),
                           *p.get("right_place", ident), label="sub_tube")
        return L.vgref_boolean({"boolunion": 0, "boolinter": 1, "boolsub": 2}[k], left, right)
    raise ValueError(k)


def oracle_unplaced(orc: Oracle, spec):
    """Create spec's shape in the C restatement."""
    p = spec.params
    k = spec.kind
    if k == "box":
        return orc.shape("box", p["dx"], p["dy"], p["dz"])
    if k == "tube":
        return orc.shape("tube", p["rmin"], p["rmax"], p["dz"], p["sphi"], p["dphi"])
    raise NotImplementedError(k)


def oracle_generic_xform(spec) -> bool:
    """Shapes whose placed volumes always use the generic transform
    (source/UnplacedPolyhedron.cpp:321-333)."""
    return spec.kind == "polyhedron"
