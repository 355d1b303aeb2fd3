"""Host-side mirror of the reference's geometry and VPlacedVolume SOA3D API.

Names, argument order and meaning follow the reference so that call sites read
alike:
  - ``Geometry.UnplacedBox(dx, dy, dz)`` ... (volumes/Unplaced*.h constructors)
  - ``Geometry.Transformation3D(tx, ty, tz, phi, theta, psi)`` (degrees,
    source/Transformation3D.cpp:36-44)
  - ``Geometry.LogicalVolume(label, unplaced)``, ``LogicalVolume.Place(t)``,
    ``LogicalVolume.PlaceDaughter(daughter, t)`` (source/LogicalVolume.cpp:60-102)
  - ``PlacedVolume.Contains(points, out)``, ``Inside``, ``DistanceToIn(points,
    dirs, step_max, out)``, ``DistanceToOut``, ``SafetyToIn``, ``SafetyToOut``,
    ``DistanceToInMinimize``, ``SafetyToInMinimize``, ``SafetyToOutMinimize``
    (volumes/PlacedVolume.h:145-250)
Every call goes through libvgb.so's C ABI.  Arrays may be numpy arrays (host
memory, staged by the library) or torch tensors on the geometry's CUDA device.
Errors raise VgbError instead of asserting.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import check

kInside, kSurface, kOutside = 0, 1, 2
kTolerance = 1e-9
kInfinity = float("inf")


def _addr(a) -> int | None:
    """Address of a contiguous array (numpy or torch) or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensors must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)!r}")


def _check_dtype(a, kind: str) -> None:
    if a is None:
        return
    want = {"f8": ("float64",), "i4": ("int32",), "u1": ("uint8", "bool")}[kind]
    name = str(a.dtype).replace("torch.", "")
    if name not in want:
        raise TypeError(f"expected dtype {want[0]}, got {name}")


def _len(a) -> int:
    return int(a.shape[0])


class SOA3D:
    """Structure-of-arrays batch of 3-vectors (base/SOA3D.h:32-39)."""

    def __init__(self, x, y, z):
        if not (_len(x) == _len(y) == _len(z)):
            raise ValueError("SOA3D components must have one length")
        for a in (x, y, z):
            _check_dtype(a, "f8")
        self.x, self.y, self.z = x, y, z

    def size(self) -> int:
        return _len(self.x)

    def __len__(self) -> int:
        return self.size()


@dataclass
class LogicalVolume:
    geometry: "Geometry"
    id: int
    label: str

    def Place(self, transformation: int) -> "PlacedVolume":
        out = ctypes.c_int32()
        check(self.geometry.L.vgb_place(self.geometry.handle, self.id, transformation, ctypes.byref(out)))
        return PlacedVolume(self.geometry, out.value, self)

    def PlaceDaughter(self, daughter: "LogicalVolume", transformation: int) -> "PlacedVolume":
        out = ctypes.c_int32()
        check(self.geometry.L.vgb_place_daughter(self.geometry.handle, self.id, daughter.id,
                                         transformation, ctypes.byref(out)))
        return PlacedVolume(self.geometry, out.value, daughter)


class PlacedVolume:
    """A placed volume; its methods are the VPlacedVolume SOA3D virtuals."""

    def __init__(self, geometry: "Geometry", pid: int, logical: LogicalVolume):
        self.geometry = geometry
        self.id = pid
        self.logical = logical

    # -- generic entry -------------------------------------------------------
    def batch(self, op: int, points: SOA3D, out, dirs: SOA3D | None = None, step_max=None,
              aux=None, daughter: int = 0, precision: int = L.PREC_FP64, stream=None) -> None:
        g = self.geometry
        g._require_closed()
        n = points.size()
        if _len(out) < n:
            raise ValueError("output shorter than the batch")
        if dirs is not None and dirs.size() != n:
            raise ValueError("directions must match the points")
        if step_max is not None:
            _check_dtype(step_max, "f8")
        _check_dtype(aux, "i4")
        d = dirs
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        check(g.L.vgb_batch(
            g.handle, self.id, op, n, _addr(points.x), _addr(points.y), _addr(points.z),
            _addr(d.x) if d else None, _addr(d.y) if d else None, _addr(d.z) if d else None,
            _addr(step_max), _addr(out), _addr(aux), daughter, precision, s))

    # -- the reference's method names ----------------------------------------
    def Contains(self, points: SOA3D, out, **kw) -> None:
        _check_dtype(out, "u1")
        self.batch(L.OP_CONTAINS, points, out, **kw)

    def Inside(self, points: SOA3D, out, **kw) -> None:
        _check_dtype(out, "i4")
        self.batch(L.OP_INSIDE, points, out, **kw)

    def DistanceToIn(self, points: SOA3D, dirs: SOA3D, step_max, out, **kw) -> None:
        _check_dtype(out, "f8")
        self.batch(L.OP_DISTANCE_TO_IN, points, out, dirs, step_max, **kw)

    def DistanceToInMinimize(self, points: SOA3D, dirs: SOA3D, daughterindex: int, out,
                             nextnodeids, **kw) -> None:
        _check_dtype(out, "f8")
        self.batch(L.OP_DISTANCE_TO_IN_MINIMIZE, points, out, dirs, None, nextnodeids,
                   daughterindex, **kw)

    def DistanceToOut(self, points: SOA3D, dirs: SOA3D, step_max, out, nextnodeindex=None,
                      **kw) -> None:
        _check_dtype(out, "f8")
        if nextnodeindex is None:
            self.batch(L.OP_DISTANCE_TO_OUT, points, out, dirs, step_max, **kw)
        else:
            self.batch(L.OP_DISTANCE_TO_OUT_NODE, points, out, dirs, step_max, nextnodeindex,
                       **kw)

    def PlacedDistanceToOut(self, points: SOA3D, dirs: SOA3D, step_max, out, **kw) -> None:
        _check_dtype(out, "f8")
        self.batch(L.OP_PLACED_DISTANCE_TO_OUT, points, out, dirs, step_max, **kw)

    def SafetyToIn(self, points: SOA3D, out, **kw) -> None:
        _check_dtype(out, "f8")
        self.batch(L.OP_SAFETY_TO_IN, points, out, **kw)

    def SafetyToInMinimize(self, points: SOA3D, safeties, **kw) -> None:
        _check_dtype(safeties, "f8")
        self.batch(L.OP_SAFETY_TO_IN_MINIMIZE, points, safeties, **kw)

    def SafetyToOut(self, points: SOA3D, out, **kw) -> None:
        _check_dtype(out, "f8")
        self.batch(L.OP_SAFETY_TO_OUT, points, out, **kw)

    def SafetyToOutMinimize(self, points: SOA3D, safeties, **kw) -> None:
        _check_dtype(safeties, "f8")
        self.batch(L.OP_SAFETY_TO_OUT_MINIMIZE, points, safeties, **kw)

    def fused(self, ops: int, points: SOA3D, outs: dict, dirs: SOA3D | None = None,
              step_max=None, dto_inside_only: bool = False, precision: int = L.PREC_FP64,
              stream=None, local_inside_only: bool = False) -> None:
        """Several ops over the same points in one pass (vgb_batch_fused).
        dto_inside_only: DistanceToOut only where Contains() holds;
        local_inside_only: DistanceToOut and SafetyToOut only there (the others
        get kInfinity)."""
        g = self.geometry
        g._require_closed()
        arr = (ctypes.c_void_p * 6)()
        for k, v in outs.items():
            arr[k] = _addr(v)
        d = dirs
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        check(g.L.vgb_batch_fused(
            g.handle, self.id, ops, points.size(), _addr(points.x), _addr(points.y),
            _addr(points.z), _addr(d.x) if d else None, _addr(d.y) if d else None,
            _addr(d.z) if d else None, _addr(step_max), arr,
            (L.FUSED_DTO_INSIDE_ONLY if dto_inside_only else 0)
            | (L.FUSED_LOCAL_INSIDE_ONLY if local_inside_only else 0), precision, s))


class Geometry:
    """A geometry under construction, then closed and resident on the device."""

    def __init__(self, library=None):
        # library: an already configured ctypes handle exposing the vgb_* ABI
        # (defaults to libvgb.so)
        self.L = library if library is not None else L.lib()
        h = ctypes.c_void_p()
        check(self.L.vgb_geometry_create(ctypes.byref(h)))
        self.handle = h
        self.closed = False
        self.world: PlacedVolume | None = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and getattr(self, "L", None) is not None:
            self.L.vgb_geometry_destroy(h)
            self.handle = None

    def _id(self, fn, *args) -> int:
        out = ctypes.c_int32()
        check(fn(self.handle, *args, ctypes.byref(out)))
        return out.value

    def _require_closed(self) -> None:
        if not self.closed:
            raise L.VgbError(L.EINVAL, "geometry is not closed")

    # -- unplaced shapes (volumes/Unplaced*.h) --------------------------------
    def UnplacedBox(self, dx, dy, dz) -> int:
        return self._id(self.L.vgb_unplaced_box, dx, dy, dz)

    def UnplacedTube(self, rmin, rmax, dz, sphi, dphi) -> int:
        return self._id(self.L.vgb_unplaced_tube, rmin, rmax, dz, sphi, dphi)

    def UnplacedCone(self, rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi) -> int:
        return self._id(self.L.vgb_unplaced_cone, rmin1, rmax1, rmin2, rmax2, dz, sphi, dphi)

    def UnplacedSphere(self, rmin, rmax, sphi, dphi, stheta, dtheta) -> int:
        return self._id(self.L.vgb_unplaced_sphere, rmin, rmax, sphi, dphi, stheta, dtheta)

    def UnplacedTorus(self, rmin, rmax, rtor, sphi, dphi) -> int:
        return self._id(self.L.vgb_unplaced_torus, rmin, rmax, rtor, sphi, dphi)

    def UnplacedPolycone(self, sphi, dphi, rmin, rmax, z) -> int:
        rmin, rmax, z = (np.ascontiguousarray(a, np.float64) for a in (rmin, rmax, z))
        return self._id(self.L.vgb_unplaced_polycone, sphi, dphi, len(z), rmin.ctypes.data,
                        rmax.ctypes.data, z.ctypes.data)

    def UnplacedPolyhedron(self, phi_start_deg, phi_delta_deg, sides, z, rmin, rmax) -> int:
        rmin, rmax, z = (np.ascontiguousarray(a, np.float64) for a in (rmin, rmax, z))
        return self._id(self.L.vgb_unplaced_polyhedron, phi_start_deg, phi_delta_deg, sides,
                        len(z), z.ctypes.data, rmin.ctypes.data, rmax.ctypes.data)

    def UnplacedTrd(self, dx1, dx2, dy1, dy2, dz) -> int:
        return self._id(self.L.vgb_unplaced_trd, dx1, dx2, dy1, dy2, dz)

    def UnplacedOrb(self, r) -> int:
        return self._id(self.L.vgb_unplaced_orb, r)

    def UnplacedParallelepiped(self, x, y, z, alpha, theta, phi) -> int:
        """Half-lengths and the three angles in degrees, as the reference takes them."""
        return self._id(self.L.vgb_unplaced_parallelepiped, x, y, z, alpha, theta, phi)

    def UnplacedParaboloid(self, rlo, rhi, dz) -> int:
        return self._id(self.L.vgb_unplaced_paraboloid, rlo, rhi, dz)

    def UnplacedTrapezoid(self, dz, theta, phi, dy1, dx1, dx2, tan_alpha1, dy2, dx3, dx4,
                          tan_alpha2) -> int:
        """UnplacedTrapezoid(pDz, pTheta, pPhi, pDy1, pDx1, pDx2, pTanAlpha1, pDy2,
        pDx3, pDx4, pTanAlpha2), angles in radians
        (volumes/UnplacedTrapezoid.h:93-95)."""
        return self._id(self.L.vgb_unplaced_trapezoid, dz, theta, phi, dy1, dx1, dx2,
                        tan_alpha1, dy2, dx3, dx4, tan_alpha2)

    def UnplacedTrapezoidFromCorners(self, corners) -> int:
        """UnplacedTrapezoid(TrapCorners_t) (volumes/UnplacedTrapezoid.h:103):
        8 corners (x, y, z), 0-3 at z = -dz, 4-7 at z = +dz."""
        c = np.ascontiguousarray(corners, np.float64).reshape(8, 3)
        return self._id(self.L.vgb_unplaced_trapezoid_corners, c.ctypes.data)

    def UnplacedTrapezoidBox(self, xbox, ybox, zbox) -> int:
        """UnplacedTrapezoid(xbox, ybox, zbox) (volumes/UnplacedTrapezoid.h:115)."""
        return self.UnplacedTrapezoid(zbox, 0., 0., ybox, xbox, xbox, 0., ybox, xbox, xbox, 0.)

    def UnplacedBooleanVolume(self, op: int, left: PlacedVolume, right: PlacedVolume) -> int:
        return self._id(self.L.vgb_unplaced_boolean, op, left.id, right.id)

    # -- placement -----------------------------------------------------------
    def Transformation3D(self, tx=0., ty=0., tz=0., phi=0., theta=0., psi=0.) -> int:
        return self._id(self.L.vgb_transformation, tx, ty, tz, phi, theta, psi)

    def Transformation3DMatrix(self, tx, ty, tz, r9) -> int:
        r = np.ascontiguousarray(r9, np.float64)
        return self._id(self.L.vgb_transformation_matrix, tx, ty, tz, r.ctypes.data)

    def LogicalVolume(self, label: str, unplaced: int) -> LogicalVolume:
        lid = self._id(self.L.vgb_logical_volume, label.encode(), unplaced)
        return LogicalVolume(self, lid, label)

    def SetWorld(self, placed: PlacedVolume) -> None:
        check(self.L.vgb_set_world(self.handle, placed.id))
        self.world = placed

    def CloseGeometry(self) -> None:
        """GeoManager::CloseGeometry + CudaManager upload (one copy per table)."""
        check(self.L.vgb_geometry_close(self.handle))
        self.closed = True

    def getMaxDepth(self) -> int:
        out = ctypes.c_int32()
        check(self.L.vgb_geometry_max_depth(self.handle, ctypes.byref(out)))
        return out.value

    def device_bytes(self) -> int:
        out = ctypes.c_int64()
        check(self.L.vgb_geometry_device_bytes(self.handle, ctypes.byref(out)))
        return out.value

    # -- ingestion and export formats ---------------------------------------
    def _sized(self, fn) -> bytes:
        n = ctypes.c_size_t()
        check(fn(self.handle, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(fn(self.handle, buf, n.value, ctypes.byref(n)))
        return buf.raw[:n.value]

    def Serialize(self) -> bytes:
        """The flat image of the geometry (vgb_geometry_serialize)."""
        return self._sized(self.L.vgb_geometry_serialize)

    def Save(self, path: str) -> None:
        check(self.L.vgb_geometry_save(self.handle, os.fsencode(path)))

    def ExportCpp(self) -> str:
        """C++ source rebuilding the geometry with VecGeom's API
        (GeomCppExporter::DumpGeometry, source/CppExporter.cpp)."""
        return self._sized(self.L.vgb_geometry_export_cpp).decode()

    @classmethod
    def _adopt(cls, library, handle) -> "Geometry":
        g = cls.__new__(cls)
        g.L = library if library is not None else L.lib()
        g.handle = handle
        g.closed = False
        g.world = None
        return g

    @classmethod
    def FromImage(cls, data: bytes, library=None) -> "Geometry":
        """A new open geometry from a flat image; ids as in the image."""
        lib = library if library is not None else L.lib()
        h = ctypes.c_void_p()
        check(lib.vgb_geometry_deserialize(data, len(data), ctypes.byref(h)))
        return cls._adopt(lib, h)

    @classmethod
    def Load(cls, path: str, library=None) -> "Geometry":
        lib = library if library is not None else L.lib()
        h = ctypes.c_void_p()
        check(lib.vgb_geometry_load(os.fsencode(path), ctypes.byref(h)))
        return cls._adopt(lib, h)


# ---------------------------------------------------------------------------
# navigation (navigation/NavStatePool.h, navigation/SimpleNavigator.h)
# ---------------------------------------------------------------------------
def _stream(stream):
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else stream


class NavStatePool:
    """NavStatePool(size, depth) on the geometry's device (navigation/NavStatePool.h:46-60).

    States keep the reference's field layout; ``to_numpy()`` returns them as a
    structured array (level, onBoundary, header, path slots holding placed ids)."""

    def __init__(self, geometry: "Geometry", n: int):
        geometry._require_closed()
        self.geometry = geometry
        h = ctypes.c_void_p()
        check(geometry.L.vgb_navpool_create(geometry.handle, n, ctypes.byref(h)))
        self.handle = h
        dev, stride, cap = ctypes.c_void_p(), ctypes.c_int64(), ctypes.c_int64()
        check(geometry.L.vgb_navpool_info(h, ctypes.byref(dev), ctypes.byref(stride),
                                          ctypes.byref(cap)))
        self.stride = stride.value
        self.n = cap.value
        self.depth = geometry.getMaxDepth()

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None:
            self.geometry.L.vgb_navpool_destroy(h)
            self.handle = None

    def dtype(self) -> np.dtype:
        return np.dtype({"names": ["level", "onBoundary", "header", "path"],
                         "formats": ["<i4", "u1", "<u4", ("<i8", (self.depth + 1,))],
                         "offsets": [0, 4, 8, 16], "itemsize": self.stride})

    def to_numpy(self, n: int | None = None, stream=None) -> np.ndarray:
        n = self.n if n is None else n
        out = np.zeros(n, self.dtype())
        check(self.geometry.L.vgb_navpool_download(self.handle, out.ctypes.data, n,
                                                   _stream(stream)))
        return out

    def from_numpy(self, states: np.ndarray, stream=None) -> None:
        states = np.ascontiguousarray(states, self.dtype())
        check(self.geometry.L.vgb_navpool_upload(self.handle, states.ctypes.data, len(states),
                                                 _stream(stream)))

    def tops(self, n: int | None = None) -> np.ndarray:
        """Placed id of Top() per state (-1 when outside)."""
        st = self.to_numpy(n)
        lvl = st["level"].astype(np.int64)
        top = np.full(len(st), -1, np.int64)
        ok = lvl > 0
        top[ok] = st["path"][np.flatnonzero(ok), lvl[ok] - 1]
        return top


class SimpleNavigator:
    """navigation/SimpleNavigator.h over device batches (torch CUDA tensors)."""

    def __init__(self, geometry: "Geometry"):
        geometry._require_closed()
        self.geometry = geometry

    def LocatePoint(self, points: SOA3D, states: NavStatePool, stream=None) -> None:
        g = self.geometry
        check(g.L.vgb_nav_locate(g.handle, points.size(), _addr(points.x), _addr(points.y),
                                 _addr(points.z), states.handle, _stream(stream)))

    def FindNextBoundaryAndStep(self, points: SOA3D, dirs: SOA3D, cur: NavStatePool,
                                nxt: NavStatePool, pstep, step, safety=None,
                                precision: int = L.PREC_FP64, stream=None) -> None:
        g = self.geometry
        for a in (pstep, step, safety):
            _check_dtype(a, "f8")
        check(g.L.vgb_nav_find_next_boundary_and_step(
            g.handle, points.size(), _addr(points.x), _addr(points.y), _addr(points.z),
            _addr(dirs.x), _addr(dirs.y), _addr(dirs.z), cur.handle, nxt.handle, _addr(pstep),
            _addr(step), _addr(safety), precision, _stream(stream)))

    def FindNextBoundaryAndStepBasket(self, points: SOA3D, dirs: SOA3D, cur: NavStatePool,
                                      nxt: NavStatePool, pstep, distances, safeties=None,
                                      nextnodes=None, stream=None) -> None:
        """The basket interface (SimpleNavigator.h:637-743 with GetSafeties);
        see vgb_nav_find_next_boundary_and_step_basket."""
        g = self.geometry
        for a in (pstep, distances, safeties):
            _check_dtype(a, "f8")
        _check_dtype(nextnodes, "i4")
        check(g.L.vgb_nav_find_next_boundary_and_step_basket(
            g.handle, points.size(), _addr(points.x), _addr(points.y), _addr(points.z),
            _addr(dirs.x), _addr(dirs.y), _addr(dirs.z), cur.handle, nxt.handle, _addr(pstep),
            _addr(distances), _addr(safeties), _addr(nextnodes), _stream(stream)))

    def Trace(self, points: SOA3D, dirs: SOA3D, pstep: float, max_steps: int, nsteps,
              next_ids=None, steps=None, safeties=None, precision: int = L.PREC_FP64,
              stream=None) -> None:
        """Steps every track to the world exit (see vgb_nav_trace)."""
        g = self.geometry
        _check_dtype(nsteps, "i4")
        _check_dtype(next_ids, "i4")
        check(g.L.vgb_nav_trace(
            g.handle, points.size(), _addr(points.x), _addr(points.y), _addr(points.z),
            _addr(dirs.x), _addr(dirs.y), _addr(dirs.z), float(pstep), int(max_steps),
            _addr(next_ids), _addr(steps), _addr(safeties), _addr(nsteps), precision,
            _stream(stream)))

    def error_flags(self) -> int:
        out = ctypes.c_uint32()
        check(self.geometry.L.vgb_nav_error_flags(self.geometry.handle, ctypes.byref(out)))
        return out.value


class ABBoxNavigator(SimpleNavigator):
    """navigation/ABBoxNavigator.h over device batches: the step culls and
    orders the daughters by ABBoxManager's aligned boxes; LocatePoint and the
    safety are SimpleNavigator's (the reference's ABBoxNavigator uses them)."""

    def FindNextBoundaryAndStep(self, points: SOA3D, dirs: SOA3D, cur: NavStatePool,
                                nxt: NavStatePool, pstep, step, safety=None,
                                stream=None) -> None:
        g = self.geometry
        for a in (pstep, step, safety):
            _check_dtype(a, "f8")
        check(g.L.vgb_abbox_nav_find_next_boundary_and_step(
            g.handle, points.size(), _addr(points.x), _addr(points.y), _addr(points.z),
            _addr(dirs.x), _addr(dirs.y), _addr(dirs.z), cur.handle, nxt.handle, _addr(pstep),
            _addr(step), _addr(safety), _stream(stream)))

    def Trace(self, points: SOA3D, dirs: SOA3D, pstep: float, max_steps: int, nsteps,
              next_ids=None, steps=None, safeties=None, stream=None) -> None:
        """Steps every track to the world exit (see vgb_abbox_nav_trace)."""
        g = self.geometry
        _check_dtype(nsteps, "i4")
        _check_dtype(next_ids, "i4")
        check(g.L.vgb_abbox_nav_trace(
            g.handle, points.size(), _addr(points.x), _addr(points.y), _addr(points.z),
            _addr(dirs.x), _addr(dirs.y), _addr(dirs.z), float(pstep), int(max_steps),
            _addr(next_ids), _addr(steps), _addr(safeties), _addr(nsteps), _stream(stream)))


def ComputeABBox(geometry: "Geometry", placed) -> np.ndarray:
    """ABBoxManager::ComputeABBox: (lower xyz, upper xyz) of a placed volume's
    aligned box in its mother's frame."""
    out = np.zeros(6)
    pid = placed.id if hasattr(placed, "id") else int(placed)
    check(geometry.L.vgb_abbox_compute(geometry.handle, pid, out.ctypes.data))
    return out


# ---------------------------------------------------------------------------
# baskets: many placed volumes in one persistent launch (vgb_basket_*)
# ---------------------------------------------------------------------------
class _Basket(ctypes.Structure):
    _fields_ = [("placed", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("offset", ctypes.c_int64), ("count", ctypes.c_int64)]


class BasketPlan:
    """A plan over baskets (placed volume, offset, count) of concatenated SOA
    arrays; ``ops`` is a mask of (1 << op) over the fused ops (Contains ...
    SafetyToOut), ``outs`` maps op -> output array of all points."""

    def __init__(self, geometry: "Geometry", baskets, ops: int, block: int = 0, tile: int = 0):
        geometry._require_closed()
        self.geometry = geometry
        arr = (_Basket * max(1, len(baskets)))()
        for k, (pv, off, cnt) in enumerate(baskets):
            arr[k].placed = pv.id if hasattr(pv, "id") else int(pv)
            arr[k].offset = int(off)
            arr[k].count = int(cnt)
        h = ctypes.c_void_p()
        check(geometry.L.vgb_basket_plan_create(geometry.handle, arr, len(baskets), ops, block,
                                                tile, ctypes.byref(h)))
        self.handle = h
        self.ops = ops

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None:
            self.geometry.L.vgb_basket_plan_destroy(h)
            self.handle = None

    def info(self) -> dict:
        pts, tiles = ctypes.c_int64(), ctypes.c_int64()
        block, tile = ctypes.c_int32(), ctypes.c_int32()
        check(self.geometry.L.vgb_basket_plan_info(self.handle, ctypes.byref(pts),
                                                   ctypes.byref(tiles), ctypes.byref(block),
                                                   ctypes.byref(tile)))
        return {"points": pts.value, "tiles": tiles.value, "block": block.value,
                "tile": tile.value}

    def _args(self, points: SOA3D, dirs, step, outs):
        arr = (ctypes.c_void_p * 6)()
        for op, a in outs.items():
            arr[op] = _addr(a)
        d = dirs
        return (_addr(points.x), _addr(points.y), _addr(points.z),
                _addr(d.x) if d else None, _addr(d.y) if d else None, _addr(d.z) if d else None,
                _addr(step), arr)

    def run(self, points: SOA3D, dirs, step, outs: dict, flags: int = 0, stream=None) -> None:
        check(self.geometry.L.vgb_basket_run(self.handle, *self._args(points, dirs, step, outs),
                                             flags, _stream(stream)))

    def tune(self, points: SOA3D, dirs, step, outs: dict, flags: int = 0, reps: int = 3,
             stream=None) -> tuple:
        b, t, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_float()
        check(self.geometry.L.vgb_basket_tune(self.handle, *self._args(points, dirs, step, outs),
                                              flags, reps, _stream(stream), ctypes.byref(b),
                                              ctypes.byref(t), ctypes.byref(ms)))
        return b.value, t.value, ms.value

    def capture(self, points: SOA3D, dirs, step, outs: dict, flags: int = 0) -> None:
        check(self.geometry.L.vgb_basket_graph_capture(
            self.handle, *self._args(points, dirs, step, outs), flags))

    def replay(self, stream=None) -> None:
        check(self.geometry.L.vgb_basket_graph_launch(self.handle, _stream(stream)))


# ---------------------------------------------------------------------------
# navigation server: continuous batching of track baskets (vgb_server_*)
# ---------------------------------------------------------------------------
class NavServer:
    """Requests of straight tracks (host arrays) served by continuous batching;
    see vgb_server_* in include/vgb.h."""

    def __init__(self, geometry: "Geometry", max_tracks: int = 0, steps_per_launch: int = 8,
                 max_steps: int = 1000, pstep: float = 1e30, precision: int = L.PREC_FP64):
        geometry._require_closed()
        self.geometry = geometry
        h = ctypes.c_void_p()
        check(geometry.L.vgb_server_create(geometry.handle, max_tracks, steps_per_launch,
                                           max_steps, pstep, precision, ctypes.byref(h)))
        self.handle = h
        mt, nb = ctypes.c_int64(), ctypes.c_int64()
        check(geometry.L.vgb_server_info(h, ctypes.byref(mt), ctypes.byref(nb)))
        self.max_tracks = mt.value
        self.device_bytes = nb.value
        self._sizes = {}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None:
            self.geometry.L.vgb_server_destroy(h)
            self.handle = None

    def submit(self, points, dirs) -> int:
        arrs = [np.ascontiguousarray(a, np.float64) for a in (*points, *dirs)]
        rid = ctypes.c_int64()
        check(self.geometry.L.vgb_server_submit(self.handle, len(arrs[0]),
                                                *(a.ctypes.data for a in arrs), ctypes.byref(rid)))
        self._sizes[rid.value] = len(arrs[0])
        return rid.value

    def step(self, max_completed: int = 4096):
        """One iteration; returns (completed request ids, live tracks, queued requests)."""
        out = (ctypes.c_int64 * max_completed)()
        nc, live, queued = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        check(self.geometry.L.vgb_server_step(self.handle, out, max_completed, ctypes.byref(nc),
                                              ctypes.byref(live), ctypes.byref(queued)))
        return [out[k] for k in range(nc.value)], live.value, queued.value

    def result(self, rid: int) -> dict:
        n = self._sizes.get(rid, 0)
        res = {"nsteps": np.zeros(n, np.int32), "x": np.zeros(n), "y": np.zeros(n),
               "z": np.zeros(n), "hash": np.zeros(n, np.uint64)}
        check(self.geometry.L.vgb_server_result(self.handle, rid,
                                                *(res[k].ctypes.data for k in
                                                  ("nsteps", "x", "y", "z", "hash"))))
        self._sizes.pop(rid, None)
        return res
