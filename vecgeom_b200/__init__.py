"""vecgeom_b200 -- B200-native implementation of VecGeom's geometry hot path.

The compute lives in libvgb.so (CUDA for sm_100a, C ABI in include/vgb.h);
this package is the Python host side that mirrors the reference API.
"""
from ._lib import (VgbError, check, lib, LIB_PATH, PREC_FP64, PREC_FP32_REFINE,  # noqa: F401
                   OP_CONTAINS, OP_INSIDE, OP_DISTANCE_TO_IN, OP_DISTANCE_TO_OUT,
                   OP_SAFETY_TO_IN, OP_SAFETY_TO_OUT, OP_DISTANCE_TO_IN_MINIMIZE,
                   OP_SAFETY_TO_IN_MINIMIZE, OP_SAFETY_TO_OUT_MINIMIZE,
                   OP_DISTANCE_TO_OUT_NODE, OP_PLACED_DISTANCE_TO_OUT)
from .geometry import (Geometry, LogicalVolume, PlacedVolume, SOA3D,  # noqa: F401
                       NavStatePool, SimpleNavigator, ABBoxNavigator, ComputeABBox,
                       BasketPlan, NavServer, kInside, kSurface, kOutside, kTolerance, kInfinity)

__all__ = ["Geometry", "LogicalVolume", "PlacedVolume", "SOA3D", "NavStatePool",
           "SimpleNavigator", "ABBoxNavigator", "ComputeABBox", "BasketPlan", "NavServer", "VgbError", "lib"]
