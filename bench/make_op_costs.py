"""Writes bench/op_costs.json: the algorithmic flops per point of every shape
operation of the benchmark workloads -- measurement infrastructure, NOT
product code.

count_ops.cu runs libvgb's shape arithmetic (written in the reference's
operation order, templated on the arithmetic type) on the host with an
op-counting number type; this script builds it, runs the benchmark inputs
through it (the same seeded point mix, 2^14 points per shape; DistanceToOut
and SafetyToOut on the points inside the shape, as the benchmark runs them)
and averages the counts per point.  Rules: + - * / sqrt count 1, a
transcendental counts 1, comparisons and selects 0; there is no FMA (the
kernels are compiled without contraction).  The identity placement of the
benchmark shapes costs no flops, as in the reference's specialised transform.

    python bench/make_op_costs.py
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from vecgeom_b200 import _lib  # noqa: E402
from vecgeom_b200 import workloads as W  # noqa: E402
from vecgeom_b200.geometry import Geometry  # noqa: E402

SO = os.path.join(ROOT, "_build", "opcount", "liboc.so")
OPS = {"contains": 0, "inside": 1, "distance_to_in": 2, "distance_to_out": 3,
       "safety_to_in": 4, "safety_to_out": 5}
LOCAL = ("distance_to_out", "safety_to_out")
BYTES = {"contains": 25, "inside": 28, "safety_to_in": 32, "safety_to_out": 32,
         "distance_to_in": 64, "distance_to_out": 64}
N = 1 << 14


def build() -> ctypes.CDLL:
    os.makedirs(os.path.dirname(SO), exist_ok=True)
    src = os.path.join(ROOT, "vecgeom_b200", "csrc")
    subprocess.run(["nvcc", "-std=c++17", "-O1", "-Xcompiler", "-fPIC", "-Xcompiler",
                    "-ffp-contract=off", "--expt-relaxed-constexpr", "-diag-suppress", "20011", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-shared", "-o", SO,
                    os.path.join(HERE, "count_ops.cu"), os.path.join(src, "geometry.cu"),
                    os.path.join(src, "unplaced.cu"), os.path.join(src, "geometry_io.cu"),
                    "-lcudart"], check=True)
    L = ctypes.CDLL(SO)
    for name, (res, args) in _lib.SIGNATURES.items():
        f = getattr(L, name, None)
        if f is not None:
            f.restype = res
            f.argtypes = args
    vp = ctypes.c_void_p
    L.oc_count.restype = ctypes.c_int
    L.oc_count.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64] + [vp] * 8
    return L


def count(L, spec, mix, seed) -> dict:
    g = Geometry(library=L)
    pv = g.LogicalVolume(spec.kind, W.build_unplaced(g, spec)).Place(g.Transformation3D())
    wl = W.make_workload(spec, N, seed, mix=mix)
    inside = spec.contains(wl.x, wl.y, wl.z)
    out = {}
    for name, op in OPS.items():
        sel = inside if name in LOCAL else np.ones(N, bool)
        arr = [np.ascontiguousarray(a[sel]) for a in (wl.x, wl.y, wl.z, wl.dx, wl.dy, wl.dz,
                                                       wl.step)]
        m = len(arr[0])
        c = np.zeros(5, np.int64)
        use_dir = name.startswith("distance")
        ptr = lambda a: a.ctypes.data  # noqa: E731
        rc = L.oc_count(g.handle, pv.id, op, m, ptr(arr[0]), ptr(arr[1]), ptr(arr[2]),
                        ptr(arr[3]) if use_dir else None, ptr(arr[4]) if use_dir else None,
                        ptr(arr[5]) if use_dir else None, ptr(arr[6]) if use_dir else None,
                        c.ctypes.data)
        if rc == -3:
            return {}
        assert rc == 0, (spec.kind, name, rc)
        per = c / max(1, m)
        out[name] = {"flops_per_point": round(float(per.sum()), 2),
                     "add": round(float(per[0]), 2), "mul": round(float(per[1]), 2),
                     "div": round(float(per[2]), 2), "sqrt": round(float(per[3]), 2),
                     "transcendental": round(float(per[4]), 2),
                     "bytes_per_point": BYTES[name],
                     "flops_per_byte": round(float(per.sum()) / BYTES[name], 3),
                     "points": m}
    return out


def main() -> None:
    L = build()
    res = {"method": __doc__.strip().splitlines()[0] + " " + " ".join(
        __doc__.strip().splitlines()[2:12]), "points_per_shape": N, "workloads": {}}
    for wname in ("box", "shapes", "heavy"):
        shapes, _, mix = W.bench_config(wname)
        res["workloads"][wname] = {}
        for si, (name, spec) in enumerate(shapes.items()):
            c = count(L, spec, mix, W.bench_seed(si))
            res["workloads"][wname][name] = c if c else "not counted (boolean components run " \
                                                        "in double only)"
            print(wname, name, {k: v["flops_per_point"] for k, v in c.items()} if c else c)
    with open(os.path.join(HERE, "op_costs.json"), "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
