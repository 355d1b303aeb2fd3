"""Write the golden vectors in tests/golden/ from the reference itself.

Runs the reference VecGeom Scalar backend (oracle/_ref/libvgref.so, built from
the reference sources by ``make -C oracle ref``) on seeded inputs and stores
inputs + outputs as .npz fixtures.  The fixtures travel with the repository,
so the parity tests need neither the reference tree nor its build.

    python tests/golden/make_golden.py [--placement NAME] [shape ...]
"""
from __future__ import annotations

import json
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from helpers import PLACEMENTS, ref_unplaced, shape_specs  # noqa: E402
from vecgeom_b200 import workloads as W  # noqa: E402

N = 512
OPS = {"contains": oracle.CONTAINS, "inside": oracle.INSIDE,
       "distance_to_in": oracle.DISTANCE_TO_IN, "distance_to_out": oracle.DISTANCE_TO_OUT,
       "safety_to_in": oracle.SAFETY_TO_IN, "safety_to_out": oracle.SAFETY_TO_OUT}


def spec_json(spec) -> str:
    p = {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in spec.params.items()}
    return json.dumps({"kind": spec.kind, "params": p})


_CR = []


def _crlibm_ref():
    if not _CR:
        _CR.append(oracle.RefLib(crlibm=True))
    return _CR[0]


def make_case(ref, name: str, spec, placement: str, seed: int) -> dict:
    wl = W.make_workload(spec, N, seed)
    # near-surface etc. are drawn in the shape's frame; move them to the mother
    # frame of the placement so Contains/Inside/DistanceToIn see the same mix
    tx, ty, tz, phi, theta, psi = PLACEMENTS[placement]
    t = ref.L.vgref_transform_euler(tx, ty, tz, phi, theta, psi)
    r12 = np.zeros(12)
    codes = np.zeros(2, np.int32)
    ref.L.vgref_transform_get(t, r12.ctypes.data, codes.ctypes.data)
    R = r12[3:].reshape(3, 3)
    T = r12[:3]
    loc = np.stack([wl.x, wl.y, wl.z])
    ldir = np.stack([wl.dx, wl.dy, wl.dz])
    # local = R^T (master - T)  =>  master = R local + T   (row-major R as stored)
    mst = (R @ loc) + T[:, None]
    mdir = R @ ldir
    unpl = ref_unplaced(ref, spec)
    lv = ref.L.vgref_logical(name.encode(), unpl)
    pv = ref.L.vgref_place(lv, t)
    pts_m = (mst[0].copy(), mst[1].copy(), mst[2].copy())
    dirs_m = (mdir[0].copy(), mdir[1].copy(), mdir[2].copy())
    pts_l = (wl.x, wl.y, wl.z)
    dirs_l = (wl.dx, wl.dy, wl.dz)
    out = {"spec": spec_json(spec), "placement": placement,
           "mx": pts_m[0], "my": pts_m[1], "mz": pts_m[2],
           "mdx": dirs_m[0], "mdy": dirs_m[1], "mdz": dirs_m[2],
           "lx": wl.x, "ly": wl.y, "lz": wl.z, "ldx": wl.dx, "ldy": wl.dy, "ldz": wl.dz,
           "step": wl.step}
    for opname, op in OPS.items():
        if op in (oracle.DISTANCE_TO_OUT, oracle.SAFETY_TO_OUT):
            pts, dirs = pts_l, dirs_l
        else:
            pts, dirs = pts_m, dirs_m
        use_dir = op in (oracle.DISTANCE_TO_IN, oracle.DISTANCE_TO_OUT)
        out[opname] = ref.batch(pv, op, pts, dirs if use_dir else None,
                                wl.step if use_dir else None)
    if spec.kind == "torus" and oracle.RefLib.available(crlibm=True):
        # the reference's torus with correctly rounded atan2/sin/cos/cbrt
        # (oracle/ref_crlibm.cpp): its distances move with the C library's last
        # bits, and these are the values of a correctly rounding library
        cr = _crlibm_ref()
        tc = cr.L.vgref_transform_euler(tx, ty, tz, phi, theta, psi)
        pvc = cr.L.vgref_place(cr.L.vgref_logical(name.encode(), ref_unplaced(cr, spec)), tc)
        out["distance_to_in_crlibm"] = cr.batch(pvc, oracle.DISTANCE_TO_IN, pts_m, dirs_m,
                                                wl.step)
        out["distance_to_out_crlibm"] = cr.batch(pvc, oracle.DISTANCE_TO_OUT, pts_l, dirs_l,
                                                 wl.step)
    if spec.kind == "sphere":
        # the reference's sphere DistanceToIn is a stub returning kInfinity
        # (volumes/kernel/SphereImplementation.h:84-93); pin it to USolids'
        # USphere::DistanceToIn (USolids/src/USphere.cc:630) instead
        out["distance_to_in_vecgeom_stub"] = out["distance_to_in"]
        out["distance_to_in"] = ref.usphere_distance_to_in(spec.params, t, pts_m, dirs_m)
    return out


def main(argv) -> None:
    only = None
    if "--placement" in argv:
        k = argv.index("--placement")
        only = argv[k + 1]
        argv = argv[:k] + argv[k + 2:]
    ref = oracle.RefLib()
    shapes = shape_specs()
    names = argv or list(shapes)
    for name in sorted(shapes):
        if name not in names:
            continue
        # the seed depends on the case name only, so adding a shape leaves the
        # other fixtures unchanged
        base = W.SEED_BASE + 10 * (zlib.crc32(name.encode()) % 100000)
        for j, placement in enumerate(PLACEMENTS):
            if only is not None and placement != only:
                continue
            case = make_case(ref, name, shapes[name], placement, base + j)
            path = os.path.join(HERE, f"{name}_{placement}.npz")
            np.savez_compressed(path, **case)
            print("wrote", os.path.relpath(path, ROOT))


if __name__ == "__main__":
    main(sys.argv[1:])
