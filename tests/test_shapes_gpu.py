"""GPU parity of the FP64 batch kernels, through the C ABI.

* against the reference's own outputs (tests/golden/*.npz, written by the
  reference Scalar backend): Contains/Inside bit-exact, distances and safeties
  within 1e-9 mm or 1e-12 relative;
* against the C oracle on larger seeded inputs, device and host buffers;
* the Minimize / node-index / placed forms against their definitions.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from helpers import (PLACEMENTS, assert_distances, assert_exact, assert_torus_distances,
                     vgb_unplaced)
from test_oracle_golden import load_case, spec_from_meta

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
VGB_SHAPES = {"box", "tube", "cone", "sphere", "trd", "torus", "polycone", "polyhedron", "boolsub",
              "orb", "parallelepiped", "paraboloid", "boolunion", "boolinter", "trapezoid",
              "trapezoidcorners"}

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def dev(a):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def spec_of_kind(kind):
    """The parity shape named `kind`, else the first one of that kind."""
    from helpers import shape_specs
    specs = shape_specs()
    return specs.get(kind) or next(s for s in specs.values() if s.kind == kind)


def build_placed(spec, placement):
    import vecgeom_b200 as V
    g = V.Geometry()
    u = vgb_unplaced(g, spec)
    lv = g.LogicalVolume(spec.kind, u)
    pv = lv.Place(g.Transformation3D(*PLACEMENTS[placement]))
    g.CloseGeometry()
    return g, pv


def run_all_ops(pv, pm, dm, pl, dl, step, on_device=True):
    import vecgeom_b200 as V
    torch = _torch()
    n = len(pm[0])
    conv = dev if on_device else np.ascontiguousarray
    P = V.SOA3D(*(conv(a) for a in pm))
    D = V.SOA3D(*(conv(a) for a in dm))
    PL = V.SOA3D(*(conv(a) for a in pl))
    DL = V.SOA3D(*(conv(a) for a in dl))
    S = conv(step)
    if on_device:
        mk = {"u1": lambda: torch.zeros(n, dtype=torch.uint8, device="cuda"),
              "i4": lambda: torch.zeros(n, dtype=torch.int32, device="cuda"),
              "f8": lambda: torch.zeros(n, dtype=torch.float64, device="cuda")}
    else:
        mk = {"u1": lambda: np.zeros(n, np.uint8), "i4": lambda: np.zeros(n, np.int32),
              "f8": lambda: np.zeros(n, np.float64)}
    out = {k: mk[t]() for k, t in (("contains", "u1"), ("inside", "i4"), ("safety_to_in", "f8"),
                                   ("safety_to_out", "f8"), ("distance_to_in", "f8"),
                                   ("distance_to_out", "f8"))}
    pv.Contains(P, out["contains"])
    pv.Inside(P, out["inside"])
    pv.SafetyToIn(P, out["safety_to_in"])
    pv.SafetyToOut(PL, out["safety_to_out"])
    pv.DistanceToIn(P, D, S, out["distance_to_in"])
    pv.DistanceToOut(PL, DL, S, out["distance_to_out"])
    if on_device:
        torch.cuda.synchronize()
        return {k: host(v) for k, v in out.items()}
    return out


def check_against(res, want, what, spec=None, local=None):
    assert_exact(res["contains"], want["contains"], f"{what} Contains")
    assert_exact(res["inside"], want["inside"], f"{what} Inside")
    for k in ("safety_to_in", "safety_to_out"):
        assert_distances(res[k], want[k], f"{what} {k}")
    if spec is not None and spec.kind == "torus":
        for k in ("distance_to_in", "distance_to_out"):
            assert_torus_distances(res[k], want[k + "_crlibm"], want[k], f"{what} {k}")
        return
    for k in ("distance_to_in", "distance_to_out"):
        assert_distances(res[k], want[k], f"{what} {k}")


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
@pytest.mark.parametrize("on_device", [True, False], ids=["device", "host"])
def test_golden_parity(path, on_device):
    d, meta = load_case(path)
    if meta["kind"] not in VGB_SHAPES:
        pytest.skip(f"{meta['kind']} not in this build")
    spec = spec_from_meta(meta)
    g, pv = build_placed(spec, str(d["placement"]))
    res = run_all_ops(pv, (d["mx"], d["my"], d["mz"]), (d["mdx"], d["mdy"], d["mdz"]),
                      (d["lx"], d["ly"], d["lz"]), (d["ldx"], d["ldy"], d["ldz"]), d["step"],
                      on_device)
    check_against(res, d, os.path.basename(path), spec,
                  ((d["lx"], d["ly"], d["lz"]), (d["ldx"], d["ldy"], d["ldz"])))


@pytest.mark.parametrize("kind", sorted(VGB_SHAPES))
def test_large_seeded_vs_reference(kind):
    """2^16 mixed points per shape, every op, against the reference itself when
    oracle/_ref is built, else against the C restatement."""
    from helpers import shape_specs
    from vecgeom_b200 import workloads as W
    spec = spec_of_kind(kind)
    wl = W.make_workload(spec, 1 << 16, W.SEED_BASE + 17)
    g, pv = build_placed(spec, "generic")
    pts = (wl.x, wl.y, wl.z)
    dirs = (wl.dx, wl.dy, wl.dz)
    res = run_all_ops(pv, pts, dirs, pts, dirs, wl.step)
    want = reference_outputs(spec, "generic", pts, dirs, wl.step)
    check_against(res, want, kind, spec, (pts, dirs))


def reference_outputs(spec, placement, pts, dirs, step):
    from helpers import ref_unplaced, oracle_unplaced, oracle_generic_xform
    want = {}
    if oracle.RefLib.available():
        ref = oracle.RefLib()
        pv = ref.placed(ref_unplaced(ref, spec), *PLACEMENTS[placement])
        call = lambda op, p, d=None, s=None: ref.batch(pv, op, p, d, s)  # noqa: E731
    else:
        orc = oracle.Oracle()
        sh = oracle_unplaced(orc, spec)
        xf = orc.xform(*PLACEMENTS[placement], generic=oracle_generic_xform(spec))
        call = lambda op, p, d=None, s=None: orc.batch(sh, xf, op, p, d, s)  # noqa: E731
    want["contains"] = call(oracle.CONTAINS, pts)
    want["inside"] = call(oracle.INSIDE, pts)
    want["safety_to_in"] = call(oracle.SAFETY_TO_IN, pts)
    want["safety_to_out"] = call(oracle.SAFETY_TO_OUT, pts)
    want["distance_to_in"] = call(oracle.DISTANCE_TO_IN, pts, dirs, step)
    if spec.kind == "sphere" and oracle.RefLib.available():
        want["distance_to_in"] = ref.usphere_distance_to_in(spec.params, ref.last_transform, pts,
                                                            dirs)
    want["distance_to_out"] = call(oracle.DISTANCE_TO_OUT, pts, dirs, step)
    if spec.kind == "torus" and oracle.RefLib.available(crlibm=True):
        cr = oracle.RefLib(crlibm=True)
        pvc = cr.placed(ref_unplaced(cr, spec), *PLACEMENTS[placement])
        want["distance_to_in_crlibm"] = cr.batch(pvc, oracle.DISTANCE_TO_IN, pts, dirs, step)
        want["distance_to_out_crlibm"] = cr.batch(pvc, oracle.DISTANCE_TO_OUT, pts, dirs, step)
    return want


@pytest.mark.parametrize("kind", sorted(VGB_SHAPES))
def test_minimize_node_and_placed_forms(kind):
    """DistanceToInMinimize / SafetyTo{In,Out}Minimize / DistanceToOut(nodeindex)
    / PlacedDistanceToOut against their definitions in
    volumes/ShapeImplementationHelper.h:637-748 and :243-270."""
    import torch
    import vecgeom_b200 as V
    from helpers import shape_specs
    from vecgeom_b200 import workloads as W
    spec = spec_of_kind(kind)
    n = 1 << 14
    wl = W.make_workload(spec, n, W.SEED_BASE + 23)
    g, pv = build_placed(spec, "generic")
    P = V.SOA3D(dev(wl.x), dev(wl.y), dev(wl.z))
    D = V.SOA3D(dev(wl.dx), dev(wl.dy), dev(wl.dz))
    step = dev(wl.step)
    dti = torch.empty(n, dtype=torch.float64, device="cuda")
    pv.DistanceToIn(P, D, step, dti)
    sti = torch.empty_like(dti)
    pv.SafetyToIn(P, sti)
    sto = torch.empty_like(dti)
    pv.SafetyToOut(P, sto)
    dto = torch.empty_like(dti)
    pv.DistanceToOut(P, D, step, dto)
    # Minimize: a running minimum seeded with a per-point value
    cur0 = torch.from_numpy(np.random.default_rng(1).uniform(0., 40., n)).cuda()
    cur = cur0.clone()
    ids = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    pv.DistanceToInMinimize(P, D, 5, cur, ids)
    torch.cuda.synchronize()
    # the DistanceToIn with step_max = cur0 must be recomputed to compare
    dti_c = torch.empty_like(dti)
    pv.DistanceToIn(P, D, cur0.clone(), dti_c)
    upd = dti_c < cur0
    assert torch.equal(cur, torch.where(upd, dti_c, cur0))
    assert torch.equal(ids, torch.where(upd, torch.full_like(ids, 5), torch.full_like(ids, -7)))
    s = cur0.clone()
    pv.SafetyToInMinimize(P, s)
    assert torch.equal(s, torch.minimum(sti, cur0))
    s = cur0.clone()
    pv.SafetyToOutMinimize(P, s)
    assert torch.equal(s, torch.minimum(sto, cur0))
    node = torch.zeros(n, dtype=torch.int32, device="cuda")
    dto2 = torch.empty_like(dti)
    pv.DistanceToOut(P, D, step, dto2, nextnodeindex=node)
    assert torch.equal(dto2, dto)
    assert torch.equal(node, torch.where(dto < step, torch.full_like(node, -1),
                                         torch.full_like(node, -2)))


def test_empty_batch_and_bad_arguments():
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    g, pv = build_placed(W.box_spec(1., 2., 3.), "identity")
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    pv.Inside(V.SOA3D(e, e, e), torch.empty(0, dtype=torch.int32, device="cuda"))
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(V.VgbError):
        pv.batch(99, V.SOA3D(x, x, x), x)
    with pytest.raises(V.VgbError):   # distances need directions
        pv.batch(V.OP_DISTANCE_TO_IN, V.SOA3D(x, x, x), x)


@pytest.mark.parametrize("kind", sorted(VGB_SHAPES))
@pytest.mark.parametrize("placement", ["identity", "generic"])
def test_fp32_refine_equals_fp64(kind, placement):
    """The FP32+refine form certifies in float only answers the FP64 form gives
    too (points outside the shape's widened box, rays missing it) and runs the
    FP64 kernels for the rest, so every op must agree bit for bit."""
    import torch
    import vecgeom_b200 as V
    from helpers import shape_specs
    from vecgeom_b200 import workloads as W
    spec = spec_of_kind(kind)
    n = 1 << 15
    wl = W.make_workload(spec, n, W.SEED_BASE + 31)
    # a far shell too: most of its rays miss, so the float screen settles them
    rng = np.random.default_rng(5)
    far = rng.normal(size=(3, n // 4))
    far *= (3. * max(spec.half) / np.linalg.norm(far, axis=0))
    x = np.concatenate([wl.x, far[0]])
    y = np.concatenate([wl.y, far[1]])
    z = np.concatenate([wl.z, far[2]])
    d = W.isotropic(np.random.default_rng(6), len(x))
    g, pv = build_placed(spec, placement)
    P = V.SOA3D(dev(x), dev(y), dev(z))
    D = V.SOA3D(dev(d[0]), dev(d[1]), dev(d[2]))
    step = torch.full((len(x),), 1e30, dtype=torch.float64, device="cuda")
    for meth, dt, args in (("Contains", torch.uint8, ()), ("Inside", torch.int32, ()),
                           ("DistanceToIn", torch.float64, (D, step)),
                           ("SafetyToIn", torch.float64, ())):
        a = torch.full((len(x),), 7, dtype=dt, device="cuda")
        b = torch.full((len(x),), 9, dtype=dt, device="cuda")
        getattr(pv, meth)(P, *args, a, precision=V.PREC_FP64)
        getattr(pv, meth)(P, *args, b, precision=V.PREC_FP32_REFINE)
        torch.cuda.synchronize()
        same = (a == b) | (torch.isnan(a) & torch.isnan(b)) if dt == torch.float64 else a == b
        assert bool(same.all()), f"{kind} {meth}: {int((~same).sum())} differ"


FUSED_OPS = {"contains": 0, "inside": 1, "distance_to_in": 2, "distance_to_out": 3,
             "safety_to_in": 4, "safety_to_out": 5}


def fused_against_per_op(spec, n, seed, on_device):
    """vgb_batch_fused over all six ops equals six vgb_batch calls, bit for bit."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    wl = W.make_workload(spec, n, seed)
    g, pv = build_placed(spec, "generic")
    pts, dirs = (wl.x, wl.y, wl.z), (wl.dx, wl.dy, wl.dz)
    want = run_all_ops(pv, pts, dirs, pts, dirs, wl.step)
    conv = dev if on_device else (lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory())
    dt = {"contains": torch.uint8, "inside": torch.int32}
    outs = {k: torch.zeros(n, dtype=dt.get(k, torch.float64),
                           device="cuda" if on_device else "cpu") for k in FUSED_OPS}
    if not on_device:
        outs = {k: v.pin_memory() for k, v in outs.items()}
    pv.fused(0x3f, V.SOA3D(*(conv(a) for a in pts)), {FUSED_OPS[k]: v for k, v in outs.items()},
             V.SOA3D(*(conv(a) for a in dirs)), conv(wl.step))
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in outs.items()}
    for k in FUSED_OPS:
        a, b = got[k], want[k]
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
        assert same.all(), f"{spec.kind} fused {k}: {np.flatnonzero(~same)[:5]}"


@pytest.mark.parametrize("kind", sorted(VGB_SHAPES))
@pytest.mark.parametrize("on_device", [True, False], ids=["device", "host"])
def test_fused_equals_per_op(kind, on_device):
    from vecgeom_b200 import workloads as W
    fused_against_per_op(spec_of_kind(kind), 1 << 14, W.SEED_BASE + 41, on_device)


@pytest.mark.parametrize("on_device", [True, False], ids=["device", "host"])
def test_fused_host_staging_across_chunks(on_device):
    """More points than one staging chunk (1 M), the last chunk ragged."""
    from vecgeom_b200 import workloads as W
    fused_against_per_op(spec_of_kind("sphere"), (1 << 20) * 2 + 4099, W.SEED_BASE + 43,
                         on_device)


@pytest.mark.parametrize("pinned", [False, True], ids=["pageable", "pinned"])
def test_batch_host_staging_across_chunks(pinned):
    """vgb_batch with host buffers over more points than the staging slots hold
    at once (3 x 2^20 + 4099: full chunks, then the halving tail, every slot
    reused) equals the device-buffer call bit for bit: a point op, a directed
    op, and a Minimize op, which also reads its outputs and node ids in."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    spec = spec_of_kind("tube")
    n = 3 * (1 << 20) + 4099
    wl = W.make_workload(spec, n, W.SEED_BASE + 53)
    g, pv = build_placed(spec, "generic")
    if pinned:
        hconv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
        hbuf = lambda a: torch.from_numpy(np.array(a)).pin_memory()  # noqa: E731
        back = lambda t: t.numpy()  # noqa: E731
    else:
        hconv = hbuf = lambda a: np.array(a)  # noqa: E731
        back = lambda t: t  # noqa: E731
    pts, dirs = (wl.x, wl.y, wl.z), (wl.dx, wl.dy, wl.dz)
    PD, DD, SD = V.SOA3D(*map(dev, pts)), V.SOA3D(*map(dev, dirs)), dev(wl.step)
    PH, DH, SH = V.SOA3D(*map(hconv, pts)), V.SOA3D(*map(hconv, dirs)), hconv(wl.step)

    ins_d = torch.empty(n, dtype=torch.int32, device="cuda")
    ins_h = hbuf(np.zeros(n, np.int32))
    pv.Inside(PD, ins_d)
    pv.Inside(PH, ins_h)
    dti_d = torch.empty(n, dtype=torch.float64, device="cuda")
    dti_h = hbuf(np.zeros(n))
    pv.DistanceToIn(PD, DD, SD, dti_d)
    pv.DistanceToIn(PH, DH, SH, dti_h)
    # Minimize: the current step is the input distance, node ids start at -1
    start = wl.step * 0.5
    min_d, ids_d = dev(start), dev(np.full(n, -1, np.int32))
    min_h, ids_h = hbuf(start), hbuf(np.full(n, -1, np.int32))
    pv.DistanceToInMinimize(PD, DD, 7, min_d, ids_d)
    pv.DistanceToInMinimize(PH, DH, 7, min_h, ids_h)
    torch.cuda.synchronize()
    for what, a, b in (("Inside", ins_h, ins_d), ("DistanceToIn", dti_h, dti_d),
                       ("DistanceToInMinimize", min_h, min_d), ("node ids", ids_h, ids_d)):
        a, b = back(a), b.cpu().numpy()
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
        assert same.all(), f"host-staged {what}: {np.flatnonzero(~same)[:5]}"
    assert (back(ids_h) == 7).any() and (back(ids_h) == -1).any()


@pytest.mark.parametrize("kind", ["tube", "sphere", "polycone", "boolsub"])
@pytest.mark.parametrize("on_device", [True, False], ids=["device", "host"])
def test_fused_local_ops_inside_only(kind, on_device):
    """VGB_FUSED_LOCAL_INSIDE_ONLY: one fused call gives every op on all points,
    with DistanceToOut and SafetyToOut equal to the per-op results where
    Contains() holds and kInfinity elsewhere."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    spec = spec_of_kind(kind)
    n = 1 << 15
    wl = W.make_workload(spec, n, W.SEED_BASE + 47)
    g, pv = build_placed(spec, "generic")
    pts, dirs = (wl.x, wl.y, wl.z), (wl.dx, wl.dy, wl.dz)
    want = run_all_ops(pv, pts, dirs, pts, dirs, wl.step)
    conv = dev if on_device else (lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory())
    dt = {"contains": torch.uint8, "inside": torch.int32}
    outs = {k: torch.zeros(n, dtype=dt.get(k, torch.float64),
                           device="cuda" if on_device else "cpu") for k in FUSED_OPS}
    if not on_device:
        outs = {k: v.pin_memory() for k, v in outs.items()}
    pv.fused(0x3f, V.SOA3D(*(conv(a) for a in pts)), {FUSED_OPS[k]: v for k, v in outs.items()},
             V.SOA3D(*(conv(a) for a in dirs)), conv(wl.step), local_inside_only=True)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in outs.items()}
    inside = want["contains"].astype(bool)
    for k in FUSED_OPS:
        a, b = got[k], want[k]
        if k in ("distance_to_out", "safety_to_out"):
            assert np.isinf(a[~inside]).all() and (a[~inside] > 0).all(), k
            a, b = a[inside], b[inside]
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else a == b
        assert same.all(), f"{kind} fused {k}: {np.flatnonzero(~same)[:5]}"
