"""Baskets: many shape instances of mixed types in one persistent launch.

The mixed-basket workload (lognormal basket sizes, the eight benchmark kinds
with lengths jittered +-20%, random Euler placements and translations) is
checked against the reference itself: every basket's shape is built in the
reference (oracle/_ref) with its own Transformation3D(tx, ty, tz, phi, theta,
psi) (source/Transformation3D.cpp:36-55) and runs the basket's points there.
The tuned launch shape and the CUDA-graph replay must not change the results.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import (assert_distances, assert_exact, assert_torus_distances, ref_unplaced,
                     reference_defined)
from vecgeom_b200 import workloads as W

DTI, STI = 1 << 2, 1 << 4  # op masks: DistanceToIn, SafetyToIn
ALL = 0x3f


def test_basket_sizes_follow_the_lognormal_clip():
    bs = W.config4_baskets(4096)
    n = np.array([b.n for b in bs])
    assert n.min() >= 16 and n.max() <= 65536
    assert 700 < np.median(n) < 1400
    kinds = {b.spec.kind for b in bs}
    assert kinds == set(W.BASKET_KINDS)


def _setup(nb, seed, max_n=3000):
    import torch
    import vecgeom_b200 as V
    bs = W.config4_baskets(nb, seed=seed)
    for b in bs:
        b.n = min(b.n, max_n)
    bs[3].n = 0  # an empty basket
    g = V.Geometry()
    placed, offsets, pts, dirs, step = W.build_baskets(g, bs)
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    P = V.SOA3D(*(dev(a) for a in pts))
    D = V.SOA3D(*(dev(a) for a in dirs))
    return g, bs, placed, offsets, P, D, dev(step)


def _outs(n, ops):
    import torch
    dt = {0: torch.uint8, 1: torch.int32}
    return {op: torch.full((n,), -3, dtype=dt.get(op, torch.float64), device="cuda")
            for op in range(6) if (ops >> op) & 1}


def _same(a, b):
    import torch
    if a.dtype == torch.float64:
        return bool(((a == b) | (torch.isnan(a) & torch.isnan(b))).all())
    return bool((a == b).all())


def _reference_baskets(bs, offsets, pts, dirs, step, ops):
    """Every basket through the reference: its jittered shape at its own Euler
    placement; sphere DistanceToIn through USolids' USphere (the reference's
    own is a stub).  Returns the outputs and the mask of points compared: the
    points on which the reference's result is defined (helpers.reference_defined,
    judged on the basket's points in its shape's frame)."""
    ref = oracle.RefLib()
    cr = oracle.RefLib(crlibm=True)
    threads = os.cpu_count() or 1
    n = len(pts[0])
    want = {op: oracle.out_array(op, n) for op in range(6) if (ops >> op) & 1}
    for op in (oracle.DISTANCE_TO_IN, oracle.DISTANCE_TO_OUT):
        if op in want:
            want[("crlibm", op)] = oracle.out_array(op, n)
    keep = np.ones(n, bool)
    for off, b in zip(offsets, bs):
        if b.n == 0:
            continue
        ok = reference_defined(b.spec, W.make_workload(b.spec, b.n, b.seed).z)
        keep[off:off + b.n] = ok
        idx = off + np.flatnonzero(ok)
        p = tuple(np.ascontiguousarray(a[idx]) for a in pts)
        d = tuple(np.ascontiguousarray(a[idx]) for a in dirs)
        s = np.ascontiguousarray(step[idx])
        rpv = ref.placed(ref_unplaced(ref, b.spec), *b.place)
        if b.spec.kind == "torus":
            cpv = cr.placed(ref_unplaced(cr, b.spec), *b.place)
            for op in (oracle.DISTANCE_TO_IN, oracle.DISTANCE_TO_OUT):
                if ("crlibm", op) in want:
                    want[("crlibm", op)][idx] = cr.batch(cpv, op, p, d, s, nthreads=threads)
        for op in [o for o in want if isinstance(o, int)]:
            if op == oracle.DISTANCE_TO_IN and b.spec.kind == "sphere":
                want[op][idx] = ref.usphere_distance_to_in(b.spec.params, ref.last_transform, p,
                                                           d, nthreads=threads)
            elif op in (oracle.DISTANCE_TO_IN, oracle.DISTANCE_TO_OUT):
                want[op][idx] = ref.batch(rpv, op, p, d, s, nthreads=threads)
            else:
                want[op][idx] = ref.batch(rpv, op, p, nthreads=threads)
    return want, keep


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.RefLib.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("ops,nb", [(DTI | STI, 320), (ALL, 96)], ids=["dti_sti", "all_ops"])
def test_baskets_match_the_reference(ops, nb):
    """nb baskets of the mixed workload (one of them empty), each with its own
    random placement and jittered parameters, against the reference."""
    import torch
    import vecgeom_b200 as V
    bs = W.config4_baskets(nb, seed=W.SEED_BASE + 41)
    for b in bs:
        b.n = min(b.n, 4096)
    bs[3].n = 0
    g = V.Geometry()
    placed, offsets, pts, dirs, step = W.build_baskets(g, bs)
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    P = V.SOA3D(*(dev(a) for a in pts))
    D = V.SOA3D(*(dev(a) for a in dirs))
    plan = V.BasketPlan(g, [(pv, o, b.n) for pv, o, b in zip(placed, offsets, bs)], ops)
    got = _outs(P.size(), ops)
    plan.run(P, D, dev(step), got)
    torch.cuda.synchronize()
    got = {op: v.cpu().numpy() for op, v in got.items()}
    want, keep = _reference_baskets(bs, offsets, pts, dirs, step, ops)
    assert (~keep).sum() < 1e-3 * len(keep)
    torus = np.zeros(len(keep), bool)
    kinds = set()
    for off, b in zip(offsets, bs):
        if b.n == 0:
            continue
        kinds.add(b.spec.kind)
        sl = slice(off, off + b.n)
        if b.spec.kind == "torus":
            torus[sl] = True
        k = keep[sl]
        what = f"basket at {off} ({b.spec.kind}, {b.n} points, placement {b.place})"
        for op in got:
            g_, w_ = got[op][sl][k], want[op][sl][k]
            if op in (oracle.CONTAINS, oracle.INSIDE):
                assert_exact(g_, w_, f"{what} op {op}")
            elif b.spec.kind != "torus" or op not in (oracle.DISTANCE_TO_IN,
                                                      oracle.DISTANCE_TO_OUT):
                assert_distances(g_, w_, f"{what} op {op}")
    # torus distances: against the reference with correctly rounded libm
    for op in set(got) & {oracle.DISTANCE_TO_IN, oracle.DISTANCE_TO_OUT}:
        t = torus & keep
        assert_torus_distances(got[op][t], want[("crlibm", op)][t], want[op][t],
                               f"torus baskets op {op}")
    assert kinds == set(W.BASKET_KINDS)


@pytest.mark.gpu
def test_tuned_shape_and_graph_replay_keep_results():
    import torch
    import vecgeom_b200 as V
    g, bs, placed, offsets, P, D, step = _setup(64, W.SEED_BASE + 43)
    plan = V.BasketPlan(g, [(pv, o, b.n) for pv, o, b in zip(placed, offsets, bs)], DTI | STI)
    first = _outs(P.size(), DTI | STI)
    plan.run(P, D, step, first)
    block, tile, ms = plan.tune(P, D, step, _outs(P.size(), DTI | STI), reps=2)
    assert block in (256, 512) and tile % block == 0 and ms > 0
    info = plan.info()
    assert (info["block"], info["tile"]) == (block, tile)
    second = _outs(P.size(), DTI | STI)
    plan.capture(P, D, step, second)
    plan.replay()
    plan.replay()
    torch.cuda.synchronize()
    for op in first:
        assert _same(first[op], second[op])


@pytest.mark.gpu
def test_basket_plan_rejects_bad_input():
    import vecgeom_b200 as V
    g, bs, placed, offsets, P, D, step = _setup(4, W.SEED_BASE + 47, max_n=64)
    with pytest.raises(V.VgbError):
        V.BasketPlan(g, [(placed[0], -1, 5)], DTI)
    with pytest.raises(V.VgbError):
        V.BasketPlan(g, [(placed[0], 0, 5)], 1 << 9)
    with pytest.raises(V.VgbError):
        V.BasketPlan(g, [(placed[0], 0, 5)], DTI, block=96)
    plan = V.BasketPlan(g, [(placed[0], 0, 5)], DTI)
    with pytest.raises(V.VgbError):
        plan.run(P, None, None, _outs(P.size(), DTI))
