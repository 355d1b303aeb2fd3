"""Baskets: many shape instances of mixed types in one persistent launch.

The basket kernel runs the same per-point functions as vgb_batch_fused, so its
results must equal, bit for bit, one fused call per basket; the tuned launch
shape and the CUDA-graph replay must not change them.
"""
import numpy as np
import pytest

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


def _per_basket(placed, offsets, bs, P, D, step, ops):
    import vecgeom_b200 as V
    n = P.size()
    ref = _outs(n, ops)
    for pv, off, b in zip(placed, offsets, bs):
        if b.n == 0:
            continue
        sl = slice(off, off + b.n)
        pv.fused(ops, V.SOA3D(P.x[sl], P.y[sl], P.z[sl]), {k: v[sl] for k, v in ref.items()},
                 dirs=V.SOA3D(D.x[sl], D.y[sl], D.z[sl]), step_max=step[sl])
    return ref


def _same(a, b):
    import torch
    if a.dtype == torch.float64:
        return bool(((a == b) | (torch.isnan(a) & torch.isnan(b))).all())
    return bool((a == b).all())


@pytest.mark.gpu
@pytest.mark.parametrize("ops", [DTI | STI, ALL], ids=["dti_sti", "all_ops"])
def test_baskets_match_per_basket_calls(ops):
    import torch
    import vecgeom_b200 as V
    g, bs, placed, offsets, P, D, step = _setup(96, W.SEED_BASE + 41)
    plan = V.BasketPlan(g, [(pv, o, b.n) for pv, o, b in zip(placed, offsets, bs)], ops)
    got = _outs(P.size(), ops)
    plan.run(P, D, step, got)
    torch.cuda.synchronize()
    want = _per_basket(placed, offsets, bs, P, D, step, ops)
    torch.cuda.synchronize()
    for op in got:
        assert _same(got[op], want[op]), f"op {op} differs"


@pytest.mark.gpu
def test_tuned_shape_and_graph_replay_keep_results():
    import torch
    import vecgeom_b200 as V
    g, bs, placed, offsets, P, D, step = _setup(64, W.SEED_BASE + 43)
    plan = V.BasketPlan(g, [(pv, o, b.n) for pv, o, b in zip(placed, offsets, bs)], DTI | STI)
    first = _outs(P.size(), DTI | STI)
    plan.run(P, D, step, first)
    block, tile, ms = plan.tune(P, D, step, _outs(P.size(), DTI | STI), reps=2)
    assert block in (128, 256, 512) and tile % block == 0 and ms > 0
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
