"""vgb_basket_run_noalloc: the basket launch for callers that cannot allocate.

Some callers cannot call cudaMalloc in the middle of their work: frameworks that
hand all of the GPU's memory to their own pool allocator when they start, and
online event loops where an allocation could stall or fail during a run.  For
them the library has one entry point that allocates nothing: it keeps its
basket tables in a fixed array compiled into the library instead of in a plan.
This file checks it through the C ABI against the allocating entry point
(vgb_basket_run through a plan), on two calls in a row, and its size limit.
It is collected last, so a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from vecgeom_b200 import workloads as W

DTI, STI = 1 << 2, 1 << 4  # op masks: DistanceToIn, SafetyToIn


class CBasket(ctypes.Structure):
    _fields_ = [("placed", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("offset", ctypes.c_int64), ("count", ctypes.c_int64)]


def _setup(nb, seed):
    import torch
    import vecgeom_b200 as V
    bs = W.config4_baskets(nb, seed=seed)
    for b in bs:
        b.n = min(b.n, 2500)
    g = V.Geometry()
    placed, offsets, pts, dirs, step = W.build_baskets(g, bs)
    g.CloseGeometry()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return g, bs, placed, offsets, [dev(a) for a in (*pts, *dirs, step)]


def _noalloc(g, table, ops, arrays, outs):
    import vecgeom_b200 as V
    L = V.lib()
    arr = (CBasket * max(1, len(table)))()
    for k, (pv, off, cnt) in enumerate(table):
        arr[k].placed, arr[k].offset, arr[k].count = pv.id, off, cnt
    o = (ctypes.c_void_p * 6)()
    for op, t in outs.items():
        o[op] = t.data_ptr()
    return L.vgb_basket_run_noalloc(g.handle, arr, len(table), ops,
                                    *(a.data_ptr() for a in arrays), o, 0, None)


def _outs(n):
    import torch
    return {2: torch.full((n,), -5., dtype=torch.float64, device="cuda"),
            4: torch.full((n,), -5., dtype=torch.float64, device="cuda")}


def _same(a, b):
    return bool(((a == b) | (a.isnan() & b.isnan())).all())


@pytest.mark.gpu
def test_noalloc_matches_the_plan_on_two_calls_in_a_row():
    import torch
    import vecgeom_b200 as V
    g, bs, placed, offsets, arrays = _setup(80, W.SEED_BASE + 61)
    n = len(arrays[0])
    table = [(pv, o, b.n) for pv, o, b in zip(placed, offsets, bs)]
    P = V.SOA3D(*arrays[:3])
    D = V.SOA3D(*arrays[3:6])
    want = _outs(n)
    V.BasketPlan(g, table, DTI | STI).run(P, D, arrays[6], want)
    # first call: every basket; second call: every other basket, in reverse,
    # over fresh outputs (the array still holds the first call's tables)
    got1 = _outs(n)
    assert _noalloc(g, table, DTI | STI, arrays, got1) == 0
    sub = table[::-2]
    got2 = _outs(n)
    assert _noalloc(g, sub, DTI | STI, arrays, got2) == 0
    torch.cuda.synchronize()
    for op in want:
        assert _same(got1[op], want[op]), f"first call, op {op}"
    covered = torch.zeros(n, dtype=torch.bool, device="cuda")
    for pv, off, cnt in sub:
        covered[off:off + cnt] = True
    for op in want:
        assert _same(got2[op][covered], want[op][covered]), f"second call, op {op}"
        assert bool((got2[op][~covered] == -5.).all()), "second call wrote outside its baskets"


@pytest.mark.gpu
def test_noalloc_at_its_limit_with_empty_baskets():
    """Exactly VGB_NOALLOC_MAX_BASKETS small baskets, every seventh one empty:
    the table kernel then scans 8 baskets per thread and fills the last prefix
    entry.  Compared with the plan on two calls in a row, the second from a
    pinned host array that is overwritten as soon as the call returns."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import _lib
    nb = _lib.NOALLOC_MAX_BASKETS
    bs = W.config4_baskets(nb, seed=W.SEED_BASE + 65)
    for b in bs:
        b.n = min(b.n, 24)
    g = V.Geometry()
    placed, offsets, pts, dirs, step = W.build_baskets(g, bs)
    g.CloseGeometry()
    arrays = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (*pts, *dirs, step)]
    n = len(arrays[0])
    table = [(pv, o, 0 if k % 7 == 3 else b.n)
             for k, (pv, o, b) in enumerate(zip(placed, offsets, bs))]
    want = _outs(n)
    V.BasketPlan(g, table, DTI | STI).run(V.SOA3D(*arrays[:3]), V.SOA3D(*arrays[3:6]),
                                          arrays[6], want)
    got1 = _outs(n)
    assert _noalloc(g, table, DTI | STI, arrays, got1) == 0
    # second call from pinned host memory, scribbled over right after the call
    L = V.lib()
    pinned = torch.empty(nb * ctypes.sizeof(CBasket), dtype=torch.uint8).pin_memory()
    arr = (CBasket * nb).from_address(pinned.data_ptr())
    for k, (pv, off, cnt) in enumerate(table):
        arr[k].placed, arr[k].offset, arr[k].count = pv.id, off, cnt
    o = (ctypes.c_void_p * 6)()
    got2 = _outs(n)
    for op, t in got2.items():
        o[op] = t.data_ptr()
    assert L.vgb_basket_run_noalloc(g.handle, arr, nb, DTI | STI,
                                    *(a.data_ptr() for a in arrays), o, 0, None) == 0
    for k in range(nb):
        arr[k].count = 0
    torch.cuda.synchronize()
    empty = torch.zeros(n, dtype=torch.bool, device="cuda")
    for k, (pv, off, cnt) in enumerate(table):
        if cnt == 0:
            empty[off:off + bs[k].n] = True
    for op in want:
        assert _same(got1[op], want[op]), f"first call, op {op}"
        assert _same(got2[op], want[op]), f"second call (pinned array), op {op}"
        assert bool((got1[op][empty] == -5.).all()), "an empty basket was written"


@pytest.mark.gpu
def test_noalloc_rejects_more_baskets_than_its_table():
    import vecgeom_b200 as V
    from vecgeom_b200 import _lib
    g, bs, placed, offsets, arrays = _setup(2, W.SEED_BASE + 63)
    n = len(arrays[0])
    table = [(placed[0], 0, 1)] * (_lib.NOALLOC_MAX_BASKETS + 1)
    st = _noalloc(g, table, DTI | STI, arrays, _outs(n))
    assert st == _lib.ENOSPC
    assert b"exceed" in V.lib().vgb_last_error()
