"""Navigation server (continuous batching) on the layered detector.

Each request's per-track results (step count, final point, FNV-1a hash of its
(next placed id, step, safety) records) must equal the reference's own
SimpleNavigator trace of the same tracks (FindNextBoundaryAndStep + GetSafety,
navigation/SimpleNavigator.h:340-596, run by oracle/_ref in a fresh process),
whether the request is served alone or while other requests of uneven sizes
arrive and finish around it.
"""
import os
import sys

import numpy as np
import pytest

import oracle
from vecgeom_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))

MAX_STEPS = 48


def fnv1a(data: bytes, h: int = 0xcbf29ce484222325) -> int:
    for b in data:
        h ^= b
        h = (h * 0x100000001b3) & 0xffffffffffffffff
    return h


def fnv_hash(ids, steps, safeties):
    """FNV-1a 64 over the little-endian bytes of (int32 id, float64 step,
    float64 safety) records."""
    return fnv1a(b"".join(np.int32(i).tobytes() + np.float64(s).tobytes() +
                          np.float64(f).tobytes() for i, s, f in zip(ids, steps, safeties)))


def test_fnv1a_known_answers():
    # published FNV-1a 64 test vectors
    assert fnv1a(b"") == 0xcbf29ce484222325
    assert fnv1a(b"a") == 0xaf63dc4c8601ec8c
    assert fnv1a(b"foobar") == 0x85944171f73967e8


def requests(sizes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k, n in enumerate(sizes):
        if k % 2:
            pts, dirs = W.isotropic_tracks(n, seed + k)
        else:
            _, dirs = W.isotropic_tracks(n, seed + k)
            pts = (rng.uniform(-1000, 1000, n), rng.uniform(-1000, 1000, n),
                   rng.uniform(-1200, 1200, n))
        out.append((pts, dirs))
    return out


def reference_truth(reqs):
    """Per request: the reference's trace results of its tracks (one traced
    batch of all requests' tracks, split back per request)."""
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_nav_golden import reference_trace_isolated
    pts = tuple(np.concatenate([r[0][j] for r in reqs]) for j in range(3))
    dirs = tuple(np.concatenate([r[1][j] for r in reqs]) for j in range(3))
    ids, steps, saf, nst = reference_trace_isolated(pts, dirs, MAX_STEPS, os.cpu_count() or 1)
    out, b = [], 0
    for r in reqs:
        m = len(r[0][0])
        sl = slice(b * MAX_STEPS, (b + m) * MAX_STEPS)
        out.append(truth_of(r[0], r[1], ids[sl], steps[sl], saf[sl], nst[b:b + m]))
        b += m
    return out


def truth_of(pts, dirs, ids, steps, saf, nst):
    n = len(pts[0])
    ids = ids.reshape(n, MAX_STEPS)
    steps = steps.reshape(n, MAX_STEPS)
    saf = saf.reshape(n, MAX_STEPS)
    hashes = np.array([fnv_hash(ids[i, :nst[i]], steps[i, :nst[i]], saf[i, :nst[i]])
                       for i in range(n)], np.uint64)
    fx = np.array(pts[0], np.float64).copy()
    fy = np.array(pts[1], np.float64).copy()
    fz = np.array(pts[2], np.float64).copy()
    for i in range(n):
        for k in range(nst[i]):
            fx[i] = fx[i] + dirs[0][i] * steps[i, k]
            fy[i] = fy[i] + dirs[1][i] * steps[i, k]
            fz[i] = fz[i] + dirs[2][i] * steps[i, k]
    return {"nsteps": nst, "hash": hashes, "x": fx, "y": fy, "z": fz}


def serve(srv, reqs, arrivals):
    """Submits request k once `arrivals[k]` iterations have run; returns results."""
    order = list(range(len(reqs)))
    pending = sorted(order, key=lambda k: arrivals[k])
    it = 0
    rid_of = {}
    results = {}
    while pending or len(results) < len(reqs):
        while pending and arrivals[pending[0]] <= it:
            k = pending.pop(0)
            rid_of[srv.submit(*reqs[k])] = k
        done, live, queued = srv.step()
        for rid in done:
            results[rid_of[rid]] = srv.result(rid)
        it += 1
        assert it < 10000
    return results


def assert_same(res, want, what):
    for key in ("nsteps", "hash", "x", "y", "z"):
        assert np.array_equal(res[key], want[key]), f"{what}: {key} differs"


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.RefLib.available(), reason="oracle/_ref not built")
def test_served_alone_and_in_the_mix_match_the_reference():
    import vecgeom_b200 as V
    sizes = [300, 17, 1000, 1, 513, 2048, 64, 777]
    reqs = requests(sizes, W.SEED_BASE + 91)
    truth = reference_truth(reqs)
    g = V.Geometry()
    W.build_detector(W.VgbBuilder(g))
    # small slot table so admission has to wait for retirements
    for precision in (0, 1):
        srv = V.NavServer(g, max_tracks=2560, steps_per_launch=5, max_steps=MAX_STEPS,
                          precision=precision)
        mixed = serve(srv, reqs, arrivals=[0, 0, 1, 2, 2, 3, 7, 9])
        for k in range(len(reqs)):
            assert_same(mixed[k], truth[k], f"request {k} in the mix (precision {precision})")
    for k in (0, 5):
        alone = serve(V.NavServer(g, max_tracks=4096, steps_per_launch=3, max_steps=MAX_STEPS),
                      [reqs[k]], arrivals=[0])
        assert_same(alone[0], truth[k], f"request {k} alone")


@pytest.mark.gpu
def test_server_capacity_and_errors():
    import vecgeom_b200 as V
    g = V.Geometry()
    W.build_detector(W.VgbBuilder(g))
    srv = V.NavServer(g, max_tracks=512, steps_per_launch=4, max_steps=MAX_STEPS)
    assert srv.max_tracks == 512
    pts, dirs = W.isotropic_tracks(600, 5)
    with pytest.raises(V.VgbError):
        srv.submit(pts, dirs)
    rid = srv.submit(*W.isotropic_tracks(0, 5))
    done, live, queued = srv.step()
    assert rid in done or srv.result(rid)["nsteps"].size == 0
    with pytest.raises(V.VgbError):
        srv.result(12345)


@pytest.mark.gpu
def test_small_request_passes_a_large_one_that_does_not_fit():
    """Admission is not strictly first come first served: with 10 chunks of
    slots, a 2048-track request (8 chunks) running and a second one queued that
    does not fit, a 64-track request that arrives after it is admitted into the
    two free chunks and finishes first."""
    import vecgeom_b200 as V
    g = V.Geometry()
    W.build_detector(W.VgbBuilder(g))
    srv = V.NavServer(g, max_tracks=2560, steps_per_launch=2, max_steps=MAX_STEPS)
    a = srv.submit(*W.isotropic_tracks(2048, W.SEED_BASE + 95))
    srv.step()
    b = srv.submit(*W.isotropic_tracks(2048, W.SEED_BASE + 96))
    c = srv.submit(*W.isotropic_tracks(64, W.SEED_BASE + 97))
    order = []
    for _ in range(10000):
        done, live, queued = srv.step()
        order += list(done)
        if len(order) == 3:
            break
    assert set(order) == {a, b, c}
    assert order.index(c) < order.index(b), order
