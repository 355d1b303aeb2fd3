"""The basket navigation interface (navigation/SimpleNavigator.h:599-743):
FindNextBoundaryAndStep over a basket, with DistanceToOut's node index,
DistanceToInMinimize over the daughters and the 1e-9 relocation push, and
GetSafeties.  Tracks start from points spread over the layered detector and
take 0-3 single steps first, so the basket step starts on boundaries too; half
of them propose a physical step of U(0, 50) mm.  Against tests/golden/nav/
basket.npz (written by the reference, tests/golden/make_nav_golden.py) and the
live reference, bit for bit:
  * CPU: Navigator::step_basket built for the host (hc_nav_basket);
  * GPU: vgb_nav_locate, vgb_nav_find_next_boundary_and_step for the prior
    steps, then vgb_nav_find_next_boundary_and_step_basket.
"""
import numpy as np
import pytest

import oracle
from make_nav_golden import basket_inputs, reference_basket_isolated
from navhelpers import (BASKET_KEYS, NAV_GOLDEN, assert_basket_equal, build, dev, host_basket,
                        load_hostcheck)


def fixture():
    d = np.load(NAV_GOLDEN + "/basket.npz")
    pts = (d["x"], d["y"], d["z"])
    dirs = (d["dx"], d["dy"], d["dz"])
    return d, pts, dirs, d["pstep"], [int(p) for p in d["priors"]]


def want_of(d, prior):
    return {k: d[f"{k}_{prior}"] for k in BASKET_KEYS}


@pytest.fixture(scope="module")
def hc():
    return load_hostcheck()


def test_host_basket_matches_fixture(hc):
    d, pts, dirs, pstep, priors = fixture()
    for prior in priors:
        got = host_basket(hc, "detector", pts, dirs, pstep, prior)
        assert_basket_equal(got, want_of(d, prior), f"host, {prior} prior steps")


def test_fixture_exercises_every_branch():
    d, _, _, _, priors = fixture()
    nodes = np.concatenate([d[f"nextnode_{p}"] for p in priors])
    bnd = np.concatenate([d[f"boundary_{p}"] for p in priors])
    assert (nodes == -1).any() and (nodes == -2).any() and (nodes >= 0).any()
    assert (bnd == 0).any() and (bnd == 1).any()


@pytest.mark.skipif(not oracle.RefLib.available(), reason="oracle/_ref not built")
def test_host_basket_matches_reference_more_tracks(hc):
    pts, dirs, pstep = basket_inputs(4000)
    want = reference_basket_isolated(pts, dirs, pstep, (0, 2, 5))
    for prior in (0, 2, 5):
        got = host_basket(hc, "detector", pts, dirs, pstep, prior)
        assert_basket_equal(got, {k: want[f"{k}_{prior}"] for k in BASKET_KEYS},
                            f"host vs reference, {prior} prior steps")


@pytest.mark.gpu
def test_gpu_basket_matches_fixture():
    import torch
    import vecgeom_b200 as V
    d, pts, dirs, pstep, priors = fixture()
    n = len(pts[0])
    g, placed = build(None, "detector", close=True)
    pos = {int(p.id): k for k, p in enumerate(placed)}
    nav = V.SimpleNavigator(g)
    D = V.SOA3D(*(dev(v) for v in dirs))
    big = torch.full((n,), 1e30, dtype=torch.float64, device="cuda")
    ps = dev(pstep)
    for prior in priors:
        a, b = V.NavStatePool(g, n), V.NavStatePool(g, n)
        P = [dev(v) for v in pts]
        nav.LocatePoint(V.SOA3D(*P), a)
        step = torch.zeros(n, dtype=torch.float64, device="cuda")
        for _ in range(prior):
            nav.FindNextBoundaryAndStep(V.SOA3D(*P), D, a, b, big, step)
            P = [P[j] + Dj * step for j, Dj in enumerate((D.x, D.y, D.z))]
            a, b = b, a
        dist = torch.zeros(n, dtype=torch.float64, device="cuda")
        saf = torch.zeros(n, dtype=torch.float64, device="cuda")
        node = torch.zeros(n, dtype=torch.int32, device="cuda")
        nav.FindNextBoundaryAndStepBasket(V.SOA3D(*P), D, a, b, ps, dist, saf, node)
        torch.cuda.synchronize()
        want = want_of(d, prior)
        inside = want["nextnode"] != -7
        got = {"px": P[0].cpu().numpy(), "py": P[1].cpu().numpy(), "pz": P[2].cpu().numpy()}
        for k in ("px", "py", "pz"):
            assert np.array_equal(got[k], want[k]), f"{k} after {prior} prior steps"
        st = b.to_numpy()
        tops = b.tops()
        new_top = np.array([pos[int(t)] if t >= 0 else -1 for t in tops], np.int32)
        checks = {"distance": dist.cpu().numpy(), "safety": saf.cpu().numpy(),
                  "nextnode": node.cpu().numpy(), "newtop": new_top,
                  "boundary": st["onBoundary"].astype(np.int32)}
        for k, v in checks.items():
            a_, b_ = v[inside], want[k][inside]
            same = (a_ == b_) | (np.isnan(a_) & np.isnan(b_)) if a_.dtype.kind == "f" else a_ == b_
            assert same.all(), f"{k} after {prior} prior steps: tracks {np.flatnonzero(~same)[:6]}"
    assert nav.error_flags() == 0
