"""CPU: the C oracle restatement against the reference's golden vectors.

tests/golden/*.npz were written by the reference VecGeom Scalar backend
(tests/golden/make_golden.py).  This pins oracle/vgb_oracle.c: Contains and
Inside bit-exact, distances and safeties within 1e-9 mm or 1e-12 relative.
"""
import glob
import json
import os

import numpy as np
import pytest

import oracle
from helpers import PLACEMENTS, assert_distances, assert_exact, oracle_unplaced, \
    oracle_generic_xform
from vecgeom_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
ORACLE_SHAPES = {"box", "tube"}


def load_case(path):
    d = np.load(path)
    meta = json.loads(str(d["spec"]))
    return d, meta


def spec_from_meta(meta):
    p = meta["params"]
    k = meta["kind"]
    ctor = {"box": W.box_spec, "tube": W.tube_spec, "cone": W.cone_spec,
            "sphere": W.sphere_spec, "torus": W.torus_spec, "trd": W.trd_spec,
            "polycone": W.polycone_spec, "polyhedron": W.polyhedron_spec,
            "boolsub": W.boolsub_spec, "orb": W.orb_spec,
            "parallelepiped": W.parallelepiped_spec, "paraboloid": W.paraboloid_spec,
            "trapezoid": W.trapezoid_spec,
            "trapezoidcorners": W.trapezoid_corners_spec}.get(k)
    if ctor is None:
        return W.boolean_spec(k, **p)
    return ctor(**p)


@pytest.fixture(scope="module")
def orc():
    oracle.build(with_ref=False)
    return oracle.Oracle()


def test_golden_fixtures_present():
    kinds = {os.path.basename(p).split("_")[0] for p in GOLDEN}
    assert {"box", "tube", "cone", "sphere", "torus", "polycone", "polyhedron", "boolsub",
            "trd"} <= kinds


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference(orc, path):
    d, meta = load_case(path)
    if meta["kind"] not in ORACLE_SHAPES:
        pytest.skip(f"oracle restatement of {meta['kind']} not present")
    spec = spec_from_meta(meta)
    shape = oracle_unplaced(orc, spec)
    xf = orc.xform(*PLACEMENTS[str(d["placement"])], generic=oracle_generic_xform(spec))
    pm = (d["mx"], d["my"], d["mz"])
    dm = (d["mdx"], d["mdy"], d["mdz"])
    pl = (d["lx"], d["ly"], d["lz"])
    dl = (d["ldx"], d["ldy"], d["ldz"])
    step = d["step"]
    assert_exact(orc.batch(shape, xf, oracle.CONTAINS, pm), d["contains"], "Contains")
    assert_exact(orc.batch(shape, xf, oracle.INSIDE, pm), d["inside"], "Inside")
    assert_distances(orc.batch(shape, xf, oracle.SAFETY_TO_IN, pm), d["safety_to_in"],
                     "SafetyToIn")
    assert_distances(orc.batch(shape, xf, oracle.SAFETY_TO_OUT, pl), d["safety_to_out"],
                     "SafetyToOut")
    assert_distances(orc.batch(shape, xf, oracle.DISTANCE_TO_IN, pm, dm, step),
                     d["distance_to_in"], "DistanceToIn")
    assert_distances(orc.batch(shape, xf, oracle.DISTANCE_TO_OUT, pl, dl, step),
                     d["distance_to_out"], "DistanceToOut")
