"""Continuous collision detection against the reference engine's own continuous-collision pass, through the C ABI.

The fixture (tests/golden/c5_ccd_hit.npz, made by tests/golden/make_golden.py) is the first step of a
serving-style request (c1 mix with 5% small circles at 200 m/s) in which the reference moved a body back: the state
entering the step ("pre."), after the spatial pass ("sp.") and after the move-back ("ccd."). Here the same state is
loaded with its stale collider poses, integrated, posed and swept. Body positions, collider world positions and
AABBs after the move-back are bit-exact (the casts follow the reference's operation order), and the colliders'
min extents equal the reference's.
"""
import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")

FIXTURE = "c5_ccd_hit.npz"


def _world(d, ccd=True):
    it, g = d["meta.iters"], d["meta.gravity"]
    mats = [tuple(r) for r in d["meta.materials"]]
    w = ag2d.World(dt=float(d["meta.dt"][0]), velocity_iterations=int(it[0]), position_iterations=int(it[1]),
                   gravity=(float(g[0]), float(g[1])), ccd=ccd)
    w.load_state(d, "pre.", mats, with_poses=True)
    return w


def _run(w, d):
    w.run_phase(ag2d.PHASE_INTEGRATE)
    w.run_phase(ag2d.PHASE_SPATIAL_FULL if int(d["sp.spatialDirty"][0]) else ag2d.PHASE_SPATIAL_DYNAMIC)
    w.run_phase(ag2d.PHASE_CCD)


def test_ccd_moves_bodies_back_like_the_reference():
    d = parity.load(FIXTURE)
    w = _world(d)
    _run(w, d)
    assert w.counters()["ccd_hits"] > 0
    for field, key in ((ag2d.BODY_COM_X, "ccd.body.comX"), (ag2d.BODY_COM_Y, "ccd.body.comY")):
        assert parity.mismatches(w.read(field), d[key]) == 0, key
    for field, key in ((ag2d.COL_WORLD_X, "ccd.col.worldPosX"), (ag2d.COL_WORLD_Y, "ccd.col.worldPosY"),
                       (ag2d.COL_AABB_MIN_X, "ccd.col.aabbMinX"), (ag2d.COL_AABB_MIN_Y, "ccd.col.aabbMinY"),
                       (ag2d.COL_AABB_MAX_X, "ccd.col.aabbMaxX"), (ag2d.COL_AABB_MAX_Y, "ccd.col.aabbMaxY")):
        assert parity.mismatches(w.read(field), d[key]) == 0, key


def test_ccd_hit_count_matches_the_reference():
    d = parity.load(FIXTURE)
    w = _world(d)
    _run(w, d)
    # Bodies the reference moved: post-CCD position differs from the position the spatial pass saw.
    sp_x = d["sp.col.worldPosX"]
    ccd_x = d["ccd.col.worldPosX"]
    body = d["pre.col.bodyIndex"]
    ref_moved = np.unique(body[(sp_x != ccd_x) | (d["sp.col.worldPosY"] != d["ccd.col.worldPosY"])])
    assert w.counters()["ccd_hits"] == ref_moved.size


def test_ccd_off_leaves_tunnelling_bodies_alone():
    d = parity.load(FIXTURE)
    w = _world(d, ccd=False)
    w.run_phase(ag2d.PHASE_INTEGRATE)
    w.run_phase(ag2d.PHASE_SPATIAL_FULL if int(d["sp.spatialDirty"][0]) else ag2d.PHASE_SPATIAL_DYNAMIC)
    assert parity.mismatches(w.read(ag2d.COL_WORLD_Y), d["sp.col.worldPosY"]) == 0
