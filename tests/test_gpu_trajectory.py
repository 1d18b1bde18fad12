"""600-step trajectory of a 256-polygon drop (c1 mix, seed 0) against the reference engine's own trajectory.

The solver's colouring changes the Gauss-Seidel order, so the two runs are not bit-identical and a falling pile
diverges chaotically in its details. The comparison is on the statistics the parity contract names, each with its
tolerance written here:
  - free fall (steps 0-39, before the bodies reach the ground): vertical momentum within 1e-4 relative, kinetic
    energy within 1e-3 relative (initial overlaps are resolved in another order, nothing else differs);
  - energy drift: the kinetic-energy peak of the fall within 5 % and reached within 10 steps of the reference's;
  - momentum: total vertical momentum at its extreme within 5 %; horizontal momentum stays below 3 % of it;
  - penetration: the deepest contact after the first 20 steps no more than 1.5 x the reference's deepest (+1 cm);
  - the settled pile: contact count over the last 100 steps within 20 % of the reference's.
The reference trajectory (tests/golden/traj_c1_n256.npz) is the compiled reference engine run by
tests/golden/make_golden.py.
"""
import json
import os

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
from ag2d import scenes  # noqa: E402


def _trajectory(steps=600):
    sc = scenes.make_c1(256, 0)
    w = ag2d.World.from_scene(sc)
    w.step(0)
    out = {k: [] for k in ("px", "py", "ke", "max_depth", "manifolds", "sleeping")}
    inv_m = inv_i = None
    for _ in range(steps):
        w.step(1)
        if inv_m is None:
            inv_m = w.read(ag2d.BODY_INV_MASS).astype(np.float64)
            inv_i = w.read(ag2d.BODY_INV_INERTIA).astype(np.float64)
        dyn = inv_m > 0
        m = np.where(dyn, 1.0 / np.where(dyn, inv_m, 1.0), 0.0)
        inertia = np.where(inv_i > 0, 1.0 / np.where(inv_i > 0, inv_i, 1.0), 0.0)
        vx = w.read(ag2d.BODY_VEL_X).astype(np.float64)
        vy = w.read(ag2d.BODY_VEL_Y).astype(np.float64)
        om = w.read(ag2d.BODY_ANGULAR_VELOCITY).astype(np.float64)
        out["px"].append(float(np.sum((m * vx)[dyn])))
        out["py"].append(float(np.sum((m * vy)[dyn])))
        out["ke"].append(float(0.5 * np.sum((m * (vx * vx + vy * vy) + inertia * om * om)[dyn])))
        man = w.read(ag2d.PREV_MANIFOLDS)
        out["max_depth"].append(float(man["depth"].max()) if man.size else 0.0)
        out["manifolds"].append(int(man.size))
        out["sleeping"].append(int(np.sum(w.read(ag2d.BODY_STATE) == 1)))
    return {k: np.asarray(v) for k, v in out.items()}


@pytest.fixture(scope="module")
def runs():
    ref = parity.load("traj_c1_n256.npz")
    gpu = _trajectory()
    out_dir = os.environ.get("AG2D_TRAJ_OUT")
    if out_dir:
        with open(os.path.join(out_dir, "traj_c1_n256_gpu.json"), "w") as f:
            json.dump({k: v.tolist() for k, v in gpu.items()}, f)
    return {k: np.asarray(ref[k], np.float64) for k in gpu}, gpu


def test_free_fall_matches(runs):
    ref, gpu = runs
    sl = slice(0, 40)
    np.testing.assert_allclose(gpu["py"][sl], ref["py"][sl], rtol=1e-4)
    np.testing.assert_allclose(gpu["ke"][sl], ref["ke"][sl], rtol=1e-3)


def test_energy_peak(runs):
    ref, gpu = runs
    assert abs(gpu["ke"].max() - ref["ke"].max()) <= 0.05 * ref["ke"].max()
    assert abs(int(np.argmax(gpu["ke"])) - int(np.argmax(ref["ke"]))) <= 10


def test_momentum(runs):
    ref, gpu = runs
    peak_ref, peak_gpu = ref["py"].min(), gpu["py"].min()
    assert abs(peak_gpu - peak_ref) <= 0.05 * abs(peak_ref)
    assert np.abs(gpu["px"]).max() <= 0.03 * abs(peak_gpu)


def test_penetration(runs):
    ref, gpu = runs
    assert gpu["max_depth"][20:].max() <= 1.5 * ref["max_depth"][20:].max() + 0.01


def test_settled_contacts(runs):
    ref, gpu = runs
    r, g = ref["manifolds"][-100:].mean(), gpu["manifolds"][-100:].mean()
    assert abs(g - r) <= 0.2 * r
