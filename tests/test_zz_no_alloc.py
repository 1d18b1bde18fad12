"""ag2d_solve_noalloc (the allocation-free solve) against the world's solver entry point, through the C ABI.

The same solver input (the reference's solver-input tap of a golden fixture) goes through AG2D_PHASE_SOLVE of a
world and through ag2d_solve_noalloc on caller-owned device tensors. Velocities, poses and impulses must agree
within 1e-6 relative (both run the same colouring and the same per-constraint arithmetic). Two calls in a row,
on two different scenes, check that the static scratch carries nothing from one call to the next. This file is
named to be collected last and passes alone or after the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

import parity

pytestmark = pytest.mark.gpu

ag2d = pytest.importorskip("ag2d")
torch = pytest.importorskip("torch")
from oracle import oraapi  # noqa: E402

RTOL, ATOL = 1e-6, 1e-7


class SolveView(ctypes.Structure):
    _fields_ = [("n_bodies", ctypes.c_uint32), ("body_velocity", ctypes.c_void_p), ("body_pose", ctypes.c_void_p),
                ("n_colliders", ctypes.c_uint32), ("collider_body", ctypes.c_void_p),
                ("collider_material", ctypes.c_void_p), ("n_materials", ctypes.c_uint32),
                ("materials", ctypes.c_void_p)]


def _lib():
    lib = ctypes.CDLL(ag2d.LIB_PATH)
    lib.ag2d_solve_noalloc.argtypes = [ctypes.POINTER(SolveView), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    lib.ag2d_solve_noalloc.restype = ctypes.c_int32
    lib.ag2d_last_error_string.restype = ctypes.c_char_p
    return lib


def _to_ag2d(m):
    out = np.zeros(m.shape[0], ag2d.MANIFOLD_DTYPE)
    for f in ("a", "b", "nx", "ny", "depth", "count"):
        out[f] = m[f]
    out["px0"], out["px1"] = m["px"][:, 0], m["px"][:, 1]
    out["py0"], out["py1"] = m["py"][:, 0], m["py"][:, 1]
    out["id0"], out["id1"] = m["id"][:, 0], m["id"][:, 1]
    out["jn0"], out["jn1"] = m["jn"][:, 0], m["jn"][:, 1]
    out["jt0"], out["jt1"] = m["jt"][:, 0], m["jt"][:, 1]
    return out


def _case(name):
    d = parity.load(name)
    if "svin.man.count" not in d:
        pytest.skip("no manifolds at this step")
    mats = [tuple(r) for r in d["meta.materials"]]
    it = d["meta.iters"]
    g = d["meta.gravity"]
    m_in = _to_ag2d(oraapi.manifolds_from_dump(d, "svin.man."))
    # Existing entry point: a world loaded with the solver input, solved by AG2D_PHASE_SOLVE.
    w = ag2d.World(dt=float(d["meta.dt"][0]), velocity_iterations=int(it[0]), position_iterations=int(it[1]),
                   gravity=(float(g[0]), float(g[1])))
    w.load_state(d, "svin.", mats)
    w.write(ag2d.MANIFOLDS, m_in)
    w.run_phase(ag2d.PHASE_SOLVE)
    want = {f: w.read(f) for f in (ag2d.BODY_VEL_X, ag2d.BODY_VEL_Y, ag2d.BODY_ANGULAR_VELOCITY, ag2d.BODY_COM_X,
                                   ag2d.BODY_COM_Y)}
    want_m = w.read(ag2d.MANIFOLDS)
    w.close()
    # The same input as caller-owned device tensors.
    b = lambda k: np.asarray(d["svin.body." + k], np.float32)
    vel = np.stack([b("velocityX"), b("velocityY"), b("angularVelocity"), b("invMass")], 1)
    pose = np.stack([b("comX"), b("comY"), b("rotation"), b("invInertia")], 1)
    mat = np.concatenate([np.asarray(mats, np.float32), np.zeros((len(mats), 1), np.float32)], 1)
    dev = torch.device("cuda:0")
    t = {
        "vel": torch.from_numpy(np.ascontiguousarray(vel)).to(dev),
        "pose": torch.from_numpy(np.ascontiguousarray(pose)).to(dev),
        "cbody": torch.from_numpy(np.asarray(d["svin.col.bodyIndex"], np.int32)).to(dev),
        "cmat": torch.from_numpy(np.asarray(d["svin.col.materialIndex"], np.int32)).to(dev),
        "mat": torch.from_numpy(np.ascontiguousarray(mat)).to(dev),
        "man": torch.from_numpy(m_in.view(np.uint8).copy()).to(dev),
        "status": torch.zeros(2, dtype=torch.int32, device=dev),
    }
    view = SolveView(vel.shape[0], t["vel"].data_ptr(), t["pose"].data_ptr(), t["cbody"].numel(),
                     t["cbody"].data_ptr(), t["cmat"].data_ptr(), mat.shape[0], t["mat"].data_ptr())
    return (int(it[0]), int(it[1])), m_in.shape[0], view, t, want, want_m


def _check(t, want, want_m):
    vel = t["vel"].cpu().numpy()
    pose = t["pose"].cpu().numpy()
    got = {ag2d.BODY_VEL_X: vel[:, 0], ag2d.BODY_VEL_Y: vel[:, 1], ag2d.BODY_ANGULAR_VELOCITY: vel[:, 2],
           ag2d.BODY_COM_X: pose[:, 0], ag2d.BODY_COM_Y: pose[:, 1]}
    for f, ref in want.items():
        np.testing.assert_allclose(got[f], ref, rtol=RTOL, atol=ATOL, err_msg=f"field {f}")
    man = t["man"].cpu().numpy().view(ag2d.MANIFOLD_DTYPE)
    for f in ("jn0", "jt0", "jn1", "jt1"):
        np.testing.assert_allclose(man[f], want_m[f], rtol=RTOL, atol=ATOL, err_msg=f)


def test_noalloc_matches_world_solver_two_calls_in_a_row():
    lib = _lib()
    stream = torch.cuda.current_stream()
    for name in ("c2_n2000_s1_step240.npz", "c1_n256_s0_step300.npz"):
        (vi, pi), n, view, t, want, want_m = _case(name)
        rc = lib.ag2d_solve_noalloc(ctypes.byref(view), t["man"].data_ptr(), n, vi, pi, stream.cuda_stream,
                                    t["status"].data_ptr())
        assert rc == 0, lib.ag2d_last_error_string()
        torch.cuda.synchronize()
        status, colors = (int(x) for x in t["status"].cpu())
        assert status == 0 and colors > 0, (status, colors)
        _check(t, want, want_m)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _lib()
    view = SolveView(16, None, None, 16, None, None, 1, None)
    rc = lib.ag2d_solve_noalloc(ctypes.byref(view), None, 16384 + 1, 8, 3, None, None)
    assert rc == ag2d.ERR_CAPACITY
    assert b"exceeds the static scratch limit 16384" in lib.ag2d_last_error_string()
    view.n_bodies = 16384 + 1
    rc = lib.ag2d_solve_noalloc(ctypes.byref(view), None, 0, 8, 3, None, None)
    assert rc == ag2d.ERR_CAPACITY
