"""The C++ facade (include/ag2d_simulation.hpp): reference-style scene code compiles against it and links to the
library. Without a device the program reports it; on a GPU it steps the scene through Simulation::update."""
import os
import shutil
import subprocess

import pytest

from conftest import LIB_DIR, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp")


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not installed")
    lib = os.path.join(LIB_DIR, "libag2d.so")
    if not os.path.exists(lib):
        pytest.skip("libag2d.so is not built")
    exe = str(tmp_path / "facade_demo")
    subprocess.run(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-L", LIB_DIR, "-lag2d",
                    f"-Wl,-rpath,{LIB_DIR}", "-o", exe], check=True)
    return exe


def test_facade_compiles_and_runs(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith(("no-device", "ok ")), out.stdout


@pytest.mark.gpu
def test_facade_steps_scene_on_gpu(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    fields = out.stdout.split()
    assert fields[0] == "ok", out.stdout
    bodies, manifolds, mean_y = int(fields[1]), int(fields[2]), float(fields[3])
    assert bodies == 68 and manifolds > 0   # ground, 60 pile bodies, a capsule, a destroyed circle, a dumbbell,
    #                                         a static hook and a three-link chain on revolute joints
    assert int(fields[6]) == 67             # colliders in the trees: 63 live bodies, four more on the dumbbell
    #                                         (its two wheels and the two convex pieces of its concave bracket)
    assert -1.0 < mean_y < 6.0   # the pile has fallen onto the ground (spawned between y = 1 and 8.5)
    found, touching = int(fields[4]), int(fields[5])   # the editor-style circle query around the pile's base
    assert 0 < touching <= found
    impacts, largest = int(fields[7]), float(fields[8])   # collision callback on the ground's collider, threshold 0.5
    assert impacts > 0 and largest >= 0.5
