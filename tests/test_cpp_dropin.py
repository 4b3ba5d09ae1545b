"""The C++ drop-in classes (include/fluid/PBFluids.h, SDFBoundary.h) compile
for a caller written against the reference's interface (CPU), and run it
(GPU)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "realtime-fsi-engine_b200", "lib")


def build(tmp_path, name="dropin_main"):
    exe = str(tmp_path / name)
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L" + LIBDIR, "-lpbf_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_dropin_caller_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_dropin_caller_runs(have_gpu, tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["particles"] == 4096 and out["nonfinite"] == 0 and out["inside_obstacle"] == 0
    assert out["contacts"] > 0 and out["closest_face"] >= 0


def test_scene_caller_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path, "scene_main"))


@pytest.mark.gpu
def test_scene_caller_runs_container_preset(have_gpu, tmp_path):
    """include/core/SceneSetup.h's loadScene from C++: the Container Cube
    preset (16,384 particles spawned inside a 4.5-unit cube held by the SDF),
    30 frames; no particle leaves the cube."""
    exe = build(tmp_path, "scene_main")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["particles"] == 16384 and out["mesh_vertices"] == 1538 and out["mesh_faces"] == 3072
    assert out["nonfinite"] == 0 and out["outside"] == 0
