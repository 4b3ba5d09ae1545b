"""The C++ drop-in classes (include/fluid/PBFluids.h, SDFBoundary.h) compile
for a caller written against the reference's interface (CPU), and run it
(GPU)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "realtime-fsi-engine_b200", "lib")


def build(tmp_path):
    exe = str(tmp_path / "dropin_main")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-Wall", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"), "-L" + LIBDIR, "-lpbf_b200",
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
