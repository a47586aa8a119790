"""The reasoning behind the per-cell candidate-leaf query of cone-shadow
marches (device.cuh dist_fast), checked on the CPU: tests/cpp/leafgrid_check
restates the grid and the exactness test over the oracle's scene and, at
points along shadow-style marches in the stress scenes, requires every
answer the test accepts to give the march what the oracle's traversal gives
it (both below the stop, or bit-equal)."""
import os
import subprocess

import pytest

from conftest import ROOT

SRCS = ["scene.cpp", "gi.cpp", "render.cpp", "diff.cpp"]


@pytest.mark.parametrize("scene", ["interflect_b200/scenes/c3_stress.rad", "tests/golden/scenes/stress.rad"])
def test_accepted_leaf_list_answers_equal_the_reference_traversal(tmp_path, scene):
    exe = str(tmp_path / "leafgrid_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "oracle"), "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "leafgrid_check.cpp")] +
                   [os.path.join(ROOT, "oracle", s) for s in SRCS] + ["-lpthread"], check=True)
    r = subprocess.run([exe, os.path.join(ROOT, scene)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "every accepted answer equals the reference traversal" in r.stdout
