"""The shading passes take pixels in 8 x 4 tiles (interflect_b200/csrc/
pixorder.h). This compiles the header for the host and checks that the order
is a permutation of the film for sizes with and without partial tiles."""
import os
import subprocess

from conftest import ROOT


def test_tile_order_is_a_permutation(tmp_path):
    exe = str(tmp_path / "pixorder_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, os.path.join(ROOT, "tests", "cpp", "pixorder_check.cpp")],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "permutation" in r.stdout
