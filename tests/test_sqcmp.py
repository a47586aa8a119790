"""The BVH query compares squared box distances instead of box distances
(interflect_b200/csrc/sqcmp.h). This compiles the same header for the host
and checks it against comparing the correctly rounded square roots on 100 M
random, near-tie, subnormal and special operands."""
import os
import subprocess

from conftest import ROOT


def test_square_root_comparisons_are_exact(tmp_path):
    exe = str(tmp_path / "sqcmp_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "sqcmp_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cases agree" in r.stdout
