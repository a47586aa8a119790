"""The device's acos and atan (interflect_b200/csrc/libm_f32.h, the fdlibm
algorithms that glibc's acosf and atanf implement) against the platform
libm on every float: the quad-light form factor (ltc.rs) and the sphere-light
extension depend on them, and the oracle calls glibc. The same header is
compiled for the host with -ffp-contract=off, as the device build disables
FMA contraction."""
import os
import subprocess

from conftest import ROOT


def test_acos_and_atan_equal_glibc_on_every_float(tmp_path):
    exe = str(tmp_path / "libm_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-pthread", "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "libm_check.cpp"), "-lm"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "every input agrees" in r.stdout
