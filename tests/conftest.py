import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
SCENES = os.path.join(ROOT, "tests", "golden", "scenes")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")


def scene_src(name: str) -> str:
    with open(os.path.join(SCENES, name if name.endswith(".rad") else name + ".rad")) as f:
        return f.read()


@pytest.fixture(scope="session", autouse=True)
def _built_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


@pytest.fixture(scope="session")
def gpu_ctx():
    import interflect_b200 as ifx
    ctx = ifx.Context(0)
    yield ctx
    ctx.close()
