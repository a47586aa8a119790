"""The bounds-checked build (libinterflect_b200_checked.so, -DIFX_CHECKED) on
the small parity cases: every scene-array index the kernels use is checked
(an out-of-range index sets a status bit, is replaced by an in-range one and
the call fails with "a bounds check failed"), and the transfer's CSR and
cluster structures are validated before the solve reads them. Run in a
child process (IFX_CHECKED=1 selects that library), its outputs must be the
normal build's, byte for byte, with no check failing. This stands in for a
memory checker, which the test does not need: the checks are in the kernels."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, scene_src

pytestmark = pytest.mark.gpu

CASES = [("product", 4000, 8, 120, 90), ("closed_box", 3000, 8, 64, 64), ("stress", 3000, 8, 80, 60),
         ("cornell", 3000, 5, 64, 64)]

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import interflect_b200 as ifx
assert ifx.LIB_PATH.endswith("_checked.so"), ifx.LIB_PATH
cases = json.loads(sys.argv[2])
out = {}
with ifx.Context(0) as ctx:
    for name, src, n, res, w, h in cases:
        ctx.upload(ifx.parse(src))
        ctx.generate(n)
        info = ctx.build(res)
        le = ctx.light_surfels()
        st = ctx.solve(16)
        ctx.grid_build()
        lin, s8, ev = ctx.render_frame(w, h)
        f = ctx.frame(w, h)
        t = ctx.transfer()
        np.savez(sys.argv[3] + "/" + name + ".npz", lin=lin, s8=s8, idx=t["idx"], w=t["w"],
                 rad=ctx.surfels()["rad"], flin=f["linear"])
        out[name] = [info.links, info.evals, le, st.iterations, ev]
print(json.dumps(out))
"""


def run_normal(name, n, res, w, h):
    import interflect_b200 as ifx
    with ifx.Context(0) as ctx:
        ctx.upload(ifx.parse(scene_src(name)))
        ctx.generate(n)
        info = ctx.build(res)
        le = ctx.light_surfels()
        st = ctx.solve(16)
        ctx.grid_build()
        lin, s8, ev = ctx.render_frame(w, h)
        f = ctx.frame(w, h)
        t = ctx.transfer()
        return [info.links, info.evals, le, st.iterations, ev], dict(
            lin=lin, s8=s8, idx=t["idx"], w=t["w"], rad=ctx.surfels()["rad"], flin=f["linear"])


def test_checked_build_passes_every_check_and_changes_nothing(tmp_path):
    lib = os.path.join(ROOT, "interflect_b200", "lib", "libinterflect_b200_checked.so")
    assert os.path.exists(lib), "build the checked library: python -m interflect_b200.build --checked"
    cases = [(name, scene_src(name), n, res, w, h) for name, n, res, w, h in CASES]
    env = dict(os.environ, IFX_CHECKED="1")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(cases), str(tmp_path)], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    for name, n, res, w, h in CASES:
        counts, arrays = run_normal(name, n, res, w, h)
        assert got[name] == counts, name
        c = np.load(tmp_path / f"{name}.npz")
        for k, v in arrays.items():
            assert c[k].tobytes() == v.tobytes(), (name, k)
