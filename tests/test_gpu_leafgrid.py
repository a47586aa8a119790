"""The per-cell leaf lists that cone-shadow marches of large BVHs use in
place of a full traversal (device.cuh dist_fast) change no result: the
stress scene (513 objects, a deep BVH) through the transfer, the light
stage and the shade with the lists on and off gives identical bytes and
counts. The parity tests against the oracle on the stress scene run with the
lists on (the default)."""
import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import scene_src

pytestmark = pytest.mark.gpu


def run(on: bool, n=6000, w=160, h=120):
    with ifx.Context(0) as ctx:
        ctx.set_leaf_grid(on)
        ctx.upload(ifx.parse(scene_src("stress")))
        ctx.generate(n)
        info = ctx.build(8)
        le = ctx.light_surfels()
        st = ctx.solve(24)
        ctx.grid_build()
        lin, s8, ev = ctx.render_frame(w, h)
        f = ctx.frame(w, h)
        t = ctx.transfer()
        d = ctx.row_diag()
        return (info, le, st, ev, f["shade_evals"]), dict(idx=t["idx"], w=t["w"], starts=t["starts"],
                                                         row_evals=d["row_evals"], lin=lin, s8=s8,
                                                         flin=f["linear"], rad=ctx.surfels()["rad"])


def test_leaf_lists_change_nothing_on_the_stress_scene():
    c1, a1 = run(True)
    c0, a0 = run(False)
    assert c1 == c0
    for k in a0:
        assert np.asarray(a1[k]).tobytes() == np.asarray(a0[k]).tobytes(), k
