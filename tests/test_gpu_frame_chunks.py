"""The one-call frame (`ifx_frame`) composes films of 2^18 pixels or more in
row chunks and copies each chunk to the host while the next is composed.
Its linear and sRGB outputs must be byte-equal to the stage-by-stage path
(`ifx_render_frame` after the GI stages), which composes the whole film in
one launch, for every output combination (linear only, sRGB only, both, into
page-locked or pageable arrays) and for film heights that do not divide into
equal chunks. The stage-by-stage path itself is pinned to the oracle by the
parity tests (main.rs:229-367)."""
import numpy as np
import pytest
import torch

import interflect_b200 as ifx
from conftest import scene_src

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = ifx.Context(0)
    c.upload(ifx.parse(scene_src("product")))
    c.generate(4000)
    yield c
    c.close()


def staged(ctx, w, h):
    ctx.build(8)
    ctx.light_surfels()
    ctx.solve(16)
    ctx.grid_build()
    lin, s8, ev = ctx.render_frame(w, h)
    return lin, s8, ev


@pytest.mark.parametrize("w,h", [(640, 480), (1000, 263)])
def test_chunked_frame_equals_the_staged_frame(ctx, w, h):
    assert w * h >= 1 << 18
    want_lin, want_s8, want_ev = staged(ctx, w, h)
    fr = ctx.frame(w, h, "beauty", max_bounces=16)
    assert fr["shade_evals"] == want_ev
    assert fr["linear"].tobytes() == want_lin.tobytes()
    assert fr["srgb"].tobytes() == want_s8.tobytes()
    # One output at a time, and into page-locked arrays.
    assert ctx.frame(w, h, "beauty", max_bounces=16, linear=False)["srgb"].tobytes() == want_s8.tobytes()
    assert ctx.frame(w, h, "beauty", max_bounces=16, srgb=False)["linear"].tobytes() == want_lin.tobytes()
    pin8 = torch.zeros((h, w, 3), dtype=torch.uint8, pin_memory=True).numpy()
    pinl = torch.zeros((h, w, 3), dtype=torch.float32, pin_memory=True).numpy()
    fr = ctx.frame(w, h, "beauty", max_bounces=16, out_linear=pinl, out_srgb=pin8)
    assert pin8.tobytes() == want_s8.tobytes() and pinl.tobytes() == want_lin.tobytes()
    assert np.shares_memory(fr["srgb"], pin8)
