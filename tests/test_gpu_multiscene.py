"""Packed multi-scene frame: many scenes' solve + shade in one persistent
cooperative launch replayed from a CUDA graph. Every scene must be
bit-identical to its own unbatched frame (ifx_light_surfels + ifx_solve +
ifx_grid_build + ifx_render_frame), whatever the packing order or the
autotuned launch shape."""
import re

import numpy as np
import pytest

import interflect_b200 as ifx
from interflect_b200.scenes.gen_scenes import packed_scenes

pytestmark = pytest.mark.gpu

BOUNCES = 24


def small(src: str, i: int) -> tuple[str, int]:
    """A packed scene scaled down for the test: 1.5k-4k surfels, 64-160 px."""
    surfels = 1500 + 500 * (i % 6)
    side = 64 + 32 * (i % 4)
    src = re.sub(r"render \{[^}]*\}",
                 f"render {{ width: {side}, height: {side}, surfels: {surfels}, bounces: {BOUNCES}, exposure: 1.0 }}",
                 src)
    return src, side


@pytest.fixture(scope="module")
def scenes():
    out = []
    for i, src in enumerate(packed_scenes(6, seed=99)):
        s, side = small(src, i)
        sc = ifx.parse(s)
        ctx = ifx.Context(0)
        ctx.upload(sc)
        ctx.generate(sc.cfg.surfels)
        ctx.build(8)
        out.append(dict(src=s, side=side, ctx=ctx, surf=ctx.surfels()))
    yield out
    for d in out:
        d["ctx"].close()


def unbatched(d, emit=None):
    ctx = ifx.Context(0)
    ctx.upload(ifx.parse(d["src"]))
    s = d["surf"]
    ctx.upload_surfels(s["p"], s["n"], s["albedo"], s["area"])
    if emit is not None:
        ctx.set_light_emission(emit)
    ctx.build(8)
    ctx.light_surfels()
    st = ctx.solve(BOUNCES)
    ctx.grid_build()
    lin, s8, _ = ctx.render_frame(d["side"], d["side"])
    ctx.close()
    return lin, s8, st


def test_packed_scenes_are_bit_identical_to_unbatched_frames(scenes):
    ms = ifx.MultiScene(0)
    for d in scenes:
        ms.add(d["ctx"], d["side"], d["side"], BOUNCES)
    grid, block = ms.build(autotune=True)
    assert grid > 0 and block in (128, 256)
    ms.run()
    for i, d in enumerate(scenes):
        lin, s8, st = ms.download(i)
        rl, r8, rst = unbatched(d)
        assert st.iterations == rst.iterations
        assert lin.tobytes() == rl.tobytes(), i
        assert s8.tobytes() == r8.tobytes(), i
    # Relighting one member is picked up by the next replay.
    e = scenes[2]["ctx"].light_emission() * np.float32(0.5)
    scenes[2]["ctx"].set_light_emission(e)
    ms.run()
    lin, _, _ = ms.download(2)
    rl, _, _ = unbatched(scenes[2], emit=e)
    assert lin.tobytes() == rl.tobytes()
    scenes[2]["ctx"].set_light_emission(e * np.float32(2.0))
    ms.close()


def test_packing_order_and_launch_shape_do_not_change_bits(scenes):
    outs = {}
    for order, tune in ((list(range(len(scenes))), False), (list(reversed(range(len(scenes)))), True)):
        ms = ifx.MultiScene(0)
        for k in order:
            ms.add(scenes[k]["ctx"], scenes[k]["side"], scenes[k]["side"], BOUNCES)
        ms.build(autotune=tune)
        ms.run()
        for pos, k in enumerate(order):
            lin, _, st = ms.download(pos)
            outs.setdefault(k, []).append((lin.tobytes(), st.iterations))
        ms.close()
    for k, v in outs.items():
        assert v[0] == v[1], k


def test_a_rerendered_member_is_refused(scenes):
    d = scenes[0]
    ms = ifx.MultiScene(0)
    ms.add(d["ctx"], d["side"], d["side"], BOUNCES)
    ms.build(autotune=False)
    ms.run()
    d["ctx"].render_frame(32, 32)
    with pytest.raises(ifx.DeviceError):
        ms.run()
    ms.close()


def test_grid_barrier_runs_out_and_the_packed_frame_recovers(scenes):
    """The packed launch's grid barriers are bounded: with no polls at all
    every CTA but the last to arrive gives up, the run returns
    IFX_ERR_TIMEOUT (no hang, no fault), and after a rebuild with the default
    budget the same packed frame is bit-identical to the unbatched frames."""
    ms = ifx.MultiScene(0)
    for d in scenes:
        ms.add(d["ctx"], d["side"], d["side"], BOUNCES)
    ms.set_wait_limit(0)
    ms.build(autotune=False)
    with pytest.raises(ifx.WaitTimeout, match="grid barrier"):
        ms.run()
    ms.set_wait_limit(None)
    ms.build(autotune=False)
    ms.run()
    for i, d in enumerate(scenes):
        lin, _, st = ms.download(i)
        rl, _, rst = unbatched(d)
        assert st.iterations == rst.iterations and lin.tobytes() == rl.tobytes(), i
    ms.close()
