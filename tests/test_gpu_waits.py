"""Failure detection on the GPU without a fault: every device-side wait is
bounded, and a test makes two of them run out on purpose by giving them no
polls at all (ifx_set_wait_limit(ctx, 0)), never by hanging or faulting
anything.

* The scene-staging wait of the ray-marching kernels (the mbarrier that the
  CTA's bulk copy of the scene program completes): with no polls every CTA
  gives up at once, records the timeout, waits for its own copy to land and
  leaves without tracing; the stage call returns IFX_ERR_TIMEOUT.
* The grid barriers of the packed multi-scene launch are exhausted the same
  way in tests/test_gpu_multiscene.py.

Afterwards the same context, with the default budget back, must produce
exactly what a fresh context produces. The reference cannot fail inside a
stage (it only validates input, scene.rs:106-148); these waits are this
implementation's own.
"""
import pytest

import interflect_b200 as ifx
from conftest import scene_src

pytestmark = pytest.mark.gpu


def run_all(ctx, w=96, h=72):
    ctx.build(8)
    le = ctx.light_surfels()
    st = ctx.solve(16)
    ctx.grid_build()
    lin, s8, ev = ctx.render_frame(w, h)
    return le, st, lin.tobytes(), s8.tobytes(), ev, ctx.surfels()["rad"].tobytes()


def test_bounded_waits_run_out_and_the_context_recovers():
    scene = ifx.parse(scene_src("closed_box"))
    with ifx.Context(0) as fresh:
        fresh.upload(scene)
        fresh.generate(3000)
        want = run_all(fresh)

    with ifx.Context(0) as ctx:
        ctx.upload(scene)
        ctx.generate(3000)
        ctx.build(8)
        ctx.set_wait_limit(0)
        # Staging wait of the light stage's kernel.
        with pytest.raises(ifx.WaitTimeout, match="bounded wait expired"):
            ctx.light_surfels()
        # Staging wait of the shading passes (both streams of ifx_frame).
        with pytest.raises(ifx.WaitTimeout, match="bounded wait expired"):
            ctx.frame(64, 48)
        ctx.set_wait_limit(None)
        # The same context, default budget: identical to a fresh context.
        ctx.upload(scene)
        ctx.generate(3000)
        assert run_all(ctx) == want
