"""Edge cases of the GPU path against the oracle: the BVH switched off
(main.rs `--no-bvh`, scene.rs:191-213's linear scan), zero bounces, a handful
of surfels (empty rows, empty matrix), extreme cluster grids and ragged or
one-pixel films. The bar is the parity bar of test_gpu_parity: integers
exact, floats within 1e-4 relative (expected bit-identical)."""
import os

import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import scene_src
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

NCPU = os.cpu_count() or 1
REL = 1e-4


@pytest.fixture(scope="module")
def ctx():
    c = ifx.Context(0)
    yield c
    c.close()


def rel_err(a, b, floor=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), floor)


def both(name, target, use_bvh=True):
    src = scene_src(name)
    o = Oracle(src, threads=NCPU)
    o.set_use_bvh(use_bvh)
    s = ifx.parse(src)
    s.set_use_bvh(use_bvh)
    return o, s


def run_pipeline(ctx, o, s, target, res, bounces, w, h, mode="beauty"):
    """Both sides through surfels -> transfer -> solve -> grid -> frame;
    returns what the test compares."""
    k = o.generate(target)
    ctx.upload(s)
    n = ctx.generate(target)
    assert n == k
    if n == 0:
        return k, None
    nc = o.build_clusters(res)
    oi = o.build_transfer()
    gi = ctx.build(res)
    assert (gi.clusters, gi.links, gi.evals) == (nc, oi["links"], oi["evals"])
    gt, ot = ctx.transfer(), o.transfer(k, oi["links"])
    assert np.array_equal(gt["starts"], ot["starts"]) and np.array_equal(gt["idx"], ot["idx"])
    assert rel_err(gt["w"], ot["w"]).max(initial=0.0) <= REL
    assert ctx.light_surfels() == o.light_surfels()
    st = ctx.solve(bounces)
    oit, ores = o.solve(bounces)
    assert st.iterations == oit
    assert rel_err(ctx.surfels()["rad"], o.surfels()["rad"]).max(initial=0.0) <= REL
    o.build_grid()
    ctx.grid_build()
    film, oev = o.render(w, h, mode)
    lin, _, gev = ctx.render_frame(w, h, mode)
    assert gev == oev
    assert rel_err(lin, film).max(initial=0.0) <= REL
    return k, (st, lin, film)


@pytest.mark.parametrize("name,target,mode", [("product", 4000, "beauty"), ("cornell", 3000, "beauty"),
                                              ("stress", 2000, "steps")])
def test_linear_scan_matches_the_oracle(ctx, name, target, mode):
    """With the BVH off every query scans objects in order on both sides."""
    o, s = both(name, target, use_bvh=False)
    run_pipeline(ctx, o, s, target, 8, 6, 64, 48, mode)


def test_zero_bounces(ctx):
    """solve.rs:57: no bounce runs, iterations 0, residual 0, radiosity the
    direct term."""
    o, s = both("closed_box", 2000)
    k, (st, _, _) = run_pipeline(ctx, o, s, 2000, 8, 0, 32, 32)
    assert st.iterations == 0 and st.residual == 0.0
    g = ctx.surfels()
    assert g["rad"].tobytes() == g["direct"].tobytes()


@pytest.mark.parametrize("target", [1, 2, 7, 33])
def test_a_handful_of_surfels(ctx, target):
    """Tiny systems: rows without links, possibly no links at all."""
    o, s = both("closed_box", target)
    run_pipeline(ctx, o, s, target, 8, 4, 24, 16)


@pytest.mark.parametrize("res", [1, 2, 64])
def test_cluster_grid_extremes(ctx, res):
    o, s = both("cornell", 3000)
    run_pipeline(ctx, o, s, 3000, res, 5, 32, 32)


@pytest.mark.parametrize("w,h", [(1, 1), (17, 3), (3, 17), (129, 1), (1, 65)])
def test_ragged_films(ctx, w, h):
    o, s = both("product", 3000)
    run_pipeline(ctx, o, s, 3000, 8, 4, w, h)


def test_fused_frame_rejects_bad_calls():
    """ifx_frame validates like the stage calls and leaves the context usable."""
    c = ifx.Context(0)
    try:
        with pytest.raises(ifx.DeviceError):
            c.frame(16, 16)  # no scene yet
        s = ifx.parse(scene_src("cornell"))
        c.upload(s)
        with pytest.raises(ifx.DeviceError):
            c.frame(16, 16)  # beauty needs surfels
        c.generate(2000)
        with pytest.raises(ifx.LimitError):
            c.frame(16, 16, cluster_res=0)
        with pytest.raises(ifx.LimitError):
            c.frame(0, 16)
        with pytest.raises(ifx.DeviceError):
            c.frame(16, 16, mode=7)
        f = c.frame(16, 16)  # still usable
        assert f["solve"].iterations > 0 and f["shade_evals"] > 0
        lin, _, ev = c.render_frame(16, 16)
        assert lin.tobytes() == f["linear"].tobytes() and ev == f["shade_evals"]
    finally:
        c.close()


def test_caller_output_arrays(ctx):
    """Outputs written into caller arrays equal freshly allocated ones; wrong
    shapes or types are refused before any device work."""
    s = ifx.parse(scene_src("cornell"))
    ctx.upload(s)
    ctx.generate(2000)
    a = ctx.frame(24, 16)
    lin = np.full((16, 24, 3), -1.0, np.float32)
    s8 = np.full((16, 24, 3), 7, np.uint8)
    b = ctx.frame(24, 16, out_linear=lin, out_srgb=s8)
    assert b["linear"] is lin and b["srgb"] is s8
    assert lin.tobytes() == a["linear"].tobytes() and s8.tobytes() == a["srgb"].tobytes()
    r8 = np.zeros((16, 24, 3), np.uint8)
    _, got, _ = ctx.render_frame(24, 16, out_srgb=r8)
    assert got is r8 and r8.tobytes() == a["srgb"].tobytes()
    for bad in (np.zeros((16, 24, 3), np.float32), np.zeros((24, 16, 3), np.uint8),
                np.zeros((16, 24, 6), np.uint8)[:, :, :3]):
        with pytest.raises(ValueError):
            ctx.frame(24, 16, out_srgb=bad)
