"""`--mode reference`: the brute-force path tracer (reference.rs, driven per
pixel by main.rs:249-258) on the GPU against the oracle's restatement.

Both sides seed one PCG32 per pixel from (y << 32) | x, draw in the same
order and compute in IEEE FP32 without contraction; the only transcendental,
the azimuth's sin/cos, comes from one host table shared by both, so the
linear film is expected bit-identical. The test bar is 1e-4 relative on every
pixel, and the bit-identical share is printed.
"""
import os
import subprocess

import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import SCENES, scene_src
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


@pytest.mark.parametrize("name,w,h,spp", [("cornell", 32, 32, 4), ("bench_sphere_only", 24, 24, 3),
                                          ("product", 40, 30, 2), ("bench_high_albedo", 20, 20, 5),
                                          ("stress", 24, 18, 1)])
def test_reference_parity(ctx, name, w, h, spp):
    src = scene_src(name)
    o = Oracle(src, threads=NCPU)
    film, _ = o.render(w, h, "reference", spp=spp)
    ctx.upload(ifx.parse(src))
    lin, s8 = ctx.render_reference(w, h, spp)
    e = rel_err(lin, film)
    exact = float(np.mean(lin == film))
    print(f"{name} {w}x{h} spp {spp}: max rel {e.max():.3e}, bit-identical {exact * 100:.4f}%")
    assert e.max() <= REL
    ref8 = o.encode(w, h, o.info()["exposure"], True)
    same = np.all(lin == film, axis=2)
    assert np.array_equal(s8[same], ref8[same])


def test_reference_camera_override(ctx):
    """A turntable camera (main.rs:492-520) reaches the path tracer too."""
    src = scene_src("cornell")
    s = ifx.parse(src)
    ctx.upload(s)
    cam = s.info.camera
    pos = (cam["look"][0] + 1.5, cam["pos"][1], cam["pos"][2] - 0.5)
    c2 = ifx.camera(pos, cam["look"], cam["up"], cam["fov"])
    lin, _ = ctx.render_reference(24, 24, 2, cam=c2, srgb=False)
    o = Oracle(src, threads=NCPU)
    film, _ = o.render(24, 24, "reference", pos=np.float32(pos), look=np.float32(cam["look"]), spp=2)
    assert rel_err(lin, film).max() <= REL


def test_reference_is_deterministic(ctx):
    ctx.upload(ifx.parse(scene_src("cornell")))
    a = ctx.render_reference(64, 48, 8)
    b = ctx.render_reference(64, 48, 8)
    assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes()


def test_reference_rejects_bad_sample_counts(ctx):
    ctx.upload(ifx.parse(scene_src("cornell")))
    for spp in (0, (1 << 20) + 1):
        with pytest.raises(ifx.LimitError):
            ctx.render_reference(8, 8, spp)
    with pytest.raises(ifx.LimitError):
        ctx.render_reference(0, 8, 4)


def test_energy_against_path_traced_ground_truth(tmp_path):
    """ci.yml:151-176: the solver's image and a 48-spp reference of every
    bench scene at 120x120 agree in total energy (compare's luma ratio in
    0.85..1.25)."""
    ratios = {}
    for name in ("bench_box_only", "bench_cornell", "bench_high_albedo", "bench_sphere_only"):
        s = os.path.join(SCENES, name + ".rad")
        a, g = tmp_path / f"a_{name}.png", tmp_path / f"g_{name}.png"
        for extra, out in (((), a), (("--mode", "reference", "--spp", "48"), g)):
            r = subprocess.run([ifx.CLI_PATH, "render", s, "-o", str(out), "-w", "120", "-h", "120", *extra],
                               capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, r.stdout + r.stderr
        r = subprocess.run([ifx.COMPARE_PATH, str(a), str(g)], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0, r.stdout + r.stderr
        line = [x for x in r.stdout.splitlines() if "ratio" in x][0]
        ratios[name] = float(line.split("ratio")[1].strip(" )"))
    print(ratios)
    assert all(0.85 < v < 1.25 for v in ratios.values()), ratios


def test_accuracy_benchmark_runs(tmp_path):
    """bench.sh's table through `python -m interflect_b200.accuracy`, small."""
    from interflect_b200 import accuracy
    r = accuracy.run(spp=16, res=64, out_dir=str(tmp_path))
    assert r["deterministic"]
    assert [x["scene"] for x in r["scenes"]] == ["box_only", "cornell", "high_albedo", "sphere_only"]
    assert all(0.8 < x["luma"] < 1.3 and 0.0 < x["ssim"] <= 1.0 for x in r["scenes"]), r["scenes"]
    assert set(r["perf_ms"]) == {"cornell", "product", "stress"}


def test_path_work_counters(ctx):
    """The counting launch of the path tracer tallies its marches and SDF
    queries without changing the image."""
    ctx.upload(ifx.parse(scene_src("cornell")))
    plain, _ = ctx.render_reference(16, 16, 2, srgb=False)
    ctx.set_work_counting(True)
    ctx.reset_work()
    counted, _ = ctx.render_reference(16, 16, 2, srgb=False)
    counts, flops = ctx.work("path")
    ctx.set_work_counting(False)
    assert counted.tobytes() == plain.tobytes()
    assert counts[12] > 0 and counts[11] >= counts[12] and flops > 0
