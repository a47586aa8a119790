"""The `compare` tool (the reference's src/bin/compare.rs): its report on
PNGs of every 8-bit colour type, checked against the same metrics computed
here with numpy, and its exit codes. Host only."""
import re
import subprocess

import numpy as np
import pytest

import interflect_b200 as ifx

PIL = pytest.importorskip("PIL.Image")


def run(*args):
    return subprocess.run([ifx.COMPARE_PATH, *map(str, args)], capture_output=True, text=True, timeout=120)


def metrics(a, b):
    """compare.rs:12-66,87-132 restated with numpy, sums in the tool's order."""
    a, b = a.astype(np.int64), b.astype(np.int64)
    d = np.abs(a - b)
    pix = d.max(axis=2)
    la = 0.2126 * a[..., 0] + 0.7152 * a[..., 1] + 0.0722 * a[..., 2]
    lb = 0.2126 * b[..., 0] + 0.7152 * b[..., 1] + 0.0722 * b[..., 2]
    h, w = la.shape
    C1, C2, tiles = 6.5025, 58.5225, []
    for y in range(0, h - 7, 8):
        for x in range(0, w - 7, 8):
            ta, tb = la[y:y + 8, x:x + 8].ravel(), lb[y:y + 8, x:x + 8].ravel()
            ma, mb = ta.mean(), tb.mean()
            va, vb = ((ta - ma) ** 2).sum() / 63, ((tb - mb) ** 2).sum() / 63
            cov = ((ta - ma) * (tb - mb)).sum() / 63
            tiles.append(((2 * ma * mb + C1) * (2 * cov + C2)) / ((ma * ma + mb * mb + C1) * (va + vb + C2)))
    return dict(ndiff=int((pix > 0).sum()), max=int(pix.max()), mean=d.sum() / d.size,
                la=la.mean(), lb=lb.mean(), ssim=np.mean(tiles) if tiles else 1.0)


def parse(out):
    g = lambda pat: re.search(pat, out).group(1)
    return dict(ndiff=int(g(r"differing px\s+(\d+)")), max=int(g(r"max abs err\s+(\d+)")),
                mean=float(g(r"mean abs err\s+([0-9.]+)")), la=float(g(r"mean luma\s+([0-9.]+)")),
                lb=float(g(r"mean luma\s+[0-9.]+ vs ([0-9.]+)")), ssim=float(g(r"SSIM\s+([0-9.]+)")))


@pytest.mark.parametrize("mode", ["RGB", "RGBA", "L", "LA", "P"])
def test_report_matches_numpy_on_every_colour_type(tmp_path, mode):
    rng = np.random.default_rng(3)
    base = rng.integers(0, 256, size=(37, 53, 3), dtype=np.uint8)
    other = base.copy()
    other[5:20, 7:30] = rng.integers(0, 256, size=(15, 23, 3), dtype=np.uint8)
    ia, ib = PIL.fromarray(base, "RGB"), PIL.fromarray(other, "RGB")
    if mode != "RGB":
        ia, ib = ia.convert(mode), ib.convert(mode)
    pa, pb = tmp_path / "a.png", tmp_path / "b.png"
    ia.save(pa)
    ib.save(pb)
    ra, rb = (np.asarray(PIL.open(p).convert("RGB")) for p in (pa, pb))
    r = run(pa, pb, "--diff", tmp_path / "d.png")
    assert r.returncode == 0, r.stderr
    got, want = parse(r.stdout), metrics(ra, rb)
    assert got["ndiff"] == want["ndiff"] and got["max"] == want["max"]
    assert got["mean"] == pytest.approx(want["mean"], abs=1e-5)
    assert got["la"] == pytest.approx(want["la"], abs=0.006) and got["lb"] == pytest.approx(want["lb"], abs=0.006)
    assert got["ssim"] == pytest.approx(want["ssim"], abs=1e-6)
    d = np.asarray(PIL.open(tmp_path / "d.png").convert("RGB"))
    assert np.array_equal(d[..., 0], np.minimum(np.abs(ra.astype(int) - rb.astype(int)).max(axis=2) * 8, 255))


def test_identical_images_and_exit_codes(tmp_path):
    img = np.full((16, 24, 3), 77, np.uint8)
    pa, pb, pc = tmp_path / "a.png", tmp_path / "b.png", tmp_path / "c.png"
    PIL.fromarray(img).save(pa)
    PIL.fromarray(img).save(pb)
    PIL.fromarray(img[:8]).save(pc)
    r = run(pa, pb)
    assert r.returncode == 0
    assert "differing px  0 (0.0000%)" in r.stdout and "SSIM          1.000000" in r.stdout
    assert run(pa, pc).returncode == 1 and "size mismatch" in run(pa, pc).stderr
    assert run(pa).returncode == 2
    assert run(pa, tmp_path / "missing.png").returncode != 0
