"""Accuracy and speed against the path-traced ground truth, as bench.sh does
it for the reference (bench.sh:1-84): every Lambertian bench scene is
rendered once by the radiosity pipeline and once by `--mode reference`
through the `interflect` CLI, then scored by the `compare` tool (SSIM and
the mean-luma energy ratio). Glossy scenes are timed without a score, and
the run ends with the determinism gate (the same frame rendered three
times must give identical PNG bytes).

    python -m interflect_b200.accuracy [--spp 512] [--res 300] [--scenes DIR]

OURS_MS and REF_MS are wall-clock times of whole CLI processes, as bench.sh
measures them: scene parse, CUDA context creation and PNG writing included.
The `total` the CLI reports (GI + shade on the device side of the process)
is printed beside them.
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import os
import re
import subprocess
import sys
import tempfile
import time

from . import CLI_PATH, COMPARE_PATH

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEFAULT_SCENES = os.path.join(_ROOT, "tests", "golden", "scenes")


def _render(scene: str, out: str, res: int, extra=()) -> tuple[float, float]:
    """(wall ms of the CLI process, the CLI's own `total` ms)."""
    t0 = time.perf_counter()
    r = subprocess.run([CLI_PATH, "render", scene, "-o", out, "-w", str(res), "-h", str(res), *extra],
                       capture_output=True, text=True)
    wall = (time.perf_counter() - t0) * 1e3
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(scene)}: {r.stderr.strip() or r.stdout.strip()}")
    m = re.search(r"total\s+(\d+) ms", r.stdout)
    return wall, float(m.group(1)) if m else float("nan")


def _compare(a: str, b: str) -> tuple[float, float]:
    r = subprocess.run([COMPARE_PATH, a, b], capture_output=True, text=True, check=True)
    ssim = float(re.search(r"SSIM\s+([0-9.]+)", r.stdout).group(1))
    luma = float(re.search(r"ratio ([0-9.]+)\)", r.stdout).group(1))
    return ssim, luma


def run(spp: int = 512, res: int = 300, scenes_dir: str = DEFAULT_SCENES, out_dir: str | None = None,
        perf_scenes=("cornell", "product", "stress"), det_res: int = 200) -> dict:
    out_dir = out_dir or tempfile.mkdtemp(prefix="ifx_accuracy_")
    os.makedirs(out_dir, exist_ok=True)
    rows = []
    print(f"{'SCENE':<22} {'OURS_MS':>10} {'REF_MS':>10} {'SPEEDUP':>9} {'SSIM':>8} {'LUMA':>8}"
          f" {'OURS_DEV':>9} {'REF_DEV':>9}")
    print("-" * 92)
    for scene in sorted(glob.glob(os.path.join(scenes_dir, "bench_*.rad"))):
        name = os.path.basename(scene)[len("bench_"):-len(".rad")]
        ours, ref = os.path.join(out_dir, f"{name}_ours.png"), os.path.join(out_dir, f"{name}_ref.png")
        ow, od = _render(scene, ours, res)
        rw, rd = _render(scene, ref, res, ("--mode", "reference", "--spp", str(spp)))
        ssim, luma = _compare(ours, ref)
        rows.append(dict(scene=name, ours_ms=ow, ref_ms=rw, speedup=rw / ow, ssim=ssim, luma=luma,
                         ours_device_ms=od, ref_device_ms=rd))
        print(f"{name:<22} {ow:>10.0f} {rw:>10.0f} {rw / ow:>8.1f}x {ssim:>8.6f} {luma:>8.3f} {od:>9.0f} {rd:>9.0f}")
    print("\nPerf-only scenes (glossy/metal, excluded from the accuracy table):")
    perf = {}
    for name in perf_scenes:
        scene = os.path.join(scenes_dir, name + ".rad")
        if not os.path.exists(scene):
            continue
        w, d = _render(scene, os.path.join(out_dir, name + ".png"), res)
        perf[name] = w
        print(f"  {name:<20} {w:>6.0f} ms   (device {d:.0f} ms)")
    print("\nDeterminism gate:")
    digests = []
    for i in range(3):
        p = os.path.join(out_dir, f"det_{i}.png")
        _render(os.path.join(scenes_dir, "cornell.rad"), p, det_res)
        with open(p, "rb") as f:
            digests.append(hashlib.md5(f.read()).hexdigest())
    deterministic = len(set(digests)) == 1
    print("  PASS  bit-identical across 3 runs" if deterministic else "  FAIL  output varies between runs")
    return dict(spp=spp, res=res, scenes=rows, perf_ms=perf, deterministic=deterministic, out_dir=out_dir)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--spp", type=int, default=int(os.environ.get("SPP", 512)))
    ap.add_argument("--res", type=int, default=int(os.environ.get("RES", 300)))
    ap.add_argument("--scenes", default=DEFAULT_SCENES, help="directory holding bench_*.rad and cornell.rad")
    ap.add_argument("--out", default=None, help="directory for the PNGs [default: a temporary one]")
    a = ap.parse_args(argv)
    r = run(a.spp, a.res, a.scenes, a.out)
    return 0 if r["deterministic"] else 1


if __name__ == "__main__":
    sys.exit(main())
