"""GPU parity on the benchmark configuration scenes: the Cornell box (C1),
the product-scale scene (C2, the 1080p headline's scene) and the stress
scene (C3), each run through the product path (`ifx_surfels_generate`, then
`ifx_frame`: transfer build, direct light, Jacobi solve, gather grid and
shade in one call) and through the oracle on the same surfels.

These scenes carry the extensions that the reference's own scenes do not
exercise: the rotated box (C1), smooth subtraction and cylinder drilling of
the bowl (C2, over sdf.rs:166-172's subtraction), and the sphere light (C2;
its form factor calls CUDA's atanf, the only transcendental on the device
that is not bit-exact with glibc). C1 and C2 run with every surfel the
configuration places; C3 runs with its surfel target reduced to 20,000 and
a 320x180 film so that the oracle finishes in seconds.

Bar: surfels, cluster ids and members, CSR starts and link column indices,
the bounce count and every SDF evaluation count bit-exact, with the rows
whose link sets differ (threshold-boundary flips) counted and printed;
link weights, radiosities and linear pixels within 1e-4 relative, with max,
RMS and the bit-identical fraction printed.
"""
import os

import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import ROOT
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

NCPU = os.cpu_count() or 1
REL = 1e-4
SCENES = os.path.join(ROOT, "interflect_b200", "scenes")

# name, surfel target (None = the scene's own), film
CASES = [
    ("c1_cornell", None, (260, 260)),
    ("c1_cornell_strict", None, (260, 260)),
    ("c2_product", None, (480, 270)),
    ("c2_product_strict", None, (480, 270)),
    ("c3_stress", 20000, (320, 180)),
]


def rel_err(a, b, floor=1e-6):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), floor)


def report(gpu, ref, what):
    e = rel_err(gpu, ref)
    exact = float(np.mean(np.asarray(gpu) == np.asarray(ref))) if np.size(ref) else 1.0
    mx = float(e.max()) if e.size else 0.0
    rms = float(np.sqrt(np.mean(e ** 2))) if e.size else 0.0
    print(f"{what}: max rel {mx:.3e}, rms {rms:.3e}, bit-identical {exact * 100:.4f}%")
    return mx


def row_mismatches(gs, gi, os_, oi, n):
    """Rows whose linked-cluster lists differ between the two CSR matrices."""
    gs, os_ = gs.astype(np.int64), os_.astype(np.int64)
    return sum(1 for i in range(n) if not np.array_equal(gi[gs[i]:gs[i + 1]], oi[os_[i]:os_[i + 1]]))


@pytest.fixture(scope="module")
def ctx():
    c = ifx.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name,target,film", CASES, ids=[c[0] for c in CASES])
def test_config_scene_frame_parity(ctx, name, target, film):
    with open(os.path.join(SCENES, name + ".rad")) as f:
        src = f.read()
    w, h = film
    s = ifx.parse(src)
    cfg = s.cfg
    target = target or cfg.surfels

    # Surfel generation (surfel.rs:147-255): count and bytes.
    o = Oracle(src, threads=NCPU)
    k = o.generate(target)
    ctx.upload(s)
    assert ctx.generate(target) == k
    g, r = ctx.surfels(), o.surfels()
    for fld in ("p", "n", "albedo", "area"):
        assert g[fld].tobytes() == r[fld].tobytes(), f"surfel {fld}"

    # The oracle's frame on those surfels.
    nc = o.build_clusters(8)
    oi = o.build_transfer()
    ole = o.light_surfels()
    oit, _ = o.solve(cfg.bounces)
    o.build_grid()
    film_o, oev = o.render(w, h, "beauty")

    # The product path: one ifx_frame call.
    fr = ctx.frame(w, h, "beauty", cluster_res=8, max_bounces=cfg.bounces)
    gi = fr["transfer"]
    print(f"{name}: {k} surfels, {nc} clusters, {gi.candidates} candidates, {gi.links} links, "
          f"{fr['solve'].iterations} bounces, film {w}x{h}")

    # Clusters (formfactor.rs:70-147): ids, members, p/n/area/radius.
    assert gi.clusters == nc
    gc, oc = ctx.clusters(nc), o.clusters(nc, k)
    assert np.array_equal(gc["offsets"], oc["offsets"]) and np.array_equal(gc["members"], oc["members"])
    for fld in ("p", "n", "area", "radius"):
        assert gc[fld].tobytes() == oc[fld].tobytes(), f"cluster {fld}"

    # Transfer (formfactor.rs:153-277): CSR structure exact, weights close.
    gt, ot = ctx.transfer(), o.transfer(k, oi["links"])
    mism = row_mismatches(gt["starts"], gt["idx"], ot["starts"], ot["idx"], k)
    print(f"{name}: threshold-boundary row mismatches {mism} of {k} rows")
    assert mism == 0
    assert gi.links == oi["links"] and gi.evals == oi["evals"] and gi.interior_rows == oi["interior_rows"]
    assert np.array_equal(gt["starts"], ot["starts"]) and np.array_equal(gt["idx"], ot["idx"])
    assert report(gt["w"], ot["w"], f"{name} link weights") <= REL
    assert abs(gi.mean_row_sum - oi["mean_row_sum"]) <= REL * abs(oi["mean_row_sum"])

    # Direct light and solve (solve.rs:27-108): counts exact, values close.
    assert fr["light_evals"] == ole
    assert fr["solve"].iterations == oit
    g, r = ctx.surfels(), o.surfels()
    assert report(g["direct"], r["direct"], f"{name} direct E") <= REL
    assert report(g["rad"], r["rad"], f"{name} radiosity") <= REL
    assert report(g["irr"], r["irr"], f"{name} irradiance") <= REL

    # Shade (main.rs:229-367): evaluations exact, linear pixels close.
    assert fr["shade_evals"] == oev
    assert report(fr["linear"], film_o, f"{name} {w}x{h} linear pixels") <= REL
    ref8 = o.encode(w, h, o.info()["exposure"], True)
    same = np.all(fr["linear"] == film_o, axis=2)
    assert np.array_equal(fr["srgb"][same], ref8[same])
    assert np.abs(fr["srgb"].astype(int) - ref8.astype(int)).max() <= 1
    if name.endswith("_strict"):
        # Reference features only: no transcendental differs, so every value
        # is expected bit-identical.
        assert fr["linear"].tobytes() == film_o.tobytes()
