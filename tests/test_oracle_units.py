"""The reference's own unit tests (27 #[test] functions in src/*.rs),
restated over the oracle. Each test names the reference test it follows."""
import math

import numpy as np
import pytest

from conftest import scene_src
from pyoracle import Oracle, OracleError, form_factor_at, srgb
import pyoracle

FAR_LIGHT = "light { verts: [[100,100,100],[101,100,100],[101,100,101],[100,100,101]], emit: [1,1,1] }\n"


def one_object(obj: str) -> Oracle:
    return Oracle(obj + "\n" + FAR_LIGHT)


# ---------------------------------------------------------------- sdf.rs --
def test_cylinder_distances_are_correct():  # sdf.rs:183-217
    o = one_object("cylinder { a: [0,0,0], b: [0,2,0], radius: 1 }")
    pts = [(3, 1, 0), (0, 5, 0), (0, -1, 0), (0, 1, 0), (1, 1, 0), (0, 2, 0)]
    want = [2.0, 3.0, 1.0, -1.0, 0.0, 0.0]
    d, _ = o.dist_mat(pts)
    assert np.all(np.abs(d - want) < 1e-4), d
    d, _ = o.dist_mat([(2, 3, 0)])
    assert abs(d[0] - math.sqrt(2)) < 1e-4


def test_cone_distances_are_correct():  # sdf.rs:219-249
    o = one_object("cone { a: [0,0,0], b: [0,2,0], radius: 1, radius_top: 0 }")
    d, _ = o.dist_mat([(0, 1, 0), (0, 3, 0), (5, 1, 0), (1, 0, 0), (0.9, 0.1, 0), (0.9, 1.8, 0)])
    assert d[0] < 0 and d[1] > 0.9 and d[2] > 3.5 and abs(d[3]) < 1e-3 and d[4] < 0 and d[5] > 0


PRIMS = ["cylinder { a: [-0.4,0.1,0.2], b: [0.5,1.3,-0.3], radius: 0.35 }",
         "cone { a: [0.2,0.0,0.1], b: [-0.1,1.6,0.4], radius: 0.5, radius_top: 0.15 }"]


def _probe(i, scale):
    f = np.float32(i)
    return np.array([np.sin(f * np.float32(0.71)) * scale, np.cos(f * np.float32(1.13)) * scale,
                     np.sin(f * np.float32(0.37)) * scale], np.float32)


@pytest.mark.parametrize("prim", PRIMS)
def test_new_primitives_never_overstate_distance(prim):  # sdf.rs:254-296
    o = one_object(prim)
    pts = np.stack([_probe(i, 3.0) for i in range(4000)])
    d, _ = o.dist_mat(pts)
    assert np.all(np.isfinite(d))
    f = np.arange(4000, dtype=np.float32)
    dirs = np.stack([np.cos(f * np.float32(2.1)), np.sin(f * np.float32(0.9)), np.cos(f * np.float32(1.7))], 1)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pos = d > 0
    stepped, _ = o.dist_mat(pts[pos] + dirs[pos] * d[pos, None])
    assert np.all(stepped > -1e-3)


@pytest.mark.parametrize("prim", PRIMS)
def test_new_primitive_bounds_enclose_the_surface(prim):  # sdf.rs:299-335
    o = one_object(prim)
    nodes, _ = o.bvh()
    lo, hi = nodes[0, 0:3], nodes[0, 3:6]
    pts = np.stack([_probe(i, 2.5) for i in range(20000)])
    d, _ = o.dist_mat(pts)
    inside = pts[d < 0]
    assert len(inside) > 0
    assert np.all(inside >= lo - 1e-4) and np.all(inside <= hi + 1e-4)


# ---------------------------------------------------------------- bvh.rs --
def scattered(n: int) -> str:  # bvh.rs:316-335
    mats = "".join(f'material "m{k}" {{ albedo: [0.5,0.5,0.5] }}\n' for k in range(4))
    objs = []
    for i in range(n):
        f = np.float32(i)
        c = (np.sin(f * np.float32(1.7)) * 4.0, np.cos(f * np.float32(2.3)) * 3.0, np.sin(f * np.float32(0.9)) * 4.0)
        r = 0.2 + (i % 5) * 0.05
        objs.append(f"sphere {{ center: [{c[0]:.9g},{c[1]:.9g},{c[2]:.9g}], radius: {r:.9g}, mat: \"m{i % 4}\" }}")
    return mats + "\n".join(objs) + "\n" + FAR_LIGHT


def test_child_indices_are_consistent_with_layout():  # bvh.rs:342-377
    nodes, _ = Oracle(scattered(200)).bvh()
    cnt = nodes[:, 7].view(np.uint32)
    right = nodes[:, 8].view(np.uint32)
    for i in range(len(nodes)):
        if cnt[i] > 0:
            continue
        l, r = i + 1, int(right[i])
        assert l < len(nodes) and r < len(nodes) and r > l
        for c in (l, r):
            assert np.all(nodes[c, 0:3] >= nodes[i, 0:3] - 1e-4) and np.all(nodes[c, 3:6] <= nodes[i, 3:6] + 1e-4)


def test_every_primitive_lands_in_exactly_one_leaf():  # bvh.rs:381-399
    nodes, order = Oracle(scattered(200)).bvh()
    seen = np.zeros(200, int)
    start, cnt = nodes[:, 6].view(np.uint32), nodes[:, 7].view(np.uint32)
    for i in range(len(nodes)):
        for k in range(int(start[i]), int(start[i] + cnt[i])):
            seen[order[k]] += 1
    assert np.all(seen == 1)


def test_pruning_agrees_with_linear_scan():  # bvh.rs:403-428
    o = Oracle(scattered(300))
    f = np.arange(3000, dtype=np.float32) * np.float32(0.037)
    pts = np.stack([np.sin(f) * 6.0, np.cos(f * np.float32(1.3)) * 5.0, np.sin(f * np.float32(0.7)) * 6.0], 1)
    fast, _ = o.dist_mat(pts)
    o.set_use_bvh(False)
    slow, _ = o.dist_mat(pts)
    assert np.all(np.abs(fast - slow) < 1e-5)


# ---------------------------------------------------------------- ltc.rs --
def ceiling_light(half, h):
    return np.array([[-half, h, -half], [half, h, -half], [half, h, half], [-half, h, half]], np.float32)


def test_dsl_winding_yields_positive_form_factor():  # ltc.rs:156-163
    assert form_factor_at(ceiling_light(1.0, 2.0), (0, 0, 0), (0, 1, 0)) > 0.05


def test_small_distant_light_matches_analytic_limit():  # ltc.rs:169-181
    half, h = 0.05, 5.0
    ff = form_factor_at(ceiling_light(half, h), (0, 0, 0), (0, 1, 0))
    expect = (2 * half) ** 2 / (math.pi * h * h)
    assert abs(ff - expect) / expect < 0.02


def test_light_below_horizon_contributes_nothing():  # ltc.rs:186-189
    assert form_factor_at(ceiling_light(1.0, -2.0), (0, 0, 0), (0, 1, 0)) < 1e-6


# -------------------------------------------------------------- trace.rs --
def _flush_shadow(extra=""):
    o = Oracle(scene_src("flush_ceiling_light") + extra)
    v = ceiling_light(0.7, 3.94)
    c = v.mean(0)
    dist = float(np.linalg.norm(c))
    a1 = np.linalg.norm(np.cross(v[1] - v[0], v[3] - v[0]))
    a2 = np.linalg.norm(np.cross(v[3] - v[2], v[1] - v[2]))
    radius = math.sqrt(0.5 * (a1 + a2) / math.pi)
    k = min(max(dist / radius, 1.5), 96.0)
    end = max(dist - radius * 1.25, 0.05)
    vis, _ = o.soft_shadow([(0, 3e-3, 0)], [c / dist], 0.015, end, k)
    return vis[0]


def test_unoccluded_floor_under_flush_light_is_not_self_shadowed():  # trace.rs:223-243
    assert _flush_shadow() > 0.9


def test_real_occluder_still_casts_shadow():  # trace.rs:247-262
    assert _flush_shadow('box { center: [0,2,0], size: [1.5,0.2,1.5], mat: "w" }\n') < 0.1


# --------------------------------------------------------- formfactor.rs --
def closed_box_transfer(n=3000):  # formfactor.rs:299-306
    o = Oracle(scene_src("closed_box"), threads=4)
    k = o.generate(n)
    assert k > 0
    nc = o.build_clusters(8)
    info = o.build_transfer()
    return o, k, nc, info


def test_closed_box_conserves_energy():  # formfactor.rs:313-328
    _, _, _, info = closed_box_transfer()
    assert 0.7 < info["mean_row_sum"] <= 1.0001


def test_transfer_matrix_is_sparse_and_well_formed():  # formfactor.rs:332-360
    o, k, nc, info = closed_box_transfer()
    t = o.transfer(k, info["links"])
    assert len(t["starts"]) == k + 1 and int(t["starts"][-1]) == len(t["idx"]) == len(t["w"])
    assert np.all(np.diff(t["starts"].astype(np.int64)) >= 0)
    assert np.all(t["idx"] < nc)
    assert info["links"] * 3 < k * nc


# -------------------------------------------------------------- solve.rs --
def test_no_interior_surfel_is_unlit():  # solve.rs:146-174
    o, k, _, _ = closed_box_transfer()
    o.light_surfels()
    o.solve(16)
    irr = o.surfels()["irr"].max(1)
    lit = irr[irr > 0]
    assert len(lit) > k / 4
    assert lit.min() > lit.max() * 1e-3


def test_solve_converges():  # solve.rs:179-196
    o, _, _, _ = closed_box_transfer()
    o.light_surfels()
    it, res = o.solve(64)
    assert res < 1e-3 and it < 64


# -------------------------------------------------------------- scene.rs --
def test_parses_a_minimal_scene():  # scene.rs:613-621
    i = Oracle(scene_src("minimal")).info()
    assert i["objects"] == 1 and i["lights"] == 1 and i["materials"] == 1


def test_comments_and_trailing_commas_are_accepted():  # scene.rs:623-627
    Oracle("# leading comment\n" + scene_src("minimal") + "\n# trailing comment\n")


def test_planes_are_excluded_from_the_bvh():  # scene.rs:631-644
    i = Oracle(scene_src("minimal") + '\nplane { normal: [0,1,0], height: 0, mat: "w" }\n').info()
    assert i["planes"] == 1 and i["objects"] == 1


MALFORMED = [("", "no `light` block"), ("wibble { }", "unknown block"), ("camera { nonsense: 5 }", "unknown camera key"),
             ("camera { fov: abc }", "expected number"), ("camera { pos: [1, 2 }", "expected number"),
             ('light { emit: [1,1,1] } sphere { mat: "nope" }', "unknown material")]


@pytest.mark.parametrize("src,expect", MALFORMED)
def test_malformed_input_errors_instead_of_panicking(src, expect):  # scene.rs:648-673
    with pytest.raises(OracleError, match=expect):
        Oracle(src)


BASE = "light { verts: [[-1,4,-1],[1,4,-1],[1,4,1],[-1,4,1]], emit: [9,9,9] }"
ABSURD = [("render { surfels: 999999999 }", "surfels"), ("render { width: 200000, height: 200000 }", "exceeds"),
          ("render { width: 0, height: 10 }", "at least 1"), ("render { bounces: 2000000000 }", "bounces"),
          ("render { exposure: 0 }", "exposure")]


@pytest.mark.parametrize("cfg,expect", ABSURD)
def test_absurd_render_settings_are_rejected(cfg, expect):  # scene.rs:680-708
    with pytest.raises(OracleError, match=expect):
        Oracle(cfg + "\n" + BASE + "\n")


@pytest.mark.parametrize("cfg", ["render { width: 3840, height: 2160, surfels: 200000, bounces: 64 }",
                                 "render { width: 1920, height: 1080 }", "render { surfels: 1 }"])
def test_realistic_settings_are_accepted(cfg):  # scene.rs:712-727
    Oracle(cfg + "\n" + BASE + "\n")


def test_bounds_enclose_geometry_without_excessive_padding():  # scene.rs:731-751
    i = Oracle(scene_src("minimal")).info()
    lo, hi = i["lo"], i["hi"]
    assert np.all(lo <= [0.5, 1.5, 2.5]) and np.all(hi >= [1.5, 4.0, 3.5])
    geom = np.array([1.5, 4.0, 3.5]) - np.array([0.5, 1.5, -1.0])
    assert np.linalg.norm(hi - lo) < np.linalg.norm(geom) * 2.0


# --------------------------------------------------------------- film.rs --
def test_srgb_transfer_hits_known_anchors():  # film.rs:74-87
    assert srgb(0.0) == 0 and srgb(1.0) == 255 and abs(srgb(0.2140) - 128) <= 1
    assert srgb(-5.0) == 0 and srgb(9.0) == 255


def test_srgb_is_monotonic():  # film.rs:89-97
    v = [srgb(i / 1000) for i in range(1001)]
    assert all(b >= a for a, b in zip(v, v[1:]))


def test_aces_maps_into_unit_range():  # film.rs:101-116
    import ctypes as C
    out = np.zeros(3, np.float32)
    vals = []
    for e in (0.0, 0.1, 0.5, 1.0, 4.0, 100.0, 1e6):
        pyoracle.lib().orc_aces(np.full(3, e, np.float32).ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
        assert np.all(out >= 0) and np.all(out <= 1)
        vals.append(out[0])
    assert vals[3] > vals[2]


def test_encode_produces_three_bytes_per_pixel():  # film.rs:118-125
    o = Oracle(scene_src("minimal"))
    o.render(4, 3, mode="normals")
    buf = o.encode(4, 3, 1.0, True)
    assert buf.shape == (3, 4, 3)
