"""The oracle against the reference's published numbers and its own
fixtures: the pin that makes the oracle trustworthy as a checker."""
import json
import os

import numpy as np

from conftest import ROOT, scene_src
from pyoracle import Oracle

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))


def test_product_scene_counts_match_readme():
    """README.md 'First render': every integer the reference prints for
    scenes/product.rad is reproduced exactly (12270 surfels, 311 clusters,
    110026 links, 12 bounces, 50 evals/px, ...)."""
    o = Oracle(scene_src("product"), threads=os.cpu_count() or 1)
    i = o.info()
    assert (i["objects"] + i["planes"], i["lights"], i["materials"], i["bvh_nodes"]) == (
        GOLDEN["objects"], GOLDEN["lights"], GOLDEN["materials"], GOLDEN["bvh_nodes"])
    assert (i["width"], i["height"]) == (GOLDEN["width"], GOLDEN["height"])
    n = o.generate(i["surfels"])
    assert n == GOLDEN["surfels_placed"] and i["surfels"] == GOLDEN["surfels_requested"]
    assert o.build_clusters(8) == GOLDEN["clusters"]
    t = o.build_transfer()
    assert t["links"] == GOLDEN["links"]
    assert f"{t['mean_row_sum']:.3f}" == GOLDEN["row_sum_3dp"]
    assert f"{t['evals'] / 1e6:.1f}" == GOLDEN["transfer_evals_M_1dp"]
    de = o.light_surfels()
    it, res = o.solve(i["bounces"])
    assert it == GOLDEN["bounces"]
    assert f"{res:.2e}".replace("e-05", "e-5") == GOLDEN["residual_3sf"]
    assert f"{de / 1e6:.1f}" == GOLDEN["solve_evals_M_1dp"]
    o.build_grid()
    _, ev = o.render(i["width"], i["height"])
    assert f"{ev / 1e6:.1f}" == GOLDEN["shade_evals_M_1dp"]
    assert round(ev / (i["width"] * i["height"])) == GOLDEN["evals_per_px"]


def test_integration_pins_cornell_and_stress():
    """TESTING.md 3.4/3.5 and ci.yml gates: sealed Cornell row-sum ~0.82 and
    > 0.7, convergence below 1e-3 in fewer than 16 bounces; stress ~0.15."""
    o = Oracle(scene_src("cornell"), threads=os.cpu_count() or 1)
    o.generate(o.info()["surfels"])
    o.build_clusters(8)
    t = o.build_transfer()
    assert t["mean_row_sum"] > 0.7 and abs(t["mean_row_sum"] - 0.82) < 0.01
    o.light_surfels()
    it, res = o.solve(o.info()["bounces"])
    assert res < 1e-3 and it < 16


def test_thread_count_invariance():
    """README.md:65-81: output is bit-identical for any thread count."""
    outs = []
    for th in (1, 3, 8):
        o = Oracle(scene_src("closed_box"), threads=th)
        o.generate(3000)
        o.build_clusters(8)
        o.build_transfer()
        o.light_surfels()
        o.solve(16)
        o.build_grid()
        film, ev = o.render(48, 32)
        outs.append((o.surfels()["rad"].tobytes(), film.tobytes(), ev))
    assert outs[0] == outs[1] == outs[2]
