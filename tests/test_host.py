"""CPU-side checks of the product boundary: the C-ABI library loads and
exports every declared entry point, the host scene stage (parser, limits,
BVH, bounds) matches the oracle bit for bit, and device entry points fail
loudly without a GPU."""
import os
import re

import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import ROOT, scene_src
from pyoracle import Oracle

HEADER = os.path.join(ROOT, "include", "interflect.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ifx_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = ifx.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(ifx.EXPORTS)


SCENES = ["product", "cornell", "stress", "closed_box", "flush_ceiling_light", "minimal", "bench_box_only",
          "bench_cornell", "bench_high_albedo", "bench_sphere_only"]


@pytest.mark.parametrize("name", SCENES)
def test_host_scene_matches_oracle(name):
    """Counts, world bounds and every BVH node bit-identical to the oracle's
    restatement of scene.rs/bvh.rs."""
    src = scene_src(name)
    s = ifx.parse(src)
    o = Oracle(src)
    oi = o.info()
    si = s.info
    assert (si.objects, si.planes, si.lights, si.materials, si.bvh_nodes) == (
        oi["objects"], oi["planes"], oi["lights"], oi["materials"], oi["bvh_nodes"])
    assert np.array(si.bounds_lo, np.float32).tobytes() == oi["lo"].tobytes()
    assert np.array(si.bounds_hi, np.float32).tobytes() == oi["hi"].tobytes()
    assert (si.cfg.width, si.cfg.height, si.cfg.surfels, si.cfg.bounces) == (
        oi["width"], oi["height"], oi["surfels"], oi["bounces"])
    nodes, order = s.bvh()
    onodes, oorder = o.bvh()
    assert nodes.tobytes() == onodes.view(np.uint32).tobytes()
    assert np.array_equal(order, oorder)


MALFORMED = [("", "no `light` block"), ("wibble { }", "unknown block `wibble`"),
             ("camera { nonsense: 5 }", "unknown camera key `nonsense`"),
             ("camera { fov: abc }", "expected number, found `abc`"),
             ("camera { pos: [1, 2 }", "expected number, found `}`"),
             ('light { emit: [1,1,1] } sphere { mat: "nope" }', "unknown material `nope`"),
             ("camera {", "unexpected end of file"), ("render { width: 0x10 }", "expected number"),
             ("camera { fov 3 }", "expected `:`, found `3`")]


@pytest.mark.parametrize("src,expect", MALFORMED)
def test_malformed_input_is_rejected_like_the_reference(src, expect):
    with pytest.raises(ifx.ParseError) as e:
        ifx.parse(src)
    assert expect in str(e.value)
    with pytest.raises(Exception) as e2:
        Oracle(src)
    assert str(e.value) == str(e2.value)


def test_limits_and_cli_overrides_are_validated():
    base = "light { verts: [[-1,4,-1],[1,4,-1],[1,4,1],[-1,4,1]], emit: [9,9,9] }"
    for cfg, expect in [("render { surfels: 999999999 }", "surfels"),
                        ("render { width: 200000, height: 200000 }", "exceeds"),
                        ("render { width: 0, height: 10 }", "at least 1"),
                        ("render { bounces: 2000000000 }", "bounces"), ("render { exposure: 0 }", "exposure")]:
        with pytest.raises(ifx.ParseError, match=expect):
            ifx.parse(cfg + "\n" + base)
    s = ifx.parse(base)
    with pytest.raises(ifx.LimitError, match="surfels"):
        s.set_cfg(surfels=999999999)
    s.set_cfg(width=3840, height=2160, surfels=200000, bounces=64)
    assert s.cfg.width == 3840 and s.cfg.surfels == 200000


def test_extension_keys_parse_identically():
    """The synthetic benchmark scenes' extensions (rotate_y, smooth,
    subtract_cylinder, sphere_light) parse the same way in product and oracle."""
    src = ('material "m" { albedo: [0.5,0.6,0.7] }\n'
           'box { center: [0,0.6,0], size: [0.6,1.2,0.6], rotate_y: 15, mat: "m" }\n'
           'sphere { center: [1,1,1], radius: 0.5, smooth: 0.05, subtract_sphere: [[1,1.3,1], 0.4],'
           ' subtract_cylinder: [[1,0,1],[1,2,1], 0.1], mat: "m" }\n'
           'sphere_light { center: [0,3,0], radius: 0.3, emit: [6,6,6] }\n')
    s, o = ifx.parse(src), Oracle(src)
    assert s.info.sphere_lights == o.info()["sphere_lights"] == 1
    assert np.array(s.info.bounds_lo, np.float32).tobytes() == o.info()["lo"].tobytes()
    assert s.bvh()[0].tobytes() == o.bvh()[0].view(np.uint32).tobytes()


@pytest.mark.skipif(ifx.cuda_available(), reason="checks the no-GPU failure path")
def test_device_calls_fail_loudly_without_a_gpu():
    with pytest.raises(ifx.DeviceError):
        ifx.Context(0)
