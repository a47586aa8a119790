"""The solve's sliced-ELL copy of the transfer (rows sorted by link count,
32-row slices, links interleaved by 4): on an irregular matrix (empty rows,
lengths not multiples of 4, a partial last slice) the solve stays
bit-identical to the oracle's CSR solve, and ifx_clusters_build gives the
oracle's clusters."""
import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import scene_src
from pyoracle import Oracle

pytestmark = pytest.mark.gpu


def test_irregular_matrix_solves_bit_exactly():
    src = scene_src("cornell")
    ctx = ifx.Context(0)
    ctx.upload(ifx.parse(src))
    n = ctx.generate(3001)
    nc = ctx.build_clusters(8)
    s = ctx.surfels()
    o = Oracle(src, threads=4)
    o.set_surfels(s["p"], s["n"], s["albedo"], s["area"])
    assert o.build_clusters(8) == nc
    gc, oc = ctx.clusters(nc), o.clusters(nc, n)
    assert gc["members"].tobytes() == oc["members"].tobytes()
    assert gc["offsets"].tobytes() == oc["offsets"].tobytes()

    rng = np.random.default_rng(4)
    lens = rng.integers(0, 203, size=n)
    lens[rng.choice(n, size=n // 7, replace=False)] = 0  # empty rows
    starts = np.zeros(n + 1, np.uint32)
    starts[1:] = np.cumsum(lens)
    idx = np.concatenate([np.sort(rng.choice(nc, size=k, replace=k > nc)) for k in lens]).astype(np.uint32)
    w = (rng.random(len(idx)) * (0.9 / 200)).astype(np.float32)
    ctx.upload_transfer(starts, idx, w)
    o.set_transfer(starts, idx, w)
    E = (rng.random((n, 3)) * 2.0).astype(np.float32)
    for bounces in (3, 40):
        ctx.set_emission(E)
        o.set_surfel_state(direct=E, irr=np.zeros_like(E), rad=E)
        gs = ctx.solve(bounces)
        oit, ores = o.solve(bounces)
        g, r = ctx.surfels(), o.surfels()
        assert gs.iterations == oit
        assert np.float32(gs.residual).tobytes() == np.float32(ores).tobytes()
        assert g["rad"].tobytes() == r["rad"].tobytes()
        assert g["irr"].tobytes() == r["irr"].tobytes()
    ctx.close()
