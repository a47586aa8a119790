"""The FP64 reference of the differentiable frame (oracle/diff.cpp) on the
CPU: its image is the oracle's f32 render (the linearisation misses no term
of main.rs:289-356), and its gradient is the derivative of its loss (FP64
central differences)."""
import os

import numpy as np
import pytest

from conftest import ROOT
from pyoracle import Oracle

K = 5
W = H = 40


def c5_src(surfels: int) -> str:
    with open(os.path.join(ROOT, "interflect_b200", "scenes", "c5_cornell_fill.rad")) as f:
        return f.read().replace("surfels: 20000", f"surfels: {surfels}")


@pytest.fixture(scope="module")
def model():
    o = Oracle(c5_src(1500), threads=os.cpu_count() or 1)
    n = o.generate(1500)
    s = o.surfels()
    rng = np.random.default_rng(5)
    # A per-surfel albedo override, as the differentiation workload uses.
    rho = np.clip(s["albedo"] + rng.normal(0.0, 0.05, s["albedo"].shape), 0.05, 0.95).astype(np.float32)
    o.set_surfels(s["p"], s["n"], rho, s["area"])
    emit = o.emission() * np.float32(0.8)
    o.set_emission(emit)
    o.build_clusters(8)
    o.build_transfer()
    o.light_surfels()
    it, _ = o.solve(K, fixed=True)
    assert it == K
    o.build_grid()
    film, _ = o.render(W, H)
    dims = o.diff_build(W, H)
    assert dims == (n, 2, W * H)
    return o, rho.astype(np.float64), emit.astype(np.float64), film


def test_fixed_bounce_solve_runs_every_bounce():
    o = Oracle(c5_src(800), threads=4)
    o.generate(800)
    o.build_clusters(8)
    o.build_transfer()
    o.light_surfels()
    it_free, _ = o.solve(200)
    o.light_surfels()
    it_fixed, res = o.solve(it_free + 7, fixed=True)
    assert it_fixed == it_free + 7 and res < 1e-4


def test_model_image_is_the_f32_render(model):
    o, rho, emit, film = model
    _, img = o.diff_loss(rho, emit, K)
    ref = film.reshape(-1, 3).astype(np.float64)
    rel = np.abs(img - ref) / np.maximum(np.abs(ref), 1e-3)
    assert rel.max() < 1e-5, rel.max()


def test_model_gradient_matches_central_differences(model):
    o, rho, emit, _ = model
    rng = np.random.default_rng(9)
    _, img = o.diff_loss(rho, emit, K)
    target = img + rng.normal(0.0, 0.05, img.shape)
    _, g_rho, g_e = o.diff_grad(rho, emit, K, target)
    h = 1e-4
    live = np.flatnonzero(np.abs(g_rho).reshape(-1) > 1e-9)
    coords = rng.choice(live, size=min(24, len(live)), replace=False)
    scale = max(np.abs(g_rho).max(), np.abs(g_e).max())
    for q in coords:
        i, c = divmod(int(q), 3)
        rp, rm = rho.copy(), rho.copy()
        rp[i, c] += h
        rm[i, c] -= h
        fd = (o.diff_loss(rp, emit, K, target)[0] - o.diff_loss(rm, emit, K, target)[0]) / (2 * h)
        assert abs(g_rho[i, c] - fd) <= 1e-6 * abs(fd) + 1e-9 * scale, (i, c, g_rho[i, c], fd)
    for l in range(emit.shape[0]):
        for c in range(3):
            ep, em = emit.copy(), emit.copy()
            ep[l, c] += h
            em[l, c] -= h
            fd = (o.diff_loss(rho, ep, K, target)[0] - o.diff_loss(rho, em, K, target)[0]) / (2 * h)
            assert abs(g_e[l, c] - fd) <= 1e-6 * abs(fd) + 1e-9 * scale, (l, c, g_e[l, c], fd)


def test_loss_is_quadratic_in_emission(model):
    """The image is affine in the emissions: L(e + t d) is an exact
    quadratic in t, which pins the emission paths of the model."""
    o, rho, emit, _ = model
    d = np.random.default_rng(3).normal(0.0, 1.0, emit.shape)
    L = [o.diff_loss(rho, emit + t * d, K)[0] for t in (-1.0, 0.0, 1.0, 2.0)]
    # Third finite difference of a quadratic vanishes.
    third = L[3] - 3 * L[2] + 3 * L[1] - L[0]
    assert abs(third) <= 1e-9 * max(abs(x) for x in L)
