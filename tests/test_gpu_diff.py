"""Differentiation on the GPU: gradients of an L2 image loss with respect to
per-surfel albedo and per-light emission through the hand-written adjoint,
behind a torch.autograd.Function harness that calls the C ABI.

Checks: the differentiable forward is the plain renderer's frame bit for bit
and the oracle's f32 frame; the adjoint gradient agrees with the FP64 CPU
reference gradient (oracle/diff.cpp) and with FP64 central differences
(h = 1e-4) on 64 seeded coordinates to 1e-3; the gradient is bit-identical
across runs. Each check runs twice: on a reduced case (96x96, 4,000
surfels, 6 bounces) and at the differentiation benchmark's own
configuration (the C5 scene at 512x512, 20,000 surfels requested, its 12
bounces)."""
import os

import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import ROOT
from pyoracle import Oracle

pytestmark = pytest.mark.gpu

FD_TOL = 1e-3  # relative agreement with FP64 central differences (h = 1e-4)
# (film side, surfels requested, bounces K): reduced, and the benchmark's.
CASES = {"reduced": (96, 4000, 6), "c5": (512, 20000, 12)}


def c5_src(surfels: int) -> str:
    with open(os.path.join(ROOT, "interflect_b200", "scenes", "c5_cornell_fill.rad")) as f:
        return f.read().replace("surfels: 20000", f"surfels: {surfels}")


@pytest.fixture(scope="module", params=list(CASES))
def setup(request):
    W, SURFELS, K = CASES[request.param]
    H = W
    src = c5_src(SURFELS)
    scene = ifx.parse(src)
    assert scene.cfg.bounces >= K
    ctx = ifx.Context(0)
    ctx.upload(scene)
    n = ctx.generate(SURFELS)
    s = ctx.surfels()
    ctx.build(8)
    info = ctx.diff_setup(W, H, K)
    assert info["surfels"] == n and info["lights"] == 2 and info["pixels"] == W * H
    assert info["gather_entries"] > 0 and info["links"] > 0
    rng = np.random.default_rng(2026)
    rho0 = s["albedo"].astype(np.float32)
    rho_t = np.clip(rho0 + rng.normal(0.0, 0.05, rho0.shape), 0.05, 0.95).astype(np.float32)
    emit0 = ctx.light_emission()
    target = ctx.diff_forward(rho_t, emit0)
    # The FP64 reference over the same surfels (the oracle's transfer and
    # grid are bit-identical to the GPU's).
    o = Oracle(src, threads=os.cpu_count() or 1)
    o.set_surfels(s["p"], s["n"], rho0, s["area"])
    o.build_clusters(8)
    o.build_transfer()
    o.build_grid()
    assert o.diff_build(W, H) == (n, 2, W * H)
    yield dict(ctx=ctx, o=o, s=s, rho0=rho0, rho_t=rho_t, emit0=emit0, target=target, n=n, src=src, W=W, H=H,
               K=K)
    ctx.close()


def test_forward_is_the_renderers_frame(setup):
    ctx, s = setup["ctx"], setup["s"]
    W, H, K = setup["W"], setup["H"], setup["K"]
    rho = setup["rho_t"]
    emit = setup["emit0"] * np.float32(1.3)
    img = ctx.diff_forward(rho, emit)
    # The plain pipeline with the same albedo and emission, K bounces.
    ctx2 = ifx.Context(0)
    ctx2.upload(ifx.parse(setup["src"]))
    ctx2.upload_surfels(s["p"], s["n"], rho, s["area"])
    ctx2.set_light_emission(emit)
    ctx2.build(8)
    ctx2.light_surfels()
    st = ctx2.solve(K)
    ctx2.grid_build()
    lin, _, _ = ctx2.render_frame(W, H)
    ctx2.close()
    # The plain solve stops at the residual test (solve.rs:96-101); where it
    # ran all K bounces its frame is the differentiable frame bit for bit.
    if st.iterations == K:
        assert img.tobytes() == lin.tobytes()
    # ... and the oracle's f32 frame.
    o = Oracle(setup["src"], threads=os.cpu_count() or 1)
    o.set_surfels(s["p"], s["n"], rho, s["area"])
    o.set_emission(emit)
    o.build_clusters(8)
    o.build_transfer()
    o.light_surfels()
    assert o.solve(K, fixed=True)[0] == K
    o.build_grid()
    film, _ = o.render(W, H)
    rel = np.abs(img - film) / np.maximum(np.abs(film), 1e-6)
    exact = np.mean(img == film)
    print(f"diff forward vs oracle: max rel {rel.max():.3e}, rms {np.sqrt(np.mean(rel ** 2)):.3e}, "
          f"exact {100 * exact:.3f}%")
    assert rel.max() <= 1e-4


def _torch_grad(ctx, rho, emit, target):
    torch = pytest.importorskip("torch")

    class SurfelFrame(torch.autograd.Function):
        """The differentiable frame as a torch op over the C ABI (host tensors)."""

        @staticmethod
        def forward(fctx, rho_t, emit_t):
            img = ctx.diff_forward(rho_t.detach().numpy(), emit_t.detach().numpy())
            return torch.from_numpy(img)

        @staticmethod
        def backward(fctx, g):
            gr, ge = ctx.diff_backward(g.contiguous().numpy())
            return torch.from_numpy(gr), torch.from_numpy(ge)

    r = torch.tensor(rho, requires_grad=True)
    e = torch.tensor(emit, requires_grad=True)
    img = SurfelFrame.apply(r, e)
    loss = ((img - torch.from_numpy(target)) ** 2).sum()
    loss.backward()
    return float(loss.detach()), r.grad.detach().numpy().copy(), e.grad.detach().numpy().copy()


def test_gradient_matches_fp64_reference_and_central_differences(setup):
    ctx, o, K = setup["ctx"], setup["o"], setup["K"]
    rho, emit, target = setup["rho0"], setup["emit0"], setup["target"]
    loss, g_rho, g_e = _torch_grad(ctx, rho, emit, target)
    t64 = target.reshape(-1, 3).astype(np.float64)
    r64, e64 = rho.astype(np.float64), emit.astype(np.float64)
    L64, gr64, ge64 = o.diff_grad(r64, e64, K, t64)
    assert abs(loss - L64) <= 1e-4 * L64
    scale = max(np.abs(gr64).max(), np.abs(ge64).max())
    # Against the FP64 CPU reference gradient, every coordinate.
    assert np.all(np.abs(g_rho - gr64) <= FD_TOL * np.abs(gr64) + 1e-6 * scale)
    assert np.all(np.abs(g_e - ge64) <= FD_TOL * np.abs(ge64) + 1e-6 * scale)
    rel = np.linalg.norm(g_rho - gr64) / np.linalg.norm(gr64)
    print(f"{setup['W']}x{setup['H']}, {setup['n']} surfels, K={K}: gradient vs FP64 reference, "
          f"global relative error {rel:.3e}, loss {loss:.6e} vs {L64:.6e}")
    assert rel < 1e-4, rel
    # Against FP64 central differences on 64 seeded coordinates: the six
    # emission coordinates and 58 albedo coordinates the frame depends on.
    rng = np.random.default_rng(64)
    live = np.flatnonzero(np.abs(gr64).reshape(-1) > 1e-6 * scale)
    picks = rng.choice(live, size=58, replace=False)
    h = 1e-4
    checked = 0
    for q in picks:
        i, c = divmod(int(q), 3)
        rp, rm = r64.copy(), r64.copy()
        rp[i, c] += h
        rm[i, c] -= h
        fd = (o.diff_loss(rp, e64, K, t64)[0] - o.diff_loss(rm, e64, K, t64)[0]) / (2 * h)
        assert abs(g_rho[i, c] - fd) <= FD_TOL * abs(fd) + 1e-6 * scale, (i, c, g_rho[i, c], fd)
        checked += 1
    for l in range(2):
        for c in range(3):
            ep, em = e64.copy(), e64.copy()
            ep[l, c] += h
            em[l, c] -= h
            fd = (o.diff_loss(r64, ep, K, t64)[0] - o.diff_loss(r64, em, K, t64)[0]) / (2 * h)
            assert abs(g_e[l, c] - fd) <= FD_TOL * abs(fd) + 1e-6 * scale, (l, c, g_e[l, c], fd)
            checked += 1
    assert checked == 64


def test_gradient_is_bit_identical_across_runs(setup):
    ctx, rho, emit, target = setup["ctx"], setup["rho0"], setup["emit0"], setup["target"]
    outs = []
    for _ in range(3):
        img = ctx.diff_forward(rho, emit)
        outs.append(ctx.diff_backward(2.0 * (img - target)))
    for gr, ge in outs[1:]:
        assert gr.tobytes() == outs[0][0].tobytes() and ge.tobytes() == outs[0][1].tobytes()


def test_prepared_state_ends_with_a_new_frame(setup):
    ctx = ifx.Context(0)
    ctx.upload(ifx.parse(setup["src"]))
    ctx.generate(1000)
    ctx.build(8)
    ctx.diff_setup(32, 32, 3)
    ctx.diff_forward()
    ctx.render_frame(32, 32)
    with pytest.raises(ifx.DeviceError):
        ctx.diff_forward()
    with pytest.raises(ValueError):
        ctx.diff_setup(32, 32, 3)
        ctx.diff_forward(rho=np.zeros((3, 3), np.float32))
    ctx.close()
