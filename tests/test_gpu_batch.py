"""Batched relighting (many emission vectors on one transfer matrix, solved
as a CSR SpMM): every right-hand side is bit-identical to its own solve, the
stop rule applies per right-hand side, and the autotuned block shape never
changes a bit."""
import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import scene_src

pytestmark = pytest.mark.gpu


def relight_rhs(n: int, R: int, seed: int = 7) -> np.ndarray:
    """R emission vectors, each 1-4 surfels-as-lights of intensity U[1, 50]
    (an RGB splat), as the batching configuration describes."""
    rng = np.random.default_rng(seed)
    E = np.zeros((R, n, 3), np.float32)
    for r in range(R):
        k = rng.integers(1, 5)
        idx = rng.choice(n, size=k, replace=False)
        E[r, idx, :] = rng.uniform(1.0, 50.0, size=(k, 1)).astype(np.float32)
    return E


@pytest.fixture(scope="module")
def cornell():
    ctx = ifx.Context(0)
    ctx.upload(ifx.parse(scene_src("cornell")))
    ctx.generate(6000)
    info = ctx.build(8)
    yield ctx, info
    ctx.close()


def test_batched_rhs_are_bit_identical_to_single_solves(cornell):
    ctx, info = cornell
    n = ctx.n_surfels
    E = relight_rhs(n, 40)
    rad, irr, it, res = ctx.solve_batched(E, 64)
    assert np.all(it >= 1) and np.all(it < 64)
    assert len(set(it.tolist())) > 1, "expected different convergence per rhs"
    for r in (0, 1, 7, 19, 39):
        ctx.set_emission(E[r])
        st = ctx.solve(64)
        s = ctx.surfels()
        assert st.iterations == it[r], r
        assert np.float32(st.residual).tobytes() == res[r].tobytes(), r
        assert s["rad"].tobytes() == rad[r].tobytes(), r
        assert s["irr"].tobytes() == irr[r].tobytes(), r


def test_batch_position_and_autotune_do_not_change_results(cornell):
    ctx, info = cornell
    n = ctx.n_surfels
    E = relight_rhs(n, 70, seed=11)
    rad_a, irr_a, it_a, _ = ctx.solve_batched(E, 32)
    # Same rhs at other batch positions and in a smaller batch.
    perm = np.random.default_rng(3).permutation(70)
    rad_b, _, it_b, _ = ctx.solve_batched(E[perm], 32)
    assert rad_b.tobytes() == rad_a[perm].tobytes() and np.array_equal(it_b, it_a[perm])
    rad_c, _, _, _ = ctx.solve_batched(E[5:9], 32)
    assert rad_c.tobytes() == rad_a[5:9].tobytes()
    best = ctx.autotune_batched(E)
    assert best in (2, 4, 8, 16)
    rad_d, irr_d, it_d, _ = ctx.solve_batched(E, 32)
    assert rad_d.tobytes() == rad_a.tobytes() and irr_d.tobytes() == irr_a.tobytes()
