"""The allocation-free Jacobi solve (ifx_solve_noalloc) against ifx_solve.

ifx_solve_noalloc is for callers that cannot let the library allocate GPU
memory (an engine that owns the whole device through its own arena, a frame
loop that cannot afford cudaMalloc's synchronisation): they pass their own
device buffers and the library's scratch is a fixed static device array.
This file runs last so that a failure here never hides the other tests'
results; it passes run alone or after them.
"""
import numpy as np
import pytest

import interflect_b200 as ifx
from conftest import scene_src

pytestmark = pytest.mark.gpu


def _dev_f4(torch, xyz, w=None):
    a = np.zeros((len(xyz), 4), np.float32)
    a[:, :3] = xyz
    if w is not None:
        a[:, 3] = w
    return torch.from_numpy(a).to("cuda:0")


def _dev_u32(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).to("cuda:0")


def test_noalloc_solve_matches_the_context_solve_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    ctx = ifx.Context(0)
    scene = ifx.parse(scene_src("closed_box"))
    ctx.upload(scene)
    ctx.generate(3000)
    info = ctx.build(8)
    ctx.light_surfels()
    s0 = ctx.surfels()  # E in direct and rad, irr = 0
    cl = ctx.clusters(info.clusters)
    tr = ctx.transfer()
    ref_stats = ctx.solve(40)
    ref = ctx.surfels()

    # The caller's own device buffers (allocated by the caller, not by the library).
    p4 = _dev_f4(torch, s0["p"], s0["area"])
    d4 = _dev_f4(torch, s0["direct"])
    a4 = _dev_f4(torch, s0["albedo"])
    cp4 = _dev_f4(torch, cl["p"], cl["area"])
    ranges = _dev_u32(torch, np.stack([cl["offsets"][:-1], cl["offsets"][1:]], 1).reshape(-1))
    members = _dev_u32(torch, cl["members"])
    starts = _dev_u32(torch, tr["starts"])
    idx = _dev_u32(torch, tr["idx"])
    w = torch.from_numpy(tr["w"]).to("cuda:0")
    irr4 = torch.zeros_like(d4)
    rad4 = torch.zeros_like(d4)
    n, nc = len(s0["area"]), info.clusters
    stream = torch.cuda.current_stream().cuda_stream

    free_after = []
    for call in range(2):
        irr4.zero_()
        rad4.copy_(d4)  # the solve starts from B = E, as after light_surfels
        torch.cuda.synchronize()
        st = ifx.solve_noalloc(0, stream, n, nc, p4.data_ptr(), d4.data_ptr(), a4.data_ptr(), irr4.data_ptr(),
                               rad4.data_ptr(), cp4.data_ptr(), ranges.data_ptr(), members.data_ptr(),
                               starts.data_ptr(), idx.data_ptr(), w.data_ptr(), 40)
        assert st.iterations == ref_stats.iterations, call
        assert np.float32(st.residual).tobytes() == np.float32(ref_stats.residual).tobytes(), call
        rad = rad4.cpu().numpy()[:, :3]
        irr = irr4.cpu().numpy()[:, :3]
        # Same kernels, same order of operations: bit-identical (tolerance 0).
        assert rad.tobytes() == ref["rad"].tobytes(), call
        assert irr.tobytes() == ref["irr"].tobytes(), call
        assert torch.cuda.current_device() == 0
        free_after.append(torch.cuda.mem_get_info(0)[0])
    # The first call may load the module that holds the static scratch; the
    # second must leave the device's free memory exactly as it found it (any
    # cudaMalloc would take at least one 2 MiB granule).
    assert free_after[1] == free_after[0], free_after
    ctx.close()


def test_noalloc_solve_refuses_misaligned_pointers_before_launching():
    """An arena offset aligned to less than a float4 is refused with an error
    (no kernel runs, so the caller's context stays usable)."""
    torch = pytest.importorskip("torch")
    buf = torch.zeros(1024, dtype=torch.float32, device="cuda:0")
    base = buf.data_ptr()
    ptrs = [base + 256 * i for i in range(11)]
    ptrs[3] += 4  # irr4 on a 4-byte boundary only
    with pytest.raises(ifx.DeviceError, match="misaligned"):
        ifx.solve_noalloc(0, 0, 8, 2, *ptrs, 4)
    ptrs[3] -= 4
    ptrs[6] += 4  # cluster_ranges on a 4-byte boundary only
    with pytest.raises(ifx.DeviceError, match="misaligned"):
        ifx.solve_noalloc(0, 0, 8, 2, *ptrs, 4)
    torch.cuda.synchronize()  # the context is still healthy


def test_noalloc_solve_rejects_more_clusters_than_its_scratch_holds():
    with pytest.raises(ifx.LimitError, match="exceed"):
        ifx.solve_noalloc(0, 0, 10, ifx.NOALLOC_MAX_CLUSTERS + 1, *([0] * 11), 4)
