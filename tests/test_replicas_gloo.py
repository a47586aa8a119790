"""The multi-GPU form of the benchmark on the CPU: N independent replicas
(one process per GPU, no data-path collective), timed as the maximum over
ranks with the work summed over ranks. Run here as world-size-2 gloo
process groups."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    import bench
    w, r, local = bench.dist_setup()
    import torch.distributed as dist
    assert dist.get_backend() == "gloo"
    # Rank r "took" (r + 1) * 10 ms and processed (r + 1) * 1000 units.
    (t_max,), (units,) = bench.allreduce_max_sum([(r + 1) * 10.0], [(r + 1) * 1000.0], w)
    bench.barrier(w)
    # The reference arm's ranks other than 0 print nothing and do no work.
    ref = bench.run_reference(type("A", (), {"workload": "c1_cornell", "steps": 1, "warmup": 0,
                                             "cpu_rows": 0.01})(), w, r) if r != 0 else None
    q.put((r, w, local, t_max, units, ref))
    dist.destroy_process_group()


def test_replicas_reduce_time_as_max_and_work_as_sum():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, local, t_max, units, ref in out:
        assert w == world and local == r
        assert t_max == 20.0 and units == 3000.0
        assert ref is None
    # Whole-job throughput: all ranks' units over the slowest rank's time.
    assert out[0][4] / (out[0][3] / 1e3) == pytest.approx(150000.0)
