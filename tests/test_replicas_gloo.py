"""Multi-rank host logic of the replica benchmark on CPU: two gloo ranks each solve an
independent small problem with the oracle (a Bloch point per rank), and the job line
takes the slowest rank's step time and counts both ranks' solves."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import time
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method="env://",
                            timeout=__import__("datetime").timedelta(seconds=120))
    P = np.vstack([np.eye(3), np.diag([np.sqrt(2), np.sqrt(3), np.sqrt(5)])])
    q = [(0.13, 0.21, 0.17), (0.05, 0.04, 0.03)][rank]
    S = O.build_q_system(1, P, q, O.material_smooth_exp(1))
    t0 = time.perf_counter()
    sol = O.solve_modes(S, nev=4, p=12, tol=1e-10, tolCG=1e-12)
    dt = time.perf_counter() - t0 + 0.05 * rank  # rank 1 is the slower replica
    line = bench.replica_line(world, rank, dt, 1, torch.device("cpu"))
    out.put((rank, dt, line, sol["lam"].tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_line_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(2)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = max(r[1] for r in res)
    for rank, dt, line, lam in res:
        assert line["n_gpus"] == 2
        assert line["seconds_per_step"] == pytest.approx(slowest, rel=1e-12)
        assert line["solves_per_s_all_gpus"] == pytest.approx(2 / slowest, rel=1e-3)
        assert all(x > 0 for x in lam)
    # the two Bloch points are different problems
    assert not np.allclose(res[0][3], res[1][3])
