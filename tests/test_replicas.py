"""The multi-GPU path of the benchmark is replicas only: every rank solves
its own seeded system, ranks meet only at the timing barrier and the
max-over-ranks reduction, and the whole-job rate is world x steps over the
slowest rank's time.  This runs that host logic with two gloo ranks on the
CPU, each rank's step being a GMRES-IR solve by the oracle."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import time

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench
    import oracle
    from mpir_b200 import kkt
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = kkt.grid3d(grid=6, seed=bench.replica_seed(11, rank))
        dist.barrier()
        t0 = time.perf_counter()
        x, st = oracle.Oracle().gmres_ir(s.n, s.Ap, s.Ai, s.Ax, s.b)
        ms = 1e3 * (time.perf_counter() - t0) + 10.0 * rank  # ranks differ in time
        dist.barrier()
        mx = bench.rank_max(dist, ms, "cpu")
        be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
        np.save(out + f".{rank}.npy", np.array([ms, mx, be, s.b[0]]))
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo(tmp_path):
    import torch.multiprocessing as tmp
    world, port = 2, _free_port()
    out = str(tmp_path / "r")
    tmp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                        start_method="spawn")
    r = [np.load(out + f".{k}.npy") for k in range(world)]
    ms = [v[0] for v in r]
    # every rank sees the slowest rank's time
    assert r[0][1] == r[1][1] == max(ms)
    # each rank solved its own system, to the benchmark's backward error
    assert r[0][3] != r[1][3]
    assert all(v[2] <= 1e-14 for v in r)
    # whole-job rate: world x steps over the slowest rank
    import bench  # noqa: F401  (path set by conftest)
    assert bench.aggregate_rate(world, 3, max(ms)) == pytest.approx(world * 3 / (max(ms) / 1e3))
