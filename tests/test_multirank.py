"""The multi-GPU plumbing of bench.py on CPU: two ranks as processes over
gloo (world size 2).  Ranks own independent scenes and exchange only the
barrier around the timed region and the max of their elapsed times, from
which rank 0 reports the whole-job rate."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    bench.WORKLOAD.update(width=48, height=36, n_views=3, n_planes=2, n_spheres=0)
    try:
        d = bench.Dist(world, backend="gloo")
        sc, images, pairs = bench.make_scene(seed=d.rank)
        d.barrier()
        elapsed = 100.0 + 50.0 * d.rank  # the slow rank sets the job time
        ms = d.max(elapsed)
        value = bench.job_mpix_per_s(d.world, 4, 3 * 48 * 36, ms)
        d.barrier()
        d.close()
        q.put((rank, ms, value, float(images[0].mean()), None))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, None, None, None, repr(e)))


def test_two_ranks_over_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, ms, value, mean, err = q.get(timeout=180)
        assert err is None, err
        out[r] = (ms, value, mean)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the max over ranks, and the same whole-job value
    assert out[0][0] == out[1][0] == 150.0
    assert out[0][1] == out[1][1] == pytest.approx(2 * 4 * 3 * 48 * 36 / 0.150 / 1e6)
    # the ranks' scenes are independent (seeded by rank)
    assert out[0][2] != out[1][2]


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(1)
    assert not d.pg and d.max(3.5) == 3.5
    d.barrier()
    d.close()
    assert bench.job_mpix_per_s(1, 2, 1_000_000, 1000.0) == pytest.approx(2.0)
    assert np.isfinite(bench.job_mpix_per_s(8, 3, 11 * 1600 * 1200, 5300.0))
