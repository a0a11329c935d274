"""View sharding of one scene over ranks (hpm-mvs_b200/scene_dist.py) on the
CPU: two gloo ranks with a stand-in per-problem solver.  Each rank solves
its share of the problems, depth maps are all-gathered before each
geometric iteration, and the result must equal the one-rank run."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hpm-mvs_b200")

# 5 views of uneven size, each view a problem with two sources
SHAPES = {0: (6, 8), 1: (5, 7), 2: (6, 8), 3: (4, 9), 4: (6, 6)}
PAIRS = [(v, [(v + 1) % 5, (v + 2) % 5]) for v in range(5)]


class FakeSolver:
    """Deterministic stand-in: pass A fills a view with its id; a geometric
    pass mixes the view's map with the means of its sources' maps."""

    def pass_a(self, p):
        import torch

        v = PAIRS[p][0]
        h, w = SHAPES[v]
        d = torch.full((h, w), float(v + 1)) + torch.arange(h * w, dtype=torch.float32).reshape(h, w) * 0.01
        return d, torch.zeros((h, w, 3)), torch.ones((h, w))

    def geom(self, p, it, depths, normal, cost):
        v, srcs = PAIRS[p]
        m = sum(float(depths[s].mean()) for s in srcs)
        return depths[v] * 0.5 + m * (it + 1), normal, cost


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, PKG)
    try:
        import torch.distributed as dist

        import scene_dist

        dist.init_process_group("gloo", rank=rank, world_size=world)
        mine, all_depth = scene_dist.run_scene_sharded(FakeSolver(), PAIRS, SHAPES, geom_iterations=2, dist=dist)
        dist.destroy_process_group()
        q.put((rank, {v: m[0].numpy() for v, m in mine.items()}, {v: d.numpy() for v, d in all_depth.items()}, None))
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put((rank, None, None, repr(e)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_scene_equals_one_rank():
    import torch.multiprocessing as mp

    sys.path.insert(0, PKG)
    import scene_dist

    one, one_all = scene_dist.run_scene_sharded(FakeSolver(), PAIRS, SHAPES, geom_iterations=2, dist=None)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r, mine, all_depth, err = q.get(timeout=180)
        assert err is None, err
        got[r] = (mine, all_depth)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(got[0][0]) == [0, 2, 4] and sorted(got[1][0]) == [1, 3]  # round-robin shares
    for r in (0, 1):
        for v, d in got[r][0].items():
            np.testing.assert_array_equal(d, one[v][0].numpy())
        assert sorted(got[r][1]) == list(range(5))
        for v, d in got[r][1].items():
            assert d.shape == SHAPES[v]
            np.testing.assert_array_equal(d, one_all[v].numpy())


def test_round_robin_shares():
    sys.path.insert(0, PKG)
    import scene_dist

    assert scene_dist.my_problems(11, 0, 4) == [0, 4, 8]
    assert scene_dist.my_problems(11, 3, 4) == [3, 7]
    assert scene_dist.my_problems(2, 2, 4) == []
    assert sum(len(scene_dist.my_problems(11, r, 4)) for r in range(4)) == 11
