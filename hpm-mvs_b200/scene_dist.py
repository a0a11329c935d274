"""One scene's views sharded over ranks (one process per GPU): the reference's
main() (main.cpp:636-677) with pass set A and each geometric iteration split
across ranks, and one exchange per iteration, an all-gather of the depth maps.

    rank r processes problems r, r + world, r + 2*world, ...
    pass set A          own problems (no exchange: a problem reads only images)
    all-gather          pass-A depth maps of every view
    geometric iter. 0   own problems, reading every view's pass-A depths
    all-gather          geometric depth maps
    geometric iter. k   own problems, reading iteration k-1's depths

The reference runs the geometric iterations view after view, so its second
iteration reads the maps of earlier views already updated in place.  Ranks
work at the same time, so here iteration k reads iteration k-1's maps of all
views; with one rank hpm_run_scene keeps the in-place order.

The per-problem work is a Solver (GpuSolver runs it through the C ABI); the
exchange is torch.distributed (NCCL over NVLink between GPUs, gloo in the
CPU tests).  Maps travel as float32 tensors on the solver's device.
"""
from __future__ import annotations

import numpy as np


def my_problems(n_problems: int, rank: int, world: int):
    return list(range(rank, n_problems, world))


class GpuSolver:
    """Per-problem passes through hpm_process_problem on one context; maps
    stay on the device (torch tensors)."""

    def __init__(self, ctx, images, cams, pairs, seed=0, pyramid_levels=-1, device="cuda"):
        import torch

        self.ctx, self.cams, self.pairs = ctx, np.asarray(cams), pairs
        self.seed, self.levels, self.device = seed, pyramid_levels, device
        self.images = [torch.as_tensor(np.asarray(i, np.float32), device=device) for i in images]
        self.torch = torch
        self._sync()

    def _sync(self):
        """Torch's stream before the C ABI reads tensors on its own stream."""
        if self.torch.device(self.device).type == "cuda":
            self.torch.cuda.current_stream(self.device).synchronize()

    def _views(self, p):
        ref, srcs = self.pairs[p]
        ids = [ref] + list(srcs)
        return ids, [self.images[i].data_ptr() for i in ids], self.cams[ids]

    def _set(self, p):
        import ctypes

        import hpm_b200 as hb

        ids, ptrs, cams = self._views(p)
        arr = (ctypes.c_void_p * len(ids))(*ptrs)
        cams = np.ascontiguousarray(cams, dtype=hb.CAMERA_DTYPE)
        self.ctx._check(hb.lib().hpm_set_views(self.ctx.handle, arr, hb._p(cams), len(ids)), "hpm_set_views")
        return ids

    def _run(self, p, *, geom, multi, seed, planes=None, costs=None, depths=None):
        import ctypes

        import hpm_b200 as hb

        torch = self.torch
        ids = self._set(p)
        h, w = self.images[ids[0]].shape
        if geom:
            arr = (ctypes.c_void_p * len(ids))(*[depths[i].data_ptr() for i in ids])
            self.ctx._check(hb.lib().hpm_set_geom_depths(self.ctx.handle, arr), "hpm_set_geom_depths")
            self.ctx._check(hb.lib().hpm_set_hypotheses(self.ctx.handle, ctypes.c_void_p(planes.data_ptr()),
                                                        ctypes.c_void_p(costs.data_ptr())), "hpm_set_hypotheses")
        d = torch.empty((h, w), dtype=torch.float32, device=self.device)
        n = torch.empty((h, w, 3), dtype=torch.float32, device=self.device)
        c = torch.empty((h, w), dtype=torch.float32, device=self.device)
        o = hb.HpmProblemOpts(int(not geom), int(geom), int(multi), int(seed), int(self.levels))
        self.ctx._check(hb.lib().hpm_process_problem(self.ctx.handle, ctypes.byref(o), ctypes.c_void_p(d.data_ptr()),
                                                     ctypes.c_void_p(n.data_ptr()), ctypes.c_void_p(c.data_ptr()),
                                                     None), "hpm_process_problem")
        return d, n, c

    def pass_a(self, p):
        return self._run(p, geom=False, multi=False, seed=self.seed + p)

    def geom(self, p, it, depths, normal, cost):
        ref = self.pairs[p][0]
        planes = self.torch.cat([normal, depths[ref][..., None]], -1).contiguous()
        self._sync()
        return self._run(p, geom=True, multi=it > 0, seed=self.seed + 1000003 * (it + 1) + p, planes=planes,
                         costs=cost, depths=depths)


def gather_maps(dist, maps, owners, shape_of, like):
    """Every view's map on every rank: rank r holds maps[v] for the views
    it owns; views are exchanged owner by owner with all_gather over a
    padded stack (one collective per round of owned views)."""
    import torch

    world = dist.get_world_size() if dist is not None else 1
    views = sorted(owners)
    if world == 1:
        return {v: maps[v] for v in views}
    out = {}
    per_rank = [[v for v in views if owners[v] == r] for r in range(world)]
    rounds = max(len(x) for x in per_rank)
    for k in range(rounds):
        shapes = [shape_of(per_rank[r][k]) if k < len(per_rank[r]) else None for r in range(world)]
        numel = max(int(np.prod(s)) for s in shapes if s is not None)
        mine = per_rank[dist.get_rank()]
        send = torch.zeros(numel, dtype=torch.float32, device=like.device)
        if k < len(mine):
            src = maps[mine[k]].reshape(-1)
            send[: src.numel()] = src
        recv = [torch.empty_like(send) for _ in range(world)]
        dist.all_gather(recv, send)
        if like.is_cuda:  # the C ABI reads the maps on its own stream next
            torch.cuda.current_stream(like.device).synchronize()
        for r in range(world):
            if shapes[r] is not None:
                out[per_rank[r][k]] = recv[r][: int(np.prod(shapes[r]))].reshape(shapes[r])
    return out


def run_scene_sharded(solver, pairs, view_shapes, *, geom_iterations=2, dist=None):
    """The scene with this rank's share of the problems.  Returns the final
    (depth, normal, cost) maps of the views this rank owns, and every view's
    final depth map (gathered)."""
    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    mine = my_problems(len(pairs), rank, world)
    owners = {pairs[p][0]: p % world for p in range(len(pairs))}
    depth, normal, cost = {}, {}, {}
    for p in mine:
        v = pairs[p][0]
        depth[v], normal[v], cost[v] = solver.pass_a(p)
    like = next(iter(depth.values())) if depth else None
    if like is None:  # a rank without problems still takes part in the exchanges
        import torch

        like = torch.zeros(1, device=getattr(solver, "device", "cpu"))
    shape = lambda v: view_shapes[v]  # noqa: E731
    all_depth = gather_maps(dist, depth, owners, shape, like)
    for it in range(geom_iterations):
        new = {}
        for p in mine:
            v = pairs[p][0]
            new[v], normal[v], cost[v] = solver.geom(p, it, all_depth, normal[v], cost[v])
        depth.update(new)
        all_depth = gather_maps(dist, depth, owners, shape, like)
    return {v: (depth[v], normal[v], cost[v]) for v in depth}, all_depth
