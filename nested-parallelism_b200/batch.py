"""Batched SSSP: the 64-instance R-MAT workload, its sharding over ranks, and
the one-launch batch run of each shard.

Workload: `count` independent R-MAT graphs (a=.57 b=.19 c=.19, no noise,
duplicates and self-loops removed), scale drawn uniformly from 12..18, edge
factor from {4, 8, 16, 32}, uint32 weights uniform in [1, 255], and a source
vertex drawn uniformly, all from one seeded generator.  The reference runs one
SSSP per process (apps/sssp/src/gpu/sssp.cpp:141); here the whole batch is one
persistent cooperative launch (nps_sssp_batch) replayed from a CUDA graph.

Multi-GPU: the instances shard with no exchange during the solve.  Ranks take
the instances of a longest-processing-time partition by work (m + n), solve
their shard in one launch, and all-gather per-instance results (FNV-1a hash of
the distances, reached count, iterations) at the end.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import Graph, Instance, Params, fnv1a, gen_rmat, sssp_batch

SCALES = (12, 18)
EDGE_FACTORS = (4, 8, 16, 32)


@dataclasses.dataclass
class BatchItem:
    index: int
    scale: int
    edge_factor: int
    graph_seed: int
    graph: Graph
    source: int


def rmat_batch(count: int = 64, seed: int = 7, scales: Tuple[int, int] = SCALES,
               edge_factors: Sequence[int] = EDGE_FACTORS, only: Sequence[int] = None) -> List[BatchItem]:
    """The batch workload.  Instance i's scale, edge factor, graph seed and
    source depend only on (seed, i); `only` builds a subset of the indices."""
    rng = np.random.default_rng(seed)
    draws = [(int(rng.integers(scales[0], scales[1] + 1)), int(rng.choice(edge_factors)),
              int(rng.integers(0, 1 << 31)), float(rng.random())) for _ in range(count)]
    keep = range(count) if only is None else only
    out = []
    for i in keep:
        scale, ef, gseed, u = draws[i]
        g = gen_rmat(scale, ef, seed=gseed)
        out.append(BatchItem(i, scale, ef, gseed, g, min(int(u * g.n), g.n - 1)))
    return out


def work_estimate(scale: int, edge_factor: int) -> int:
    """Work of an instance before it is generated: n + generated edges."""
    return (1 << scale) * (1 + edge_factor)


def shard(work: Sequence[int], world: int) -> List[List[int]]:
    """Longest-processing-time partition of instance indices into `world` shards
    (largest first onto the least-loaded shard; ties by lower shard index)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        r = min(range(world), key=lambda s: (loads[s], s))
        parts[r].append(i)
        loads[r] += int(work[i])
    return [sorted(p) for p in parts]


def shard_indices(count: int, seed: int, world: int, rank: int, scales=SCALES, edge_factors=EDGE_FACTORS):
    """Indices of the instances rank `rank` solves (the same on every rank)."""
    rng = np.random.default_rng(seed)
    draws = [(int(rng.integers(scales[0], scales[1] + 1)), int(rng.choice(edge_factors)),
              int(rng.integers(0, 1 << 31)), float(rng.random())) for _ in range(count)]
    return shard([work_estimate(s, ef) for s, ef, _, _ in draws], world)[rank]


class DeviceBatch:
    """Device copies of a list of BatchItems and their Instance descriptors."""

    def __init__(self, items: Sequence[BatchItem], device):
        import torch
        self.items = list(items)
        self.keep = []
        self.instances = []
        for it in self.items:
            g = it.graph
            t = [torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(device)
                 for a in (g.row_ptr, g.col, g.w)]
            dist = torch.empty(g.n, dtype=torch.int32, device=device)
            self.keep.append((*t, dist))
            self.instances.append(Instance(t[0], t[1], t[2], dist, g.n, g.m, it.source))

    def run(self, params: Params, use_graph: bool = True, stream=None):
        return sssp_batch(self.instances, params, use_graph=use_graph, stream=stream)

    def distances(self) -> List[np.ndarray]:
        return [k[3].cpu().numpy().view(np.uint32).copy() for k in self.keep]

    def results(self) -> List[Dict]:
        out = []
        for it, d in zip(self.items, self.distances()):
            reached = d < 0x40000000
            out.append({"index": it.index, "fnv1a": fnv1a(d), "reached": int(reached.sum()),
                        "m_reached": int(np.diff(it.graph.row_ptr)[reached].sum())})
        return out


def gather_results(local: List[Dict], group=None) -> List[Dict]:
    """All-gather per-instance result dicts over torch.distributed (any backend);
    returns them sorted by instance index on every rank."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return sorted(local, key=lambda r: r["index"])
    world = dist.get_world_size(group)
    got: List[List[Dict]] = [None] * world  # type: ignore[list-item]
    dist.all_gather_object(got, local, group=group)
    return sorted((r for part in got for r in part), key=lambda r: r["index"])
