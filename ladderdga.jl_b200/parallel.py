"""Multi-GPU plumbing: one process per GPU, independent parameter points per rank.

The reference distributes one parameter point over Julia worker processes by bosonic frequency
(``gen_ω_part``, parallelization_helpers.jl:49-53) and scans parameter points (U, β) in separate
runs.  Here one B200 holds a whole parameter point (the chain of the largest configuration needs
~125 MB of HBM), so the unit of distribution is the parameter point: every rank runs the complete
chain for its share of the points and the ranks meet only to gather results and to take the
maximum of their step times.  There is no data-path collective.

The frequency partitions of the reference are kept (``par_partition``, ``gen_ω_part``,
``gen_νω_part``) because the parallel API of ``core`` reports them, and because they define the
split a caller would use to shard one point by ω.

Uneven batches (points with different Nν) are balanced by a longest-processing-time greedy over
the BSE work of each point (N_q · N_ω · Nν³ per channel), which dominates the chain.
"""
from __future__ import annotations

import heapq
from typing import Any, Callable, Sequence


def par_partition(set_, N: int) -> list[range]:
    """Index ranges of ``set_`` split into ``N`` (almost) equal contiguous segments, the first
    ``len % N`` one longer (parallelization_helpers.jl:22-29).  0-based ranges."""
    n = set_ if isinstance(set_, int) else len(set_)
    if N > n:
        raise RuntimeError(f"Cannot split set of length {n} into {N} partitions.")
    N = 1 if N <= 0 else N
    s, r = divmod(n, N)
    return [range(i * s + min(i, r), (i + 1) * s + min(i + 1, r)) for i in range(N)]


def gen_ω_part(sP, N: int):
    """``(ωi_range, ωi_part)``: the bosonic grid as (index, ωn) pairs and its partition over ``N``
    workers (parallelization_helpers.jl:49-53).  Indices are 0-based."""
    ωi_range = [(i, wn) for i, wn in enumerate(range(-sP.n_iω, sP.n_iω + 1))]
    return ωi_range, par_partition(ωi_range, N)


def gen_νω_part(sP, N: int):
    """``(ωνi_range, ωνi_part)`` over (ωn, νn, ωi, νi) with the shift of ν by ⌊shift·ωn/2⌋
    (parallelization_helpers.jl:36-42)."""
    rng = []
    nv = sP.n_iν + getattr(sP, "n_iν_shell", 0)
    for wi, wn in enumerate(range(-sP.n_iω, sP.n_iω + 1)):
        off = int(sP.shift * wn / 2)  # trunc, as Julia's trunc(Int, ·)
        for vi, vn in enumerate(range(-nv - off, nv - off)):
            rng.append((wn, vn, wi, vi))
    return rng, par_partition(rng, N)


def gen_ν_part(νGrid, sP, N: int) -> list[list[tuple[int, int, int, int]]]:
    """``gen_ν_part`` (parallelization_helpers.jl:62-68): ``νGrid`` (the EoM's νn, e.g.
    ``range(0, n_iν)``) split into ``N`` segments; each segment's list of (ωi, ωn, νi, νn) over the
    box whose νn lies in the segment, sorted by νn (stable, so ω ascends within one νn).  νn is the
    shifted frequency νn − ⌊shift·ωn/2⌋ (trunc); ωi and νi are 0-based here."""
    grid = list(νGrid)
    parts = par_partition(grid, N)
    cells = []
    for vi, j in enumerate(range(-sP.n_iν, sP.n_iν)):          # Julia's comprehension: ω fastest
        for wi, wn in enumerate(range(-sP.n_iω, sP.n_iω + 1)):
            cells.append((wi, wn, vi, j - int(sP.shift * wn / 2)))
    out = []
    for seg in parts:
        keep = set(grid[i] for i in seg)
        out.append(sorted((c for c in cells if c[3] in keep), key=lambda c: c[3]))
    return out


def gen_ν_part_slices(data, index_list):
    """``gen_ν_part_slices`` (parallelization_helpers.jl:81-102): ``data`` [Nq, Nν, Nω] rearranged
    for one segment of ``gen_ν_part`` -> (res [Nq, Nω, len(νn_list)] with zeros where a (ω, νn) is
    not in the box, νn_list, ωn_ranges)."""
    import numpy as np
    data = np.asarray(data)
    νn = [c[3] for c in index_list]
    νn_list = list(dict.fromkeys(νn))                            # unique, first-seen order
    res = np.zeros((data.shape[0], data.shape[2], len(νn_list)), dtype=data.dtype, order="F")
    ωn_ranges = []
    for v in νn_list:
        sl = [c[1] for c in index_list if c[3] == v]
        ωn_ranges.append(range(sl[0], sl[-1] + 1))
    k, cur = 0, index_list[0][3]
    for wi, _, vi, vn in index_list:
        if vn != cur:
            cur = vn
            k += 1
        res[:, wi, k] = data[:, vi, wi]
    return res, νn_list, ωn_ranges


def point_weight(n_nu: int, n_q: int, n_w: int) -> float:
    """Relative cost of one parameter point: the two BSE channels, N_q N_ω matrices of Nν³."""
    return float(n_q) * float(n_w) * float(n_nu) ** 3


def balance_points(weights: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Assign points to ranks, heaviest first, each to the least-loaded rank (ties: lower rank,
    then lower point index).  Deterministic, so every rank computes the same assignment without
    communication.  Each rank's list is in ascending point order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    out: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    return [sorted(x) for x in out]


def rank_points(weights: Sequence[float], rank: int, world: int) -> list[int]:
    """The points of ``rank`` in a ``world``-rank job (``balance_points``)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside 0..{world - 1}")
    return balance_points(weights, world)[rank]


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float, group=None, device=None) -> float:
    """Maximum of ``value`` over the ranks of the default (or given) process group; the value
    itself without one.  ``device``: where the reduction tensor lives (a CUDA device for NCCL,
    None = CPU for gloo)."""
    dist = _dist()
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_points(local: dict, group=None) -> dict:
    """Merge the per-rank ``{point index: result}`` dicts on every rank (all_gather_object).  A
    point reported by two ranks is an assignment error and raises."""
    dist = _dist()
    if dist is None:
        return dict(local)
    parts: list[Any] = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, dict(local), group=group)
    merged: dict = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"point {k} was computed by more than one rank")
            merged[k] = v
    return merged


def run_points(weights: Sequence[float], run_one: Callable[[int], Any], group=None) -> dict:
    """Run ``run_one(i)`` for this rank's share of the points and return every point's result on
    every rank, in point order.  Without a process group all points run here."""
    dist = _dist()
    rank, world = (dist.get_rank(group), dist.get_world_size(group)) if dist else (0, 1)
    mine = rank_points(weights, rank, world)
    local = {i: run_one(i) for i in mine}
    merged = gather_points(local, group)
    missing = set(range(len(weights))) - set(merged)
    if missing:
        raise RuntimeError(f"points without a result: {sorted(missing)}")
    return {i: merged[i] for i in range(len(weights))}
