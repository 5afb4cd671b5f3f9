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

import numpy as np
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


# ------------------------------------------------------------------------------------------------
# One parameter point sharded by bosonic frequency (the reference's worker split: gen_ω_part,
# parallelization_helpers.jl:49-53, used by calc_bubble_par / calc_χγ_par / calc_Σ_par,
# ladderDGATools.jl:46-245).  Every rank computes the bubble, both BSE channels and λ₀ on its ω
# block (par_partition of 0..Nω-1), the ranks assemble the whole χ_m and χ_d (one all-reduce each,
# every rank contributing its block and zeros elsewhere: exact), run the λm Newton on the whole χ
# (every rank the same kernel on the same data: the same λm), form their ω block's part of
# Σ_ladder, and sum those parts with one all-reduce; the tail and Hartree terms come from rank 0
# only.  The μ fit and the energies then run on every rank on the same Σ_ladder.  The exchanged
# data are N_q N_ω doubles per channel and N_q νmax complex values: 0.3 MB each on the 3D 32³ point.
# ------------------------------------------------------------------------------------------------
class HandleStages:
    """The sharded chain's stages on a library handle (``core.lDΓAHelper``), through the C ABI.
    Exchange buffers are torch tensors on ``device`` (a CUDA device for NCCL, the CPU for gloo);
    the library reads and writes them directly (host or device pointers)."""

    def __init__(self, h):
        self.h = h
        self.ctx = h.ctx
        self.Nq, self.Nnu, self.Nw = self.ctx.Nq, self.ctx.Nnu, self.ctx.Nw

    @staticmethod
    def _ptr(t):
        import ctypes as C
        return C.c_void_p(t.data_ptr())

    def set_shard(self, w_lo: int, w_hi: int, constants: bool) -> None:
        self.ctx.call("ldga_set_omega_shard", int(w_lo), int(w_hi), int(bool(constants)))

    def bubble(self) -> None:
        self.ctx.call("ldga_bubble", None)

    def bse(self, ch: int) -> None:
        import ctypes as C
        from ._lib import as_fc, ptr
        nfb = C.c_int32(0)
        Γ = self.h.Γ_m if ch == 0 else self.h.Γ_d
        self.ctx.call("ldga_bse", ch, ptr(as_fc(Γ)), None, None, C.byref(nfb))

    def lambda0(self) -> None:
        from ._lib import ptr
        h = self.h
        self.ctx.call("ldga_F_from_chi", ptr(h.χDMFT_m), ptr(h.gImp), len(h.gImp), None)
        self.ctx.call("ldga_lambda0", None, None)

    def get_chi(self, ch: int, buf) -> None:
        from . import _lib
        self.ctx.call("ldga_get", _lib.GET_CHI, ch, self._ptr(buf))

    def set_chi(self, ch: int, buf) -> None:
        self.ctx.call("ldga_set_chi", ch, self._ptr(buf))

    def lambda_m(self) -> tuple[float, int]:
        import ctypes as C
        s = C.c_double()
        self.ctx.call("ldga_sum_kw", 1, 0.0, 0, C.byref(s))
        rhs = 2.0 * self.h.imp_density - s.value
        lam, its = C.c_double(), C.c_int32()
        self.ctx.call("ldga_lambda_m", rhs, C.byref(lam), C.byref(its))
        return lam.value, its.value

    def eom(self, lam_m: float, numax: int, out) -> None:
        self.ctx.call("ldga_eom", float(lam_m), 0.0, int(numax), 1, self.h.χloc_m_sum, self._ptr(out))

    def finish(self, lam_m: float, numax: int, sigma) -> dict:
        from .core import G_from_Σladder, calc_E
        h = self.h
        S = sigma.cpu().numpy().view(np.complex128)[..., 0].T.copy()          # [Nq, numax]
        mu, G = G_from_Σladder(S, h.Σ_loc, h.kG, h.mP, h.sP, fix_n=True, h=h)
        off = -h.sP.fft_range[0]
        ek, ep = calc_E(G[:, off:off + numax], S, mu, h.kG, h.mP, h=h)
        return {"lambda_m": lam_m, "mu": mu, "E_kin": ek, "E_pot1": ep, "Sigma_ladder": S}


def λm_chain_omega_sharded(stages, group=None, numax: int | None = None) -> dict:
    """The λm chain (run_minimal.jl: bubble -> χ, γ of m and d -> λ₀ -> λm_correction_full,
    conditions_new.jl:174-190) of one parameter point with its bosonic frequencies split over the
    ranks of ``group`` (all stages of ``stages`` on this rank's block).  Without a process group
    the whole range runs here.  Returns λm, the Newton iterations, μ, the energies and Σ_ladder
    (the same on every rank) and this rank's block."""
    import torch
    dist = _dist()
    rank, world = (dist.get_rank(group), dist.get_world_size(group)) if dist else (0, 1)
    backend = dist.get_backend(group) if dist else "gloo"
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    nq, nnu, nw = stages.Nq, stages.Nnu, stages.Nw
    block = par_partition(nw, world)[rank]
    numax = nnu // 2 if numax is None else int(numax)
    stages.set_shard(block.start, block.stop, rank == 0)
    try:
        stages.bubble()
        stages.bse(0)
        stages.bse(1)
        stages.lambda0()
        for ch in (0, 1):
            buf = torch.zeros((nw, nq), dtype=torch.float64, device=dev)     # column-major [q, ω]
            stages.get_chi(ch, buf)
            buf[: block.start] = 0.0                                           # other ranks' blocks
            buf[block.stop:] = 0.0
            if dist:
                dist.all_reduce(buf, group=group)
            stages.set_chi(ch, buf)
        lam, its = stages.lambda_m()
        sigma = torch.zeros((numax, nq, 2), dtype=torch.float64, device=dev)  # column-major [q, ν] complex
        stages.eom(lam, numax, sigma)
        if dist:
            dist.all_reduce(sigma, group=group)
        res = stages.finish(lam, numax, sigma)
    finally:
        stages.set_shard(0, nw, True)
    res["newton_iterations"] = its
    res["block"] = (block.start, block.stop)
    return res
