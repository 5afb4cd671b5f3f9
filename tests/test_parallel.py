"""Multi-rank host logic (CPU, gloo): frequency partitions of the reference's parallel helpers,
point balancing for uneven batches, and the gather / max-over-ranks path that ``bench.py --gpus N``
and batch runs take, with two real processes."""
import itertools
import os
import socket

import numpy as np
import pytest

import ladderdga_b200  # noqa: F401  (registers the package)
from ladderdga_b200 import parallel as P
from ladderdga_b200 import synthetic as S


class _SP:
    def __init__(self, n_iω, n_iν, shift=False, n_iν_shell=0):
        self.n_iω, self.n_iν, self.shift, self.n_iν_shell = n_iω, n_iν, shift, n_iν_shell


def _julia_partition(n, N):
    """The reference's formula verbatim in 1-based form (parallelization_helpers.jl:28)."""
    s, r = divmod(n, N)
    return [list(range(i * s + 1 + (i < r) * i + (i >= r) * r, (i + 1) * s + (i < r) * (i + 1) + (i >= r) * r + 1))
            for i in range(N)]


@pytest.mark.parametrize("n,N", [(21, 1), (21, 2), (21, 4), (41, 8), (8, 8), (10, 3), (61, 7)])
def test_par_partition_matches_reference_formula(n, N):
    got = [[i + 1 for i in r] for r in P.par_partition(n, N)]
    assert got == _julia_partition(n, N)
    assert sorted(itertools.chain.from_iterable(got)) == list(range(1, n + 1))


def test_par_partition_errors():
    with pytest.raises(RuntimeError):
        P.par_partition(3, 4)
    assert P.par_partition(5, 0) == [range(0, 5)]


def test_gen_omega_and_nu_omega_parts():
    sp = _SP(n_iω=10, n_iν=10)
    rng, part = P.gen_ω_part(sp, 4)
    assert [wn for _, wn in rng] == list(range(-10, 11))
    assert [len(p) for p in part] == [6, 5, 5, 5]
    rng2, part2 = P.gen_νω_part(_SP(n_iω=2, n_iν=3, shift=True), 3)
    assert len(rng2) == 5 * 6
    # shifted fermionic window for ωn = -2: ν = -3+1 .. 2+1
    assert [v for (w, v, _, _) in rng2 if w == -2] == list(range(-2, 4))
    assert [v for (w, v, _, _) in rng2 if w == 1] == list(range(-3, 3))   # trunc(1/2) = 0
    assert sum(len(p) for p in part2) == len(rng2)


def test_balance_points_is_a_cover_and_near_optimal():
    pts = S.batch_points(16, ns=8)
    w = [P.point_weight(2 * p["n_iv"], 15, 2 * p["n_iw"] + 1) for p in pts]
    for world in (1, 2, 3, 4):
        parts = P.balance_points(w, world)
        flat = sorted(itertools.chain.from_iterable(parts))
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        # list scheduling (Graham): makespan <= total / m + (1 - 1/m) max w
        assert max(loads) <= sum(w) / world + (1.0 - 1.0 / world) * max(w) + 1e-6 * sum(w)
        assert parts == P.balance_points(w, world)   # deterministic
    with pytest.raises(ValueError):
        P.rank_points(w, 2, 2)


def test_balance_small_exhaustive():
    rng = np.random.default_rng(3)
    w = list(rng.integers(1, 50, size=7).astype(float))
    best = min(max(sum(w[i] for i in range(7) if a[i] == r) for r in range(2)) for a in itertools.product((0, 1), repeat=7))
    parts = P.balance_points(w, 2)
    assert max(sum(w[i] for i in p) for p in parts) <= 4.0 / 3.0 * best + 1e-9


def test_without_process_group_everything_runs_here():
    out = P.run_points([3.0, 1.0, 2.0], lambda i: i * i)
    assert out == {0: 0, 1: 1, 2: 4}
    assert P.max_over_ranks(2.5) == 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, weights, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import ldga_ref as R
        kG = R.gen_kGrid("2Dsc-1.0", 6)

        def one(i):
            # a CPU stand-in for one parameter point: the oracle's kMult-weighted mean of a
            # point-dependent function on the irreducible wedge
            f = np.cos(0.3 * (i + 1) * np.asarray(kG.eps))
            return float(np.sum(kG.kMult * f) / np.sum(kG.kMult))

        res = P.run_points(weights, one)
        mine = P.rank_points(weights, rank, world)
        t = P.max_over_ranks(float(rank + 1) * 1.5)
        q.put((rank, res, mine, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_batch():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    weights = [P.point_weight(n, 45, n + 1) for n in (16, 30, 60, 120, 16, 30)]
    procs = [ctx.Process(target=_worker, args=(r, world, port, weights, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    outs.sort()
    from oracle import ldga_ref as R
    kG = R.gen_kGrid("2Dsc-1.0", 6)
    serial = {i: float(np.sum(kG.kMult * np.cos(0.3 * (i + 1) * np.asarray(kG.eps))) / np.sum(kG.kMult))
              for i in range(len(weights))}
    for rank, res, mine, t in outs:
        assert res == serial                      # every rank holds every point, bitwise
        assert t == 3.0                           # max over ranks of 1.5 * (rank + 1)
    assert sorted(outs[0][2] + outs[1][2]) == list(range(len(weights)))
    assert set(outs[0][2]).isdisjoint(outs[1][2])
    # the Nν = 120 point outweighs all others together: its rank takes nothing else
    heavy = 0 if 3 in outs[0][2] else 1
    assert outs[heavy][2] == [3]


def test_gen_nu_part_reference_case():
    """test/parallelization_helpers.jl:5-12 (sP_grid_s1 = SimulationParameters(4, 5, 2, true, ...)):
    three segments; the first holds νn = 0, 1 over the whole ω grid -4:4."""
    sp = _SP(n_iω=4, n_iν=5, shift=True)
    t = P.gen_ν_part(range(0, sp.n_iν), sp, 3)
    assert len(t) == 3
    data = np.random.default_rng(5).standard_normal((3, 2 * sp.n_iν, 2 * sp.n_iω + 1)) + 0j
    res, νn, ωn = P.gen_ν_part_slices(data, t[0])
    assert νn == [0, 1]
    assert ωn[0] == range(-4, 5)
    assert res.shape == (3, 9, 2)
    # every (ω, νn) cell of the segment carries the box value at its shifted ν index
    for wi, wn, vi, vn in t[0]:
        assert res[:, wi, νn.index(vn)].tolist() == data[:, vi, wi].tolist()
        assert vn == (vi - sp.n_iν) - int(sp.shift * wn / 2)
    # the segments cover the requested νn exactly once per (ω, νn) in the box
    seen = [(c[0], c[3]) for seg in t for c in seg]
    assert len(seen) == len(set(seen))
    assert {c[3] for seg in t for c in seg} == set(range(0, sp.n_iν))
