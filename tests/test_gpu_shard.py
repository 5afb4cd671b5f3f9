"""ω-sharded parameter point on the GPU (ldga_set_omega_shard and parallel.λm_chain_omega_sharded).

The reference splits one point's bosonic frequencies over workers (gen_ω_part / par_partition,
parallelization_helpers.jl:22-53; calc_bubble_par / calc_χγ_par / calc_Σ_par, ladderDGATools.jl:46-245).
Here every shard's stages run on the library's kernels restricted to its ω block:

* one process, the shards one after another on one handle: χ_m, χ_d, γ and λ₀ of every block equal the
  unsharded run bit for bit (each (q, ω) matrix is solved the same way), and the shards' Σ_ladder parts,
  the tail and Hartree terms added once, sum to the unsharded Σ_ladder;
* two processes on this GPU joined by gloo (host collectives: no kernel waits on another process):
  the driver's λm, μ, energies and Σ_ladder against the unsharded chain and the FP64 oracle;
* entry points that need every frequency refuse a sharded handle.
"""
import ctypes as C
import os
import socket

import numpy as np
import pytest

import ladderdga_b200 as L
from ladderdga_b200 import _lib
from ladderdga_b200 import parallel as P
from ladderdga_b200 import synthetic as S

pytestmark = pytest.mark.gpu

SMALL = dict(dim=3, ns=8, beta=5.0, U=1.2, n_iv=4, n_iw=4, seed=77)


def _arrays(ctx):
    nq, nnu, nw = ctx.Nq, ctx.Nnu, ctx.Nw
    out = {}
    for name, what, ch, real in (("chi_m", _lib.GET_CHI, 0, True), ("chi_d", _lib.GET_CHI, 1, True),
                                 ("gamma_m", _lib.GET_GAMMA, 0, False), ("gamma_d", _lib.GET_GAMMA, 1, False),
                                 ("lambda0", _lib.GET_LAMBDA0, 0, False), ("chi0", _lib.GET_CHI0, 0, False)):
        a = np.empty((nq, nw), order="F") if real else _lib.cplx_out((nq, nnu, nw))
        ctx.call("ldga_get", what, ch, _lib.ptr(a))
        out[name] = a
    return out


def _sigma(st, lam, numax):
    import torch
    s = torch.zeros((numax, st.Nq, 2), dtype=torch.float64)
    st.eom(lam, numax, s)
    return s.numpy().view(np.complex128)[..., 0].T.copy()


@pytest.mark.parametrize("inp_kw,prec", [(None, L.PREC_MIXED), (SMALL, L.PREC_FP64)])
def test_shards_one_after_another_equal_the_whole_point(require_gpu, inp_kw, prec):
    inp = S.config_input(3) if inp_kw is None else S.make_input(**inp_kw)
    h = L.setup_synthetic(inp, precision=prec)
    ctx = h.ctx
    st = P.HandleStages(h)
    st.bubble(); st.bse(0); st.bse(1); st.lambda0()
    whole = _arrays(ctx)
    lam, _ = st.lambda_m()
    numax = ctx.Nnu // 2
    s_whole = _sigma(st, lam, numax)
    for world in (2, 3):
        blocks = P.par_partition(ctx.Nw, world)
        got = {k: np.full_like(v, np.nan) for k, v in whole.items()}
        for b in blocks:
            st.set_shard(b.start, b.stop, False)
            st.bubble(); st.bse(0); st.bse(1); st.lambda0()
            a = _arrays(ctx)
            for k in got:
                got[k][..., b.start:b.stop] = a[k][..., b.start:b.stop]
        for k in got:
            assert np.array_equal(got[k], whole[k]), (world, k)        # bit for bit
        # the handle holds every block's χ now: Σ parts per block, the constant terms once
        parts = []
        for r, b in enumerate(blocks):
            st.set_shard(b.start, b.stop, r == 0)
            parts.append(_sigma(st, lam, numax))
        st.set_shard(0, ctx.Nw, True)
        s_sum = np.sum(parts, axis=0)
        assert np.max(np.abs(s_sum - s_whole)) <= 1e-13 * np.max(np.abs(s_whole)), world


def test_sharded_handle_refuses_whole_range_entry_points(require_gpu):
    h = L.setup_synthetic(S.make_input(**SMALL))
    ctx = h.ctx
    lib = ctx.lib
    assert lib.ldga_set_omega_shard(ctx.h, 3, 3, 1) == _lib.LDGA_ERR_ARG            # empty
    assert lib.ldga_set_omega_shard(ctx.h, 0, ctx.Nw + 1, 1) == _lib.LDGA_ERR_ARG    # outside
    ctx.call("ldga_set_omega_shard", 2, 5, 0)
    z = np.zeros(4 * ctx.Nnu * ctx.Nnu * ctx.Nw)
    st = lib.ldga_chain_m(ctx.h, _lib.ptr(z), 4, _lib.ptr(z), _lib.ptr(z), _lib.ptr(z), _lib.ptr(z), 4, 0.5, 0.1, 0,
                          None, None, None, None)
    assert st == _lib.LDGA_ERR_STATE
    assert b"shard" in lib.ldga_last_error(ctx.h)
    lm, ld, its = C.c_double(), C.c_double(), C.c_int32()
    st = lib.ldga_lambda_dm(ctx.h, 0.1, 2, 1e-4, 1e-8, 10, C.byref(lm), C.byref(ld), C.byref(its), None, None, None,
                            None)
    assert st == _lib.LDGA_ERR_STATE
    ctx.call("ldga_set_omega_shard", 0, ctx.Nw, 1)                                   # whole again


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        h = L.setup_synthetic(S.make_input(**SMALL))
        res = P.λm_chain_omega_sharded(P.HandleStages(h))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_processes_gloo_on_one_gpu(require_gpu):
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = sorted([q.get(timeout=600) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # the unsharded chain on the same GPU, and the oracle
    h = L.setup_synthetic(S.make_input(**SMALL))
    whole = P.λm_chain_omega_sharded(P.HandleStages(h))
    from oracle import ldga_ref as R
    ref = R.run_chain(S.make_input(**SMALL), lambda_type="m")["result"]
    for rank, res in outs:
        assert res["lambda_m"] == whole["lambda_m"]                      # the same χ: the same Newton
        assert abs(res["lambda_m"] - ref.lam_m) <= 1e-10
        for other in (whole["Sigma_ladder"], np.asarray(ref.Sigma_ladder)):
            assert np.max(np.abs(res["Sigma_ladder"] - other)) <= 1e-10 * np.max(np.abs(other))
        assert abs(res["mu"] - ref.mu) <= 1e-10
        assert abs(res["E_kin"] - ref.EKin) <= 1e-10 * max(1.0, abs(ref.EKin))
        assert abs(res["E_pot1"] - ref.EPot_p1) <= 1e-10 * max(1.0, abs(ref.EPot_p1))
    assert np.array_equal(outs[0][1]["Sigma_ladder"], outs[1][1]["Sigma_ladder"])
