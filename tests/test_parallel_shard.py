"""One parameter point sharded by bosonic frequency over two and three gloo ranks on the CPU: the host logic of
``parallel.λm_chain_omega_sharded`` (the reference's ω partition over workers, gen_ω_part /
par_partition, parallelization_helpers.jl:22-53, with calc_bubble_par / calc_χγ_par / calc_Σ_par,
ladderDGATools.jl:46-245).

The stages run on a stand-in for the library handle built on the oracle (test infrastructure): it
computes each stage the way the oracle does and exposes only what the driver exchanges -- this
rank's block of χ_m / χ_d and this rank's ω part of Σ_ladder, with the tail and Hartree terms where
the driver asks for them.  The driver's partition, the χ assembly, the Σ all-reduce and the shared
λm / μ / energies must then reproduce the oracle's unsharded λm chain (conditions_new.jl:174-190).
"""
import os
import socket

import numpy as np
import pytest

import ladderdga_b200  # noqa: F401  (registers the package)
from ladderdga_b200 import parallel as P
from ladderdga_b200 import synthetic as S

INP = dict(dim=2, ns=8, beta=5.0, U=1.2, n_iv=4, n_iw=4, seed=31)


class OracleStages:
    """The sharded chain's stages on the oracle: every stage is computed whole, and the driver sees
    only this rank's block (get_chi) and this rank's part of Σ_ladder (eom)."""

    def __init__(self, inp):
        from oracle import ldga_ref as R
        self.R = R
        self.h = R.setup_ldga(inp)
        h = self.h
        self.Nq, self.Nnu, self.Nw = h.kG.Nq, 2 * h.sP.n_iv, 2 * h.sP.n_iw + 1
        self.block, self.constants = range(0, self.Nw), True
        self.calls = []

    def set_shard(self, lo, hi, constants):
        self.block, self.constants = range(lo, hi), bool(constants)
        self.calls.append(("shard", lo, hi, bool(constants)))

    def bubble(self):
        h, R = self.h, self.R
        self.chi0 = R.calc_bubble(h.ghat, h.grhat, h.kG, h.mP, h.sP)

    def bse(self, ch):
        h, R = self.h, self.R
        x, g = R.calc_chi_gamma("m" if ch == 0 else "d", h.Gamma_m if ch == 0 else h.Gamma_d, self.chi0, h.mP, h.sP)
        setattr(self, f"x{ch}", x)
        setattr(self, f"g{ch}", g)

    def lambda0(self):
        h, R = self.h, self.R
        self.l0 = R.calc_lambda0(self.chi0, R.F_m_of(h), h.mP, h.sP)

    def get_chi(self, ch, buf):
        # the whole array, as the library returns it; outside this rank's block its entries are
        # not this rank's to give: poison them so that a driver which forgot to mask them fails
        x = np.array(getattr(self, f"x{ch}").T)                  # [ω, q]
        mask = np.ones(self.Nw, bool)
        mask[self.block.start:self.block.stop] = False
        x[mask] = np.nan
        buf.copy_(__import__("torch").from_numpy(x))

    def set_chi(self, ch, buf):
        setattr(self, f"gathered{ch}", buf.numpy().T.copy())    # [q, ω]

    def lambda_m(self):
        h, R = self.h, self.R
        self.cm = R.ChiT(self.gathered0, h.mP.beta, tail_c=[0, 0, h.mP.Ekin_DMFT])
        self.cd = R.ChiT(self.gathered1, h.mP.beta, tail_c=[0, 0, h.mP.Ekin_DMFT])
        rhs = R.lambda_m_rhs(h.imp_density, self.cm, self.cd, h.kG, h.mP, h.sP)
        lam, _ = R.lambda_m_correction(self.cm, rhs, h.kG, h.mP, h.sP)
        return lam, 0

    def eom(self, lam, numax, out):
        h, R = self.h, self.R
        cm = self.cm.copy()
        R.chi_lambda_inplace(cm, lam)
        parts = R.calc_Sigma_w(R.eom, cm.data, self.g0, self.cd.data, self.g1, self.l0, h.grhat, h.kG, h.mP.U,
                               h.sP, numax)
        S = parts[:, :, self.block.start:self.block.stop].sum(axis=2) / h.mP.beta
        if self.constants:
            tail = -h.mP.U * (R.sum_kw(h.kG, cm) - h.chiloc_m_sum) / R.iv_array(h.mP.beta, range(numax))
            S = S + tail[None, :] + h.mP.n * h.mP.U / 2.0
        v = np.ascontiguousarray(S.T).view(np.float64).reshape(numax, self.Nq, 2)
        out.copy_(__import__("torch").from_numpy(v))

    def finish(self, lam, numax, sigma):
        h, R = self.h, self.R
        S = sigma.numpy().view(np.complex128)[..., 0].T.copy()
        mu, G = R.G_from_Sigma_ladder(S, h.sigma_loc, h.kG, h.mP, h.sP.fft_range, fix_n=True)
        off = -h.sP.fft_range[0]
        ek, ep = R.calc_E(G[:, off:off + numax], S, mu, h.kG, h.mP)
        return {"lambda_m": lam, "mu": mu, "E_kin": ek, "E_pot1": ep, "Sigma_ladder": S}


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
        st = OracleStages(S.make_input(**INP))
        res = P.λm_chain_omega_sharded(st)
        q.put((rank, res, st.calls))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_omega_sharded_chain_matches_unsharded_oracle(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import ldga_ref as R
    ref = R.run_chain(S.make_input(**INP), lambda_type="m")["result"]
    nw = 2 * INP["n_iw"] + 1
    blocks = [o[1]["block"] for o in outs]
    assert blocks == [(r.start, r.stop) for r in P.par_partition(nw, world)]
    for rank, res, calls in outs:
        assert calls[0] == ("shard", *blocks[rank], rank == 0)      # constants on rank 0 only
        assert calls[-1] == ("shard", 0, nw, True)                   # the handle is left whole
        assert res["lambda_m"] == ref.lam_m                            # the same χ: the same Newton
        s_ref = np.asarray(ref.Sigma_ladder)
        assert np.max(np.abs(res["Sigma_ladder"] - s_ref)) <= 1e-12 * np.max(np.abs(s_ref))
        assert abs(res["mu"] - ref.mu) <= 1e-12
        assert abs(res["E_kin"] - ref.EKin) <= 1e-12 * max(1.0, abs(ref.EKin))
        assert abs(res["E_pot1"] - ref.EPot_p1) <= 1e-12 * max(1.0, abs(ref.EPot_p1))
    # every rank holds the same result, bit for bit
    for _, res, _ in outs[1:]:
        assert np.array_equal(res["Sigma_ladder"], outs[0][1]["Sigma_ladder"])


def test_omega_sharded_chain_without_process_group():
    """No process group: the whole ω range runs here, and the result is the oracle's chain."""
    from oracle import ldga_ref as R
    st = OracleStages(S.make_input(**INP))
    res = P.λm_chain_omega_sharded(st)
    ref = R.run_chain(S.make_input(**INP), lambda_type="m")["result"]
    assert res["block"] == (0, 2 * INP["n_iw"] + 1)
    assert res["lambda_m"] == ref.lam_m
    assert np.max(np.abs(res["Sigma_ladder"] - ref.Sigma_ladder)) <= 1e-12 * np.max(np.abs(ref.Sigma_ladder))
