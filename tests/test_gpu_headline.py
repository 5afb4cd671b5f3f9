"""GPU parity at the benchmarked sizes, through the C ABI, against the FP64 oracle.

* Configuration 3 (3D sc 32^3, 969 irreducible q, beta = 20, U = 1.5, Nnu = 40, Nw = 41): the headline
  workload in MIXED mode, run as the benchmark runs it -- autotuned BSE, the whole lambda_m chain in
  one ldga_chain_m call, captured in a CUDA graph and replayed -- and every compiled configuration of
  the preconditioned BSE at this size.
* Configuration 2 (2D 64^2, 561 irreducible q, beta = 30, U = 2, Nnu = 60, Nw = 61): lambda_dm in FP64
  and in MIXED mode.

Tolerances: elementwise relative 1e-10 (denominator max(|oracle|, 1e-6 max|oracle|)) for chi0, chi_r,
gamma_r, lambda0, Sigma_ladder and G_ladder; absolute 1e-10 for mu; relative 1e-10 for the energies.
lambda_m of configuration 3 is not a parity quantity: newton_right (LambdaCorrection/helpers.jl:133-153)
with the derivative df_c1 of conditions_new.jl:150-153, which carries the chi tail constants, walks
away from f's root left of 0 into the poles of f (the synthetic chi_m < 0 at large |w|), where its
iterates depend on the rounding of the sums.  There the device's lambda_m is checked to be a root of
the oracle's f, and the lambda-dependent outputs are compared at the oracle's lambda_m.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

import ladderdga_b200 as L
from ladderdga_b200 import _lib
from ladderdga_b200 import synthetic as S
from oracle import ldga_ref as R

pytestmark = pytest.mark.gpu

RTOL = 1e-10
FLOOR = 1e-6


def rel(a, b):
    """Elementwise relative difference max |a - b| / max(|b|, FLOOR max|b|)."""
    a, b = np.asarray(a), np.asarray(b)
    m = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), FLOOR * m)))


def device_arrays(ctx):
    nq, nnu, nw = ctx.Nq, ctx.Nnu, ctx.Nw

    def get(what, ch=0, real=False):
        out = np.empty((nq, nw), order="F") if real else _lib.cplx_out((nq, nnu, nw))
        ctx.call("ldga_get", what, ch, _lib.ptr(out))
        return out

    return {"chi0": get(_lib.GET_CHI0), "chi_m": get(_lib.GET_CHI, _lib.CH_M, True),
            "chi_d": get(_lib.GET_CHI, _lib.CH_D, True), "gamma_m": get(_lib.GET_GAMMA, _lib.CH_M),
            "gamma_d": get(_lib.GET_GAMMA, _lib.CH_D), "lambda0": get(_lib.GET_LAMBDA0)}


def chi_rel(a, ref, r):
    """Componentwise error of chi_r(q, w) = Re sum_nu y_nu / beta^2: |a - chi| divided by the magnitude
    of the summed terms, sum_nu |y_nu| / beta^2 with y = gamma chi0 (1 + s U chi) from the oracle.  Where
    the terms cancel, no FP64 evaluation of the sum is more accurate than that magnitude allows."""
    mP = ref["h"].mP
    s = 1.0 if r == "m" else -1.0
    chi = ref[f"chi_{r}"].data
    y = ref[f"gamma_{r}"] * ref["chi0"] * (1.0 + s * mP.U * chi)[:, None, :]
    scale = np.abs(y).sum(axis=1) / mP.beta ** 2
    return float(np.max(np.abs(np.asarray(a) - chi) / np.maximum(scale, 1e-300)))


def check_arrays(dev, ref, what):
    for k in ("chi0", "lambda0", "gamma_m", "gamma_d"):
        assert rel(dev[k], ref[k]) < RTOL, (what, k, rel(dev[k], ref[k]))
    for r in ("m", "d"):
        assert chi_rel(dev[f"chi_{r}"], ref, r) < RTOL, (what, r, chi_rel(dev[f"chi_{r}"], ref, r))


def set_oracle_inputs(ctx, ref):
    """The oracle's chi, gamma and lambda0 as the handle's EoM inputs (each later stage alone)."""
    ctx.call("ldga_set_chi", _lib.CH_M, _lib.ptr(np.asfortranarray(ref["chi_m"].data)))
    ctx.call("ldga_set_chi", _lib.CH_D, _lib.ptr(np.asfortranarray(ref["chi_d"].data)))
    ctx.call("ldga_set_gamma", _lib.CH_M, _lib.ptr(_lib.as_fc(ref["gamma_m"])))
    ctx.call("ldga_set_gamma", _lib.CH_D, _lib.ptr(_lib.as_fc(ref["gamma_d"])))
    ctx.call("ldga_set_lambda0", _lib.ptr(_lib.as_fc(ref["lambda0"])))


def g_ladder(h, sigma=None):
    """μ fit, G_ladder and energies on the device from the handle's Σ_ladder (or the given one)."""
    ctx = h.ctx
    if sigma is not None:
        ctx.call("ldga_set_sigma", _lib.ptr(_lib.as_fc(sigma)), sigma.shape[1])
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))
    mu, ek, ep, n = (C.c_double() for _ in range(4))
    ctx.call("ldga_g_ladder", None, 0, 1, h.mP.μ, C.byref(mu), _lib.ptr(G), C.byref(ek), C.byref(ep), C.byref(n))
    return G, mu.value, ek.value, ep.value


class ChainM:
    """ldga_chain_m from pinned host buffers, as the benchmark's end-to-end leg calls it: the buffers
    are allocated once, so the second call with use_graph captures the chain and later ones replay it."""

    def __init__(self, h):
        import torch
        self.h, self.ctx = h, h.ctx

        def pinned(a):
            v = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(-1, order="F")).view(np.float64)
            return torch.from_numpy(v.copy()).pin_memory()

        self.src = [pinned(x) for x in (h.Σ_loc, h.Γ_m, h.Γ_d, h.χDMFT_m, h.gImp)]
        self.numax = h.sP.n_iν
        self.S_out = torch.zeros(self.ctx.Nq * self.numax * 2, dtype=torch.float64).pin_memory()
        self.sc = (C.c_double * 8)()

    def __call__(self, use_graph):
        h, p = self.h, [C.c_void_p(t.data_ptr()) for t in self.src]
        self.ctx.call("ldga_chain_m", p[0], len(h.Σ_loc), p[1], p[2], p[3], p[4], len(h.gImp), h.imp_density,
                      h.χloc_m_sum, use_graph, C.c_void_p(self.S_out.data_ptr()), None, None, self.sc)
        S_ = self.S_out.numpy().view(np.complex128).reshape((self.ctx.Nq, self.numax), order="F").copy()
        return list(self.sc), S_


def at_lambda(h, lam_m, lam_d=0.0, numax=None):
    """EoM, μ fit, G_ladder and energies on the device at the given λ (the chain's last stages)."""
    ctx = h.ctx
    numax = h.sP.n_iν if numax is None else numax
    Sg = _lib.cplx_out((ctx.Nq, numax))
    ctx.call("ldga_eom", lam_m, lam_d, numax, 1, h.χloc_m_sum, _lib.ptr(Sg))
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))
    mu, ek, ep, n = (C.c_double() for _ in range(4))
    ctx.call("ldga_g_ladder", None, 0, 1, h.mP.μ, C.byref(mu), _lib.ptr(G), C.byref(ek), C.byref(ep), C.byref(n))
    return Sg, G, mu.value, ek.value, ep.value


@pytest.fixture(scope="module")
def cfg3(require_gpu):
    R.set_workers(os.cpu_count() or 1)
    inp = S.config_input(3)
    return inp, R.run_chain(inp, lambda_type="m")


def test_config3_mixed_chain_graph(cfg3):
    """The benchmarked call: autotuned MIXED BSE, ldga_chain_m eager then captured and replayed."""
    inp, ref = cfg3
    h = L.setup_synthetic(inp, precision=L.PREC_MIXED)
    lib = h.ctx.lib
    try:
        h.ctx.call("ldga_bubble", None)
        for t in ("m", "d"):
            L.autotune_bse(h, t, reps=2)
        name = lib.ldga_bse_config_name(h.ctx.Nnu, L.PREC_MIXED, -1).decode()
        assert name.startswith("iter"), name            # the preconditioned solve is what runs here
        res = ref["result"]
        rh, cm = ref["h"], ref["chi_m"]
        rhs = 2 * rh.imp_density - R.sum_kw(rh.kG, ref["chi_d"])
        run = ChainM(h)
        for use_graph in (0, 1, 1, 1):                  # eager, capture, replay
            sc, S_chain = run(use_graph)
            dev = device_arrays(h.ctx)
            check_arrays(dev, ref, (name, use_graph))
            # λm: a root of the oracle's f (which root newton_right reaches is not a parity quantity)
            lam = sc[0]
            f = R.sum_kw(rh.kG, cm, transform=lambda x: R.chi_lambda(x, lam)) - rhs
            scale = R.sum_kw(rh.kG, cm, transform=lambda x: np.abs(R.chi_lambda(x, lam)))
            assert abs(f) <= 1e-9 * max(1.0, scale), (lam, f)
            # the chain's Σ_ladder is the EoM at its own λ
            Sg, _, mu, _, ep = at_lambda(h, lam)
            assert rel(S_chain, Sg) < 1e-12 and abs(mu - sc[1]) < 1e-12
        # the λ-dependent stages at the oracle's λm, each from the oracle's inputs: the EoM from its χ,
        # γ and λ₀, then the μ fit, G_ladder and the energies from its Σ_ladder.  (λm = 29.59 lies
        # beyond the first pole of χ_λ, where 1/(1 + λχ) amplifies upstream rounding differences.)
        set_oracle_inputs(h.ctx, ref)
        Sg = _lib.cplx_out((h.ctx.Nq, h.sP.n_iν))
        h.ctx.call("ldga_eom", res.lam_m, 0.0, h.sP.n_iν, 1, h.χloc_m_sum, _lib.ptr(Sg))
        assert rel(Sg, res.Sigma_ladder) < RTOL
        G, mu, ek, ep = g_ladder(h, res.Sigma_ladder)
        assert rel(G, res.G_ladder) < RTOL
        assert abs(mu - res.mu) < 1e-10
        assert abs(ek - res.EKin) <= RTOL * max(1.0, abs(res.EKin))
        assert abs(ep - res.EPot_p1) <= RTOL * max(1.0, abs(res.EPot_p1))
    finally:
        L.tune_reset()


def test_config3_chain_pivoted_fallback_of_every_matrix(cfg3):
    """The chain's two-channel BSE with every matrix handed to the pivoted FP64 solve: with the sweep
    limit at 0 (LDGA_ITER_SWEEPS=0 when the handle is made) the preconditioned iteration stops after
    its first residual, appends every matrix (q + Nq w) to its channel's list, and one pivoted launch
    re-solves both lists.  χ and γ of both channels against the oracle at the parity tolerance (the
    first residual alone is far from it), eager, captured and replayed; λm a root of the oracle's f."""
    import tempfile
    inp, ref = cfg3
    fd, path = tempfile.mkstemp()
    os.write(fd, f"bse 40 {L.PREC_MIXED} iter8x2dm2ns:3\n".encode())
    os.close(fd)
    os.environ["LDGA_ITER_SWEEPS"] = "0"
    try:
        L.tune_reset()
        L.tune_load(path)
        h = L.setup_synthetic(inp, precision=L.PREC_MIXED)
    finally:
        del os.environ["LDGA_ITER_SWEEPS"]
        os.unlink(path)
    try:
        rh, cm = ref["h"], ref["chi_m"]
        rhs = 2 * rh.imp_density - R.sum_kw(rh.kG, ref["chi_d"])
        run = ChainM(h)
        h.ctx.call("ldga_bse_sweeps", None, None)      # clear the sweep counters
        for use_graph in (0, 1, 1):
            sc, S_chain = run(use_graph)
            passes, warps = C.c_int64(), C.c_int64()
            h.ctx.call("ldga_bse_sweeps", C.byref(passes), C.byref(warps))
            assert warps.value > 0 and passes.value == warps.value, (passes.value, warps.value)   # one sweep
            dev = device_arrays(h.ctx)
            check_arrays(dev, ref, ("all pivoted", use_graph))
            lam = sc[0]
            f = R.sum_kw(rh.kG, cm, transform=lambda x: R.chi_lambda(x, lam)) - rhs
            scale = R.sum_kw(rh.kG, cm, transform=lambda x: np.abs(R.chi_lambda(x, lam)))
            assert abs(f) <= 1e-9 * max(1.0, scale), (lam, f)
            Sg, _, mu, _, _ = at_lambda(h, lam)
            assert rel(S_chain, Sg) < 1e-12 and abs(mu - sc[1]) < 1e-12
    finally:
        L.tune_reset()


def test_config3_every_mixed_bse_configuration(cfg3):
    """Every compiled MIXED configuration at Nnu = 40 (the autotuner's candidates) on the headline
    input: χ_r and γ_r against the oracle, no matrix left to the pivoted fallback."""
    import tempfile
    inp, ref = cfg3
    h = L.setup_synthetic(inp, precision=L.PREC_MIXED)
    lib = h.ctx.lib
    nnu = h.ctx.Nnu
    names = []
    while lib.ldga_bse_config_name(nnu, L.PREC_MIXED, len(names)):
        names.append(lib.ldga_bse_config_name(nnu, L.PREC_MIXED, len(names)).decode())
    chi0 = L.calc_bubble(h)
    assert rel(chi0.data, ref["chi0"]) < RTOL
    try:
        for nm in names:
            fd, path = tempfile.mkstemp()
            os.write(fd, f"bse {nnu} {L.PREC_MIXED} {nm}\n".encode())
            os.close(fd)
            L.tune_reset()
            L.tune_load(path)
            os.unlink(path)
            for r in ("m", "d"):
                x, g = L.calc_χγ(r, h, chi0)
                assert chi_rel(x.data, ref, r) < RTOL, (nm, r, chi_rel(x.data, ref, r))
                assert rel(g.data, ref[f"gamma_{r}"]) < RTOL, (nm, r, rel(g.data, ref[f"gamma_{r}"]))
                if nm.startswith("iter"):
                    assert x.n_fallback == 0, (nm, r, x.n_fallback)
    finally:
        L.tune_reset()


@pytest.fixture(scope="module")
def cfg2(require_gpu):
    R.set_workers(os.cpu_count() or 1)
    inp = S.config_input(2)
    return inp, R.run_chain(inp, lambda_type=None)


def test_config2_every_mixed_bse_configuration(cfg2):
    """Every compiled MIXED configuration at Nν = 60 on configuration 2's matrices -- the preconditioned
    iteration on tiles padded to 64 (the default) and the LU forms: χ_r and γ_r against the oracle,
    no matrix left to the pivoted fallback by the iteration."""
    import tempfile
    inp, ref = cfg2
    h = L.setup_synthetic(inp, precision=L.PREC_MIXED)
    lib = h.ctx.lib
    nnu = h.ctx.Nnu
    names = []
    while lib.ldga_bse_config_name(nnu, L.PREC_MIXED, len(names)):
        names.append(lib.ldga_bse_config_name(nnu, L.PREC_MIXED, len(names)).decode())
    assert names[0].startswith("iter") and "64" in names[0]
    chi0 = L.calc_bubble(h)
    assert rel(chi0.data, ref["chi0"]) < RTOL
    try:
        for nm in names:
            fd, path = tempfile.mkstemp()
            os.write(fd, f"bse {nnu} {L.PREC_MIXED} {nm}\n".encode())
            os.close(fd)
            L.tune_reset()
            L.tune_load(path)
            os.unlink(path)
            for r in ("m", "d"):
                x, g = L.calc_χγ(r, h, chi0)
                assert chi_rel(x.data, ref, r) < RTOL, (nm, r, chi_rel(x.data, ref, r))
                assert rel(g.data, ref[f"gamma_{r}"]) < RTOL, (nm, r, rel(g.data, ref[f"gamma_{r}"]))
                if nm == names[0]:
                    assert x.n_fallback == 0, (nm, r, x.n_fallback)
    finally:
        L.tune_reset()


@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_MIXED])
def test_config2_lambda_dm(cfg2, prec):
    """Configuration 2 as specified: both channels and λdm, in FP64 and in MIXED mode.  The arrays
    before λ against the oracle; the device's (λm, λd) is a root of the ORACLE's λdm residual
    (conditions_new.jl:250-276) to the Newton's atol 1e-8, and Σ_ladder, G_ladder, μ and the energies
    at that root equal the oracle's there."""
    inp, ref = cfg2
    h = L.setup_synthetic(inp, precision=prec)
    chi0 = L.calc_bubble(h)
    xm, gm = L.calc_χγ("m", h, chi0)
    xd, gd = L.calc_χγ("d", h, chi0)
    l0 = L.calc_λ0(chi0, h)
    dev = device_arrays(h.ctx)
    check_arrays(dev, ref, prec)
    res = L.λdm_correction(xm, gm, xd, gd, l0, h)
    assert res.sc_converged, (res.λm, res.λd)
    # reference properties (test/full_run.jl:151-165): PP and E_pot consistency at the root
    assert abs(res.PP_p2 - 0.25) < 1e-8
    assert abs(res.EPot_p1 - res.EPot_p2) < 1e-8
    numax = res.Σ_ladder.shape[1]
    hr = ref["h"]
    state = {"mu": hr.mP.mu}
    n, mu, ek, ep1, ep2, lhs_c1, Sr, Gr = R.lambda_dm_residual(np.array([res.λm, res.λd]), ref["chi_m"],
                                                               ref["gamma_m"], ref["chi_d"], ref["gamma_d"],
                                                               ref["lambda0"], hr, numax, state)
    rhs_c1 = hr.mP.n / 2 * (1 - hr.mP.n / 2)
    assert math.hypot(lhs_c1 - rhs_c1, ep1 - ep2) < 1e-8, (lhs_c1 - rhs_c1, ep1 - ep2)
    assert rel(res.Σ_ladder, Sr) < RTOL
    assert abs(res.μ - mu) < 1e-10
    for a, b in ((res.EPot_p2, ep2), (res.PP_p2, lhs_c1)):
        assert abs(a - b) <= RTOL * max(1.0, abs(b)), (a, b)
    # G_ladder = 1/(iν + μ - ε_k - Σ) amplifies Σ's differences near the Fermi surface: the μ fit,
    # G_ladder and the energies are compared from the oracle's Σ_ladder
    G, mu2, ek2, ep2_ = g_ladder(h, Sr)
    assert rel(G, Gr) < RTOL
    assert abs(mu2 - mu) < 1e-10
    for a, b in ((ek2, ek), (ep2_, ep1)):
        assert abs(a - b) <= RTOL * max(1.0, abs(b)), (a, b)
