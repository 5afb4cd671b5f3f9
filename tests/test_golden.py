"""The ladder chain against the committed golden fixtures (tests/golden/chain_*.npz, written by
tests/golden/make_golden.py from the FP64 oracle).

CPU tests: the synthetic generator still produces the fixtures' inputs, the oracle still reproduces
the fixtures, and the oracle's results obey the reference's full-run properties
(test/full_run.jl:57-61, 110-165).  GPU tests: the CUDA path through the C ABI reproduces the
fixtures in every BSE precision mode (relative 1e-10; lambda absolute 1e-10; lambda_dm 1e-8, the
tolerance its 2-D Newton stops at).
"""
from pathlib import Path

import numpy as np
import pytest

import ladderdga_b200 as L
from ladderdga_b200 import synthetic as S
from oracle import ldga_ref as R
from tests.golden.make_golden import CASES, input_digest

GOLD = Path(__file__).resolve().parent / "golden"
RTOL = 1e-10
ATOL_LAMBDA = 1e-10
ATOL_LAMBDA_DM = 1e-8


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", params=list(CASES))
def gold(request):
    name = request.param
    return name, S.make_input(**CASES[name]), dict(np.load(GOLD / f"chain_{name}.npz"))


# ------------------------------------------------------------------------------ CPU
def test_inputs_unchanged(gold):
    name, inp, g = gold
    assert str(g["digest"]) == input_digest(inp), f"synthetic inputs of {name} changed: regenerate the fixtures"


def test_oracle_reproduces_fixture(gold):
    name, inp, g = gold
    m = R.run_chain(inp, lambda_type="m")
    assert rel(m["chi0"], g["chi0"]) < 1e-13
    for r in ("m", "d"):
        assert rel(m[f"chi_{r}"].data, g[f"chi_{r}"]) < 1e-12
        assert rel(m[f"gamma_{r}"], g[f"gamma_{r}"]) < 1e-12
    assert rel(m["lambda0"], g["lambda0"]) < 1e-12
    res = m["result"]
    assert abs(res.lam_m - g["lm_scalars"][0]) < 1e-11
    assert rel(res.Sigma_ladder, g["lm_sigma"]) < 1e-11


def test_oracle_properties(gold):
    """test/full_run.jl: Pauli sum rule after lambda_m; PP and E_pot consistency after lambda_dm;
    Sigma reproducible from the returned lambda; chi unchanged by chi_lambda!/reset!; Sigma parts sum."""
    name, inp, g = gold
    m = R.run_chain(inp, lambda_type=None)
    h = m["h"]
    lam_m, lam_d = g["lm_scalars"][0], g["ldm_scalars"][1]
    # Pauli sum rule: sum_kw chi_m^lambda = 2 imp_density - sum_kw chi_d
    cm = R.chi_lambda(m["chi_m"].data, lam_m)
    lhs = R.sum_kw(h.kG, R.ChiT(cm, h.mP.beta, tail_c=m["chi_m"].tail_c))
    assert abs(lhs - (2 * h.imp_density - R.sum_kw(h.kG, m["chi_d"]))) < 1e-9
    # lambda_dm root: PP_p2 = n/2 (1 - n/2) and E_pot,1 = E_pot,2
    s = g["ldm_scalars"]
    assert s[9] == 1.0
    assert abs(s[8] - 0.25) < 1e-7 and abs(s[5] - s[6]) < 1e-7
    # Sigma from the returned lambda_m
    S_re = R.calc_Sigma(m["chi_m"], m["gamma_m"], m["chi_d"], m["gamma_d"], h.chiloc_m_sum, m["lambda0"], h.grhat,
                        h.kG, h.mP, h.sP, numax=g["lm_sigma"].shape[1], lam_m=lam_m)
    assert rel(S_re, g["lm_sigma"]) < 1e-12
    # chi_lambda! followed by reset! restores chi (reset! applies the inverse map, so up to rounding)
    before = m["chi_m"].data.copy()
    R.chi_lambda_inplace(m["chi_m"], 0.7)
    assert m["chi_m"].lam == 0.7
    R.reset(m["chi_m"])
    assert m["chi_m"].lam == 0.0 and rel(m["chi_m"].data, before) < 1e-14
    # Sigma parts add up to Sigma (test/full_run.jl:57-61)
    P = R.calc_Sigma_parts(m["chi_m"], m["gamma_m"], m["chi_d"], m["gamma_d"], h.chiloc_m_sum, m["lambda0"], h.grhat,
                           h.kG, h.mP, h.sP, lam_m=lam_m)
    S_full = R.calc_Sigma(m["chi_m"], m["gamma_m"], m["chi_d"], m["gamma_d"], h.chiloc_m_sum, m["lambda0"], h.grhat,
                          h.kG, h.mP, h.sP, lam_m=lam_m, tc=True)
    assert rel(P.sum(axis=2), S_full) < 1e-12


# ------------------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("prec", [L.PREC_FP64_INV, L.PREC_FP64, L.PREC_MIXED])
def test_cuda_chain_matches_fixture(gold, prec, require_gpu):
    name, inp, g = gold
    h = L.setup_synthetic(inp, precision=prec)
    chi0 = L.calc_bubble(h)
    xm, gm = L.calc_χγ("m", h, chi0)
    xd, gd = L.calc_χγ("d", h, chi0)
    l0 = L.calc_λ0(chi0, h)
    assert rel(np.asarray(h.gLoc), g["gloc"]) < 1e-14
    assert abs(h.χloc_m_sum - float(g["chiloc_m_sum"])) < 1e-12
    assert abs(h.imp_density - float(g["imp_density"])) < 1e-12
    assert rel(chi0.data, g["chi0"]) < RTOL
    assert rel(xm.data, g["chi_m"]) < RTOL and rel(xd.data, g["chi_d"]) < RTOL
    assert rel(gm.data, g["gamma_m"]) < RTOL and rel(gd.data, g["gamma_d"]) < RTOL
    assert rel(np.asarray(l0), g["lambda0"]) < RTOL
    res = L.λ_correction("m", xm, gm, xd, gd, l0, h)
    s = g["lm_scalars"]
    assert abs(res.λm - s[0]) < ATOL_LAMBDA
    assert abs(res.μ - s[2]) < 1e-10
    assert rel(res.Σ_ladder, g["lm_sigma"]) < RTOL
    for got, want in ((res.EKin, s[4]), (res.EPot_p1, s[5]), (res.EPot_p2, s[6]), (res.PP_p2, s[8])):
        assert abs(got - want) <= RTOL * max(1.0, abs(want))


@pytest.mark.gpu
def test_cuda_lambda_dm_matches_fixture(gold, require_gpu):
    name, inp, g = gold
    h = L.setup_synthetic(inp)
    chi0 = L.calc_bubble(h)
    xm, gm = L.calc_χγ("m", h, chi0)
    xd, gd = L.calc_χγ("d", h, chi0)
    l0 = L.calc_λ0(chi0, h)
    res = L.λdm_correction(xm, gm, xd, gd, l0, h)
    s = g["ldm_scalars"]
    assert res.sc_converged
    assert abs(res.λm - s[0]) < ATOL_LAMBDA_DM and abs(res.λd - s[1]) < ATOL_LAMBDA_DM
    assert abs(res.PP_p2 - 0.25) < 1e-7 and abs(res.EPot_p1 - res.EPot_p2) < 1e-7
    assert rel(res.Σ_ladder, g["ldm_sigma"]) < 1e-7
