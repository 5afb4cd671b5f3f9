"""Real DMFT inputs: the JLD2 reader, ``readConfig``, the impurity-file step of ``setup_LDGA`` and
``calc_E_ED`` on LadderDGA.jl's own test fixture (test/test_data/b1u2_ED_data.jld2, frozen as
tests/golden/b1u2_dmft.npz by tests/golden/make_dmft_fixture.py), and the CUDA ladder chain on it.

Known answers from the reference's tests: ``calc_E_ED`` on the fixture gives E_kin ≈ -0.10448 and
E_pot ≈ 2 · 0.14177 (atol 1e-3, test/thermodynamics.jl:1-5); the file's own E_kin_DMFT is the
same kinetic energy.  The local BSE with Γ_r = −Γ_file reproduces the file's χ_r (the consistency
the reference's setup relies on, runHelpers.jl:91-98, 137-140).
"""
import copy
import os
from pathlib import Path

import numpy as np
import pytest

import ladderdga_b200 as L
from ladderdga_b200 import inputs as I
from ladderdga_b200 import jld2
from oracle import ldga_ref as R

GOLD = Path(__file__).resolve().parent / "golden"
NPZ = GOLD / "b1u2_dmft.npz"
CFG = GOLD / "b1u2_plain.toml"
# The reference's own DMFT fixture (test/test_data/b1u2_ED_data.jld2 of LadderDGA.jl), when a checkout
# of the reference is named by LDGA_REFERENCE_DIR; the frozen copy above is used otherwise.
REF_JLD2 = os.path.join(os.environ.get("LDGA_REFERENCE_DIR", ""), "test", "test_data", "b1u2_ED_data.jld2")
EK_REF, EP_REF = -0.1044800085350687, 2 * 0.14176922807732420     # test/thermodynamics.jl:3-4
RTOL = 1e-10


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def setup():
    _, mP, sP, env, kgs = L.readConfig(str(CFG))
    return mP, sP, env, kgs, I.load_impurity_input(env.inputVars, kgs[0], mP, sP)


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD / "chain_b1u2.npz"))


# ------------------------------------------------------------------------------ CPU
@pytest.mark.skipif(not os.path.isfile(REF_JLD2), reason="LDGA_REFERENCE_DIR does not name a LadderDGA.jl checkout")
def test_jld2_reader_matches_frozen_fixture():
    """Every key the plain path reads comes out of the HDF5 container bit for bit as frozen, with
    Julia's shapes (Γ_r, χ_r: [Nω, Nν, Nν] before permutedims)."""
    f = jld2.jldopen(REF_JLD2)
    z = np.load(NPZ)
    assert set(f.keys()) >= set(z.files)
    for k in z.files:
        a, b = np.asarray(f[k]), z[k]
        assert a.shape == b.shape and a.dtype == b.dtype, k
        assert np.array_equal(a, b), k
    assert f["Γsp"].shape == (21, 20, 20) and f["gImp"].shape == (84,)
    assert f["χ_sp_asympt"].shape == (32769,)
    assert I.calc_E_ED(REF_JLD2)[0] == pytest.approx(EK_REF, abs=1e-3)
    with pytest.raises(KeyError):
        f["no such key"]


def test_calc_E_ED_known_answer():
    """test/thermodynamics.jl:1-5 on the package and on the oracle."""
    ek, ep = I.calc_E_ED(str(NPZ))
    assert ek == pytest.approx(EK_REF, abs=1e-3) and ep == pytest.approx(EP_REF, abs=1e-3)
    z = np.load(NPZ)
    eko, epo = R.calc_E_ED(z["ϵₖ"], z["Vₖ"], z["gImp"], float(z["U"]), float(z["nden"]), float(z["μ"]),
                           float(z["β"]))
    assert eko == pytest.approx(ek, rel=1e-14) and epo == pytest.approx(ep, rel=1e-14)
    # the file's DMFT kinetic energy is the same sum
    assert ek == pytest.approx(float(z["E_kin_DMFT"]), abs=1e-8)


def test_readConfig(setup):
    mP, sP, env, kgs, inp = setup
    z = np.load(NPZ)
    assert (mP.U, mP.μ, mP.β, mP.n) == (2.0, 1.0, 1.0, 1.0)
    assert mP.sVk == pytest.approx(float(np.sum(z["Vₖ"] ** 2)), rel=1e-15)
    assert mP.Ekin_DMFT == float(z["E_kin_DMFT"]) and mP.Epot_DMFT == float(z["E_pot_DMFT"])
    assert (sP.n_iω, sP.n_iν, sP.n_iν_shell, sP.shift) == (10, 10, 0, True)
    assert sP.χ_helper is None and sP.fft_range == range(-40, 41)      # 2 (n_iν + n_iω)
    assert sP.dbg_full_eom_omega is True and sP.usable_prct_reduction == 0.0
    assert kgs == [("3Dsc-0.2041241452319315", 10)]
    assert env.inputVars == str(NPZ) and env.loglevel == "Debug" and env.logfile == "stderr"


def test_readConfig_options_and_errors(tmp_path):
    text = CFG.read_text()
    # the fixture's own choice: χ asymptotics from BSE_SC.jl -> a helper that setup_LDGA refuses
    direct = text.replace('"nothing"', '"direct"', 1).replace("chi_asympt_shell = 0", "chi_asympt_shell = 2")
    p = tmp_path / "direct.toml"
    p.write_text(direct.replace('inputDir = "."', f'inputDir = "{GOLD}"'))
    _, mP, sP, env, kgs = L.readConfig(str(p))
    assert isinstance(sP.χ_helper, I.BSEAsymptoticsHelper) and sP.n_iν_shell == 2
    assert sP.fft_range == range(-40, 41)                 # only "asympt" widens the box
    with pytest.raises(NotImplementedError):
        L.setup_LDGA(kgs[0], mP, sP, env)
    # a TOML string instead of a file; "conv" grids
    s = text.replace('inputDir = "."', f'inputDir = "{GOLD}"').replace("Nk = [10]", 'Nk = "conv"')
    _, _, _, _, kgs = L.readConfig(s)
    assert kgs == [("3Dsc-0.2041241452319315", 0)]
    with pytest.raises(RuntimeError, match="smoothing"):
        L.readConfig(s.replace('omega_smoothing = "nothing"', 'omega_smoothing = "spline"'))
    with pytest.raises(SystemExit) as e:
        L.readConfig(s.replace("b1u2_dmft.npz", "missing.jld2"))
    assert e.value.code == 2


def test_impurity_input_layout(setup):
    """permutedims(·, (2, 3, 1)), Γ_r = −Γ_file, Σ_loc = Σ_Dyson(g0, gImp); the local BSE with
    these Γ_r reproduces the file's χ_r at every ω."""
    mP, sP, env, kgs, inp = setup
    z = np.load(NPZ)
    assert inp.gamma_m.shape == (20, 20, 21) and inp.gamma_m.flags.f_contiguous
    assert np.array_equal(inp.gamma_m[3, 5, 7], -z["Γsp"][7, 3, 5])
    assert np.array_equal(inp.chi_loc_d[3, 5, 7], z["χDMFTch"][7, 3, 5])
    assert np.allclose(inp.sigma_loc, 1 / z["g0"] - 1 / z["gImp"], rtol=1e-15)
    h = R.setup_ldga(inp)
    for w in range(21):
        for r, Γ, χ in (("m", inp.gamma_m, inp.chi_loc_m), ("d", inp.gamma_d, inp.chi_loc_d)):
            X = np.linalg.inv(Γ[:, :, w] + np.diag(1.0 / h.chi0_loc[0, :, w]))
            assert rel(X, χ[:, :, w]) < 1e-12, (r, w)
    with pytest.raises(ValueError, match="DimensionMismatch"):
        small = copy.copy(sP)
        small.n_iν = 8
        I.load_impurity_input(env.inputVars, kgs[0], mP, small)


def test_oracle_reproduces_dmft_fixture(setup, gold):
    mP, sP, env, kgs, inp = setup
    m = R.run_chain(inp, lambda_type="m")
    assert rel(m["chi_m"].data, gold["chi_m"]) < 1e-12 and rel(m["chi_d"].data, gold["chi_d"]) < 1e-12
    assert rel(m["h"].G_irr, gold["gloc"]) < 1e-14
    for k, a in (("chi0", m["chi0"]), ("gamma_m", m["gamma_m"]), ("gamma_d", m["gamma_d"]),
                 ("lambda0", m["lambda0"])):
        assert abs(a.sum() - gold[f"{k}_sum"]) <= 1e-11 * np.sqrt(gold[f"{k}_abs2"]) * a.size ** 0.5, k
    res = m["result"]
    assert abs(res.lam_m - gold["lm_scalars"][0]) < 1e-11
    assert rel(res.Sigma_ladder, gold["lm_sigma"]) < 1e-11
    # Pauli sum rule at the λm root
    h = m["h"]
    cm = R.ChiT(R.chi_lambda(m["chi_m"].data, res.lam_m), mP.β, tail_c=m["chi_m"].tail_c)
    assert abs(R.sum_kw(h.kG, cm) - (2 * h.imp_density - R.sum_kw(h.kG, m["chi_d"]))) < 1e-10
    # the λdm Newton finds no root on this input (its residual stays O(1)): recorded as NaN
    assert np.all(np.isnan(gold["ldm_root"]))


# ------------------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("prec", [L.PREC_FP64, L.PREC_MIXED])
def test_cuda_chain_on_dmft_input(setup, gold, prec, require_gpu):
    """readConfig → setup_LDGA (impurity file) → bubble → χ, γ (m, d) → λ₀ → λm correction on the
    GPU against the oracle's fixture on the same real inputs."""
    _, mP, sP, env, kgs = L.readConfig(str(CFG))
    h = L.setup_LDGA(kgs[0], mP, sP, env, precision=prec)
    assert abs(h.χloc_m_sum - float(gold["chiloc_m_sum"])) < 1e-12
    assert abs(h.imp_density - float(gold["imp_density"])) < 1e-12
    assert rel(np.asarray(h.gLoc), gold["gloc"]) < 1e-14
    chi0 = L.calc_bubble(h)
    xm, gm = L.calc_χγ("m", h, chi0)
    xd, gd = L.calc_χγ("d", h, chi0)
    l0 = L.calc_λ0(chi0, h)
    samples = [tuple(s) for s in (
        (0, 0, 0), (0, 9, 10), (0, 10, 10), (3, 4, 7), (17, 19, 20), (55, 12, 3), (28, 0, 14))]
    for k, a in (("chi0", chi0.data), ("gamma_m", gm.data), ("gamma_d", gd.data), ("lambda0", np.asarray(l0))):
        got = np.array([a[s] for s in samples])
        assert rel(got, gold[f"{k}_samples"]) < RTOL, k
        assert abs(a.sum() - gold[f"{k}_sum"]) <= RTOL * np.sqrt(gold[f"{k}_abs2"] * a.size), k
    assert rel(xm.data, gold["chi_m"]) < RTOL and rel(xd.data, gold["chi_d"]) < RTOL
    res = L.λ_correction("m", xm, gm, xd, gd, l0, h)
    s = gold["lm_scalars"]
    assert abs(res.λm - s[0]) < 1e-10
    assert abs(res.μ - s[2]) < 1e-10
    assert rel(res.Σ_ladder, gold["lm_sigma"]) < RTOL
    for got, want in ((res.EKin, s[4]), (res.EPot_p1, s[5]), (res.EPot_p2, s[6]), (res.PP_p2, s[8])):
        assert abs(got - want) <= RTOL * max(1.0, abs(want))
