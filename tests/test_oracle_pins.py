"""The oracle and the package's host helpers against the reference's own known answers.

Each value below is read from LadderDGA.jl's test suite (file:line given per test).  The same checks
run on the oracle (oracle/ldga_ref.py) and on the package's host-side mirror (ladderdga_b200).
"""
import math

import numpy as np
import pytest

import ladderdga_b200 as L
from oracle import ldga_ref as R


# ------------------------------------------------------------------------------ GFTools.jl
def test_filling_known_answer():
    """test/GFTools.jl:29-33: filling(G, kG_1, 1.1, 1.2, 1.3) ≈ 1.1706318843228878 on the 2x2 grid."""
    beta, mu, U = 1.3, 1.2, 1.1                      # mP_1 = ModelParameters(1.1, 1.2, 1.3, ...)
    target = 1.1706318843228878
    kG = R.gen_kGrid("2dsc-1.0", 2)
    G = np.array([[R.G_from_Sigma(n, beta, mu, e, 0.0) for n in range(50)] for e in kG.eps])
    assert R.filling_kG(G, kG, U, mu, beta) == pytest.approx(target, rel=1e-15)
    kP = L.gen_kGrid("2Dsc-1.0", 2)
    Gp = np.array([[L.G_from_Σ(n, beta, mu, e, 0.0) for n in range(50)] for e in kP.ϵkGrid])
    assert L.filling(Gp, kP, U, mu, beta) == pytest.approx(target, rel=1e-15)


def test_G_shell_sum_vs_naive():
    """test/GFTools.jl:25-32: the trigamma shell sum vs the naive sum (rtol 0.01)."""
    nu = R.iv_array(11.1, range(-50, 50))
    naive = float(np.real(np.sum(1.0 / nu**2)) / 11.1 + 11.1 / 4)
    assert R.G_shell_sum(50, 11.1) == pytest.approx(naive, rel=0.01)
    assert L.G_shell_sum(50, 11.1) == pytest.approx(naive, rel=0.01)
    for N in (1, 5, 50, 300):
        assert L.G_shell_sum(N, 7.3) == pytest.approx(R.G_shell_sum(N, 7.3), rel=1e-13)


def test_matsubara_arrays_and_G_from_sigma():
    """test/GFTools.jl:1-21."""
    assert np.allclose(L.iν_array(5.0, range(3)), 1j * np.array([1, 3, 5]) * math.pi / 5.0)
    assert np.allclose(L.iω_array(5.0, range(3)), 1j * np.array([0, 2, 4]) * math.pi / 5.0)
    mf1 = 3j * math.pi / 1.3
    assert L.G_from_Σ(1, 1.3, 1.2, 1.3, 1.4 + 0j) == pytest.approx(1 / (mf1 + 1.2 - 1.3 - 1.4))
    assert L.G_from_Σ(mf1, 1.2, 1.3, 1.4 + 0j) == pytest.approx(1 / (mf1 + 1.2 - 1.3 - 1.4))
    assert L.Σ_Dyson([1.1 + 0j], [1.2 + 0j])[0] == pytest.approx(1 / 1.1 - 1 / 1.2)


# ------------------------------------------------------------------- LambdaCorrection/helpers.jl
def test_chi_lambda():
    """test/LambdaCorrection/helpers.jl:1-13."""
    assert R.chi_lambda(1.0, 0.0) == 1.0 and L.χ_λ(1.0, 0.0) == 1.0
    assert R.chi_lambda(1.0, 1.0) == 0.5 and L.χ_λ(1.0, 1.0) == 0.5
    c = L.χT([[1.0, 2.0, 1.0]], 1.0)
    t = L.χ_λ(c, 1.1)
    L.χ_λ_(c, 1.1)
    assert np.allclose(c.data, t.data) and c.λ == 1.1
    L.reset_(c)
    assert np.allclose(c.data, [[1.0, 2.0, 1.0]]) and c.λ == 0.0


def test_newton_right_roots():
    """test/LambdaCorrection/helpers.jl:15-24: root 1 of 2x^3 + x - 3; 2-D [1, 0]."""
    f = lambda x: 2 * x**3 + x - 3   # noqa: E731
    df = lambda x: 6 * x**2 + 1      # noqa: E731
    f2 = lambda x: np.array([2 * x[0]**3 + x[0] - 3, x[1]])   # noqa: E731
    for impl in (R, L):
        nr = impl.newton_right
        assert nr(f, df, 0.0, -1.0) == pytest.approx(1.0)
        assert nr(f, df, -0.9, -1.0) == pytest.approx(1.0)
    assert L.newton_right(f, 0.0, -1.0) == pytest.approx(1.0)
    assert np.allclose(R.newton_right_nd(f2, [0.0, 0.0], [-1.0, -1.0]), [1.0, 0.0])
    assert np.allclose(L.newton_right(f2, [0.0, 0.0], [-1.0, -1.0]), [1.0, 0.0])


def test_newton_right_quirk_matches():
    """The 1-D iteration, including its back-off branch, is identical in oracle and package."""
    # sum of chi/(lam*chi+1) minus a target: the shape of the lambda_m residual, pole at lam = -1/0.8
    chis = np.array([0.8, 0.5, 0.2])
    f = lambda x: float(np.sum(chis / (x * chis + 1)) - 0.9)          # noqa: E731
    df = lambda x: float(-np.sum(chis**2 / (x * chis + 1) ** 2))      # noqa: E731
    for start, lo in ((0.0, -1.2), (-1.1, -1.2), (5.0, -1.2)):
        got = L.newton_right(f, df, start, lo)
        assert got == R.newton_right(f, df, start, lo)
        assert abs(f(got)) < 1e-12


# --------------------------------------------------------------------------------- DataTypes.jl
def _tail_case():
    wn = 2j * np.arange(-100, 101) * math.pi / 11.1
    t3 = np.zeros((4, len(wn)), dtype=np.complex128)
    with np.errstate(divide="ignore", invalid="ignore"):
        for r in range(4):
            t3[r] = 1.2 / wn + 2.3 / wn**2
    t3[:, 100] = 0.0
    return wn, t3


def test_sum_identities():
    """test/DataTypes.jl:30-67: sum_ω / sum_kω / sum_ωk identities and update_tail!."""
    wn, t3 = _tail_case()
    kGo = R.gen_kGrid("3Dsc-1.1", 2)
    kGp = L.gen_kGrid("3Dsc-1.1", 2)
    direct = np.real(t3.sum(axis=1))
    direct3 = np.sum(np.real(t3) ** 3, axis=1)
    # oracle
    c2 = R.ChiT(np.real(t3), 1.0, tail_c=[0.0, 0.0, 0.0])
    c = R.ChiT(np.real(t3), 1.0, tail_c=[0.0, 0.0, 2.3])
    assert np.allclose(R.sum_w(c2), direct)
    assert kGo.kintegrate(direct) == pytest.approx(R.sum_kw(kGo, c2))
    assert kGo.kintegrate(direct) == pytest.approx(R.sum_wk(kGo, c2))
    assert kGo.kintegrate(direct3) == pytest.approx(R.sum_kw(kGo, c2, transform=lambda x: x**3))
    assert R.sum_kw(kGo, c) == pytest.approx(R.sum_wk(kGo, c))
    # package host data type
    p2 = L.χT(np.real(t3), 1.0, tail_c=[0.0, 0.0, 0.0])
    p = L.χT(np.real(t3), 1.0, tail_c=[0.0, 0.0, 2.3])
    assert np.allclose(L.sum_ω(p2), direct)
    assert kGp.kintegrate(direct) == pytest.approx(L.sum_kω(kGp, p2))
    assert kGp.kintegrate(direct) == pytest.approx(L.sum_ωk(kGp, p2))
    assert kGp.kintegrate(direct3) == pytest.approx(L.sum_kω(kGp, p2, transform=lambda x: x**3))
    assert L.sum_kω(kGp, p) == pytest.approx(L.sum_ωk(kGp, p))
    # update_tail! moves the c2 tail from 2.3 to 4.0 (test/DataTypes.jl:47-56)
    pt = L.χT(np.real(t3), 1.0, tail_c=[0.0, 0.0, 2.3])
    with pytest.raises(ValueError):
        L.update_tail_(pt, [0, 1.0, 4.0], wn)
    L.update_tail_(pt, [0, 0.0, 4.0], wn)
    assert np.real(pt.data[0, -1] * wn[-1] ** 2) == pytest.approx(4.0)
    assert pt.tail_c == [0.0, 0.0, 4.0] and np.all(np.isfinite(pt.data))
    ot = R.ChiT(np.real(t3), 1.0, tail_c=[0.0, 0.0, 2.3])
    R.update_tail(ot, [0, 0.0, 4.0], wn)
    assert np.allclose(ot.data, pt.data)


def test_chiT_basics():
    """test/DataTypes.jl:1-13, 40-45."""
    t2 = L.χT(np.random.default_rng(0).standard_normal((3, 5)), 1.2, tail_c=[0, 0, 1.0])
    assert list(t2.indices_ω) == [-2, -1, 0, 1, 2]
    assert np.allclose(L.ωn_grid(t2), 2 * math.pi * 1j * np.arange(-2, 3) / 1.2)
    t = L.χT(np.arange(1.0, 13.0).reshape(3, 4, order="F"), 1.0)
    assert t[0, 0] == 1 and t.shape == (3, 4) and t.β == 1.0
    t[0, 0] = -11
    assert t[0, 0] == -11


# ------------------------------------------------------------------------------------ GFFit.jl
@pytest.mark.parametrize("impl", ["oracle", "package"])
def test_find_usable_interval(impl):
    """test/GFFit.jl:39-55 (1-based index ranges)."""
    f = R.find_usable_chi_interval if impl == "oracle" else (lambda *a, **k: list(L.find_usable_χ_interval(*a, **k)))
    t0 = [0.6, 0.7, 0.8, 0.9, 1.0, 0.9, 0.8, 0.7, 0.6]
    t1 = [0.8, 0.7, 0.8, 0.9, 1.0, 0.9, 0.8, 0.7, 0.8]
    t2 = [-0.8, 0.7, 0.8, 0.9, 1.0, 0.9, 0.8, 0.7, -0.8]
    t3 = [-0.8, 0.7, 0.8, 0.9, 1.0, 0.9, 0.8, 0.7, -0.8, -0.9]
    t4 = [-0.8, 0.3, -0.2]
    assert list(f(t1)) == list(range(2, 9))
    assert list(f(t1, reduce_range_prct=0.0)) == list(range(2, 9))
    assert list(f(t1, reduce_range_prct=0.50)) == list(range(3, 8))
    assert list(f(t2, reduce_range_prct=0.0)) == list(range(2, 9))
    with pytest.raises(ValueError):
        f(t3)
    assert list(f(t0, reduce_range_prct=0.0)) == list(range(1, 10))
    assert list(f(t2, sum_type="full", reduce_range_prct=0.5)) == list(range(1, 10))
    assert list(f(t2, sum_type=(2, 8), reduce_range_prct=0.5)) == list(range(2, 9))
    assert list(f([-1.0, -2.0, -1.0])) == [2]
    assert list(f(t4, reduce_range_prct=0.9)) == [2]


def test_usable_indices():
    """test/GFFit.jl:57-60 with χ_1, χ_2 of test/runtests.jl:11-12."""
    sP_1 = L.SimulationParameters(1, 2, 3, True, None, range(1, 4), 0.1, False)
    x1 = L.χT([[1.1, 1.2, 1.1], [2.1, 2.3, 2.1]], 1.0)
    x2 = L.χT([[-1.1, 1.2, 1.1], [2.1, 2.3, 2.1]], 1.0, full_range=False, reduce_range_prct=0.0)
    assert list(L.usable_ωindices(sP_1, x1)) == [1, 2, 3]
    assert list(L.usable_ωindices(sP_1, x1, x2)) == [2]


# ---------------------------------------------------------------------------------- helpers.jl
def test_reduce_range():
    """test/helpers.jl:1-11."""
    cases = [((1, 3), 1.0, (2, 2)), ((1, 4), 1.0, (2, 3)), ((1, 5), 1.0, (3, 3)), ((1, 6), 1.0, (3, 4)),
             ((1, 10), 0.2, (2, 9)), ((1, 20), 0.1, (2, 19)), ((1, 21), 0.1, (2, 20)), ((1, 20), 0.5, (6, 15)),
             ((1, 21), 0.5, (6, 16))]
    for rng, p, out in cases:
        assert R.reduce_range(rng, p) == out
        r = L.reduce_range(range(rng[0], rng[1] + 1), p)
        assert (r[0], r[-1]) == out


def test_index_functions():
    """test/helpers.jl:13-22 with sP_1, sP_grid_s0/s1 of test/runtests.jl:6-16."""
    sP_1 = L.SimulationParameters(1, 2, 3, True, None, range(1, 4), 0.1, False)
    assert list(L.νnGrid(4, sP_1)) == list(range(-7, 3))
    assert L.q0_index(L.gen_kGrid("2Dsc-1.0", 2)) == 0       # 1 in Julia's 1-based indexing
    for shift in (False, True):
        sP = L.SimulationParameters(4, 5, 2, shift, None, range(1, 4), 0.1, False)
        grid = [[(i, j - int(int(shift) * i / 2)) for j in range(-5, 5)] for i in range(-4, 5)]
        for wi in range(1, 2 * sP.n_iω + 2):
            v0 = L.ν0Index_of_ωIndex(wi, sP)
            assert grid[wi - 1][v0 - 1][1] == 0
            assert R.nu0_index_of_w_index(wi, R.SimulationParameters(4, 5, 2, shift, None, range(1, 4), 0.1, False)) == v0


# ----------------------------------------------------------------------------- LapackWrapper.jl
@pytest.mark.parametrize("N", range(8, 14))
def test_inverse_vs_lapack(N):
    """test/LapackWrapper.jl:9-36: the oracle's BSE inverse is LAPACK's (getrf + getri)."""
    import scipy.linalg as sl
    rng = np.random.default_rng(N)
    A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    lu, piv = sl.lu_factor(A)
    Ainv = sl.lu_solve((lu, piv), np.eye(N))
    assert np.allclose(np.linalg.inv(A), Ainv)


# ------------------------------------------------------------------------- Dispersions contract
@pytest.mark.parametrize("dim,ns", [(2, 2), (2, 6), (2, 8), (3, 4), (3, 6)])
def test_conv_fft_vs_direct(dim, ns):
    """conv_fft!(fft(A), fft(reverse(B))) + conv_post == (1/N_k) sum_k A(k) B(k+q) on the wedge."""
    kG = R.KGrid(dim, ns)
    rng = np.random.default_rng(dim * 100 + ns)
    A = rng.standard_normal(kG.Nq) + 1j * rng.standard_normal(kG.Nq)
    B = rng.standard_normal(kG.Nq) + 1j * rng.standard_normal(kG.Nq)
    ah, _ = R.G_fft(kG, A[:, None])
    _, brh = R.G_fft(kG, B[:, None])
    assert np.allclose(R.conv_fft(kG, ah[..., 0], brh[..., 0]), R.conv_direct(kG, A, B), atol=1e-13)


@pytest.mark.parametrize("kind,ns,nq", [("2Dsc-1.0", 16, 45), ("2Dsc-1.0", 64, 561), ("3Dsc-1.0", 32, 969),
                                        ("3Dsc-1.0", 10, 56), ("2Dsc-1.0", 48, 325)])
def test_kgrid_wedge(kind, ns, nq):
    """Irreducible point counts (test/loadFortranData.jl:6 for 3D) and package == oracle wedge."""
    p = L.gen_kGrid(kind, ns)
    o = R.gen_kGrid(kind, ns)
    assert len(p.kMult) == nq == o.Nq
    assert p.kMult.sum() == p.Nk
    assert np.array_equal(p.wedge, o.wedge) and np.array_equal(p.kMult, o.kMult)
    assert np.allclose(p.ϵkGrid, o.eps, atol=1e-15)
    assert np.all(p.wedge[0] == 0)


def test_chi_lambda_three_argument_form():
    """test/LambdaCorrection/helpers.jl:9-12: χ_λ!(χ, χ, λ) equals χ_λ(χ, λ); reset! restores."""
    c = L.χT([[1.0, 2.0, 1.0]], 1.0)
    t = L.χ_λ(c, 1.1)
    L.χ_λ_(c, c, 1.1)
    assert np.allclose(c.data, t.data) and c.λ == 1.1
    L.reset_(c)
    assert np.allclose(c.data, [[1.0, 2.0, 1.0]]) and c.λ == 0.0
    d = L.χT([[0.0, 0.0, 0.0]], 1.0)
    L.χ_λ_(d, c, 0.5)                                      # into another χT: d.λ = c.λ + λ
    assert np.allclose(d.data, np.array([[1.0, 2.0, 1.0]]) / (0.5 * np.array([[1.0, 2.0, 1.0]]) + 1))
    assert d.λ == 0.5 and c.λ == 0.0
    arr = np.zeros(3)
    L.χ_λ_(arr, np.array([1.0, 2.0, 1.0]), 1.0)
    assert arr.tolist() == [0.5, 2.0 / 3.0, 0.5]


def test_chi0_asym_coeffs_known_answer():
    """test/DataTypes.jl:16-27 with mP_1 = ModelParameters(1.1, 1.2, 1.3, 1.4, 1.5, 1.6, 1.7): the local
    tail coefficients, and the empty ω mesh that χ₀T refuses (ArgumentError)."""
    U, mu, beta, n, sVk = 1.1, 1.2, 1.3, 1.4, 1.5
    c1_ref = U * n / 2 - mu
    c3_ref = c1_ref * c1_ref + sVk + U**2 * (n / 2) * (1 - n / 2)
    mP = L.ModelParameters(U, mu, beta, n, sVk, 1.6, 1.7)
    kG = L.gen_kGrid("2Dsc-1.0", 2)
    c1, c2, c3 = L.χ0Asym_coeffs(kG, True, mP)
    assert c1 == pytest.approx(c1_ref) and c2[0] == pytest.approx(c1 ** 2) and c3 == pytest.approx(c3_ref)
    o1, o2, o3 = R.chi0_asym_coeffs(R.gen_kGrid("2Dsc-1.0", 2), True, R.ModelParameters(U, mu, beta, n, sVk, 1.6, 1.7))
    assert (o1, o2[0], o3) == pytest.approx((c1, c2[0], c3))
    td = (np.arange(1, 25).reshape(3, 2, 4, order="F")).astype(np.complex128)
    t = L.χ0T(td, beta, range(1, 5), 1, True)
    assert np.array_equal(t.data, td)
    with pytest.raises(ValueError):
        L.χ0T(td, beta, range(1, -1), 1, True)


@pytest.mark.parametrize("kind,ns", [("2Dsc-1.0", 6), ("3Dsc-0.7", 4), ("2Dsc-1.0-0.2-0.05", 8)])
def test_chi0_asym_coeffs_lattice(kind, ns):
    """Lattice tail coefficients: the package's FFT correlation against the oracle's O(N_k²) sum."""
    mP = L.ModelParameters(1.3, 0.4, 7.0, 0.9, 0.2, 0.0, 0.0)
    c1, c2, c3 = L.χ0Asym_coeffs(L.gen_kGrid(kind, ns), False, mP)
    o1, o2, o3 = R.chi0_asym_coeffs(R.gen_kGrid(kind, ns), False, R.ModelParameters(1.3, 0.4, 7.0, 0.9, 0.2, 0.0, 0.0))
    assert c1 == pytest.approx(o1, abs=1e-14) and c3 == pytest.approx(o3, rel=1e-14)
    assert np.allclose(c2, o2, rtol=1e-13, atol=1e-14)
    # q = 0 is the k-mean of t1²: c2[q0] = c3 - U² n/2 (1 - n/2)
    assert c2[0] == pytest.approx(c3 - 1.3**2 * 0.45 * 0.55, rel=1e-13)
