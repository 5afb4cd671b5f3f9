"""Host-side logic of the package without a GPU: the synthetic input generator, the k-grid and
frequency helpers, and the parameter structs, against known answers and the oracle."""
import math

import numpy as np
import pytest

import ladderdga_b200 as L
from ladderdga_b200 import synthetic as S
from oracle import ldga_ref as R


def test_splitmix64_known_answer():
    # the published SplitMix64 sequence from state 0
    assert [int(x) for x in S.splitmix64(0, 3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_and_gaussian_moments():
    u = S.uniform01(5, 200000)
    assert u.min() > 0 and u.max() < 1 and abs(u.mean() - 0.5) < 5e-3
    z = S.complex_gaussian(6, 200000)
    assert abs(np.mean(z.real)) < 1e-2 and abs(np.var(z.real) - 1) < 2e-2 and abs(np.var(z.imag) - 1) < 2e-2


def test_synthetic_input_is_deterministic_and_hermitian():
    a = S.make_input(dim=2, ns=8, beta=5.0, U=1.0, n_iv=4, n_iw=4, seed=81)
    b = S.make_input(dim=2, ns=8, beta=5.0, U=1.0, n_iv=4, n_iw=4, seed=81)
    c = S.make_input(dim=2, ns=8, beta=5.0, U=1.0, n_iv=4, n_iw=4, seed=82)
    assert np.array_equal(a.gamma_m, b.gamma_m) and not np.array_equal(a.gamma_m, c.gamma_m)
    # Sigma_loc(i nu) = U/2 + (U^2/4)/(i nu + 0.5 i sgn nu), n >= 0
    nu = (2 * np.arange(len(a.sigma_loc)) + 1) * math.pi / a.beta
    assert np.allclose(a.sigma_loc, a.U / 2 + (a.U**2 / 4) / (1j * nu + 0.5j))
    assert a.mu == a.U / 2 and a.n == 1.0
    # the correlated part C_r of chi_loc is Hermitian in (nu, nu') at every omega
    for chi in (a.chi_loc_m, a.chi_loc_d):
        d = np.array([np.diag(np.diag(chi[:, :, w])) for w in range(chi.shape[2])]).transpose(1, 2, 0)
        off = chi - d
        assert np.allclose(off, np.conj(off.transpose(1, 0, 2)))


def test_configurations():
    for cfg, (dim, ns, beta, U, n) in {1: (2, 16, 10.0, 1.0, 10), 2: (2, 64, 30.0, 2.0, 30), 3: (3, 32, 20.0, 1.5, 20),
                                       4: (2, 48, 20.0, 1.5, 20)}.items():
        c = S.CONFIGS[cfg]
        assert (c["dim"], c["ns"], c["beta"], c["U"], c["n_iv"], c["n_iw"]) == (dim, ns, beta, U, n, n)


@pytest.mark.parametrize("dim,ns", [(2, 4), (2, 7), (3, 4), (3, 5)])
def test_dispersion_and_wedge(dim, ns):
    eps = S.dispersion_full(dim, ns)
    k = 2 * np.pi * np.arange(ns) / ns
    cs = np.cos(k)
    if dim == 2:
        want = -2 * (cs[:, None] + cs[None, :])
    else:
        want = -2 * (cs[:, None, None] + cs[None, :, None] + cs[None, None, :])
    assert np.allclose(eps, want)
    kG = L.gen_kGrid(f"{dim}Dsc-1.0", ns)
    full = eps.reshape(-1)
    assert kG.kintegrate(kG.ϵkGrid) == pytest.approx(full.mean(), abs=1e-14)
    assert kG.kintegrate(kG.ϵkGrid**2) == pytest.approx((full**2).mean())


def test_kgrid_expand_reduce_roundtrip():
    kG = R.gen_kGrid("3Dsc-1.0", 6)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(kG.Nq)
    full = kG.expand(x)
    assert full.shape == (6, 6, 6)
    assert np.allclose(kG.reduce(full), x)
    # the full-grid array is invariant under the point group (axis permutations and reflections)
    assert np.allclose(full, full.transpose(1, 0, 2)) and np.allclose(full, full.transpose(2, 1, 0))
    assert np.allclose(full, np.roll(full[::-1], 1, axis=0))


def test_G_shell_sum_trigamma_against_scipy():
    for beta in (1.0, 10.0, 40.0):
        for N in (1, 3, 10, 120):
            assert L.G_shell_sum(N, beta) == pytest.approx(R.G_shell_sum(N, beta), rel=1e-13)


def test_parameter_structs_mirror_reference():
    mP = L.ModelParameters(1.5, 0.75, 20.0, 1.0, 0.0, 0.1, 0.2)
    assert (mP.U, mP.μ, mP.β, mP.n) == (1.5, 0.75, 20.0, 1.0)
    assert mP.mu == mP.μ and mP.beta == mP.β
    sP = L.SimulationParameters(4, 5, 0, False, None, range(-19, 19), 0.1, False)
    assert (sP.n_iω, sP.n_iν) == (4, 5)
    with pytest.raises(Exception):
        L.calc_χγ("x", None, None)             # error("Unkown type") for r not in {m, d}


def test_matsubara_helpers_match_oracle():
    for shift in (False, True):
        sp_o = R.SimulationParameters(3, 4, 0, shift, None, range(-20, 20), 0.1, False)
        sp_p = L.SimulationParameters(3, 4, 0, shift, None, range(-20, 20), 0.1, False)
        for wi in range(1, 2 * 3 + 2):
            assert L.ν0Index_of_ωIndex(wi, sp_p) == R.nu0_index_of_w_index(wi, sp_o)
