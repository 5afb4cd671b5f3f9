"""CPU FP64 oracle for the lDGA ladder hot path -- TEST INFRASTRUCTURE ONLY.

This module is a NumPy/SciPy restatement of LadderDGA.jl v0.15.1's plain path
(``chi_helper = nothing``): bubble -> Bethe-Salpeter (m, d) -> lambda_0 -> EoM -> lambda
correction.  It is used only by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` as the checker; the product (``ladderdga.jl_b200``) never imports it.

Parity status
-------------
* PINNED against the reference's own known answers (tests/test_oracle_pins.py):
  ``filling`` on the 2x2 grid = 1.1706318843228878 (test/GFTools.jl:33), chi_lambda and
  ``newton_right`` roots (test/LambdaCorrection/helpers.jl:1-24), the Matsubara-sum identities
  (test/DataTypes.jl:47-67), ``find_usable_chi_interval`` cases (test/GFFit.jl:39-55),
  ``reduce_range`` (test/helpers.jl:1-11), frequency index maps (test/helpers.jl:13-22),
  ``calc_E_ED`` on the reference's DMFT fixture (test/thermodynamics.jl:1-5: E_kin ≈ -0.10448 and
  E_pot ≈ 0.28354, atol 1e-3; the fixture is read by ``ladderdga_b200.jld2`` and frozen as
  tests/golden/b1u2_dmft.npz).
* UNPINNED for the bubble / BSE / EoM / lambda chain: the reference ships no golden vectors for
  them (test/ladderDGATools.jl is empty, test/full_run.jl asserts properties only) and Julia is
  not installed, so it cannot be run.  Those functions are restated from the source lines cited
  below and cross-checked by O(N_k^2) direct sums and the reference's property tests.

The k-grid arithmetic lives in the un-vendored Dispersions.jl 0.8.9 (Manifest.toml:194-200).
It is restated from its call-site contract: ``kintegrate`` is the kMult-weighted mean over the
irreducible points (DataTypes.jl:230-241), ``expandKArr``/``reduceKArr`` map between the
irreducible wedge and the full periodic grid, and ``conv_fft!`` / ``conv_post(_add)!`` form the
normalised circular convolution conv(A,B)(q) = (1/N_k) sum_k A(k) B(k+q) from ``fft(A)`` and
``fft(reverse(B))`` (BSETools.jl:165, ladderDGATools_singleCore.jl:13-26, runHelpers.jl:127-128).
The irreducible wedge is the simple-cubic point group reduction q_x >= q_y (>= q_z) >= 0 with
q_i <= N/2, ordered lexicographically (q = 0 first, matching ``q0_index == 1`` in
test/helpers.jl:15).  The same convention is used by the GPU library.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft
from scipy.special import polygamma

_WORKERS = 1


def set_workers(n: int) -> None:
    """Thread count for the oracle's FFTs (the CPU baseline uses all host cores)."""
    global _WORKERS
    _WORKERS = max(1, int(n))


# =============================================================================================
# k-grid: restatement of Dispersions.jl's gen_kGrid / kintegrate / expandKArr / reduceKArr
# =============================================================================================
class KGrid:
    """Simple-cubic k-grid with the point-group-irreducible wedge (Dispersions.jl contract)."""

    def __init__(self, dim: int, ns: int, t: float = 1.0, tp: float = 0.0, tpp: float = 0.0):
        self.dim, self.Ns, self.t, self.tp, self.tpp = dim, ns, t, tp, tpp
        self.Nk = ns ** dim
        M = ns // 2 + 1
        if dim == 2:
            wedge = [(a, b) for a in range(M) for b in range(a + 1)]
        elif dim == 3:
            wedge = [(a, b, c) for a in range(M) for b in range(a + 1) for c in range(b + 1)]
        else:
            raise ValueError("dim must be 2 or 3")
        self.wedge = np.array(wedge, dtype=np.int64)
        self.Nq = len(wedge)
        widx = {w: i for i, w in enumerate(wedge)}
        # full grid index -> irreducible index
        grids = np.meshgrid(*([np.arange(ns)] * dim), indexing="ij")
        folded = [np.minimum(g, ns - g) % ns for g in grids]
        # ns - 0 = ns -> fold to 0 handled by % ns above only for g == 0
        folded = [np.where(g == 0, 0, f) for g, f in zip(grids, folded)]
        st = np.sort(np.stack(folded, axis=-1), axis=-1)[..., ::-1]
        self.full_to_irr = np.empty((ns,) * dim, dtype=np.int64)
        for pos in np.ndindex(*((ns,) * dim)):
            self.full_to_irr[pos] = widx[tuple(int(x) for x in st[pos])]
        self.kMult = np.bincount(self.full_to_irr.reshape(-1), minlength=self.Nq).astype(np.float64)
        k = 2.0 * math.pi * self.wedge / ns
        if dim == 2:
            self.eps = (-2.0 * t * (np.cos(k[:, 0]) + np.cos(k[:, 1]))
                        - 4.0 * tp * np.cos(k[:, 0]) * np.cos(k[:, 1])
                        - 2.0 * tpp * (np.cos(2 * k[:, 0]) + np.cos(2 * k[:, 1])))
        else:
            self.eps = -2.0 * t * np.cos(k).sum(axis=1)

    @property
    def gridshape(self):
        return (self.Ns,) * self.dim

    def expand(self, arr_irr: np.ndarray) -> np.ndarray:
        """``expandKArr``: irreducible values -> full grid (leading axis q -> gridshape)."""
        return np.asarray(arr_irr)[self.full_to_irr]

    def reduce(self, arr_full: np.ndarray) -> np.ndarray:
        """``reduceKArr``: full grid -> values at the wedge representatives."""
        idx = tuple(self.wedge[:, d] for d in range(self.dim))
        return arr_full[idx]

    def kintegrate(self, arr: np.ndarray, axis: int = 0):
        """kMult-weighted mean over the irreducible axis (DataTypes.jl:230-241 usage)."""
        a = np.moveaxis(np.asarray(arr), axis, 0)
        return np.tensordot(self.kMult, a, axes=(0, 0)) / self.Nk


def gen_kGrid(kind: str, ns: int) -> KGrid:
    """Parse the reference's grid strings ``"2Dsc-t"``, ``"3Dsc-t"``, ``"2Dsc-t-tp-tpp"``."""
    head, *params = kind.split("-")
    dim = int(head[0])
    vals = [float(p) for p in params] + [0.0, 0.0]
    return KGrid(dim, ns, vals[0], vals[1], vals[2])


def conv_fft(kG: KGrid, a_hat: np.ndarray, b_rhat: np.ndarray) -> np.ndarray:
    """Dispersions ``conv_fft!`` + ``conv_post``: (1/N_k) sum_k A(k) B(k+q) at the wedge q.

    ``a_hat = fft(A)``, ``b_rhat = fft(reverse(B))`` on the full grid (leading grid axes, any
    trailing batch axes).  ifft(a_hat*b_rhat)(m) = sum_k A(k) B(k-m-1), so the value at q sits at
    m = N-1-q in every axis.
    """
    d = kG.dim
    prod = a_hat * b_rhat
    res = sfft.ifftn(prod, axes=tuple(range(d)), workers=_WORKERS)
    idx = tuple((kG.Ns - 1 - kG.wedge[:, i]) % kG.Ns for i in range(d))
    return res[idx] / kG.Nk


def conv_direct(kG: KGrid, A_irr: np.ndarray, B_irr: np.ndarray) -> np.ndarray:
    """O(N_k^2) direct sum (1/N_k) sum_k A(k) B(k+q) -- cross-check for ``conv_fft``."""
    A = kG.expand(A_irr).reshape(-1)
    Bf = kG.expand(B_irr)
    out = np.empty(kG.Nq, dtype=np.complex128)
    grid = np.stack(np.meshgrid(*([np.arange(kG.Ns)] * kG.dim), indexing="ij"), -1).reshape(-1, kG.dim)
    for qi, q in enumerate(kG.wedge):
        sh = (grid + q) % kG.Ns
        out[qi] = np.sum(A * Bf[tuple(sh[:, i] for i in range(kG.dim))]) / kG.Nk
    return out


# =============================================================================================
# Parameter structs (Config.jl:39-75) and Matsubara helpers (helpers.jl, GFTools.jl)
# =============================================================================================
@dataclass
class ModelParameters:
    U: float
    mu: float
    beta: float
    n: float
    sVk: float
    Epot_DMFT: float
    Ekin_DMFT: float


@dataclass
class SimulationParameters:
    n_iw: int
    n_iv: int
    n_iv_shell: int
    shift: bool
    chi_helper: object
    fft_range: range
    usable_prct_reduction: float
    dbg_full_eom_omega: bool


def nu_grid(wn: int, sP: SimulationParameters):
    """``nuGrid`` (helpers.jl:20)."""
    return np.arange(-sP.n_iv - sP.n_iv_shell, sP.n_iv + sP.n_iv_shell) - int(sP.shift) * int(wn / 2)


def one_to_freq(wi: int, vi: int, sP: SimulationParameters):
    """``OneToIndex_to_Freq`` (helpers.jl:46-50) with 1-based indices."""
    wn = wi - sP.n_iw - 1
    vn = (vi - sP.n_iv - 1) - int(sP.shift) * int(wn / 2)
    return wn, vn


def nu0_index_of_w_index(wi: int, sP: SimulationParameters) -> int:
    """``nu0Index_of_omegaIndex`` (helpers.jl:58), 1-based."""
    return sP.n_iv + int(sP.shift) * int((wi - sP.n_iw - 1) / 2) + 1


def reduce_range(rng, red_prct: float):
    """``reduce_range`` (helpers.jl:141-146); ``rng`` is a 1-based Julia range as (first, last)."""
    first, last = rng
    length = last - first + 1
    sub = math.floor(length / 2 * red_prct)
    lst = max(last - sub, math.ceil(length / 2 + (length % 2 == 0)))
    fst = min(first + sub, math.ceil(length / 2))
    return fst, lst


def iv_array(beta: float, grid) -> np.ndarray:
    return np.array([1j * ((2.0 * n + 1) * math.pi / beta) for n in grid], dtype=np.complex128)


def iw_array(beta: float, grid) -> np.ndarray:
    return np.array([1j * ((2.0 * n) * math.pi / beta) for n in grid], dtype=np.complex128)


# =============================================================================================
# Green's functions (GFTools.jl)
# =============================================================================================
def G_from_Sigma(nn, beta: float, mu: float, eps, sigma):
    """``G_from_Σ`` (GFTools.jl:85-86)."""
    return 1.0 / (1j * (2 * nn + 1) * math.pi / beta + mu - eps - sigma)


def G_shell_sum(N: int, beta: float) -> float:
    """``G_shell_sum`` (GFTools.jl:281-283) with the trigamma function."""
    return float((polygamma(1, N + 0.5) - polygamma(1, 0.5 - N)) * beta / (4 * math.pi**2) + beta / 4)


def filling(G: np.ndarray, U: float, mu: float, beta: float, shell: float | None = None) -> float:
    """``filling(G, U, mu, beta[, shell])`` (GFTools.jl:235-243)."""
    if shell is None:
        shell = G_shell_sum(len(G) // 2, beta)
    return 2 * (np.real(np.sum(G)) / beta + 0.5 + mu * shell) / (1 + U * shell)


def filling_kG(G: np.ndarray, kG: KGrid, U: float, mu: float, beta: float) -> float:
    """``filling(G::Matrix, kG, U, mu, beta)`` (GFTools.jl:245-247)."""
    return filling(kG.kintegrate(G, 0), U, mu, beta)


def filling_pos(Gk: np.ndarray, U: float, mu: float, beta: float, improved_sum: bool = True) -> float:
    """``filling_pos`` on a k-integrated G over nu_n = 0..N-1 (GFTools.jl:255-269)."""
    sG = np.sum(Gk)
    if not improved_sum:
        return 2 * np.real(sG + np.conj(sG)) / beta + 1
    shell = G_shell_sum(len(Gk) + 1, beta)
    return 2 * (np.real(sG + np.conj(sG)) / beta + 0.5 + mu * shell) / (1 + U * shell)


def subtract_tail(inp, c: float, iw, power: int):
    """``subtract_tail`` (GFTools.jl:293-312)."""
    out = np.array(inp, dtype=np.complex128, copy=True)
    for n in range(len(out)):
        if iw[n] != 0:
            out[n] = inp[n] - c / (iw[n] ** power)
    return out


def G_from_Sigma_ladder(Sigma_ladder: np.ndarray, sigma_loc: np.ndarray, kG: KGrid,
                        mP: ModelParameters, fft_range: range, fix_n: bool = True,
                        mu: float | None = None, improved_sum: bool = True):
    """``G_from_Σladder!`` (GFTools.jl:154-186) -> (mu, G[Nq, fft_range]).

    ``Sigma_ladder`` is [Nq, numax] over nu_n = 0..numax-1; ``sigma_loc`` covers nu_n = 0..L.
    The reference solves for mu with Roots.find_zero(f, mu, atol=1e-8).  This restatement uses a
    bracket-safeguarded Newton iteration with the analytic derivative dG/dmu = -G^2 and solves to
    machine precision, so that the GPU path (same method) agrees to ~1e-14.
    """
    mu = mP.mu if mu is None else mu
    numax = Sigma_ladder.shape[1]
    L = fft_range[-1]
    nn = np.arange(numax)
    ivn = 1j * (2 * nn + 1) * math.pi / mP.beta
    eps = kG.eps[:, None]

    def f_df(m):
        G = 1.0 / (ivn[None, :] + m - eps - Sigma_ladder)
        Gk = kG.kintegrate(G, 0)
        dGk = kG.kintegrate(-G * G, 0)
        shell = G_shell_sum(numax + 1, mP.beta)
        sG, dsG = np.sum(Gk), np.sum(dGk)
        f = 2 * (2 * np.real(sG) / mP.beta + 0.5 + m * shell) / (1 + mP.U * shell) - mP.n
        df = 2 * (2 * np.real(dsG) / mP.beta + shell) / (1 + mP.U * shell)
        return f, df

    if fix_n:
        mu = mu_newton(f_df, mu)
    G = np.empty((kG.Nq, len(fft_range)), dtype=np.complex128)
    off = -fft_range[0]
    if not np.isnan(mu):
        for n in range(0, L + 1):
            sig = Sigma_ladder[:, n] if n < numax else sigma_loc[n]
            G[:, n + off] = G_from_Sigma(n, mP.beta, mu, kG.eps, sig)
    else:
        G[:, off:] = np.nan
    # negative frequencies by conjugation (GFTools.jl:183-184)
    for j in range(off):
        G[:, j] = np.conj(G[:, off + (L - 1) - j])
    return mu, G


def mu_newton(f_df, mu0: float, tol: float = 1e-14, maxit: int = 100) -> float:
    """Safeguarded Newton for the filling condition (shared method with the GPU path).

    Newton steps with the analytic derivative; once a sign change is seen the iterate is kept
    inside the bracket (bisection fallback).  Stops when |f| < tol, the step is below
    1e-15*(1+|mu|), or after ``maxit`` steps.  Returns NaN if f is not finite.
    """
    mu = mu0
    lo, hi = -np.inf, np.inf
    for _ in range(maxit):
        f, df = f_df(mu)
        if not np.isfinite(f):
            return float("nan")
        if abs(f) < tol:
            return mu
        if f > 0:
            hi = min(hi, mu)
        else:
            lo = max(lo, mu)
        step = f / df if df != 0 else 0.0
        new = mu - step
        if not (lo < new < hi) or not np.isfinite(new):
            if np.isfinite(lo) and np.isfinite(hi):
                new = 0.5 * (lo + hi)
            else:
                new = mu - np.sign(f) * max(1.0, abs(step))
        if abs(new - mu) <= 1e-15 * (1 + abs(mu)):
            return new
        mu = new
    return mu


# =============================================================================================
# Setup (runHelpers.jl:113-187): G, its FFTs, local BSE, imp_density
# =============================================================================================
def lattice_G(kG: KGrid, sigma_loc: np.ndarray, mP: ModelParameters, fft_range: range) -> np.ndarray:
    """gLoc[q, nu] on the irreducible grid for nu in fft_range (runHelpers.jl:118-126)."""
    out = np.empty((kG.Nq, len(fft_range)), dtype=np.complex128)
    for j, vn in enumerate(fft_range):
        s = np.conj(sigma_loc[-vn - 1]) if vn < 0 else sigma_loc[vn]
        out[:, j] = G_from_Sigma(vn, mP.beta, mP.mu, kG.eps, s)
    return out


def G_fft(kG: KGrid, G_irr: np.ndarray):
    """``fft(G)`` and ``fft(reverse(G))`` on the full grid for every column (runHelpers.jl:127-128).

    Returns arrays of shape gridshape + (Nf,).
    """
    d = kG.dim
    full = kG.expand(G_irr)                       # gridshape + (Nf,)
    ghat = sfft.fftn(full, axes=tuple(range(d)), workers=_WORKERS)
    rev = full[(slice(None, None, -1),) * d]
    grhat = sfft.fftn(rev, axes=tuple(range(d)), workers=_WORKERS)
    return ghat, grhat


def calc_bubble(ghat, grhat, kG: KGrid, mP: ModelParameters, sP: SimulationParameters,
                w_subset=None) -> np.ndarray:
    """``calc_bubble`` (BSETools.jl:157-172): chi0[q, nu, w] = -beta conv(G_nu, G_{nu+w}).

    ``ghat``/``grhat`` are indexed by position in ``sP.fft_range``.
    """
    nnu = 2 * (sP.n_iv + sP.n_iv_shell)
    nw = 2 * sP.n_iw + 1
    off = -sP.fft_range[0]
    ws = range(nw) if w_subset is None else w_subset
    data = np.zeros((kG.Nq, nnu, nw), dtype=np.complex128)
    for wi in ws:
        wn = wi - sP.n_iw
        vr = np.arange(-(sP.n_iv + sP.n_iv_shell), sP.n_iv + sP.n_iv_shell) - int(sP.shift * wn / 2)
        a = ghat[..., vr + off]
        b = grhat[..., vr + wn + off]
        data[:, :, wi] = conv_fft(kG, a, b) * (-mP.beta)
    return data


def local_bubble(gimp_off, mP: ModelParameters, sP: SimulationParameters) -> np.ndarray:
    """``calc_bubble`` on the one-point grid (runHelpers.jl:138): -beta G(nu) G(nu+w)."""
    nnu, nw = 2 * sP.n_iv, 2 * sP.n_iw + 1
    out = np.empty((1, nnu, nw), dtype=np.complex128)
    for wi in range(nw):
        for vi in range(nnu):
            wn, vn = one_to_freq(wi + 1, vi + 1, sP)
            out[0, vi, wi] = -mP.beta * gimp_off(vn) * gimp_off(vn + wn)
    return out


def F_from_chi(chi: np.ndarray, gimp_off, sP: SimulationParameters, beta: float, diag_term: bool = True):
    """``F_from_χ`` (BSETools.jl:40-53)."""
    nnu, _, nw = chi.shape
    F = np.empty_like(chi)
    for wi in range(nw):
        for vpi in range(nnu):
            wn, vpn = one_to_freq(wi + 1, vpi + 1, sP)
            for vi in range(nnu):
                _, vn = one_to_freq(wi + 1, vi + 1, sP)
                num = chi[vi, vpi, wi] + (vn == vpn and diag_term) * beta * gimp_off(vn) * gimp_off(wn + vn)
                den = gimp_off(vn) * gimp_off(wn + vn) * gimp_off(vpn) * gimp_off(wn + vpn)
                F[vi, vpi, wi] = -num / den
    return F


def calc_chi_gamma(rtype: str, Gamma: np.ndarray, chi0: np.ndarray, mP: ModelParameters,
                   sP: SimulationParameters, w_subset=None):
    """``calc_χγ`` plain branch (BSETools.jl:192-248) with LAPACK inversion (``inv!``).

    Returns (chi[Nq, Nw] real, gamma[Nq, Nnu, Nw] complex).
    """
    if rtype == "d":
        s = -1
    elif rtype == "m":
        s = 1
    else:
        raise ValueError("Unkown type")
    Nq = chi0.shape[0]
    nnu = 2 * sP.n_iv
    nw = chi0.shape[2]
    chi = np.zeros((Nq, nw))
    gam = np.zeros((Nq, nnu, nw), dtype=np.complex128)
    ws = range(nw) if w_subset is None else w_subset
    sh = sP.n_iv_shell
    for wi in ws:
        A = np.broadcast_to(Gamma[:, :, wi], (Nq, nnu, nnu)).copy()
        idx = np.arange(nnu)
        A[:, idx, idx] += 1.0 / chi0[:, sh + idx, wi]
        X = np.linalg.inv(A)
        chi[:, wi] = np.real(X.sum(axis=(1, 2))) / mP.beta**2
        colsum = X.sum(axis=1)                      # sum over the first index nu'
        gam[:, :, wi] = colsum / (chi0[:, :nnu, wi] * (1.0 + s * mP.U * chi[:, wi])[:, None])
    return chi, gam


def calc_chi_gamma_vjp(rtype: str, Gamma: np.ndarray, chi0: np.ndarray, mP: ModelParameters,
                       chi_bar=None, gamma_bar=None):
    """Adjoint of ``calc_chi_gamma`` (the reference's calc_χγ with inv!, BSETools.jl:192-248) for a real
    loss: upstream chi_bar [Nq, Nw] (real) and gamma_bar [Nq, Nnu, Nw] (dL/dRe + i dL/dIm) ->
    (Gamma_bar [Nnu, Nnu, Nw], chi0_bar [Nq, Nnu, Nw]) in the same convention.  Written from the
    forward's matrix calculus with numpy's dense solver: the FP64 reference gradient of the adjoint.
    With A = Gamma + diag(1/chi0) (the reference's matrix), X = A^-1, u = X^T 1 (the column sums):
    chi = Re sum u / beta^2, gamma = u / (chi0 (1 + s U chi)), and dX = -X dA X."""
    s = -1 if rtype == "d" else 1
    Nq, nnu, nw = chi0.shape
    beta, U = mP.beta, mP.U
    xb = np.zeros((Nq, nw)) if chi_bar is None else np.asarray(chi_bar, dtype=np.float64)
    gb = np.zeros((Nq, nnu, nw), dtype=np.complex128) if gamma_bar is None else np.asarray(gamma_bar)
    Gbar = np.zeros_like(Gamma, dtype=np.complex128)
    c0bar = np.zeros((Nq, nnu, nw), dtype=np.complex128)
    idx = np.arange(nnu)
    one = np.ones(nnu)
    for wi in range(nw):
        A = np.broadcast_to(Gamma[:, :, wi], (Nq, nnu, nnu)).copy()
        d = 1.0 / chi0[:, :, wi]
        A[:, idx, idx] += d
        u = np.linalg.solve(np.transpose(A, (0, 2, 1)), np.broadcast_to(one, (Nq, nnu))[..., None])[..., 0]
        chi = np.real(u.sum(axis=1)) / beta**2
        rf = 1.0 / (1.0 + s * U * chi)
        g = gb[:, :, wi]
        s1 = np.sum(np.real(np.conj(g) * u * d), axis=1)
        xbt = xb[:, wi] - s * U * rf**2 * s1
        ubar = np.conj(d * rf[:, None]) * g + (xbt / beta**2)[:, None]
        # u = A^-T 1: dL = Re <ubar, du>, du = -A^-T dA^T u  ->  Abar = -conj(u) z^T with A^* z = ubar
        z = np.linalg.solve(np.conj(A), ubar[..., None])[..., 0]
        Abar = -np.einsum("qa,qb->qab", np.conj(u), z)
        Gbar[:, :, wi] = Abar.sum(axis=0)
        dbar = Abar[:, idx, idx] + np.conj(u * rf[:, None]) * g
        c0bar[:, :, wi] = -np.conj(d * d) * dbar
    return Gbar, c0bar


def calc_lambda0(chi0: np.ndarray, F: np.ndarray, mP: ModelParameters, sP: SimulationParameters):
    """``calc_λ0`` plain branch (BSETools.jl:129-141): lambda0[q,nu',w] = chi0 * sum_nu F / beta^2."""
    sh = sP.n_iv_shell
    core = chi0[:, sh:chi0.shape[1] - sh, :]
    colF = F.sum(axis=0)                            # [nu', w]
    return core * colF[None, :, :] / mP.beta**2


# =============================================================================================
# chi data type and Matsubara sums (DataTypes.jl:177-308)
# =============================================================================================
class ChiT:
    """``χT`` (DataTypes.jl:177-194): physical susceptibility with c2 tail and lambda."""

    def __init__(self, data: np.ndarray, beta: float, tail_c=(), full_range: bool = True,
                 reduce_range_prct: float = 0.0):
        self.data = np.array(data, dtype=np.float64)
        self.beta = beta
        nw = self.data.shape[1]
        self.indices_w = np.arange(nw) - math.ceil(nw / 2) + 1
        self.tail_c = [float(x) for x in tail_c]
        self.lam = 0.0
        if full_range:
            self.usable_w = np.arange(nw)
        else:
            self.usable_w = find_usable_chi_interval_mat(self.data, reduce_range_prct)

    def wn_grid(self):
        return 2j * math.pi * self.indices_w / self.beta

    def copy(self):
        c = ChiT.__new__(ChiT)
        c.data, c.beta, c.indices_w = self.data.copy(), self.beta, self.indices_w.copy()
        c.tail_c, c.lam, c.usable_w = list(self.tail_c), self.lam, self.usable_w.copy()
        return c


def chi_lambda(x, lam: float):
    """``χ_λ`` (LambdaCorrection/helpers.jl:18)."""
    return x / (lam * x + 1)


def dchi_lambda(x, lam: float):
    """``dχ_λ`` (LambdaCorrection/helpers.jl:61)."""
    return -chi_lambda(x, lam) ** 2


def chi_lambda_inplace(chi: ChiT, lam: float) -> None:
    """``χ_λ!`` (LambdaCorrection/helpers.jl:38-53)."""
    if lam == 0.0:
        return
    if not np.isfinite(lam):
        return
    chi.data = chi_lambda(chi.data, lam)
    chi.lam = chi.lam + lam


def reset(chi: ChiT) -> None:
    """``reset!`` (LambdaCorrection/helpers.jl:64-70): apply chi_lambda(-lam)."""
    if chi.lam != 0:
        chi.data = chi_lambda(chi.data, -chi.lam)
        chi.lam = 0.0


def _wn2_tail(chi: ChiT, wslice):
    wn = chi.wn_grid()[wslice]
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.real(chi.tail_c[2] / wn**2)
    t[~np.isfinite(t)] = 0.0
    return t


def sum_kw_raw(kG: KGrid, chi: np.ndarray, beta: float, c2: float, wn2_tail, transform=None) -> float:
    """``sum_kω(kG, χ::Matrix, β, c2, ωn2_tail; transform)`` (DataTypes.jl:230-249)."""
    res = 0.0
    norm = np.sum(kG.kMult)
    for i, wt in enumerate(wn2_tail):
        if transform is None:
            res += kG.kintegrate(chi[:, i]) - wt
        else:
            res += np.sum(transform(chi[:, i]) * kG.kMult) / norm - wt
    return (res + (-beta**2 / 12) * c2) / beta


def sum_kw(kG: KGrid, chi: ChiT, force_full_range: bool = False, transform=None, lam: float = float("nan")) -> float:
    """``sum_kω(kG, χT; ...)`` (DataTypes.jl:215-228)."""
    if chi.lam != 0 and not np.isnan(lam):
        raise RuntimeError("χ already λ-corrected, but external λ provided!")
    if not np.isnan(lam):
        transform = (lambda x, l=lam: chi_lambda(x, l))
    ws = np.arange(chi.data.shape[1]) if force_full_range else chi.usable_w
    t = _wn2_tail(chi, ws)
    return sum_kw_raw(kG, chi.data[:, ws], chi.beta, chi.tail_c[2], t, transform)


def sum_w_vec(wn_arr, chi_vec, tail_c, beta: float) -> float:
    """``sum_ω(ωn_arr, χ, tail_c, β)`` (DataTypes.jl:294-308)."""
    if not math.isclose(sum(tail_c), tail_c[2]):
        raise RuntimeError("sum_ω only implemented for 1/ω^2")
    res = 0.0
    for n in range(len(chi_vec)):
        if wn_arr[n] != 0:
            res += chi_vec[n] - np.real(tail_c[2] / wn_arr[n] ** 2)
        else:
            res += chi_vec[n]
    return (res + tail_c[2] * (-beta**2 / 12)) / beta


def sum_w(chi: ChiT, force_full_range: bool = False) -> np.ndarray:
    """``sum_ω(χT)`` (DataTypes.jl:277-292)."""
    ws = np.arange(chi.data.shape[1]) if force_full_range else chi.usable_w
    wn = chi.wn_grid()[ws]
    return np.array([sum_w_vec(wn, chi.data[q, ws], chi.tail_c, chi.beta) for q in range(chi.data.shape[0])])


def sum_wk(kG: KGrid, chi: ChiT, force_full_range: bool = False, lam: float = float("nan")) -> float:
    """``sum_ωk`` (DataTypes.jl:257-264)."""
    lam_check = (not np.isnan(lam)) and lam != 0
    if chi.lam != 0 and lam_check:
        raise RuntimeError("χ already λ-corrected, but external λ provided!")
    c = chi
    if lam_check:
        c = chi.copy()
        chi_lambda_inplace(c, lam)
    return float(kG.kintegrate(sum_w(c, force_full_range)))


def update_tail(chi: ChiT, new_tail_c, wn_grid) -> None:
    """``update_tail!`` (DataTypes.jl:315-345)."""
    new_tail_c = [float(x) for x in new_tail_c]
    if len(new_tail_c) != len(chi.tail_c):
        raise ValueError("length of new tail coefficient array must be the same as the old one")
    if len(wn_grid) != chi.data.shape[1]:
        raise ValueError("length of ωnGrid must be the same as for χ")
    if not all(np.isfinite(new_tail_c)):
        raise ValueError("One or more tail coefficients are not finite!")
    if sum(new_tail_c) != new_tail_c[2]:
        raise ValueError("update tail only implemented for c_2 coefficient!")
    lam_bak = chi.lam
    if lam_bak != 0:
        reset(chi)
    zero = [i for i, w in enumerate(wn_grid) if abs(w) < 1e-10]
    if chi.tail_c[2] != new_tail_c[2]:
        for wi in range(chi.data.shape[1]):
            if wi in zero:
                continue
            chi.data[:, wi] += np.real((new_tail_c[2] - chi.tail_c[2]) / wn_grid[wi] ** 2)
        chi.tail_c[2] = new_tail_c[2]
    chi_lambda_inplace(chi, lam_bak)


# =============================================================================================
# Usable ranges (GFFit.jl:31-84)
# =============================================================================================
def find_usable_chi_interval(chi_w, sum_type="common", reduce_range_prct: float = 0.1):
    """``find_usable_χ_interval`` (GFFit.jl:31-69); returns 1-based indices as a list."""
    chi_w = np.asarray(chi_w, dtype=np.float64)
    n = len(chi_w)
    if n % 2 == 0:
        raise ValueError("Finding a usable interval is only implemented for uneven size of χ_ω!")
    mid = math.ceil(n / 2)
    if sum_type == "full":
        return list(range(1, n + 1))
    if isinstance(sum_type, tuple):
        return list(range(sum_type[0], sum_type[1] + 1))
    darr = np.diff(chi_w)
    if chi_w[mid - 1] < 0.0:
        return [mid]
    r1 = 0
    while r1 < mid - 1 and chi_w[mid - r1 - 2] > 0 and chi_w[mid + r1] > 0:
        r1 += 1
    r2 = 0
    while r2 < mid - 1 and darr[mid - r2 - 2] > 0 and darr[mid + r2 - 1] < 0:
        r2 += 1
    rng = math.ceil(min(r1, r2) * (1 - reduce_range_prct))
    return list(range(mid - rng, mid + rng + 1))


def find_usable_chi_interval_mat(chi_qw: np.ndarray, reduce_range_prct: float = 0.1):
    """Matrix version (GFFit.jl:71-73), 0-based indices."""
    sets = [set(find_usable_chi_interval(row, reduce_range_prct=0.1)) for row in chi_qw]
    inter = sorted(set.intersection(*sets))
    return np.array([i - 1 for i in inter], dtype=np.int64)


# =============================================================================================
# lambda helpers (LambdaCorrection/helpers.jl)
# =============================================================================================
def newton_right(f, df, start: float, xmin: float, nsteps: int = 100, atol: float = 1e-13) -> float:
    """1-D ``newton_right`` (LambdaCorrection/helpers.jl:133-153), iteration-for-iteration."""
    delta = 1e-4
    x0 = start
    xi = x0
    i = 1
    while True:
        fi = f(xi)
        dfii = 1.0 / df(xi)
        xi = x0 - dfii * fi
        if abs(fi) < atol:
            break
        if xi < xmin:
            x0 = xmin + delta + abs(xmin - x0) / 2
        else:
            x0 = xi
        if i >= nsteps:
            break
        i += 1
    return xi


def fd_step(x: float) -> float:
    """FiniteDiff forward-difference step: max(sqrt(eps)*|x|, sqrt(eps))."""
    r = math.sqrt(np.finfo(np.float64).eps)
    return max(r * abs(x), r)


def fd_jacobian(f, x: np.ndarray) -> np.ndarray:
    """Forward-difference Jacobian (FiniteDiff.finite_difference_jacobian default, Val(:forward))."""
    fx = np.asarray(f(x), dtype=np.float64)
    J = np.empty((len(fx), len(x)))
    for j in range(len(x)):
        e = fd_step(x[j])
        x1 = x.copy()
        x1[j] += e
        J[:, j] = (np.asarray(f(x1)) - fx) / e
    return J


def newton_right_nd(f, start, xmin, nsteps: int = 500, atol: float = 1e-8, max_reset: int = 5,
                    reset_backoff: float = 1.0, jac=None):
    """N-D ``newton_right`` (LambdaCorrection/helpers.jl:165-208) with an FD Jacobian."""
    jac = fd_jacobian if jac is None else jac
    start = np.array(start, dtype=np.float64)
    xmin = np.array(xmin, dtype=np.float64)
    xi = start.copy()
    i = 1
    reset_i = 1
    bis_fail = False
    while True:
        fi = np.asarray(f(xi), dtype=np.float64)
        dfii = np.linalg.inv(jac(f, xi))
        xi_last = xi.copy()
        xi = xi - dfii @ fi
        for l in range(len(xi)):
            if xi[l] < xmin[l]:
                xi[l] = xmin[l] + abs(xi_last[l] - xmin[l]) / 2
                if abs(xi_last[l] - xmin[l]) / 2 < 1e-8:
                    bis_fail = True
        if bis_fail or not np.all(np.isfinite(fi)):
            bis_fail = False
            if reset_i >= max_reset:
                raise RuntimeError(f"λ root-finding returned NaN after {i} iterations and {max_reset} resets.")
            reset_i += 1
            xi = start + reset_i * reset_backoff * np.abs(xmin)
        if abs(np.linalg.norm(fi)) < atol:
            break
        if i >= nsteps:
            break
        i += 1
    return xi


def get_lambda_min(chi_data: np.ndarray) -> float:
    """``get_λ_min`` (LambdaCorrection/helpers.jl:217-220)."""
    nh = math.ceil(chi_data.shape[1] / 2) - 1
    return float(-np.min(1.0 / chi_data[:, nh]))


def lambda_m_rhs(imp_density: float, chi_m: ChiT, chi_d: ChiT, kG: KGrid, mP: ModelParameters,
                 sP: SimulationParameters, lam_d: float = float("nan"), lambda_rhs: str = "native") -> float:
    """``λm_rhs`` (LambdaCorrection/helpers.jl:234-255)."""
    if chi_d.lam != 0 and not np.isnan(lam_d):
        raise RuntimeError("Stopping λ rhs calculation")
    chi_d_sum = sum_kw(kG, chi_d, lam=lam_d)
    if (sP.chi_helper is not None and lambda_rhs == "native") or lambda_rhs == "fixed":
        return mP.n * (1 - mP.n / 2) - chi_d_sum
    if not np.isfinite(imp_density):
        raise ValueError("imp_density argument is not finite!")
    return 2 * imp_density - chi_d_sum


# =============================================================================================
# EoM (ladderDGATools.jl:147-160, 260; ladderDGATools_singleCore.jl:49-136)
# =============================================================================================
def eom(U, gm, gd, xm, xd, l0):
    """``eom`` (ladderDGATools.jl:260)."""
    return U * (gm * 1.5 * (1 + U * xm) - gd * 0.5 * (1 - U * xd) - 1.5 + 0.5 + l0)


EOM_PARTS = {
    "chi_m": lambda U, gm, gd, xm, xd, l0: U * (gm * 1.5 * (U * xm)),
    "gamma_m": lambda U, gm, gd, xm, xd, l0: U * (gm * 1.5) + 0 * gd,
    "chi_d": lambda U, gm, gd, xm, xd, l0: -U * (gd * 0.5 * (-U * xd)),
    "gamma_d": lambda U, gm, gd, xm, xd, l0: -U * (gd * 0.5) + 0 * gm,
    "rest_01": lambda U, gm, gd, xm, xd, l0: (-U * 1.0 + 0.0j) + 0 * gm,
    "rest": lambda U, gm, gd, xm, xd, l0: U * l0,
}


def calc_Sigma_w(eomf, chi_m: np.ndarray, gamma_m, chi_d: np.ndarray, gamma_d, lambda0, grhat,
                 kG: KGrid, U: float, sP: SimulationParameters, numax: int):
    """``calc_Σ_ω!`` (ladderDGATools_singleCore.jl:28-69): returns [Nq, numax, Nw] per-omega parts."""
    nw = chi_m.shape[1]
    off = -sP.fft_range[0]
    d = kG.dim
    out = np.zeros((kG.Nq, numax, nw), dtype=np.complex128)
    for wi in range(nw):
        wn = wi - sP.n_iw
        v0 = nu0_index_of_w_index(wi + 1, sP) - 1            # 0-based
        vlist = list(range(v0, 2 * sP.n_iv))[:numax]
        if not vlist:
            continue
        vl = np.array(vlist)
        K = eomf(U, gamma_m[:, vl, wi], gamma_d[:, vl, wi], chi_m[:, wi][:, None], chi_d[:, wi][:, None],
                 lambda0[:, vl, wi])                              # [Nq, nv]
        Kf = kG.expand(K)                                         # grid + (nv,)
        Khat = sfft.fftn(Kf, axes=tuple(range(d)), workers=_WORKERS)
        nii = np.arange(len(vlist))
        g = grhat[..., nii + wn + off]
        out[:, : len(vlist), wi] = conv_fft(kG, Khat, g)
    return out


def calc_Sigma_vjp(Sigma_bar, chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, G_irr, kG: KGrid,
                   mP: ModelParameters, sP: SimulationParameters, numax: int, lam_m: float = 0.0, lam_d: float = 0.0,
                   tc: bool = True):
    """Adjoint of ``calc_Σ`` (ladderDGATools_singleCore.jl:49-136) at (λm, λd) for a real loss:
    Sigma_bar [Nq, numax] (dL/dRe + i dL/dIm of the stored irreducible values) ->
    (chi_m_bar, gamma_m_bar, chi_d_bar, gamma_d_bar, lambda0_bar).  The convolution's adjoint is the
    full-grid correlation with conj(G), evaluated by FFT like the forward (conv_fft):
    Kbar(p) = kMult(p)/beta (1/N_k) sum_k Sbar_full(k) conj(G(k + p)), Sbar_full = Sbar/kMult expanded."""
    U, beta = mP.U, mP.beta
    d = kG.dim
    cmv = chi_m.data if lam_m == 0.0 else chi_lambda(chi_m.data, lam_m)
    cdv = chi_d.data if lam_d == 0.0 else chi_lambda(chi_d.data, lam_d)
    nw = cmv.shape[1]
    off = -sP.fft_range[0]
    gmb = np.zeros_like(gamma_m, dtype=np.complex128)
    gdb = np.zeros_like(gamma_d, dtype=np.complex128)
    l0b = np.zeros_like(lambda0, dtype=np.complex128)
    xmb = np.zeros(cmv.shape)
    xdb = np.zeros(cdv.shape)
    Sf = kG.expand(np.asarray(Sigma_bar) / kG.kMult[:, None])
    Shat = sfft.fftn(Sf, axes=tuple(range(d)), workers=_WORKERS)
    for wi in range(nw):
        wn = wi - sP.n_iw
        v0 = nu0_index_of_w_index(wi + 1, sP) - 1
        vlist = list(range(v0, 2 * sP.n_iv))[:numax]
        if not vlist:
            continue
        vl = np.array(vlist)
        nii = np.arange(len(vlist))
        Gc = np.conj(kG.expand(G_irr[:, nii + wn + off]))
        rev = Gc[(slice(None, None, -1),) * d]
        grc = sfft.fftn(rev, axes=tuple(range(d)), workers=_WORKERS)
        Kbar = conv_fft(kG, Shat[..., nii], grc) * kG.kMult[:, None] / beta
        gm, gd = gamma_m[:, vl, wi], gamma_d[:, vl, wi]
        gmb[:, vl, wi] = (1.5 * U * (1.0 + U * cmv[:, wi]))[:, None] * Kbar
        gdb[:, vl, wi] = (-0.5 * U * (1.0 - U * cdv[:, wi]))[:, None] * Kbar
        l0b[:, vl, wi] = U * Kbar
        xmb[:, wi] += np.sum(np.real(np.conj(Kbar) * 1.5 * U * U * gm), axis=1)
        xdb[:, wi] += np.sum(np.real(np.conj(Kbar) * 0.5 * U * U * gd), axis=1)
    if tc:
        # tail -U (sum_kω χm^λ - χloc_m_sum)/(iν_n): d/dχm^λ(q, ω) of sum_kω is kMult(q)/(β N_k)
        wnu = (2 * np.arange(numax) + 1) * math.pi / beta
        sbar = U * float(np.sum(np.imag(np.asarray(Sigma_bar)) / wnu[None, :]))
        xmb += sbar * kG.kMult[:, None] / (beta * kG.Nk)
    xmb /= (lam_m * chi_m.data + 1.0) ** 2
    xdb /= (lam_d * chi_d.data + 1.0) ** 2
    return xmb, gmb, xdb, gdb, l0b


def calc_Sigma(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, chi_m_sum: float, lambda0, grhat,
               kG: KGrid, mP: ModelParameters, sP: SimulationParameters, numax: int | None = None,
               lam_m: float = 0.0, lam_d: float = 0.0, tc: bool = True) -> np.ndarray:
    """``calc_Σ`` (ladderDGATools_singleCore.jl:114-136) -> Sigma_ladder[Nq, 0:numax-1]."""
    numax = sP.n_iv if numax is None else numax
    if chi_m.lam != 0 and lam_m != 0:
        raise RuntimeError(f"Stopping self energy calculation: λm = {lam_m} AND χm.λ = {chi_m.lam}")
    if chi_d.lam != 0 and lam_d != 0:
        raise RuntimeError(f"Stopping self energy calculation: λd = {lam_d} AND χd.λ = {chi_d.lam}")
    cm, cd = chi_m.copy(), chi_d.copy()
    if lam_m != 0.0:
        chi_lambda_inplace(cm, lam_m)
    if lam_d != 0.0:
        chi_lambda_inplace(cd, lam_d)
    return calc_Sigma_inner(cm, gamma_m, cd, gamma_d, chi_m_sum, lambda0, grhat, kG, mP, sP, numax, tc)


def calc_Sigma_inner(cm: ChiT, gamma_m, cd: ChiT, gamma_d, chi_m_sum, lambda0, grhat, kG, mP, sP,
                     numax: int, tc: bool = True) -> np.ndarray:
    """``calc_Σ!`` (ladderDGATools_singleCore.jl:71-81) on already lambda-corrected chi."""
    parts = calc_Sigma_w(eom, cm.data, gamma_m, cd.data, gamma_d, lambda0, grhat, kG, mP.U, sP, numax)
    S = parts.sum(axis=2)
    hartree = mP.n * mP.U / 2.0
    tail = (-mP.U * (sum_kw(kG, cm) - chi_m_sum) if tc else 0.0) / iv_array(mP.beta, range(numax))
    return S / mP.beta + tail[None, :] + hartree


def calc_Sigma_parts(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, chi_m_sum, lambda0, grhat, kG,
                     mP, sP, lam_m: float = 0.0, lam_d: float = 0.0, tc: bool = True) -> np.ndarray:
    """``calc_Σ_parts`` (ladderDGATools_singleCore.jl:153-189) -> [Nq, n_iv, 7]."""
    cm, cd = chi_m.copy(), chi_d.copy()
    if lam_m != 0.0:
        chi_lambda_inplace(cm, lam_m)
    if lam_d != 0.0:
        chi_lambda_inplace(cd, lam_d)
    numax = sP.n_iv
    hartree = mP.n * mP.U / 2.0
    tail = (-mP.U * (sum_kw(kG, cm) - chi_m_sum) if tc else 0.0) / iv_array(mP.beta, range(numax))
    out = np.zeros((kG.Nq, numax, 7), dtype=np.complex128)
    for j, key in enumerate(["chi_m", "gamma_m", "chi_d", "gamma_d", "rest_01", "rest"]):
        p = calc_Sigma_w(EOM_PARTS[key], cm.data, gamma_m, cd.data, gamma_d, lambda0, grhat, kG, mP.U, sP, numax)
        out[:, :, j] = p.sum(axis=2) / mP.beta
    out[:, :, 5] += hartree
    out[:, :, 6] = tail[None, :]
    return out


# =============================================================================================
# thermodynamics (thermodynamics.jl:142-168)
# =============================================================================================
def calc_E(G_nu: np.ndarray, Sigma: np.ndarray, mu: float, kG: KGrid, mP: ModelParameters):
    """``calc_E(G, Σ, μ, kG, mP)``: G and Sigma given over nu_n = 0..numax-1 -> (E_kin, E_pot)."""
    numax = min(G_nu.shape[1], Sigma.shape[1])
    ivn = iv_array(mP.beta, range(numax))
    hartree = mP.n * mP.U / 2
    eps = kG.eps
    ekin_tc = eps + hartree - mu
    epot_tc = mP.U**2 * 0.5 * mP.n * (1 - 0.5 * mP.n) + hartree * (eps + hartree - mu)
    tail = 1.0 / ivn**2
    epot_tail = epot_tc[:, None] * tail[None, :]
    ekin_tail = ekin_tc[:, None] * tail[None, :]
    epot_tail_inv = (mP.beta / 2) * hartree + (mP.beta / 2) * (-mP.beta / 2) * epot_tc
    ekin_tail_inv = (mP.beta / 2) * eps * (1 + -mP.beta * ekin_tc)
    G = G_nu[:, :numax]
    S = Sigma[:, :numax]
    epot_full = np.real(G * S - epot_tail)
    ekin_full = eps[:, None] * np.real(G - ekin_tail)
    E_kin = kG.kintegrate(4 * ekin_full.sum(axis=1) + ekin_tail_inv) / mP.beta
    E_pot = kG.kintegrate(2 * epot_full.sum(axis=1) + epot_tail_inv) / mP.beta
    return float(E_kin), float(E_pot)


def chi0_asym_coeffs(kG: KGrid, local_tail: bool, mP: ModelParameters):
    """``χ₀Asym_coeffs`` (DataTypes.jl:110-124) -> (c1, c2[q], c3); the lattice c2 is the
    convolution (1/N_k) sum_k t1(k) t1(k+q) of t1 = eps_k + Un/2 - mu (Dispersions ``conv_noPlan``)."""
    t2 = mP.U**2 * (mP.n / 2) * (1 - mP.n / 2)
    if local_tail:
        c1 = mP.U * mP.n / 2 - mP.mu
        return c1, [c1 * c1], c1 * c1 + mP.sVk + t2
    t1 = kG.eps + mP.U * mP.n / 2 - mP.mu
    c2 = np.real(conv_direct(kG, t1.astype(np.complex128), t1.astype(np.complex128)))
    return float(kG.kintegrate(t1)), c2, float(kG.kintegrate(t1**2)) + t2


def calc_E_ED(eps_k, V_k, gimp, U: float, n: float, mu: float, beta: float):
    """``calc_E_ED`` (thermodynamics.jl:46-64): Anderson-impurity energies from the bath and G_imp.
    Delta(nu) = sum_k V_k^2 / (i nu - eps_k), Sigma = i nu - Delta - 1/G + mu, with the 1/nu^2
    tails (sum V_k^2 and U^2/2 n(1-n/2) - Sigma_H (Sigma_H - mu)) summed analytically."""
    eps_k = np.asarray(eps_k, dtype=np.float64)
    V_k = np.asarray(V_k, dtype=np.float64)
    gimp = np.asarray(gimp, dtype=np.complex128)
    vk = float(np.sum(V_k**2))
    s_h = n * U / 2
    epot_tail = U**2 / 2 * n * (1 - n / 2) - s_h * (s_h - mu)
    ivn = iv_array(beta, range(len(gimp)))
    delta = np.array([np.sum(V_k * V_k / (iv - eps_k)) for iv in ivn])
    sigma = ivn - delta - 1.0 / gimp + mu
    e_kin = float(np.sum(2 * np.real(gimp * delta - vk / ivn**2)))
    e_pot = float(np.sum(2 * np.real(gimp * sigma - epot_tail / ivn**2)))
    return e_kin * (2 / beta) - (beta / 2) * vk, e_pot / beta + 0.5 * s_h - (beta / 4) * epot_tail


# =============================================================================================
# Helper struct and setup (runHelpers.jl:28-201)
# =============================================================================================
@dataclass
class Helper:
    """``lDΓAHelper`` subset used on the hot path."""
    sP: SimulationParameters
    mP: ModelParameters
    kG: KGrid
    sigma_loc: np.ndarray
    imp_density: float
    G_irr: np.ndarray
    ghat: np.ndarray
    grhat: np.ndarray
    Gamma_m: np.ndarray
    Gamma_d: np.ndarray
    chiloc_m_sum: float
    chi_loc_m: np.ndarray
    chi_loc_d: np.ndarray
    chi_m_loc: ChiT
    gamma_m_loc: np.ndarray
    chi_d_loc: ChiT
    gamma_d_loc: np.ndarray
    chi0_loc: np.ndarray
    gimp: np.ndarray
    extra: dict = field(default_factory=dict)

    def gimp_off(self, n: int) -> complex:
        return self.gimp[n] if n >= 0 else np.conj(self.gimp[-n - 1])


def setup_ldga(inp, usable_prct_reduction: float = 0.0) -> Helper:
    """``setup_LDGA`` (runHelpers.jl:85-201) from a ``SyntheticInput`` instead of the JLD2 file."""
    kG = KGrid(inp.dim, inp.ns, inp.t)
    mP = ModelParameters(inp.U, inp.mu, inp.beta, inp.n, inp.sVk, inp.Epot_DMFT, inp.Ekin_DMFT)
    L = 2 * (inp.n_iv + inp.n_iw)
    sP = SimulationParameters(inp.n_iw, inp.n_iv, 0, inp.shift, None, range(-L, L + 1),
                              usable_prct_reduction, False)
    G_irr = lattice_G(kG, inp.sigma_loc, mP, sP.fft_range)
    ghat, grhat = G_fft(kG, G_irr)
    rm = max(abs(sP.fft_range[0]), abs(sP.fft_range[-1]))
    gimp = np.asarray(inp.gimp[:rm])

    def goff(n):
        return gimp[n] if n >= 0 else np.conj(gimp[-n - 1])

    F_m = F_from_chi(inp.chi_loc_m, goff, sP, mP.beta)
    chi0_loc = local_bubble(goff, mP, sP)
    xm, gm = calc_chi_gamma("m", inp.gamma_m, chi0_loc, mP, sP)
    xd, gd = calc_chi_gamma("d", inp.gamma_d, chi0_loc, mP, sP)
    chi_m_loc = ChiT(xm, mP.beta, tail_c=[0, 0, mP.Ekin_DMFT])
    chi_d_loc = ChiT(xd, mP.beta, tail_c=[0, 0, mP.Ekin_DMFT])
    chiloc_m_sum = float(np.real(sum_w(chi_m_loc)[0]))
    nw = 2 * inp.n_iw + 1
    chi_loc_m_w = np.array([np.sum(inp.chi_loc_m[:, :, w]) / mP.beta**2 for w in range(nw)])
    chi_loc_d_w = np.array([np.sum(inp.chi_loc_d[:, :, w]) / mP.beta**2 for w in range(nw)])
    um = find_usable_chi_interval(np.real(chi_loc_m_w), reduce_range_prct=sP.usable_prct_reduction)
    ud = find_usable_chi_interval(np.real(chi_loc_d_w), reduce_range_prct=sP.usable_prct_reduction)
    loc = sorted(set(um) & set(ud))
    iwn = 1j * 2 * np.arange(-inp.n_iw, inp.n_iw + 1) * math.pi / mP.beta
    li = np.array(loc) - 1
    chi_upup = 0.5 * (chi_loc_m_w + chi_loc_d_w)[li]
    chi_upup_sub = subtract_tail(chi_upup, mP.Ekin_DMFT, iwn[li], 2)
    imp_density = float(np.real(np.sum(chi_upup_sub)) / mP.beta - mP.Ekin_DMFT * mP.beta / 12)
    h = Helper(sP, mP, kG, np.asarray(inp.sigma_loc), imp_density, G_irr, ghat, grhat,
               inp.gamma_m, inp.gamma_d, chiloc_m_sum, inp.chi_loc_m, inp.chi_loc_d,
               chi_m_loc, gm, chi_d_loc, gd, chi0_loc, gimp)
    h.extra["F_m"] = F_m
    return h


def F_m_of(h: Helper) -> np.ndarray:
    return h.extra["F_m"]


# =============================================================================================
# lambda corrections (LambdaCorrection/conditions_new.jl)
# =============================================================================================
def lambda_m_correction(chi_m: ChiT, rhs: float, kG: KGrid, mP: ModelParameters, sP: SimulationParameters,
                        validate_threshold: float = 1e-8):
    """``λm_correction`` (conditions_new.jl:144-172) -> (lambda_m, validation)."""
    lam_min = get_lambda_min(chi_m.data)
    chir = chi_m.data[:, chi_m.usable_w]
    iwn = 1j * 2 * np.arange(-sP.n_iw, sP.n_iw + 1)[chi_m.usable_w] * math.pi / mP.beta
    with np.errstate(divide="ignore", invalid="ignore"):
        wn2_tail = np.real(chi_m.tail_c[2] / iwn**2)
    wn2_tail[np.abs(iwn) < 1e-10] = 0.0

    def f(l):
        return sum_kw_raw(kG, chir, chi_m.beta, chi_m.tail_c[2], wn2_tail, lambda x: chi_lambda(x, l)) - rhs

    def df(l):
        return sum_kw_raw(kG, chir, chi_m.beta, chi_m.tail_c[2], wn2_tail, lambda x: dchi_lambda(x, l))

    lam = newton_right(f, df, 0.0, lam_min)
    c = chi_m.copy()
    chi_lambda_inplace(c, lam)
    check = sum_kw(kG, c)
    check2 = sum_wk(kG, c)
    validation = abs(rhs - check) <= validate_threshold and abs(rhs - check2) <= validate_threshold
    return lam, validation


@dataclass
class LambdaResult:
    """``λ_result`` (conditions_new.jl:13-46)."""
    lam_m: float
    lam_d: float
    type: str
    converged: bool
    sc_converged: bool
    EKin: float
    EPot_p1: float
    EPot_p2: float
    PP_p1: float
    PP_p2: float
    G_ladder: np.ndarray | None
    Sigma_ladder: np.ndarray | None
    mu: float
    n: float


def lambda_m_correction_full(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, h: Helper,
                             numax: int = -1, validate_threshold: float = 1e-8) -> LambdaResult:
    """``λm_correction_full`` (conditions_new.jl:174-190)."""
    numax = gamma_m.shape[1] // 2 if numax < 0 else numax
    rhs = lambda_m_rhs(h.imp_density, chi_m, chi_d, h.kG, h.mP, h.sP)
    lam, valid = lambda_m_correction(chi_m, rhs, h.kG, h.mP, h.sP, validate_threshold)
    S = calc_Sigma(chi_m, gamma_m, chi_d, gamma_d, h.chiloc_m_sum, lambda0, h.grhat, h.kG, h.mP, h.sP,
                   numax=numax, lam_m=lam)
    mu, G = G_from_Sigma_ladder(S, h.sigma_loc, h.kG, h.mP, h.sP.fft_range, fix_n=True)
    off = -h.sP.fft_range[0]
    ek, ep1 = calc_E(G[:, off:off + numax], S, mu, h.kG, h.mP)
    rhs_c1 = h.mP.n / 2 * (1 - h.mP.n / 2)
    xm_sum = sum_kw(h.kG, chi_m, lam=lam)
    xd_sum = sum_kw(h.kG, chi_d)
    lhs_c1 = (xd_sum + xm_sum) / 2
    ep2 = (h.mP.U / 2) * (xd_sum - xm_sum) + h.mP.U * (h.mP.n / 2 * h.mP.n / 2)
    return LambdaResult(lam, chi_d.lam, "m", valid, True, ek, ep1, ep2, rhs_c1, lhs_c1, G, S, mu, h.mP.n)


def gen_nu_w_indices(chi_m: ChiT, chi_d: ChiT, mP, sP, full: bool = False):
    """``gen_νω_indices`` (LambdaCorrection/helpers.jl:280-289)."""
    if sP.dbg_full_eom_omega:
        wind = np.arange(chi_m.data.shape[1])
    else:
        wind = np.array(sorted(set(chi_m.usable_w.tolist()) & set(chi_d.usable_w.tolist())))
    numax = sP.n_iv if full else min(sP.n_iv, math.floor(3 * len(wind) / 8))
    return wind, numax


def lambda_dm_residual(lam, chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, h: Helper, numax: int,
                       state: dict, tc: bool = True):
    """``residual_vals`` (conditions_new.jl:250-270) -> (n, mu, E_kin, E_pot1, E_pot2, lhs_c1, S, G)."""
    mP, kG = h.mP, h.kG
    if lam[0] > 1e5 or lam[1] > 1e5:
        return (float("nan"),) * 6 + (None, None)
    cm, cd = chi_m.copy(), chi_d.copy()
    chi_lambda_inplace(cm, float(lam[0]))
    chi_lambda_inplace(cd, float(lam[1]))
    S = calc_Sigma_inner(cm, gamma_m, cd, gamma_d, h.chiloc_m_sum, lambda0, h.grhat, kG, mP, h.sP, numax, tc)
    mu, G = G_from_Sigma_ladder(S, h.sigma_loc, kG, mP, h.sP.fft_range, fix_n=True, mu=state["mu"])
    state["mu"] = mu
    off = -h.sP.fft_range[0]
    ek, ep1 = calc_E(G[:, off:off + numax], S, mu, kG, mP)
    n = filling_pos(kG.kintegrate(G[:, off:off + numax], 0), mP.U, mu, mP.beta)
    xm_sum = sum_kw(kG, cm)
    xd_sum = sum_kw(kG, cd)
    lhs_c1 = (xd_sum + xm_sum) / 2
    ep2 = (mP.U / 2) * (xd_sum - xm_sum) + mP.U * (mP.n / 2 * mP.n / 2)
    return n, mu, ek, ep1, ep2, lhs_c1, S, G


def lambda_dm_correction(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, h: Helper,
                         numax: int = -1, lam_min_delta: float = 1e-4, validate_threshold: float = 1e-8,
                         lam_init=(0.0, 0.0), atol: float = 1e-8, nsteps: int = 500, mu0: float | None = None):
    """``λdm_correction`` (conditions_new.jl:219-324), plain (non-sc) branch -> LambdaResult.
    ``mu0``: starting μ of the μ fits (the reference's keyword μ, default mP.μ)."""
    if chi_m.lam != 0 or chi_d.lam != 0:
        raise RuntimeError("λ parameter already set. Aborting λdm calculation")
    mP = h.mP
    wind, nu_auto = gen_nu_w_indices(chi_m, chi_d, mP, h.sP)
    numax = nu_auto if numax < 1 else min(nu_auto, numax)
    rhs_c1 = mP.n / 2 * (1 - mP.n / 2)
    state = {"mu": mP.mu if mu0 is None else mu0}

    def residual_f(lam):
        r = lambda_dm_residual(lam, chi_m, gamma_m, chi_d, gamma_d, lambda0, h, numax, state)
        return np.array([r[5] - rhs_c1, r[3] - r[4]])

    lmt = get_lambda_min(chi_m.data)
    ldt = get_lambda_min(chi_d.data)
    xmin = np.array([lmt + lam_min_delta * abs(lmt), ldt + lam_min_delta * abs(ldt)])
    try:
        root = newton_right_nd(residual_f, np.array(lam_init, dtype=float), xmin, nsteps=nsteps, atol=atol)
    except RuntimeError:
        root = np.array([np.nan, np.nan])
    if np.all(np.isfinite(root)):
        n, mu, ek, ep1, ep2, lhs, S, G = lambda_dm_residual(root, chi_m, gamma_m, chi_d, gamma_d, lambda0,
                                                             h, numax, state)
        conv = abs(rhs_c1 - lhs) <= validate_threshold and abs(ep1 - ep2) <= validate_threshold
        return LambdaResult(float(root[0]), float(root[1]), "dm", True, conv, ek, ep1, ep2, rhs_c1, lhs,
                            G, S, mu, n)
    return LambdaResult(float(root[0]), float(root[1]), "dm", True, False, *(float("nan"),) * 5,
                        None, None, float("nan"), float("nan"))


def _sc_loop(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, mu: float, h: Helper, lm: float, ld: float,
             lam_types: bool, redo_dm: bool, numax: int, maxit: int, mixing: float, conv_abs: float, fit_mu: bool,
             update_chi_tail: bool):
    """The loop of ``run_sc!`` (conditions_new.jl:409-556) on deep copies of chi and G: EoM at (lm, ld)
    -> mixing -> G_from_Σladder! (μ fit) -> calc_E -> G_rfft! (the next EoM's G transform), until both
    potential energies change by less than conv_abs or maxit iterations; :dm types (redo_dm) re-solve
    λdm from the second iteration.  With update_chi_tail the finished loop is followed by the χ tail
    update (update_tail! with c2 = E_kin on both channels) and restarted (it = 1) until the sum rules
    hold to conv_abs or 20 tail updates (conditions_new.jl:519-545).  lam_types: run_sc! takes the λ of
    its first iteration from χ.λ (types :m, :dm, :pre_m, :pre_dm), which is 0 after the first pass, so
    a restarted loop begins at λ = 0 there; for :fix the given λ stays.
    Returns (λm, λd, rhs_c1, lhs_c1, E_pot_1, E_pot_2, E_kin, n, μ, converged, it, Σ, G)."""
    import dataclasses
    mP, kG, sP = h.mP, h.kG, h.sP
    off = -sP.fft_range[0]
    grhat = h.grhat
    xm, xd = chi_m.copy(), chi_d.copy()
    wgrid = xm.wn_grid()
    S = np.zeros((kG.Nq, numax), dtype=np.complex128)
    G = None
    rhs_c1 = mP.n / 2 * (1 - mP.n / 2)

    def sums(lm_, ld_):
        cm, cd = xm.copy(), xd.copy()
        chi_lambda_inplace(cm, lm_)
        chi_lambda_inplace(cd, ld_)
        a, b = sum_kw(kG, cm), sum_kw(kG, cd)
        return (b + a) / 2, (mP.U / 2) * (b - a) + mP.U * (mP.n / 2 * mP.n / 2)

    lhs_c1, E_pot_2 = sums(lm, ld)
    E_pot_1, E_kin, n = np.inf, np.inf, float("nan")
    converged = False
    it = 1
    tail_it = 1
    while True:
        while True:
            if it > 1 and redo_dm:
                hc = dataclasses.replace(h, grhat=grhat)
                r = lambda_dm_correction(xm, gamma_m, xd, gamma_d, lambda0, hc, numax=numax, lam_min_delta=1e-4,
                                         lam_init=(lm, ld), mu0=mu)
                lm, ld, mu = r.lam_m, r.lam_d, r.mu
                if not (np.isfinite(lm) and np.isfinite(ld)):
                    break
            S_work = S.copy()
            cm, cd = xm.copy(), xd.copy()
            chi_lambda_inplace(cm, lm)
            chi_lambda_inplace(cd, ld)
            S = calc_Sigma_inner(cm, gamma_m, cd, gamma_d, h.chiloc_m_sum, lambda0, grhat, kG, mP, sP, numax, True)
            if mixing != 0 and it > 1:
                S = (1 - mixing) * S + mixing * S_work
            mu, G = G_from_Sigma_ladder(S, h.sigma_loc, kG, mP, sP.fft_range, fix_n=fit_mu, mu=mu)
            if np.isnan(mu):
                break
            E_pot_1_old, E_pot_2_old = E_pot_1, E_pot_2
            E_kin, E_pot_1 = calc_E(G[:, off:off + numax], S, mu, kG, mP)
            n = filling_pos(kG.kintegrate(G[:, off:off + numax], 0), mP.U, mu, mP.beta)
            _, grhat = G_fft(kG, G)
            lhs_c1, E_pot_2 = sums(lm, ld)
            if abs(E_pot_1 - E_pot_1_old) < conv_abs and abs(E_pot_2 - E_pot_2_old) < conv_abs:
                converged = True
                break
            if it >= maxit:
                break
            it += 1
        if not update_chi_tail:
            break
        if not np.isfinite(E_kin):
            E_pot_1 = float("nan")
        else:
            update_tail(xm, [0, 0, E_kin], wgrid)
            update_tail(xd, [0, 0, E_kin], wgrid)
        lhs_c1, E_pot_2 = sums(lm, ld)
        if tail_it >= 20 or (abs(E_pot_1 - E_pot_2) < conv_abs and abs(lhs_c1 - rhs_c1) < conv_abs):
            break
        it = 1
        if lam_types:
            lm, ld = 0.0, 0.0
        tail_it += 1
    return lm, ld, rhs_c1, lhs_c1, E_pot_1, E_pot_2, E_kin, n, mu, converged, it, S, G


def run_sc(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, mu: float, h: Helper, type: str = "fix",
           lam_m: float = 0.0, lam_d: float = 0.0, numax: int = -1, maxit: int = 100, mixing: float = 0.2,
           conv_abs: float = 1e-8, fit_mu: bool = True, lam_min_delta: float = 1e-4,
           update_chi_tail: bool = False) -> LambdaResult:
    """``run_sc`` (conditions_new.jl:342-407) with its loop ``run_sc!`` (:409-556), tc = true.  Returns
    the reference's λ_result (its positional order: converged <- sc_converged)."""
    mP, kG, sP = h.mP, h.kG, h.sP
    wind, nu_auto = gen_nu_w_indices(chi_m, chi_d, mP, sP)
    numax = nu_auto if numax < 1 else min(nu_auto, numax)
    if type == "pre_m":
        rhs = lambda_m_rhs(h.imp_density, chi_m, chi_d, kG, mP, sP)
        lam_m, valid = lambda_m_correction(chi_m, rhs, kG, mP, sP)
        lam_d = 0.0
    elif type == "pre_dm":
        r = lambda_dm_correction(chi_m, gamma_m, chi_d, gamma_d, lambda0, h, numax=numax,
                                 lam_min_delta=lam_min_delta, validate_threshold=conv_abs)
        lam_m, lam_d, valid = r.lam_m, r.lam_d, r.sc_converged
    else:
        valid = True
    nan = float("nan")
    if not (valid and np.isfinite(lam_m) and np.isfinite(lam_d)):
        return LambdaResult(nan, nan, type, False, False, nan, nan, nan, nan, nan, None, None, nan, nan)
    if update_chi_tail and type == "fix" and (lam_m != 0 or lam_d != 0):
        # run_sc! sums the λ-corrected χ with the external λ = 0 of :fix after the tail update
        raise RuntimeError("χ already λ-corrected, but external λ provided!")
    lm, ld, rhs_c1, lhs_c1, E_pot_1, E_pot_2, E_kin, n, mu, converged, it, S, G = _sc_loop(
        chi_m, gamma_m, chi_d, gamma_d, lambda0, mu, h, lam_m, lam_d, type in ("m", "dm", "pre_m", "pre_dm"),
        type in ("dm", "pre_dm"), numax, maxit, mixing, conv_abs, fit_mu, update_chi_tail)
    if type == "fix":
        lm, ld = 0.0, 0.0      # run_sc! returns its loop-local λ, never set for :fix
    conv = (converged and np.isfinite(lhs_c1) and np.isfinite(E_pot_2) and abs(rhs_c1 - lhs_c1) <= conv_abs
            and abs(E_pot_1 - E_pot_2) <= conv_abs)
    res = LambdaResult(float(lm), float(ld), type, converged, conv, float(E_kin), float(E_pot_1), float(E_pot_2),
                       rhs_c1, float(lhs_c1), G, S, float(mu), float(n))
    res.iterations = it
    return res


def lambda_dm_sc_correction(chi_m: ChiT, gamma_m, chi_d: ChiT, gamma_d, lambda0, h: Helper, sc_max_it: int,
                            sc_mixing: float = 0.2, sc_conv: float = 1e-8, numax: int = -1,
                            lam_min_delta: float = 1e-4, validate_threshold: float = 1e-8, atol: float = 1e-8,
                            nsteps: int = 500) -> LambdaResult:
    """``λdm_correction`` with sc_max_it > 0 (conditions_new.jl:272-283, 290-324): every residual is the
    self-consistent loop ``run_sc!`` at fixed (λm, λd), from the handle's G and μ = mP.μ, with at most
    sc_max_it iterations; the root of [PP_2 - n/2(1 - n/2), E_pot,1 - E_pot,2] by the 2-D newton_right."""
    if chi_m.lam != 0 or chi_d.lam != 0:
        raise RuntimeError("λ parameter already set. Aborting λdm calculation")
    mP = h.mP
    wind, nu_auto = gen_nu_w_indices(chi_m, chi_d, mP, h.sP)
    numax = nu_auto if numax < 1 else min(nu_auto, numax)
    rhs_c1 = mP.n / 2 * (1 - mP.n / 2)

    def vals(lam):
        return _sc_loop(chi_m, gamma_m, chi_d, gamma_d, lambda0, mP.mu, h, float(lam[0]), float(lam[1]), False,
                        False, numax, sc_max_it, sc_mixing, sc_conv, True, False)

    def residual_f(lam):
        r = vals(lam)
        return np.array([r[3] - rhs_c1, r[4] - r[5]])

    lmt = get_lambda_min(chi_m.data)
    ldt = get_lambda_min(chi_d.data)
    xmin = np.array([lmt + lam_min_delta * abs(lmt), ldt + lam_min_delta * abs(ldt)])
    try:
        root = newton_right_nd(residual_f, np.array([0.0, 0.0]), xmin, nsteps=nsteps, atol=atol)
    except RuntimeError:
        root = np.array([np.nan, np.nan])
    nan = float("nan")
    if not np.all(np.isfinite(root)):
        return LambdaResult(float(root[0]), float(root[1]), "dm_sc", True, False, nan, nan, nan, nan, nan, None,
                            None, nan, nan)
    lm, ld, rhs_c1, lhs_c1, ep1, ep2, ek, n, mu, sc_conv_, it, S, G = vals(root)
    conv = abs(rhs_c1 - lhs_c1) <= validate_threshold and abs(ep1 - ep2) <= validate_threshold
    return LambdaResult(float(root[0]), float(root[1]), "dm_sc", True, conv, ek, ep1, ep2, rhs_c1, lhs_c1, G, S,
                        mu, n)


# =============================================================================================
# whole chain (scripts/run_minimal.jl:7-14)
# =============================================================================================
def run_chain(inp, lambda_type: str = "m", w_subset=None):
    """setup -> bubble -> chi,gamma (m, d) -> lambda_0 -> lambda correction."""
    h = setup_ldga(inp)
    chi0 = calc_bubble(h.ghat, h.grhat, h.kG, h.mP, h.sP)
    xm, gm = calc_chi_gamma("m", h.Gamma_m, chi0, h.mP, h.sP)
    xd, gd = calc_chi_gamma("d", h.Gamma_d, chi0, h.mP, h.sP)
    chi_m = ChiT(xm, h.mP.beta, tail_c=[0, 0, h.mP.Ekin_DMFT])
    chi_d = ChiT(xd, h.mP.beta, tail_c=[0, 0, h.mP.Ekin_DMFT])
    l0 = calc_lambda0(chi0, F_m_of(h), h.mP, h.sP)
    if lambda_type == "m":
        res = lambda_m_correction_full(chi_m, gm, chi_d, gd, l0, h)
    elif lambda_type == "dm":
        res = lambda_dm_correction(chi_m, gm, chi_d, gd, l0, h)
    else:
        res = None
    return dict(h=h, chi0=chi0, chi_m=chi_m, gamma_m=gm, chi_d=chi_d, gamma_d=gd, lambda0=l0, result=res)
