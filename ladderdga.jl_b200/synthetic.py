"""Seeded synthetic DMFT inputs for the lDGA ladder path.

The reference reads a local (impurity) solution from a JLD2 file in ``setup_LDGA``
(LadderDGA.jl ``src/runHelpers.jl:89-111``): the local generalized susceptibilities
``chiDMFTsp/ch``, the local irreducible vertices ``Gamma_sp/ch``, the impurity Green's
function and the local self-energy.  No such file exists for the benchmark configurations,
so this module generates a seeded, physically shaped stand-in with the same array shapes:

* dispersion   eps_k = -2t (cos kx + cos ky [+ cos kz])              (simple cubic, N^d grid)
* self-energy  Sigma_loc(i nu) = U/2 + (U^2/4) / (i nu + 0.5 i sgn nu)  (half filling, mu = U/2)
* G_imp(nu)    = <1/(i nu + mu - eps_k - Sigma_loc(nu))>_k               (k-average on the full grid)
* chi_r,loc    = -beta G_imp(nu) G_imp(nu+w) delta_{nu nu'} + s_r C(nu,nu',w),  s_d=+1, s_m=-1,
  C a complex Gaussian scaled by U/beta^2/(1+|n-n'|), Hermitian-symmetrised in (nu,nu')
* Gamma_r      = chi_r,loc^{-1} - diag(1/chi0_loc), so that the reference's local
  Bethe-Salpeter step (``calc_chi_gamma`` on the one-point grid) reproduces chi_r,loc.

Random numbers: SplitMix64 -> Box-Muller, seed = 1000*config + point index.  The stream is
pure integer arithmetic, so every consumer (host library, tests, CPU baseline) that calls
this module sees bit-identical inputs.

Array conventions follow the reference (Julia, column-major, first index fastest): a
``[Nnu, Nnu, Nw]`` Julia array is returned as a numpy array of that shape in Fortran order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """First ``n`` outputs of the SplitMix64 generator started at ``seed`` (uint64 array)."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int) -> np.ndarray:
    """``n`` doubles in the open interval (0, 1) from the top 53 bits of SplitMix64."""
    z = splitmix64(seed, n) >> np.uint64(11)
    return (z.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def complex_gaussian(seed: int, n: int) -> np.ndarray:
    """``n`` complex normals (unit variance per component) by Box-Muller on SplitMix64."""
    u = uniform01(seed, 2 * n)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    th = 2.0 * math.pi * u2
    return r * np.cos(th) + 1j * (r * np.sin(th))


def dispersion_full(dim: int, ns: int, t: float = 1.0, tp: float = 0.0, tpp: float = 0.0) -> np.ndarray:
    """eps_k on the full ``ns^dim`` grid, k_i = 2 pi n_i / ns (array shape (ns,)*dim, index [nx,ny(,nz)])."""
    k = 2.0 * math.pi * np.arange(ns) / ns
    c = np.cos(k)
    if dim == 2:
        cx, cy = c[:, None], c[None, :]
        c2 = np.cos(2.0 * k)
        return (-2.0 * t * (cx + cy) - 4.0 * tp * cx * cy
                - 2.0 * tpp * (c2[:, None] + c2[None, :]))
    if dim == 3:
        if tp != 0.0 or tpp != 0.0:
            raise ValueError("3D simple cubic supports nearest-neighbour hopping only")
        return -2.0 * t * (c[:, None, None] + c[None, :, None] + c[None, None, :])
    raise ValueError(f"unsupported lattice dimension {dim}")


@dataclass
class SyntheticInput:
    """Everything ``setup_LDGA`` would read from the impurity file, plus model/simulation scalars."""
    dim: int
    ns: int
    t: float
    beta: float
    U: float
    mu: float
    n: float
    n_iw: int
    n_iv: int
    shift: bool
    Ekin_DMFT: float
    Epot_DMFT: float
    sVk: float
    sigma_loc: np.ndarray          # Sigma_loc(n) for n = 0..len-1 (positive Matsubara indices)
    gimp: np.ndarray               # G_imp(n) for n = 0..rm-1
    chi_loc_m: np.ndarray          # [Nnu, Nnu, Nw] complex, Fortran order
    chi_loc_d: np.ndarray
    gamma_m: np.ndarray            # Gamma_m [Nnu, Nnu, Nw]
    gamma_d: np.ndarray
    seed: int = 0
    tags: dict = field(default_factory=dict)

    @property
    def fft_range(self) -> range:
        L = 2 * (self.n_iv + self.n_iw)
        return range(-L, L + 1)

    @property
    def kgrid_kind(self) -> str:
        return f"{self.dim}Dsc-{self.t}"


def _freq(w_i: int, v_i: int, n_iw: int, n_iv: int, shift: bool):
    """0-based index pair -> Matsubara integers (reference ``OneToIndex_to_Freq``, helpers.jl:46-50)."""
    wn = w_i - n_iw
    vn = (v_i - n_iv) - (int(shift) * int(wn / 2))
    return wn, vn


def make_input(dim: int, ns: int, beta: float, U: float, n_iv: int, n_iw: int, seed: int,
               t: float = 1.0, shift: bool = False, C_add=None) -> SyntheticInput:
    """Build the seeded local inputs for one parameter point.

    C_add ([Nnu, Nnu, Nw] complex, optional) is added to the symmetrised vertex noise C before the
    local susceptibilities and vertices are formed (a perturbation for gradient checks with respect to
    C); the C used is returned in ``tags["C"]``."""
    mu = U / 2.0
    nden = 1.0
    L = 2 * (n_iv + n_iw)
    rm = L
    nsig = 2 * L + 2
    nvals = np.arange(nsig)
    iv = 1j * (2 * nvals + 1) * math.pi / beta
    sigma_loc = U / 2.0 + (U * U / 4.0) / (iv + 0.5j)

    eps = dispersion_full(dim, ns, t).reshape(-1)
    # G_imp(n) = <G(k, n)>_k over the full grid, n = 0..rm-1
    gimp = np.empty(rm, dtype=np.complex128)
    for nn in range(rm):
        gimp[nn] = np.mean(1.0 / (iv[nn] + mu - eps - sigma_loc[nn]))

    def g_of(nn: int) -> complex:
        return gimp[nn] if nn >= 0 else np.conj(gimp[-nn - 1])

    nnu, nw = 2 * n_iv, 2 * n_iw + 1
    chi0_loc = np.empty((nnu, nw), dtype=np.complex128)
    vn_tab = np.empty((nnu, nw), dtype=np.int64)
    for wi in range(nw):
        for vi in range(nnu):
            wn, vn = _freq(wi, vi, n_iw, n_iv, shift)
            vn_tab[vi, wi] = vn
            chi0_loc[vi, wi] = -beta * g_of(vn) * g_of(vn + wn)

    g = complex_gaussian(seed, nnu * nnu * nw).reshape((nnu, nnu, nw), order="F")
    dv = np.abs(vn_tab[:, None, :] - vn_tab[None, :, :]).astype(np.float64)
    C = g * (U / beta**2) / (1.0 + dv)
    C = 0.5 * (C + np.conj(np.transpose(C, (1, 0, 2))))
    if C_add is not None:
        C = C + np.asarray(C_add, dtype=np.complex128).reshape(C.shape, order="F")

    chi_m = np.zeros((nnu, nnu, nw), dtype=np.complex128, order="F")
    chi_d = np.zeros((nnu, nnu, nw), dtype=np.complex128, order="F")
    gam_m = np.zeros((nnu, nnu, nw), dtype=np.complex128, order="F")
    gam_d = np.zeros((nnu, nnu, nw), dtype=np.complex128, order="F")
    for wi in range(nw):
        d0 = np.diag(chi0_loc[:, wi])
        chi_d[:, :, wi] = d0 + C[:, :, wi]
        chi_m[:, :, wi] = d0 - C[:, :, wi]
        inv_d0 = np.diag(1.0 / chi0_loc[:, wi])
        gam_d[:, :, wi] = np.linalg.inv(chi_d[:, :, wi]) - inv_d0
        gam_m[:, :, wi] = np.linalg.inv(chi_m[:, :, wi]) - inv_d0

    # DMFT kinetic energy (the chi tail coefficient c2): the kinetic part of the reference's
    # calc_E (thermodynamics.jl:142-168) for G(k, nu) = 1/(i nu + mu - eps_k - Sigma_loc(nu)),
    # nu_n = 0..L-1, evaluated on the full grid.
    sig_h = nden * U / 2.0
    Ekin = 0.0
    acc = np.zeros_like(eps)
    tail_c = eps + sig_h - mu
    for nn in range(L):
        Gk = 1.0 / (iv[nn] + mu - eps - sigma_loc[nn])
        acc += eps * np.real(Gk - tail_c / (iv[nn] ** 2))
    tail_inv = (beta / 2.0) * eps * (1.0 - beta * tail_c)
    Ekin = float(np.mean(4.0 * acc + tail_inv) / beta)
    sVk = float(np.mean(eps * eps))

    return SyntheticInput(dim=dim, ns=ns, t=t, beta=beta, U=U, mu=mu, n=nden, n_iw=n_iw,
                          n_iv=n_iv, shift=shift, Ekin_DMFT=Ekin, Epot_DMFT=0.0, sVk=sVk,
                          sigma_loc=sigma_loc, gimp=gimp, chi_loc_m=chi_m, chi_loc_d=chi_d,
                          gamma_m=gam_m, gamma_d=gam_d, seed=seed, tags={"C": C})


# The five benchmark configurations (lattice, temperature, coupling, frequency box).
CONFIGS = {
    1: dict(dim=2, ns=16, beta=10.0, U=1.0, n_iv=10, n_iw=10),
    2: dict(dim=2, ns=64, beta=30.0, U=2.0, n_iv=30, n_iw=30),
    3: dict(dim=3, ns=32, beta=20.0, U=1.5, n_iv=20, n_iw=20),
    4: dict(dim=2, ns=48, beta=20.0, U=1.5, n_iv=20, n_iw=20),
}


def config_input(cfg: int, point: int = 0, **override) -> SyntheticInput:
    """Seeded inputs of benchmark configuration ``cfg`` (seed = 1000*cfg + point)."""
    kw = dict(CONFIGS[cfg])
    kw.update(override)
    return make_input(seed=1000 * cfg + point, **kw)


def batch_points(n_points: int = 64, ns: int = 32, cfg: int = 5):
    """Uneven batch: U ~ U[0.5, 3], beta in {5,10,20,40}, Nnu = 2 round(1.5 beta) (half-even)."""
    u = uniform01(1000 * cfg, n_points)
    out = []
    betas = (5.0, 10.0, 20.0, 40.0)
    for p in range(n_points):
        U = 0.5 + 2.5 * float(u[p])
        beta = betas[p % 4]
        n_iv = int(round(1.5 * beta))       # Python round is half-even: 7.5 -> 8
        out.append(dict(dim=2, ns=ns, beta=beta, U=U, n_iv=n_iv, n_iw=n_iv, seed=1000 * cfg + p))
    return out
