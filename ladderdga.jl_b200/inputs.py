"""Impurity (DMFT) inputs: ``readConfig`` (IO.jl:29-128), the file-reading part of ``setup_LDGA``
(runHelpers.jl:87-112) and ``calc_E_ED`` (thermodynamics.jl:37-64).

The reference reads a TOML configuration and a JLD2 file of DMFT impurity data (vertices Γ_r,
generalized susceptibilities χ_r, G_imp, the bath G_0 or Σ_loc, the Anderson parameters ϵₖ, Vₖ and
the scalars U, μ, β, n, the DMFT energies and the frequency box).  Here the JLD2 file is read by
``jld2.py``; an ``.npz`` archive with the same keys is accepted as well, so that the inputs can
travel where the original file does not.

``load_impurity_input`` turns the file into the object ``core.setup_LDGA`` consumes: the same
fields as a ``synthetic.SyntheticInput`` (the lattice, the model scalars, Σ_loc(n) and G_imp(n) for
n >= 0, and χ_r, Γ_r as [Nν, Nν, Nω] complex arrays in the reference's axis order after
``permutedims(·, (2, 3, 1))`` and the sign flip of Γ).
"""
from __future__ import annotations

import math
import os
import sys
import tomllib
from dataclasses import dataclass

import numpy as np

from . import jld2
from .synthetic import SyntheticInput


@dataclass
class EnvironmentVars:
    """``EnvironmentVars`` (Config.jl:80-101)."""
    inputDir: str
    inputVars: str
    loglevel: str
    logfile: str


@dataclass
class BSEAsymptoticsHelper:
    """Stands for the reference's ``BSE_Asym_Helper`` / ``BSE_SC_Helper`` /
    ``BSE_Asym_Helper_Approx2`` (IO.jl:95-108), which come from BSE_SC.jl.  The asymptotic
    improvement is not part of the plain ladder path built here: ``setup_LDGA`` rejects a
    configuration that selects one.  The object keeps what the reference would have passed."""
    method: str
    n_iν_shell: int
    χsp_asympt: np.ndarray | None = None
    χch_asympt: np.ndarray | None = None
    χpp_asympt: np.ndarray | None = None


class ImpurityInput(SyntheticInput):
    """The DMFT impurity data of one parameter point, in the layout ``setup_LDGA`` consumes."""


def open_input(path):
    """A read-only mapping over an impurity file: ``.jld2`` (HDF5) or ``.npz`` with the same keys."""
    if str(path).endswith(".npz"):
        z = np.load(path, allow_pickle=False)
        return {k: (z[k].item() if z[k].ndim == 0 else np.asfortranarray(z[k])) for k in z.files}
    return jld2.jldopen(path, "r")


def _has(f, key: str) -> bool:
    return key in f


def readConfig(cfg_in: str):
    """``readConfig`` (IO.jl:29-128): ``(workerpool, mP, sP, env, kGrids)`` from a TOML file or a
    TOML string.  ``workerpool`` is None (one GPU holds a whole parameter point).  The model
    scalars, the frequency box and the χ asymptotics come from the impurity file named by
    ``[Environment] inputVars``; a missing file ends the program with status 2, as the reference
    does (``Base.exit(2)``)."""
    from .core import ModelParameters, SimulationParameters
    try:
        is_file = os.path.isfile(cfg_in)
    except (TypeError, ValueError):
        is_file = False
    if is_file:
        with open(cfg_in, "rb") as fh:
            tml = tomllib.load(fh)
    else:
        tml = tomllib.loads(cfg_in)
    sim = tml["Simulation"]
    smoothing = sim["omega_smoothing"].lower()
    if smoothing not in ("nothing", "range", "full"):
        raise RuntimeError(f'Unrecognized smoothing type "{smoothing}"')
    dbg = tml.get("Debug", {})
    dbg_full_eom_omega = bool(dbg.get("full_EoM_omega", False))

    envt = tml["Environment"]
    if os.path.isabs(envt["inputDir"]):
        input_dir = envt["inputDir"]
    else:
        base = os.path.dirname(cfg_in) if is_file else os.getcwd()
        input_dir = os.path.abspath(os.path.join(base, envt["inputDir"]))
    loglevel = envt["loglevel"]
    env = EnvironmentVars(input_dir, os.path.join(input_dir, envt["inputVars"]),
                          loglevel[:1].upper() + loglevel[1:].lower(), envt["logfile"].lower())
    if not os.path.isfile(env.inputVars):
        print(f"ERROR: input file at location {env.inputVars} not found!", file=sys.stderr)
        raise SystemExit(2)

    f = open_input(env.inputVars)
    if _has(f, "E_kin_DMFT"):
        EPot_DMFT, EKin_DMFT = float(f["E_pot_DMFT"]), float(f["E_kin_DMFT"])
    else:
        print("Warning: Could not find E_kin_DMFT, E_pot_DMFT key in input", file=sys.stderr)
        EPot_DMFT = EKin_DMFT = 0.0
    if _has(f, "U"):
        U, μ, β, nden = (float(f[k]) for k in ("U", "μ", "β", "nden"))
    else:
        print("Warning: Reading Hubbard Parameters from config. These should be supplied through the "
              "input jld2!", file=sys.stderr)
        m = tml["Model"]
        U, μ, β, nden = float(m["U"]), float(m["mu"]), float(m["beta"]), float(m["nden"])
    Vk = np.asarray(f["Vₖ"], dtype=np.float64)
    mP = ModelParameters(U, μ, β, nden, float(np.sum(Vk ** 2)), EPot_DMFT, EKin_DMFT)
    nBose, nFermi = int(f["grid_nBose"]), int(f["grid_nFermi"])
    shift = bool(f["grid_shift"])

    method = sim["chi_asympt_method"].lower()
    asympt_sc = 1 if method == "asympt" else 0
    Nν_shell = int(sim["chi_asympt_shell"])
    Nν_full = nFermi + asympt_sc * Nν_shell
    freq_r = 2 * (Nν_full + nBose)
    fft_range = range(-freq_r, freq_r + 1)
    if method in ("asympt", "direct", "direct_approx2"):
        def asym(key):
            return np.asarray(f[key]) / β ** 2 if _has(f, key) else None
        χ_helper = BSEAsymptoticsHelper(method, Nν_shell, asym("χ_sp_asympt"), asym("χ_ch_asympt"),
                                        asym("χ_pp_asympt"))
    elif method == "nothing":
        χ_helper = None
    else:
        print(f"Error: could not parse chi_asympt_method {sim['chi_asympt_method']}. "
              "Options are: asympt/direct/nothing", file=sys.stderr)
        χ_helper = None
    sP = SimulationParameters(nBose, nFermi, Nν_shell, shift, χ_helper, fft_range,
                              float(sim["usable_prct_reduction"]), dbg_full_eom_omega)
    Nk = sim["Nk"]
    if isinstance(Nk, str) and Nk.strip().lower() == "conv":
        kGrids = [(tml["Model"]["kGrid"], 0)]
    else:
        kGrids = [(tml["Model"]["kGrid"], int(n)) for n in Nk]
    return None, mP, sP, env, kGrids


def _permute(a, shape) -> np.ndarray:
    """``permutedims(a, (2, 3, 1))`` into a zero array of the box's shape (runHelpers.jl:91-98)."""
    a = np.asarray(a, dtype=np.complex128)
    p = np.transpose(a, (1, 2, 0))
    if p.shape != shape:
        raise ValueError(f"DimensionMismatch: impurity array of shape {p.shape} for a box of {shape}")
    return np.asfortranarray(p)


def load_impurity_input(source, kGridStr, mP, sP) -> ImpurityInput:
    """The ``jldopen(env.inputVars)`` block of ``setup_LDGA`` (runHelpers.jl:87-112) for the plain
    path (no ν shell): χ_m = χDMFTsp, χ_d = χDMFTch, Γ_m = −Γsp, Γ_d = −Γch, each permuted to
    [ν, ν′, ω]; Σ_loc = Σ_Dyson(g0, gImp) when the file has ``g0``, else ``SigmaLoc``.
    ``source``: a path (``.jld2`` / ``.npz``) or an open mapping."""
    from .core import Σ_Dyson
    f = open_input(source) if isinstance(source, (str, os.PathLike)) else source
    shape = (2 * sP.n_iν, 2 * sP.n_iν, 2 * sP.n_iω + 1)
    χm, χd = _permute(f["χDMFTsp"], shape), _permute(f["χDMFTch"], shape)
    Γm, Γd = -_permute(f["Γsp"], shape), -_permute(f["Γch"], shape)
    gimp = np.asarray(f["gImp"], dtype=np.complex128)
    if _has(f, "g0"):
        Σ_loc = Σ_Dyson(np.asarray(f["g0"], dtype=np.complex128), gimp)
    else:
        Σ_loc = np.asarray(f["SigmaLoc"], dtype=np.complex128)
    kind, ns = kGridStr
    head, *params = kind.split("-")
    t = float(params[0]) if params else 1.0
    return ImpurityInput(dim=int(head[0]), ns=int(ns), t=t, beta=mP.β, U=mP.U, mu=mP.μ, n=mP.n,
                         n_iw=sP.n_iω, n_iv=sP.n_iν, shift=bool(sP.shift), Ekin_DMFT=mP.Ekin_DMFT,
                         Epot_DMFT=mP.Epot_DMFT, sVk=mP.sVk, sigma_loc=Σ_loc, gimp=gimp,
                         chi_loc_m=χm, chi_loc_d=χd, gamma_m=Γm, gamma_d=Γd, seed=0,
                         tags={"source": str(source) if isinstance(source, (str, os.PathLike)) else "mapping"})


def calc_E_ED(*args):
    """``calc_E_ED`` (thermodynamics.jl:37-64): kinetic and potential energy of the Anderson
    impurity from its bath (ϵₖ, Vₖ) and G_imp, with the 1/ν² tails summed analytically.
    ``calc_E_ED(path)`` reads ϵₖ, Vₖ, gImp, U, nden, μ, β from an impurity file;
    ``calc_E_ED(ϵₖ, Vₖ, GImp, mP)`` or ``calc_E_ED(ϵₖ, Vₖ, GImp, U, n, μ, β)`` take them directly."""
    if len(args) == 1:
        f = open_input(args[0])
        return calc_E_ED(f["ϵₖ"], f["Vₖ"], f["gImp"], f["U"], f["nden"], f["μ"], f["β"])
    if len(args) == 4:
        ϵₖ, Vₖ, GImp, mP = args
        return calc_E_ED(ϵₖ, Vₖ, GImp, mP.U, mP.n, mP.μ, mP.β)
    ϵₖ, Vₖ, GImp, U, n, μ, β = args
    ϵₖ = np.asarray(ϵₖ, dtype=np.float64)
    Vₖ = np.asarray(Vₖ, dtype=np.float64)
    GImp = np.asarray(GImp, dtype=np.complex128)
    U, n, μ, β = float(U), float(n), float(μ), float(β)
    vk = float(np.sum(Vₖ ** 2))
    Σ_hartree = n * U / 2
    E_pot_tail = U ** 2 / 2 * n * (1 - n / 2) - Σ_hartree * (Σ_hartree - μ)
    E_kin_tail = vk
    E_kin = 0.0
    E_pot = 0.0
    for m in range(len(GImp)):
        iν = 1j * (2 * m + 1) * math.pi / β
        Δ = np.sum((Vₖ * np.conj(Vₖ)) / (iν - ϵₖ))
        Σ = iν - Δ - 1.0 / GImp[m] + μ
        E_kin += 2 * (GImp[m] * Δ - E_kin_tail / iν ** 2).real
        E_pot += 2 * (GImp[m] * Σ - E_pot_tail / iν ** 2).real
    E_kin = E_kin * (2 / β) - (β / 2) * E_kin_tail
    E_pot = E_pot * (1 / β) + 0.5 * Σ_hartree - (β / 4) * E_pot_tail
    return E_kin, E_pot
