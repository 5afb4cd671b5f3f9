"""Host-side mirror of LadderDGA.jl's ladder API on top of the CUDA library.

Names, argument meaning and error behaviour follow the reference (``src/LadderDGA.jl:6-38`` exports):
``setup_LDGA``, ``calc_bubble``, ``calc_χγ``, ``calc_λ0``, ``calc_Σ``, ``calc_Σ_parts``, ``sum_kω``,
``sum_ω``, ``sum_ωk``, ``χ_λ``/``χ_λ!``/``reset!``, ``λm_correction``, ``λdm_correction``,
``λ_correction``, ``G_from_Σladder``, ``calc_E``, ``filling_pos``, ...  Julia's mutating ``f!`` is
spelled ``f_`` here (``χ_λ_``, ``reset_``); every name also has an ASCII alias.

Arrays keep the reference's index order and memory layout: ``χ0.data[q, ν, ω]``,
``χ.data[q, ω]``, ``γ.data[q, ν, ω]``, ``Σ_ladder[q, ν_n]`` (ν_n = 0..νmax-1), as numpy arrays in
Fortran order (first index fastest, the Julia layout the C ABI expects).

Where work happens: every ladder-chain operation on objects produced by this module (bubble, BSE,
λ0, EoM, the λ sums and root finders, μ fit, energies) runs on the GPU through libldga_b200; the
arrays stay in device memory and are copied to the host only when ``.data`` is read.  Objects a
user builds directly from host arrays (``χT(data, β)`` without a device binding) use the host
implementation of the reference's Matsubara-sum data type, as in DataTypes.jl.
"""
from __future__ import annotations

import math
import warnings
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import _lib
from ._lib import (CH_D, CH_M, PREC_FP64, PREC_FP64_INV, PREC_MIXED, SC_LAMBDA_TYPE, SC_REDO_DM,
                   SC_UPDATE_CHI_TAIL, Context, LdgaError, as_fc, ptr)

_CH = {"m": CH_M, "d": CH_D, ":m": CH_M, ":d": CH_D}


def _channel(type_) -> int:
    key = str(type_).lstrip(":")
    if key not in ("m", "d"):
        raise ValueError("Unkown type")
    return _CH[key]


# =============================================================================================
# parameter structs (Config.jl:39-75)
# =============================================================================================
@dataclass
class ModelParameters:
    """``ModelParameters`` (Config.jl:39-47)."""
    U: float
    μ: float
    β: float
    n: float
    sVk: float = 0.0
    Epot_DMFT: float = 0.0
    Ekin_DMFT: float = 0.0

    @property
    def mu(self) -> float:
        return self.μ

    @property
    def beta(self) -> float:
        return self.β


@dataclass
class SimulationParameters:
    """``SimulationParameters`` (Config.jl:66-75)."""
    n_iω: int
    n_iν: int
    n_iν_shell: int
    shift: bool
    χ_helper: object
    fft_range: range
    usable_prct_reduction: float = 0.0
    dbg_full_eom_omega: bool = False

    @property
    def n_iw(self) -> int:
        return self.n_iω

    @property
    def n_iv(self) -> int:
        return self.n_iν

    @property
    def n_iv_shell(self) -> int:
        return self.n_iν_shell


# =============================================================================================
# k-grid (Dispersions.jl gen_kGrid contract)
# =============================================================================================
class KGrid:
    """Point-group-reduced simple-cubic grid: ``kMult``, ``ϵkGrid``, ``Nk``, ``Ns``, ``kintegrate``.

    The wedge (q_x >= q_y [>= q_z] >= 0, q_i <= N/2, lexicographic, q = 0 first) is the same one the
    GPU library uses; ``kGrid`` holds the wedge k-vectors.
    """

    def __init__(self, kind: str, ns: int):
        head, *params = kind.split("-")
        dim = int(head[0])
        if head[1:].lower() != "dsc":
            raise ValueError(f"only simple cubic grids are built, got {kind!r}")
        vals = [float(p) for p in params] + [0.0, 0.0, 0.0]
        self.kind, self.dim, self.Ns = kind, dim, ns
        self.t, self.tp, self.tpp = vals[0], vals[1], vals[2]
        M = ns // 2 + 1
        if dim == 2:
            w = [(a, b) for a in range(M) for b in range(a + 1)]
        elif dim == 3:
            w = [(a, b, c) for a in range(M) for b in range(a + 1) for c in range(b + 1)]
        else:
            raise ValueError("dimension must be 2 or 3")
        self.wedge = np.array(w, dtype=np.int64).reshape(-1, dim)
        fold = np.minimum(np.arange(ns), (ns - np.arange(ns)) % ns)
        mult = {}
        for idx in np.ndindex(*((ns,) * dim)):
            key = tuple(sorted((int(fold[i]) for i in idx), reverse=True))
            mult[key] = mult.get(key, 0) + 1
        self.kMult = np.array([mult[tuple(x)] for x in w], dtype=np.float64)
        k = 2.0 * math.pi * self.wedge / ns
        if dim == 2:
            self.ϵkGrid = (-2.0 * self.t * (np.cos(k[:, 0]) + np.cos(k[:, 1]))
                           - 4.0 * self.tp * np.cos(k[:, 0]) * np.cos(k[:, 1])
                           - 2.0 * self.tpp * (np.cos(2 * k[:, 0]) + np.cos(2 * k[:, 1])))
        else:
            self.ϵkGrid = -2.0 * self.t * np.cos(k).sum(axis=1)
        self.kGrid = k
        self.Nk = ns ** dim

    @property
    def eps(self) -> np.ndarray:
        return self.ϵkGrid

    def full_to_irr(self) -> np.ndarray:
        """Wedge index of every point of the full grid (``expandKArr``'s map), shape gridshape."""
        if getattr(self, "_f2i", None) is None:
            widx = {tuple(int(v) for v in w): i for i, w in enumerate(self.wedge)}
            ns = self.Ns
            fold = np.minimum(np.arange(ns), (ns - np.arange(ns)) % ns)
            out = np.empty((ns,) * self.dim, dtype=np.int64)
            for idx in np.ndindex(*out.shape):
                out[idx] = widx[tuple(sorted((int(fold[i]) for i in idx), reverse=True))]
            self._f2i = out
        return self._f2i

    def gridshape(self):
        return (self.Ns,) * self.dim

    def kintegrate(self, arr, axis: int = 0):
        a = np.moveaxis(np.asarray(arr), axis, 0)
        return np.tensordot(self.kMult, a, axes=(0, 0)) / self.Nk


def gen_kGrid(kind: str, ns: int) -> KGrid:
    """``gen_kGrid`` (Dispersions.jl): ``"2Dsc-t"``, ``"3Dsc-t"``, ``"2Dsc-t-tp-tpp"``."""
    return KGrid(kind, ns)


def kintegrate(kG: KGrid, arr, axis: int = 0):
    return kG.kintegrate(arr, axis)


def q0_index(kG: KGrid) -> int:
    """``q0_index`` (helpers.jl:27), 0-based."""
    return int(np.flatnonzero(np.all(kG.wedge == 0, axis=1))[0])


# =============================================================================================
# frequency helpers (helpers.jl:20-67, GFTools.jl:31-47)
# =============================================================================================
def νnGrid(ωn: int, sP: SimulationParameters) -> np.ndarray:
    return np.arange(-sP.n_iν - sP.n_iν_shell, sP.n_iν + sP.n_iν_shell) - int(sP.shift) * int(ωn / 2)


def OneToIndex_to_Freq(ωi: int, νi: int, sP: SimulationParameters):
    """1-based index pair -> Matsubara integers (helpers.jl:46-50)."""
    ωn = ωi - sP.n_iω - 1
    νn = (νi - sP.n_iν - 1) - int(sP.shift) * int(ωn / 2)
    return ωn, νn


def ν0Index_of_ωIndex(ωi: int, sP: SimulationParameters) -> int:
    """1-based index of ν_n = 0 at bosonic index ``ωi`` (helpers.jl:58)."""
    return sP.n_iν + int(sP.shift) * int((ωi - sP.n_iω - 1) / 2) + 1


def ω0_index(x) -> int:
    """1-based index of ω = 0 (helpers.jl:35-37)."""
    if isinstance(x, SimulationParameters):
        return x.n_iω + 1
    data = x.data if isinstance(x, χT) else np.asarray(x)
    return math.ceil(data.shape[1] / 2)


def iν_array(β: float, grid) -> np.ndarray:
    if isinstance(grid, int):
        grid = range(grid)
    return np.array([1j * ((2.0 * el + 1) * math.pi / β) for el in grid], dtype=np.complex128)


def iω_array(β: float, grid) -> np.ndarray:
    if isinstance(grid, int):
        grid = range(grid)
    return np.array([1j * ((2.0 * el) * math.pi / β) for el in grid], dtype=np.complex128)


def reduce_range(rng: range, red_prct: float) -> range:
    """``reduce_range`` (helpers.jl:141-146) on 1-based Julia ranges given as Python ranges."""
    first, last, length = rng[0], rng[-1], len(rng)
    sub = math.floor(length / 2 * red_prct)
    lst = max(last - sub, math.ceil(length / 2 + (length % 2 == 0)))
    fst = min(first + sub, math.ceil(length / 2))
    return range(fst, lst + 1)


# =============================================================================================
# device-backed arrays and the Matsubara data types (DataTypes.jl)
# =============================================================================================
class DeviceArray:
    """A reference-layout array held in the GPU handle; ``np.asarray`` / ``.data`` copy it to the host."""

    def __init__(self, ctx: Context, fetch: Callable[[], np.ndarray], shape, dtype=np.complex128):
        self._ctx, self._fetch, self.shape, self.dtype = ctx, fetch, tuple(shape), dtype
        self._host = None

    @property
    def data(self) -> np.ndarray:
        if self._host is None:
            self._host = self._fetch()
        return self._host

    def __array__(self, dtype=None, copy=None):
        a = self.data
        return a.astype(dtype) if dtype is not None else a

    def __getitem__(self, idx):
        return self.data[idx]

    def __len__(self):
        return self.shape[0]


class χ0T:
    """``χ0T`` (DataTypes.jl:52-69): bubble with axes (q, ν, ω).  ``asym`` is not built (plain path)."""

    def __init__(self, data, β: float, ωnGrid, n_iν: int, shift: bool, ν_shell_size: int = 0, ctx=None):
        ωs = list(ωnGrid)
        if len(ωs) == 0 or ωs[-1] < ωs[0]:
            raise ValueError("Cannot construct χ₀ array with empty frequency mesh!")   # DataTypes.jl:92-94
        self._dev = data if isinstance(data, DeviceArray) else None
        self._data = None if self._dev is not None else as_fc(data)
        self.β = β
        self.axis_types = {"q": 0, "ν": 1, "ω": 2}
        νg = np.arange(-n_iν, n_iν)
        self.indices_νω = [[(int(j - int(shift * i / 2)), int(i)) for i in ωnGrid] for j in νg]
        self.ν_shell_size = ν_shell_size
        self._ctx = ctx
        self.asym = None

    @property
    def data(self) -> np.ndarray:
        return self._dev.data if self._dev is not None else self._data

    @property
    def shape(self):
        return self._dev.shape if self._dev is not None else self._data.shape

    def size(self, axis=None):
        return self.shape if axis is None else self.shape[axis]

    def __getitem__(self, idx):
        return self.data[idx]


def χ0Asym_coeffs(kG: KGrid, local_tail: bool, mP: ModelParameters):
    """``χ₀Asym_coeffs`` (DataTypes.jl:110-124): tail coefficients (c1, c2[q], c3) of the bubble's
    asymptotics.  Local: c1 = Un/2 − μ, c2 = [c1²], c3 = c1² + sVk + U² n/2 (1 − n/2).  Lattice, with
    t1(k) = ε_k + Un/2 − μ: c1 = ⟨t1⟩_k, c2(q) = (1/N_k) Σ_k t1(k) t1(k+q), c3 = ⟨t1²⟩_k + U² n/2 (1 − n/2).
    The asymptotic array itself (χ₀Asym) needs BSE_SC.jl's shell sums and is not built."""
    t2 = mP.U ** 2 * (mP.n / 2) * (1 - mP.n / 2)
    if local_tail:
        c1 = mP.U * mP.n / 2 - mP.μ
        return c1, [c1 * c1], c1 * c1 + mP.sVk + t2
    t1 = np.asarray(kG.ϵkGrid, dtype=np.float64) + mP.U * mP.n / 2 - mP.μ
    full = t1[kG.full_to_irr()]
    F = np.fft.fftn(full)
    corr = np.fft.ifftn(np.conj(F) * F).real / kG.Nk
    c2 = corr[tuple(kG.wedge[:, d] for d in range(kG.dim))]
    return float(kintegrate(kG, t1)), c2, float(kintegrate(kG, t1 ** 2)) + t2


def core(χ0: χ0T) -> np.ndarray:
    """``core`` (DataTypes.jl:77-79)."""
    s = χ0.ν_shell_size
    return χ0.data[:, s:χ0.data.shape[1] - s, :]


class χT:
    """``χT`` (DataTypes.jl:177-194): physical susceptibility [q, ω] with c₂ tail and λ.

    A χT returned by ``calc_χγ`` is bound to its GPU handle and channel; the device keeps the
    λ = 0 data and applies χ_λ on the fly, so ``χ_λ_``/``reset_`` cost no device work and cannot
    drift.  The host ``data`` follows the reference's in-place semantics.
    """

    def __init__(self, data, β: float, indices_ω=None, tail_c=(), full_range: bool = True,
                 reduce_range_prct: float = 0.0):
        self._data = np.array(np.asarray(data, dtype=np.float64), order="F", copy=True)
        self.β = float(β)
        nw = self._data.shape[1]
        self.indices_ω = (np.arange(nw) + 1 - math.ceil(nw / 2)) if indices_ω is None else np.asarray(indices_ω)
        self.tail_c = [float(x) for x in tail_c]
        self.λ = 0.0
        self.axis_types = {"q": 0, "ω": 1}
        if full_range:
            self.usable_ω = np.arange(nw)
        else:
            self.usable_ω = find_usable_χ_interval(self._data, reduce_range_prct=reduce_range_prct) - 1
        self._ctx = None
        self._ch = None
        self._dev_λ = 0.0        # λ of the device copy
        self._dirty = False      # host data edited through __setitem__

    # -- binding to a GPU handle
    def _bind(self, ctx: Context, ch: int) -> "χT":
        self._ctx, self._ch, self._dev_λ, self._dirty = ctx, ch, 0.0, False
        return self

    def _device_λ(self, extra: float = 0.0) -> float:
        """λ to hand to the kernels so that they see χ_λ(data_pristine, self.λ + extra)."""
        if self._ctx is None:
            raise RuntimeError("χT is not bound to a GPU handle")
        if self._dirty:
            self._ctx.call("ldga_set_chi", self._ch, ptr(self._data))
            self._dev_λ = self.λ
            self._dirty = False
        return self.λ + extra - self._dev_λ

    @property
    def data(self) -> np.ndarray:
        v = self._data.view()
        v.flags.writeable = False
        return v

    @property
    def shape(self):
        return self._data.shape

    def size(self, axis=None):
        return self.shape if axis is None else self.shape[axis]

    def __getitem__(self, idx):
        return self._data[idx]

    def __setitem__(self, idx, val):
        self._data[idx] = val
        self._dirty = self._ctx is not None

    def __len__(self):
        return self._data.shape[0]

    def copy(self) -> "χT":
        c = χT.__new__(χT)
        c._data = self._data.copy(order="F")
        c.β, c.indices_ω, c.tail_c, c.λ = self.β, self.indices_ω.copy(), list(self.tail_c), self.λ
        c.axis_types, c.usable_ω = dict(self.axis_types), self.usable_ω.copy()
        c._ctx, c._ch, c._dev_λ, c._dirty = self._ctx, self._ch, self._dev_λ, self._dirty
        return c


class γT:
    """``γT`` (DataTypes.jl:358-364): triangular vertex [q, ν, ω] (device-resident)."""

    def __init__(self, data, ctx: Context | None = None, ch: int | None = None):
        self._dev = data if isinstance(data, DeviceArray) else None
        self._data = None if self._dev is not None else as_fc(data)
        self.axis_types = {"q": 0, "ν": 1, "ω": 2}
        self._ctx, self._ch = ctx, ch
        self._dirty = False

    @property
    def data(self) -> np.ndarray:
        if self._data is None:
            self._data = np.array(self._dev.data, order="F", copy=True)
        return self._data

    @property
    def shape(self):
        return self._dev.shape if self._dev is not None else self._data.shape

    def size(self, axis=None):
        return self.shape if axis is None else self.shape[axis]

    def __getitem__(self, idx):
        return self.data[idx]

    def __setitem__(self, idx, val):
        self.data[idx] = val
        self._dirty = True

    def _sync(self):
        if self._dirty and self._ctx is not None:
            self._ctx.call("ldga_set_gamma", self._ch, ptr(self._data))
            self._dirty = False


def ωn_grid(χ: χT) -> np.ndarray:
    """``ωn_grid`` (DataTypes.jl:201)."""
    return 2j * math.pi * χ.indices_ω / χ.β


def _wn2_tail(χ: χT, ws) -> np.ndarray:
    wn = ωn_grid(χ)[ws]
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.real(χ.tail_c[2] / wn**2)
    t[~np.isfinite(t)] = 0.0
    return t


def _full_range(χ: χT) -> bool:
    return len(χ.usable_ω) == χ.shape[1]


def _sum_kω_host(kG: KGrid, χdata: np.ndarray, β: float, c2: float, ωn2_tail, transform=None) -> float:
    """``sum_kω(kG, χ::Matrix, β, c2, ωn2_tail; transform)`` (DataTypes.jl:230-249), host data."""
    res = 0.0
    norm = float(np.sum(kG.kMult))
    for i, wt in enumerate(ωn2_tail):
        if transform is None:
            res += kG.kintegrate(χdata[:, i]) - wt
        else:
            res += float(np.sum(np.array([transform(x) for x in χdata[:, i]]) * kG.kMult)) / norm - wt
    return (res + (-β**2 / 12) * c2) / β


def sum_kω(kG: KGrid, χ, *args, ωn_arr=None, force_full_range: bool = False, transform=None,
           λ: float = float("nan")) -> float:
    """``sum_kω`` (DataTypes.jl:215-249).

    Forms: ``sum_kω(kG, χ::χT; λ=NaN, transform=None)`` and
    ``sum_kω(kG, χ::ndarray, β, c2, ωn2_tail; transform=None)``.
    """
    if not isinstance(χ, χT):
        β, c2, tail = args
        return _sum_kω_host(kG, np.asarray(χ, dtype=np.float64), β, c2, tail, transform)
    if χ.λ != 0 and not math.isnan(λ):
        raise RuntimeError("χ already λ-corrected, but external λ provided!")
    if len(χ.tail_c) == 3 and not (χ.tail_c[0] == 0 and χ.tail_c[1] == 0):
        raise RuntimeError("sum_kω only implemented for ω^2 tail!")
    if not math.isnan(λ) and transform is not None:
        raise RuntimeError("Only transformation OR λ value should be given!")
    extra = 0.0 if math.isnan(λ) else λ
    ws = np.arange(χ.shape[1]) if force_full_range else χ.usable_ω
    if χ._ctx is not None and transform is None and (force_full_range or _full_range(χ)):
        out = _lib.C.c_double()
        χ._ctx.call("ldga_sum_kw", χ._ch, χ._device_λ(extra), 0, _lib.C.byref(out))
        return out.value
    tf = transform
    if not math.isnan(λ):
        tf = (lambda x, l=λ: χ_λ(x, l))
    return _sum_kω_host(kG, χ._data[:, ws], χ.β, χ.tail_c[2], _wn2_tail(χ, ws), tf)


def sum_ω(χ, *args, force_full_range: bool = False):
    """``sum_ω(χ::χT)`` per q, or ``sum_ω(ωn_arr, χ::Vector, tail_c, β)`` (DataTypes.jl:277-308)."""
    if not isinstance(χ, χT):
        ωn_arr, vec, tail_c, β = χ, args[0], args[1], args[2]
        return _sum_ω_vec(ωn_arr, vec, tail_c, β)
    ws = np.arange(χ.shape[1]) if force_full_range else χ.usable_ω
    wn = ωn_grid(χ)[ws]
    return np.array([_sum_ω_vec(wn, χ._data[q, ws], χ.tail_c, χ.β) for q in range(χ.shape[0])])


def _sum_ω_vec(ωn_arr, vec, tail_c, β: float) -> float:
    if not math.isclose(sum(tail_c), tail_c[2]):
        raise RuntimeError("sum_ω only implemented for 1/ω^2, but other tail coefficients are non-zero!")
    res = 0.0
    for n in range(len(vec)):
        if ωn_arr[n] != 0:
            res += vec[n] - np.real(tail_c[2] / (ωn_arr[n] ** 2))
        else:
            res += vec[n]
    return (res + tail_c[2] * (-β**2 / 12)) / β


def sum_ωk(kG: KGrid, χ: χT, force_full_range: bool = False, λ: float = float("nan")) -> float:
    """``sum_ωk`` (DataTypes.jl:257-264)."""
    λc = (not math.isnan(λ)) and λ != 0
    if χ.λ != 0 and λc:
        raise RuntimeError("χ already λ-corrected, but external λ provided!")
    extra = λ if λc else 0.0
    if χ._ctx is not None and (force_full_range or _full_range(χ)):
        out = _lib.C.c_double()
        χ._ctx.call("ldga_sum_wk", χ._ch, χ._device_λ(extra), _lib.C.byref(out))
        return out.value
    c = χ.copy()
    if λc:
        χ_λ_(c, λ)
    return float(kG.kintegrate(sum_ω(c, force_full_range=force_full_range)))


def update_tail_(χ: χT, new_tail_c, ωnGrid) -> None:
    """``update_tail!`` (DataTypes.jl:315-345)."""
    new_tail_c = [float(x) for x in new_tail_c]
    if len(new_tail_c) != len(χ.tail_c):
        raise ValueError(f"length of new tail coefficient array ({len(new_tail_c)}) must be the same as the old one ({len(χ.tail_c)})!")
    if len(ωnGrid) != χ.shape[1]:
        raise ValueError("length of ωnGrid must be the same as for χ")
    if not all(np.isfinite(new_tail_c)):
        raise ValueError("One or more tail coefficients are not finite!")
    if sum(new_tail_c) != new_tail_c[2]:
        raise ValueError("update tail only implemented for c_2 coefficient!")
    λ_bak = χ.λ
    if λ_bak != 0:
        reset_(χ)
    if χ.tail_c[2] != new_tail_c[2]:
        for wi in range(χ.shape[1]):
            if abs(ωnGrid[wi]) < 1e-10:
                continue
            χ._data[:, wi] += np.real((new_tail_c[2] - χ.tail_c[2]) / ωnGrid[wi] ** 2)
        χ._dirty = χ._ctx is not None
        χ.tail_c[2] = new_tail_c[2]
    χ_λ_(χ, λ_bak)


# =============================================================================================
# λ transform (LambdaCorrection/helpers.jl:18-70)
# =============================================================================================
def χ_λ(χ, λ: float):
    """``χ_λ``: scalar / array -> χ/(λχ + 1); χT -> new χT with λ applied."""
    if isinstance(χ, χT):
        c = χ.copy()
        χ_λ_(c, λ)
        return c
    return χ / (λ * χ + 1)


def dχ_λ(χ, λ: float):
    """``dχ_λ`` (LambdaCorrection/helpers.jl:61-62)."""
    return -χ_λ(χ, λ) ** 2


def χ_λ_(*args) -> None:
    """``χ_λ!`` (LambdaCorrection/helpers.jl:38-53): ``χ_λ_(χ, λ)`` in place, accumulating χ.λ;
    ``χ_λ_(χ_new, χ, λ)`` writes χ's corrected values into χ_new (χ_new.λ = χ.λ + λ); both also for
    plain arrays (``χ_λ_(res, χ, λ)``).  λ = 0 leaves the data untouched."""
    if len(args) == 2:
        χ_new, χ, λ = args[0], args[0], args[1]
    elif len(args) == 3:
        χ_new, χ, λ = args
    else:
        raise TypeError("χ_λ_(χ, λ) or χ_λ_(χ_new, χ, λ)")
    if isinstance(χ_new, χT) != isinstance(χ, χT):
        raise TypeError("χ_λ_: both arguments χT, or both arrays")
    src = χ._data if isinstance(χ, χT) else χ
    dst = χ_new._data if isinstance(χ_new, χT) else χ_new
    if λ != 0.0:
        if not math.isfinite(λ):
            print(f"WARNING. SKIPPING λ correction because {λ} is not finite!")
            return
        dst[...] = src / (λ * src + 1)
    if isinstance(χ_new, χT):
        χ_new.λ = χ.λ + λ
        if χ_new is not χ and χ_new._ctx is not None:
            χ_new._dirty = True      # its device copy holds other data: upload before the next use


def reset_(χ: χT) -> None:
    """``reset!`` (LambdaCorrection/helpers.jl:64-70)."""
    if χ.λ != 0:
        λ = -χ.λ
        χ._data[:, :] = χ._data / (λ * χ._data + 1)
        χ.λ = 0.0


def get_λ_min(χ) -> float:
    """``get_λ_min`` (LambdaCorrection/helpers.jl:217-220)."""
    if isinstance(χ, χT) and χ._ctx is not None and χ.λ == χ._dev_λ and not χ._dirty:
        out = _lib.C.c_double()
        χ._ctx.call("ldga_lambda_min", χ._ch, _lib.C.byref(out))
        return out.value
    data = χ.data if isinstance(χ, χT) else np.asarray(χ)
    nh = math.ceil(data.shape[1] / 2) - 1
    return float(-np.min(1.0 / data[:, nh]))


# =============================================================================================
# root finding (LambdaCorrection/helpers.jl:133-208) -- generic host versions for user functions;
# the λ corrections themselves run their Newton loops on the device.
# =============================================================================================
def _fd_step(x: float) -> float:
    r = math.sqrt(np.finfo(np.float64).eps)
    return max(r * abs(x), r)


def newton_right(f, df=None, start=None, min_=None, nsteps: int | None = None, atol: float | None = None, **kw):
    """``newton_right``: 1-D with optional derivative, or N-D with a forward-difference Jacobian."""
    if start is None or min_ is None:
        # called as newton_right(f, start, min)
        start, min_, df = df, start, None
    if np.ndim(start) == 0:
        if df is None:
            df = (lambda x: (f(x + _fd_step(x)) - f(x)) / _fd_step(x))
        nsteps = 100 if nsteps is None else nsteps
        atol = 1e-13 if atol is None else atol
        δ = 1e-4
        x0 = float(start)
        xi = x0
        i = 1
        while True:
            fi = f(xi)
            dfii = 1 / df(xi)
            xi = x0 - dfii * fi
            if abs(fi) < atol:
                break
            if xi < min_:
                x0 = min_ + δ + abs(min_ - x0) / 2
            else:
                x0 = xi
            if i >= nsteps:
                break
            i += 1
        return xi
    return _newton_right_nd(f, np.asarray(start, float), np.asarray(min_, float),
                            nsteps=500 if nsteps is None else nsteps, atol=1e-8 if atol is None else atol, **kw)


def _newton_right_nd(f, start, xmin, nsteps=500, atol=1e-8, max_reset=5, reset_backoff=1.0, verbose=False):
    def jac(x):
        fx = np.asarray(f(x), float)
        J = np.empty((len(fx), len(x)))
        for j in range(len(x)):
            e = _fd_step(x[j])
            x1 = x.copy()
            x1[j] += e
            J[:, j] = (np.asarray(f(x1), float) - fx) / e
        return J

    xi = start.copy()
    i, reset_i, bis_fail = 1, 1, False
    while True:
        fi = np.asarray(f(xi), float)
        dfii = np.linalg.inv(jac(xi))
        last = xi.copy()
        xi = xi - dfii @ fi
        for l in range(len(xi)):
            if xi[l] < xmin[l]:
                xi[l] = xmin[l] + abs(last[l] - xmin[l]) / 2
                if abs(last[l] - xmin[l]) / 2 < 1e-8:
                    print("WARNING: Bisection step is smaller than 1e-8. This indicates faulty data or no solution.")
                    bis_fail = True
        if bis_fail or not np.all(np.isfinite(fi)):
            bis_fail = False
            if reset_i >= max_reset:
                raise RuntimeError(f"λ root-finding returned NaN after {i} iterations and {max_reset} resets. min values are {xmin}")
            reset_i += 1
            xi = start + reset_i * reset_backoff * np.abs(xmin)
        if abs(np.linalg.norm(fi)) < atol:
            break
        if i >= nsteps:
            break
        i += 1
    return xi


# =============================================================================================
# usable ranges (GFFit.jl:31-84)
# =============================================================================================
def find_usable_χ_interval(χ_ω, sum_type="common", reduce_range_prct: float = 0.1) -> np.ndarray:
    """``find_usable_χ_interval`` (GFFit.jl:31-73); returns 1-based indices like the reference."""
    χ_ω = np.asarray(χ_ω, dtype=np.float64)
    if χ_ω.ndim == 2:
        sets = [set(find_usable_χ_interval(row, reduce_range_prct=0.1).tolist()) for row in χ_ω]
        return np.array(sorted(set.intersection(*sets)), dtype=np.int64)
    n = len(χ_ω)
    if n % 2 == 0:
        raise ValueError("Finding a usable interval is only implemented for uneven size of χ_ω!")
    mid = math.ceil(n / 2)
    if sum_type == "full":
        return np.arange(1, n + 1)
    if isinstance(sum_type, tuple):
        return np.arange(sum_type[0], sum_type[1] + 1)
    darr = np.diff(χ_ω)
    if χ_ω[mid - 1] < 0.0:
        return np.array([mid])
    r1 = 0
    while r1 < mid - 1 and χ_ω[mid - r1 - 2] > 0 and χ_ω[mid + r1] > 0:
        r1 += 1
    r2 = 0
    while r2 < mid - 1 and darr[mid - r2 - 2] > 0 and darr[mid + r2 - 1] < 0:
        r2 += 1
    rng = math.ceil(min(r1, r2) * (1 - reduce_range_prct))
    return np.arange(mid - rng, mid + rng + 1)


def usable_ωindices(sP: SimulationParameters, *χs: χT) -> np.ndarray:
    """``usable_ωindices`` (GFFit.jl:81-84); 1-based indices."""
    if sP.dbg_full_eom_omega:
        return np.arange(1, χs[0].shape[1] + 1)
    s = set((χs[0].usable_ω + 1).tolist())
    for c in χs[1:]:
        s &= set((c.usable_ω + 1).tolist())
    return np.array(sorted(s), dtype=np.int64)


# =============================================================================================
# Green's function helpers (GFTools.jl)
# =============================================================================================
def G_from_Σ(ind, β, μ=None, ϵₖ=None, Σ=None):
    """``G_from_Σ(ind, β, μ, ϵk, Σ)`` or ``G_from_Σ(mf, μ, ϵk, Σ)`` (GFTools.jl:85-86)."""
    if Σ is None:
        mf, μ_, ϵ_, Σ_ = ind, β, μ, ϵₖ
        return 1.0 / (mf + μ_ - ϵ_ - Σ_)
    return 1.0 / (1j * (2 * ind + 1) * math.pi / β + μ - ϵₖ - Σ)


def G_shell_sum(N: int, β: float) -> float:
    """``G_shell_sum`` (GFTools.jl:281-283): psi_1(1/2-N) = pi^2 - psi_1(N+1/2) (reflection)."""
    a = _trigamma(N + 0.5)
    return ((a - (math.pi**2 - a)) * β / (4 * math.pi**2) + β / 4)


def _trigamma(x: float) -> float:
    """psi_1(x), x > 0: recurrence to x >= 8, then the asymptotic series (A&S 6.4.12)."""
    acc = 0.0
    while x < 8.0:
        acc += 1.0 / (x * x)
        x += 1.0
    x2 = 1.0 / (x * x)
    s = 1.0 / x + x2 / 2.0 + (1.0 / 6.0 - x2 * (1.0 / 30.0 - x2 * (1.0 / 42.0 - x2 * (1.0 / 30.0 - x2 * (
        5.0 / 66.0 - x2 * (691.0 / 2730.0 - x2 * (7.0 / 6.0))))))) / (x * x * x)
    return acc + s


def filling(G, *args):
    """``filling`` (GFTools.jl:223-247)."""
    if len(args) == 1:
        n = 2 * np.sum(G) / args[0] + 1
        if np.imag(n) > 1e-8:
            raise RuntimeError("Error: Imaginary part of filling is larger than 10^-8")
        return float(np.real(n))
    if isinstance(args[0], KGrid):
        kG, U, μ, β = args
        return filling(kG.kintegrate(np.asarray(G), 0), U, μ, β)
    U, μ, β = args[:3]
    shell = args[3] if len(args) > 3 else G_shell_sum(len(G) // 2, β)
    return float(2 * (np.real(np.sum(G)) / β + 0.5 + μ * shell) / (1 + U * shell))


def filling_pos(G, *args, improved_sum: bool = True) -> float:
    """``filling_pos`` (GFTools.jl:255-273)."""
    if isinstance(args[0], KGrid):
        kG, U, μ, β = args
        return filling_pos(kG.kintegrate(np.asarray(G), 0), U, μ, β, improved_sum=improved_sum)
    U, μ, β = args[:3]
    sG = np.sum(G)
    if len(args) > 3:
        shell = args[3]
    elif not improved_sum:
        return float(2 * np.real(sG + np.conj(sG)) / β + 1)
    else:
        shell = G_shell_sum(len(G) + 1, β)
    return float(2 * (np.real(sG + np.conj(sG)) / β + 0.5 + μ * shell) / (1 + U * shell))


def subtract_tail(inp, c: float, iω, power: int) -> np.ndarray:
    """``subtract_tail`` (GFTools.jl:293-312)."""
    out = np.array(inp, dtype=np.complex128, copy=True)
    for n in range(len(out)):
        if iω[n] != 0:
            out[n] = inp[n] - c / (iω[n] ** power)
    return out


def Σ_Dyson(GBath, GImp) -> np.ndarray:
    """``Σ_Dyson`` (GFTools.jl:195-210)."""
    return 1.0 / np.asarray(GBath) - 1.0 / np.asarray(GImp)


# =============================================================================================
# lDΓAHelper and setup (runHelpers.jl:28-201)
# =============================================================================================
@dataclass
class lDΓAHelper:
    """``lDΓAHelper`` (runHelpers.jl:28-49).  ``gLoc_fft``/``gLoc_rfft`` live on the GPU as the
    symmetry-reduced transform of G; ``gLoc`` is G on the irreducible k-points over fft_range."""
    sP: SimulationParameters
    mP: ModelParameters
    kG: KGrid
    Σ_ladderLoc: np.ndarray
    Σ_loc: np.ndarray
    imp_density: float
    gLoc: DeviceArray
    Γ_m: np.ndarray
    Γ_d: np.ndarray
    χloc_m_sum: float
    χDMFT_m: np.ndarray
    χDMFT_d: np.ndarray
    χ_m_loc: χT
    γ_m_loc: γT
    χ_d_loc: χT
    γ_d_loc: γT
    χ0Loc: χ0T
    gImp: np.ndarray
    ctx: Context = field(repr=False, default=None)
    ctx_loc: Context = field(repr=False, default=None)

    def gimp_at(self, n: int) -> complex:
        g = self.gImp
        return g[n] if n >= 0 else np.conj(g[-n - 1])


def _local_G(gimp: np.ndarray, fft_range: range) -> np.ndarray:
    """G_imp over fft_range as a [1, Nf] array (runHelpers.jl:135-136); beyond the data: 0."""
    out = np.zeros((1, len(fft_range)), dtype=np.complex128, order="F")
    rm = len(gimp)
    for j, n in enumerate(fft_range):
        if 0 <= n < rm:
            out[0, j] = gimp[n]
        elif n < 0 and -n - 1 < rm:
            out[0, j] = np.conj(gimp[-n - 1])
    return out


def setup_LDGA(kGridStr, mP: ModelParameters, sP: SimulationParameters, inputs, precision: int = PREC_FP64,
               device: int = 0, silent: bool = True) -> lDΓAHelper:
    """``setup_LDGA`` (runHelpers.jl:85-201).

    ``inputs``: the ``EnvironmentVars`` of ``readConfig`` (the impurity file ``env.inputVars`` is
    read as the reference does, ``inputs.load_impurity_input``), or any object with ``sigma_loc``
    (Σ_loc(n), n >= 0), ``gimp`` (G_imp(n), n >= 0), ``chi_loc_m``/``chi_loc_d`` and
    ``gamma_m``/``gamma_d`` ([Nν, Nν, Nω] complex), e.g. ``synthetic.make_input``.
    """
    from .inputs import EnvironmentVars, load_impurity_input
    kind, ns = kGridStr
    kG = gen_kGrid(kind, ns)
    if sP.χ_helper is not None or sP.n_iν_shell != 0:
        raise NotImplementedError("only the plain path (χ_helper = nothing, n_iν_shell = 0) is built; "
                                  "the χ asymptotics helpers come from BSE_SC.jl")
    if isinstance(inputs, EnvironmentVars):
        inputs = load_impurity_input(inputs.inputVars, kGridStr, mP, sP)
    fr = sP.fft_range
    rm = max(abs(fr[0]), abs(fr[-1]))
    Σ_loc = np.ascontiguousarray(np.asarray(inputs.sigma_loc, dtype=np.complex128))
    gimp = np.ascontiguousarray(np.asarray(inputs.gimp, dtype=np.complex128)[:rm])
    χDMFT_m, χDMFT_d = as_fc(inputs.chi_loc_m), as_fc(inputs.chi_loc_d)
    Γ_m, Γ_d = as_fc(inputs.gamma_m), as_fc(inputs.gamma_d)

    # lattice handle: G(k, ν) on the device and its transform (runHelpers.jl:113-130)
    ctx = Context(kG.dim, ns, kG.t, kG.tp, kG.tpp, mP, sP, precision, device)
    ctx.call("ldga_gloc", ptr(Σ_loc), len(Σ_loc), None)
    gloc = DeviceArray(ctx, lambda: _fetch_gloc(ctx, Σ_loc), (ctx.Nq, ctx.Nf))

    # local quantities on the one-point grid (runHelpers.jl:132-163)
    ctx_loc = Context(kG.dim, 1, kG.t, kG.tp, kG.tpp, mP, sP, precision, device)
    ctx_loc.call("ldga_set_gloc", ptr(_local_G(gimp, fr)))
    ctx_loc.call("ldga_bubble", None)
    χ0Loc = χ0T(DeviceArray(ctx_loc, lambda: _fetch(ctx_loc, "chi0"), (1, ctx.Nnu, ctx.Nw)), mP.β,
                range(-sP.n_iω, sP.n_iω + 1), sP.n_iν, sP.shift, ctx=ctx_loc)
    χ_m_loc, γ_m_loc = _bse(ctx_loc, CH_M, Γ_m, mP)
    χ_d_loc, γ_d_loc = _bse(ctx_loc, CH_D, Γ_d, mP)
    ctx_loc.call("ldga_F_from_chi", ptr(χDMFT_m), ptr(gimp), len(gimp), None)
    ctx_loc.call("ldga_lambda0", None, None)
    χloc_m_sum = float(np.real(sum_ω(χ_m_loc)[0]))
    Σ_ladderLoc = np.empty((1, sP.n_iν), dtype=np.complex128, order="F")
    ctx_loc.call("ldga_eom", 0.0, 0.0, sP.n_iν, 1, χloc_m_sum, ptr(Σ_ladderLoc))
    if np.any(np.isnan(Σ_ladderLoc)):
        warnings.warn("Σ_ladderLoc contains NaN")

    # F_m for λ0 on the lattice handle (BSETools.jl:35-38)
    ctx.call("ldga_F_from_chi", ptr(χDMFT_m), ptr(gimp), len(gimp), None)

    # usable ranges and impurity density (runHelpers.jl:146-187)
    nw = 2 * sP.n_iω + 1
    χLoc_m_ω = np.array([np.sum(χDMFT_m[:, :, w]) / mP.β**2 for w in range(nw)])
    χLoc_d_ω = np.array([np.sum(χDMFT_d[:, :, w]) / mP.β**2 for w in range(nw)])
    um = find_usable_χ_interval(np.real(χLoc_m_ω), reduce_range_prct=sP.usable_prct_reduction)
    ud = find_usable_χ_interval(np.real(χLoc_d_ω), reduce_range_prct=sP.usable_prct_reduction)
    loc = np.array(sorted(set(um.tolist()) & set(ud.tolist()))) - 1
    iωn = 1j * 2 * np.arange(-sP.n_iω, sP.n_iω + 1) * math.pi / mP.β
    χupup = 0.5 * (χLoc_m_ω + χLoc_d_ω)[loc]
    χupup_sub = subtract_tail(χupup, mP.Ekin_DMFT, iωn[loc], 2)
    imp_density = float(np.real(np.sum(χupup_sub)) / mP.β - mP.Ekin_DMFT * mP.β / 12)
    if not silent:
        print(f"Inputs Read. imp_density = {imp_density}, χloc_m_sum = {χloc_m_sum}")

    h = lDΓAHelper(sP, mP, kG, Σ_ladderLoc, Σ_loc, imp_density, gloc, Γ_m, Γ_d, χloc_m_sum, χDMFT_m,
                   χDMFT_d, χ_m_loc, γ_m_loc, χ_d_loc, γ_d_loc, χ0Loc, gimp, ctx=ctx, ctx_loc=ctx_loc)
    _CTX_BY_GRID[id(kG)] = ctx
    _HELPER_BY_GRID[id(kG)] = h
    return h


def _fetch(ctx: Context, what: str, ch: int = 0) -> np.ndarray:
    """Copy a device-resident array of the handle to the host (ldga_get)."""
    if what == "chi0":
        out = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
        ctx.call("ldga_get", _lib.GET_CHI0, 0, ptr(out))
    elif what == "gamma":
        out = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
        ctx.call("ldga_get", _lib.GET_GAMMA, ch, ptr(out))
    elif what == "lambda0":
        out = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
        ctx.call("ldga_get", _lib.GET_LAMBDA0, 0, ptr(out))
    elif what == "gloc":
        out = _lib.cplx_out((ctx.Nq, ctx.Nf))
        ctx.call("ldga_get", _lib.GET_GLOC, 0, ptr(out))
    else:
        raise KeyError(what)
    return out


def _fetch_gloc(ctx: Context, Σ_loc: np.ndarray) -> np.ndarray:
    return _fetch(ctx, "gloc")


def setup_synthetic(inp, precision: int = PREC_FP64, device: int = 0, usable_prct_reduction: float = 0.0) -> lDΓAHelper:
    """``setup_LDGA`` from a ``synthetic.SyntheticInput`` (parameters taken from it)."""
    mP = ModelParameters(inp.U, inp.mu, inp.beta, inp.n, inp.sVk, inp.Epot_DMFT, inp.Ekin_DMFT)
    L = 2 * (inp.n_iv + inp.n_iw)
    sP = SimulationParameters(inp.n_iw, inp.n_iv, 0, inp.shift, None, range(-L, L + 1), usable_prct_reduction, False)
    return setup_LDGA((inp.kgrid_kind, inp.ns), mP, sP, inp, precision=precision, device=device)


# =============================================================================================
# ladder functions (BSETools.jl, ladderDGATools_singleCore.jl)
# =============================================================================================
def calc_bubble(h: lDΓAHelper) -> χ0T:
    """``calc_bubble(h)`` (BSETools.jl:153-172); the result stays on the GPU."""
    ctx = h.ctx
    ctx.call("ldga_bubble", None)
    dev = DeviceArray(ctx, lambda: _fetch(ctx, "chi0"), (ctx.Nq, ctx.Nnu, ctx.Nw))
    return χ0T(dev, h.mP.β, range(-h.sP.n_iω, h.sP.n_iω + 1), h.sP.n_iν, h.sP.shift, ctx=ctx)


def _bse(ctx: Context, ch: int, Γ, mP, χ0: χ0T | None = None):
    if χ0 is not None and χ0._ctx is not ctx:
        ctx.call("ldga_set_chi0", ptr(as_fc(χ0.data)))
    χ = np.empty((ctx.Nq, ctx.Nw), dtype=np.float64, order="F")
    nfb = _lib.C.c_int32()
    ctx.call("ldga_bse", ch, ptr(as_fc(Γ)) if Γ is not None else None, ptr(χ), None, _lib.C.byref(nfb))

    def fetch_gamma():
        return _fetch(ctx, "gamma", ch)

    c = χT(χ, mP.β, tail_c=[0.0, 0.0, mP.Ekin_DMFT])._bind(ctx, ch)
    c.n_fallback = nfb.value
    g = γT(DeviceArray(ctx, fetch_gamma, (ctx.Nq, ctx.Nnu, ctx.Nw)), ctx, ch)
    return c, g


def calc_χγ(type_, h_or_Γ, χ0: χ0T, *args):
    """``calc_χγ(type, h, χ0)`` or ``calc_χγ(type, Γr, χ0, kG, mP, sP)`` (BSETools.jl:188-248)."""
    ch = _channel(type_)
    if isinstance(h_or_Γ, lDΓAHelper):
        h = h_or_Γ
        Γ = h.Γ_m if ch == CH_M else h.Γ_d
        ctx, mP = h.ctx, h.mP
    else:
        Γ = h_or_Γ
        ctx = χ0._ctx
        mP = args[1]
        if ctx is None:
            raise RuntimeError("calc_χγ: χ0 must come from calc_bubble on a GPU handle")
    χ, γ = _bse(ctx, ch, Γ, mP, χ0)
    _log_q0_χ_check(ctx, χ, type_)
    return χ, γ


def calc_χγ_vjp(type_, h: lDΓAHelper, χ̄=None, γ̄=None):
    """Vector-Jacobian product of ``calc_χγ(type, h, χ0)`` (BSETools.jl:192-248) at its last call on
    the GPU handle: upstream gradients of a real loss with respect to χ_r.data [Nq, Nω] and
    γ_r.data [Nq, Nν, Nω] (complex: ∂L/∂Re + i ∂L/∂Im; None = 0) -> (Γ̄_r [Nν, Nν, Nω], χ̄₀ [Nq, Nν, Nω])."""
    ch = _channel(type_)
    ctx = h.ctx
    xb = None if χ̄ is None else np.asfortranarray(np.asarray(χ̄, dtype=np.float64))
    gb = None if γ̄ is None else as_fc(γ̄)
    Gb = _lib.cplx_out((ctx.Nnu, ctx.Nnu, ctx.Nw))
    c0b = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
    nf = _lib.C.c_int32()
    ctx.call("ldga_bse_vjp", ch, ptr(xb), ptr(gb), ptr(Gb), ptr(c0b), _lib.C.byref(nf))
    if nf.value:
        warnings.warn(f"calc_χγ_vjp: {nf.value} adjoint solves above the backward-error threshold")
    return Gb, c0b


def autotune_bse(h: lDΓAHelper, type_="m", reps: int = 3) -> tuple[int, float]:
    """Time the compiled BSE configurations for this handle's box size and precision mode on its
    current χ₀ and Γ_r, and use the fastest from now on (``ldga_autotune_bse``).  The channel's χ
    and γ are left as ``calc_χγ`` would leave them.  Returns (configuration index, ms per launch)."""
    ctx = h.ctx
    ch = _channel(type_)
    Γ = h.Γ_m if ch == CH_M else h.Γ_d
    ctx.call("ldga_bse", ch, ptr(as_fc(Γ)), None, None, None)
    v, ms = _lib.C.c_int32(), _lib.C.c_double()
    ctx.call("ldga_autotune_bse", ch, int(reps), _lib.C.byref(v), _lib.C.byref(ms))
    return v.value, ms.value


def tune_save(path) -> None:
    """Write the recorded BSE configuration choices (``ldga_tune_save``)."""
    lib = _lib.load()
    if lib.ldga_tune_save(str(path).encode()) != _lib.LDGA_OK:
        raise OSError(lib.ldga_last_error(None).decode())


def tune_load(path) -> None:
    """Read BSE configuration choices written by ``tune_save`` (``ldga_tune_load``)."""
    lib = _lib.load()
    if lib.ldga_tune_load(str(path).encode()) != _lib.LDGA_OK:
        raise OSError(lib.ldga_last_error(None).decode())


def tune_reset() -> None:
    """Forget the recorded BSE configuration choices (``ldga_tune_reset``)."""
    _lib.load().ldga_tune_reset()


def _log_q0_χ_check(ctx: Context, χ: χT, type_) -> None:
    """``log_q0_χ_check`` (helpers.jl:114-121), kept as a returned value instead of a log line."""
    q0 = 0
    ωs = [i for i in range(χ.shape[1]) if i != (χ.shape[1] - 1) // 2]
    χ.q0_check = abs(float(np.sum(χ._data[q0, ωs])))


def F_from_χ(type_, h: lDΓAHelper) -> np.ndarray:
    """``F_from_χ(:m, h)`` (BSETools.jl:35-38, 40-53), computed on the device."""
    if _channel(type_) != CH_M:
        raise RuntimeError("only F_m tested!")
    ctx = h.ctx
    F = _lib.cplx_out((ctx.Nnu, ctx.Nnu, ctx.Nw))
    ctx.call("ldga_F_from_chi", ptr(h.χDMFT_m), ptr(h.gImp), len(h.gImp), ptr(F))
    return F


def calc_λ0(χ0: χ0T, h: lDΓAHelper, Fr=None) -> DeviceArray:
    """``calc_λ0(χ0, h)`` plain branch (BSETools.jl:109-144); stays on the GPU."""
    ctx = h.ctx
    if χ0._ctx is not ctx:
        ctx.call("ldga_set_chi0", ptr(as_fc(χ0.data)))
    if Fr is None:
        ctx.call("ldga_F_from_chi", ptr(h.χDMFT_m), ptr(h.gImp), len(h.gImp), None)
        ctx.call("ldga_lambda0", None, None)
    else:
        ctx.call("ldga_lambda0", ptr(as_fc(Fr)), None)

    arr = DeviceArray(ctx, lambda: _fetch(ctx, "lambda0"), (ctx.Nq, ctx.Nnu, ctx.Nw))
    arr._is_lambda0 = True
    return arr


def _prepare_eom(h: lDΓAHelper, χm: χT, γm: γT, χd: χT, γd: γT, λ0) -> None:
    ctx = h.ctx
    for c, ch in ((χm, CH_M), (χd, CH_D)):
        if c._ctx is not ctx:
            ctx.call("ldga_set_chi", ch, ptr(np.asfortranarray(c._data)))
            c._bind(ctx, ch)
            c._dev_λ = c.λ
    for g, ch in ((γm, CH_M), (γd, CH_D)):
        if g._ctx is not ctx:
            ctx.call("ldga_set_gamma", ch, ptr(as_fc(g.data)))
            g._ctx, g._ch = ctx, ch
        g._sync()
    if not (isinstance(λ0, DeviceArray) and λ0._ctx is ctx):
        ctx.call("ldga_set_lambda0", ptr(as_fc(np.asarray(λ0))))


def calc_Σ(χm: χT, γm: γT, χd: χT, γd: γT, λ0, h: lDΓAHelper, νmax: int | None = None, λm: float = 0.0,
           λd: float = 0.0, tc: bool = True) -> np.ndarray:
    """``calc_Σ`` (ladderDGATools_singleCore.jl:108-136) -> Σ_ladder[q, ν_n], ν_n = 0..νmax-1."""
    νmax = h.sP.n_iν if νmax is None else νmax
    if χm.λ != 0 and λm != 0:
        raise RuntimeError(f"Stopping self energy calculation: λm = {λm} AND χm.λ = {χm.λ}")
    if χd.λ != 0 and λd != 0:
        raise RuntimeError(f"Stopping self energy calculation: λd = {λd} AND χd.λ = {χd.λ}")
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    out = _lib.cplx_out((h.ctx.Nq, νmax))
    h.ctx.call("ldga_eom", χm._device_λ(λm), χd._device_λ(λd), νmax, int(bool(tc)), h.χloc_m_sum, ptr(out))
    return out


def calc_Σ_vjp(Σ̄, χm: χT, γm: γT, χd: χT, γd: γT, λ0, h: lDΓAHelper, νmax: int | None = None, λm: float = 0.0,
               λd: float = 0.0, tc: bool = True):
    """Vector-Jacobian product of ``calc_Σ`` (ladderDGATools_singleCore.jl:108-136) on the GPU handle:
    the upstream gradient of a real loss with respect to Σ_ladder [Nq, νmax] (∂L/∂Re + i ∂L/∂Im)
    -> (χ̄m, γ̄m, χ̄d, γ̄d, λ̄₀) with respect to the arrays calc_Σ reads (χ before the λ correction)."""
    S = as_fc(Σ̄)
    νmax = S.shape[1] if νmax is None else νmax
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    ctx = h.ctx
    xmb = np.empty((ctx.Nq, ctx.Nw), order="F")
    xdb = np.empty((ctx.Nq, ctx.Nw), order="F")
    gmb = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
    gdb = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
    l0b = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
    ctx.call("ldga_eom_vjp", χm._device_λ(λm), χd._device_λ(λd), νmax, int(bool(tc)), ptr(S), ptr(xmb), ptr(gmb),
             ptr(xdb), ptr(gdb), ptr(l0b))
    return xmb, gmb, xdb, gdb, l0b


def chain_vjp_Γ(h: lDΓAHelper, Σ̄, χm: χT, γm: γT, χd: χT, γd: γT, λ0, νmax: int | None = None, λm: float = 0.0,
                λd: float = 0.0, tc: bool = True) -> dict:
    """Adjoint of the ladder chain's BSE → EoM part at fixed λ: for a real loss L(Σ_ladder) with
    Σ̄ = ∂L/∂Σ_ladder [Nq, νmax], the gradients with respect to the local vertices Γ_m, Γ_d
    [Nν, Nν, Nω], the bubble χ₀ (both channels' BSE) and λ₀, all computed on the GPU handle.
    χm, γm, χd, γd must be the outputs of the handle's last ``calc_χγ`` calls (the BSE adjoint
    rebuilds its forward solution from them)."""
    xmb, gmb, xdb, gdb, l0b = calc_Σ_vjp(Σ̄, χm, γm, χd, γd, λ0, h, νmax=νmax, λm=λm, λd=λd, tc=tc)
    Gmb, c0m = calc_χγ_vjp("m", h, xmb, gmb)
    Gdb, c0d = calc_χγ_vjp("d", h, xdb, gdb)
    return {"Γ_m": Gmb, "Γ_d": Gdb, "χ0": c0m + c0d, "λ0": l0b}


def gloc_vjp(h: lDΓAHelper, χ̄0=None, λ̄0=None, Σ̄=None, λm: float = 0.0, λd: float = 0.0, νmax: int | None = None):
    """Vector-Jacobian product of the lattice G(k, ν) = 1/(iν + μ - ε_k - Σ_loc(ν)) through the bubble
    (χ̄₀), λ₀ = χ₀ Σ_ν F / β² (λ̄₀, F fixed) and the EoM's direct use of G (Σ̄ at λm, λd)
    -> (Σ̄_loc [len(Σ_loc)], Ḡ [Nq, Nf]); μ, G_imp and the local vertices are held fixed."""
    ctx = h.ctx
    c0 = None if χ̄0 is None else as_fc(χ̄0)
    l0 = None if λ̄0 is None else as_fc(λ̄0)
    S = None if Σ̄ is None else as_fc(Σ̄)
    nu = 0 if S is None else (S.shape[1] if νmax is None else νmax)
    ns = len(h.Σ_loc)
    slb = np.empty(ns, dtype=np.complex128)
    gb = _lib.cplx_out((ctx.Nq, ctx.Nf))
    ctx.call("ldga_gloc_vjp", ptr(c0), ptr(l0), ptr(S), float(λm), float(λd), int(nu), int(ns), ptr(slb), ptr(gb))
    return slb, gb


def chain_vjp_Σloc(h: lDΓAHelper, Σ̄, χm: χT, γm: γT, χd: χT, γd: γT, λ0, νmax: int | None = None, λm: float = 0.0,
                   λd: float = 0.0, tc: bool = True) -> dict:
    """``chain_vjp_Γ`` continued to the lattice self-energy: the gradient of a real loss L(Σ_ladder)
    at fixed λ with respect to Σ_loc (through G, the bubble, both BSE channels, λ₀ and the EoM),
    plus the vertex gradients.  G_imp, F_m and the local vertices are held fixed."""
    out = chain_vjp_Γ(h, Σ̄, χm, γm, χd, γd, λ0, νmax=νmax, λm=λm, λd=λd, tc=tc)
    slb, gb = gloc_vjp(h, out["χ0"], out["λ0"], Σ̄, λm=λm, λd=λd, νmax=νmax)
    out["Σ_loc"], out["G"] = slb, gb
    return out


def chain_vjp(h: lDΓAHelper, Σ̄, χm: χT, γm: γT, χd: χT, γd: γT, λ0, νmax: int | None = None, λm: float = 0.0,
              λd: float = 0.0, tc: bool = True) -> dict:
    """``chain_vjp_Σloc`` in one device call (``ldga_chain_vjp``): every intermediate gradient stays
    on the GPU.  Returns Γ_m, Γ_d [Nν, Nν, Nω], Σ_loc [len(Σ_loc)] and χ0 [Nq, Nν, Nω], the total
    gradient with respect to the bubble (both BSE channels and λ₀), plus the count of adjoint solves
    above the backward-error threshold."""
    S = as_fc(Σ̄)
    νmax = S.shape[1] if νmax is None else νmax
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    ctx = h.ctx
    Gm = _lib.cplx_out((ctx.Nnu, ctx.Nnu, ctx.Nw))
    Gd = _lib.cplx_out((ctx.Nnu, ctx.Nnu, ctx.Nw))
    c0 = _lib.cplx_out((ctx.Nq, ctx.Nnu, ctx.Nw))
    slb = np.empty(len(h.Σ_loc), dtype=np.complex128)
    nf = _lib.C.c_int32()
    ctx.call("ldga_chain_vjp", ptr(S), χm._device_λ(λm), χd._device_λ(λd), νmax, int(bool(tc)), ptr(Gm), ptr(Gd),
             len(slb), ptr(slb), ptr(c0), _lib.C.byref(nf))
    if nf.value:
        warnings.warn(f"chain_vjp: {nf.value} adjoint solves above the backward-error threshold")
    return {"Γ_m": Gm, "Γ_d": Gd, "Σ_loc": slb, "χ0": c0, "n_flagged": nf.value}


def epot_vjp(h: lDΓAHelper, Σ, μ: float) -> np.ndarray:
    """∂E_pot,1/∂Σ_ladder [Nq, νmax] (complex gradient) of ``calc_E`` on ``G_from_Σladder!`` with μ
    following the filling condition (``ldga_epot_vjp``)."""
    S = as_fc(Σ)
    out = _lib.cplx_out(S.shape)
    h.ctx.call("ldga_epot_vjp", S.shape[1], float(μ), ptr(S), ptr(out))
    return out


def λdm_vjp(h: lDΓAHelper, χm: χT, γm: γT, χd: χT, γd: γT, λ0, res: "λ_result", Σ̄=None, Ē: float = 0.0) -> dict:
    """Gradient of L = f(Σ_ladder) + Ē·E_pot,1 evaluated at the λdm root (``λdm_correction``,
    conditions_new.jl:207-324) with respect to Γ_m, Γ_d, Σ_loc, χ₀ and λ₀, including the implicit
    dependence of (λm, λd) on them: with F(λ) = [PP_2 - n/2(1-n/2), E_pot,1 - E_pot,2] = 0,
        dL/dθ = ∂L/∂θ + wᵀ ∂F/∂θ,   Jᵀ w = -∂L/∂λ,   J = ∂F/∂λ (analytic, 2 x 2).
    Σ̄ = ∂f/∂Σ_ladder [Nq, νmax] at the root (None = 0).  ``res`` is the λ_result of the λdm call on
    this handle; χm, χd are the unshifted (λ = 0) susceptibilities it was computed from."""
    if χm.λ != 0 or χd.λ != 0:
        raise RuntimeError("λdm_vjp: χ must be unshifted (λ = 0), as for λdm_correction")
    ctx = h.ctx
    S = as_fc(res.Σ_ladder)
    nu = S.shape[1]
    lm, ld, mu = float(res.λm), float(res.λd), float(res.μ)
    U, β = h.mP.U, h.mP.β
    kmult = np.asarray(ctx.kmult)
    SE = epot_vjp(h, S, mu)
    SL = (np.zeros_like(SE) if Σ̄ is None else as_fc(Σ̄)) + Ē * SE
    oL = calc_Σ_vjp(SL, χm, γm, χd, γd, λ0, h, νmax=nu, λm=lm, λd=ld)
    oE = calc_Σ_vjp(SE, χm, γm, χd, γd, λ0, h, νmax=nu, λm=lm, λd=ld)
    xm, xd = np.asarray(χm.data), np.asarray(χd.data)
    dL = np.array([-np.sum(oL[0] * xm**2), -np.sum(oL[2] * xd**2)])
    dE1 = np.array([-np.sum(oE[0] * xm**2), -np.sum(oE[2] * xd**2)])
    # d sum_kω(χ^λ)/dλ = -(1/β) Σ_ω ⟨(χ^λ)²⟩_q exactly.  (The reference's λm Newton, which the
    # library mirrors in ldga_sum_kw's derivative mode, also subtracts the χ tail constants there;
    # the implicit derivative needs the true one.)
    nk = float(np.sum(kmult))
    dsm = -float(np.sum(kmult[:, None] * (xm / (lm * xm + 1.0)) ** 2)) / (β * nk)
    dsd = -float(np.sum(kmult[:, None] * (xd / (ld * xd + 1.0)) ** 2)) / (β * nk)
    J = np.array([[0.5 * dsm, 0.5 * dsd], [dE1[0] + 0.5 * U * dsm, dE1[1] - 0.5 * U * dsd]])
    w = np.linalg.solve(J.T, -dL)
    # ∂s/∂χ(q, ω) of sum_kω at λ for the unshifted χ
    dsm_dx = (kmult[:, None] / (β * nk)) / (lm * xm + 1.0) ** 2
    dsd_dx = (kmult[:, None] / (β * nk)) / (ld * xd + 1.0) ** 2
    xmb = oL[0] + w[1] * oE[0] + (0.5 * w[0] + 0.5 * U * w[1]) * dsm_dx
    xdb = oL[2] + w[1] * oE[2] + (0.5 * w[0] - 0.5 * U * w[1]) * dsd_dx
    gmb, gdb, l0b = oL[1] + w[1] * oE[1], oL[3] + w[1] * oE[3], oL[4] + w[1] * oE[4]
    Gmb, c0m = calc_χγ_vjp("m", h, xmb, gmb)
    Gdb, c0d = calc_χγ_vjp("d", h, xdb, gdb)
    slb, gb = gloc_vjp(h, c0m + c0d, l0b, SL + w[1] * SE, λm=lm, λd=ld, νmax=nu)
    # the EoM's tail term -U (sum_kω χm^λ - χloc_m_sum)/(iν_n) (ladderDGATools_singleCore.jl:133):
    # ∂Σ(q, n)/∂χloc_m_sum = U/(iν_n), through L directly and through E_pot,1 of the λ condition
    ivn = 1j * (2 * np.arange(nu) + 1) * math.pi / β
    sbar_tot = SL + w[1] * SE
    s_bar = float(np.real(np.sum(np.conj(sbar_tot) * (U / ivn)[None, :])))
    out = {"Γ_m": Gmb, "Γ_d": Gdb, "Σ_loc": slb, "χ0": c0m + c0d, "λ0": l0b, "χloc_m_sum": s_bar,
           "w": w, "J": J, "∂L/∂λ": dL}
    out.update(local_vertex_vjp(h, Gmb, Gdb, l0b, s_bar))
    return out


def local_vertex_vjp(h: lDΓAHelper, Γ̄m, Γ̄d, λ̄0, χ̄loc_m_sum: float = 0.0) -> dict:
    """The gradient continued from the lattice inputs to the local susceptibilities χ_loc,r = χDMFT_r
    (setup_LDGA, runHelpers.jl:132-187): Γ_r = χ_loc,r⁻¹ - diag(1/χ₀,loc) per ω (the identity the local
    Bethe-Salpeter step of the reference's setup reproduces), F_m = F_from_χ(χ_loc,m)
    (BSETools.jl:40-53) through λ₀ = χ₀ Σ_ν F / β² (BSETools.jl:129-141), and χloc_m_sum = the tail-
    corrected sum_ω of the local χ_m, whose ω-terms are Re Σ_νν' χ_loc,m / β².  G_imp is held fixed.
        χ̄_loc,r = -χ_loc,r⁻ᴴ Γ̄_r χ_loc,r⁻ᴴ  (+ for m: conj(∂F/∂χ) F̄ + χ̄loc_m_sum / β³),
        F̄[ν, ν', ω] = Σ_q conj(χ₀[q, ν', ω]) λ̄₀[q, ν', ω] / β².
    For the synthetic inputs χ_loc,d = χ₀,loc + C and χ_loc,m = χ₀,loc - C, so C̄ = χ̄_loc,d - χ̄_loc,m.
    Gradients use ā = ∂L/∂Re a + i ∂L/∂Im a."""
    sP, β = h.sP, h.mP.β
    Xm, Xd = as_fc(h.χDMFT_m), as_fc(h.χDMFT_d)
    nnu, _, nw = Xm.shape
    c0 = np.asarray(_fetch(h.ctx, "chi0"))
    Fbar_col = np.einsum("qvw,qvw->vw", np.conj(c0), as_fc(λ̄0)) / β**2          # [ν', ω]
    out_m = np.empty_like(Xm)
    out_d = np.empty_like(Xd)
    for wi in range(nw):
        Ym, Yd = np.linalg.inv(Xm[:, :, wi]), np.linalg.inv(Xd[:, :, wi])
        out_m[:, :, wi] = -Ym.conj().T @ as_fc(Γ̄m)[:, :, wi] @ Ym.conj().T
        out_d[:, :, wi] = -Yd.conj().T @ as_fc(Γ̄d)[:, :, wi] @ Yd.conj().T
        # F_m = -(χ + δ β g1 g2)/(g1 g2 g3 g4): ∂F/∂χ = -1/(g1 g2 g3 g4); F̄[ν, ν', ω] = Fbar_col[ν', ω]
        g = np.empty((nnu, 2), dtype=np.complex128)
        for vi in range(nnu):
            wn, vn = OneToIndex_to_Freq(wi + 1, vi + 1, sP)
            g[vi] = (h.gimp_at(vn), h.gimp_at(vn + wn))
        den = (g[:, 0] * g[:, 1])[:, None] * (g[:, 0] * g[:, 1])[None, :]
        out_m[:, :, wi] += np.conj(-1.0 / den) * Fbar_col[None, :, wi]
    out_m += χ̄loc_m_sum / β**3
    return {"χ_loc_m": out_m, "χ_loc_d": out_d, "C": out_d - out_m}


def calc_Σ_parts(χm: χT, γm: γT, χd: χT, γd: γT, λ0, h: lDΓAHelper, tc: bool = True, λm: float = 0.0,
                 λd: float = 0.0) -> np.ndarray:
    """``calc_Σ_parts`` (ladderDGATools_singleCore.jl:149-189) -> [q, ν_n, 7]."""
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    out = _lib.cplx_out((h.ctx.Nq, h.sP.n_iν, 7))
    h.ctx.call("ldga_eom_parts", χm._device_λ(λm), χd._device_λ(λd), int(bool(tc)), h.χloc_m_sum, ptr(out))
    return out


def G_from_Σladder(Σ_ladder: np.ndarray, Σloc, kG: KGrid, mP: ModelParameters, sP: SimulationParameters,
                   fix_n: bool = False, μ: float | None = None, h: lDΓAHelper | None = None):
    """``G_from_Σladder`` (GFTools.jl:154-186) -> (μ, G_ladder[q, fft_range]) on the device."""
    ctx = h.ctx if h is not None else _current_ctx(kG)
    μ = mP.μ if μ is None else μ
    S = as_fc(Σ_ladder)
    ctx.call("ldga_set_sigma", ptr(S), S.shape[1])
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))
    out = [_lib.C.c_double() for _ in range(4)]
    Σl = np.ascontiguousarray(np.asarray(Σloc, dtype=np.complex128))
    st = ctx.lib.ldga_g_ladder(ctx.h, ptr(Σl), len(Σl), int(bool(fix_n)), μ, _lib.C.byref(out[0]), ptr(G),
                               _lib.C.byref(out[1]), _lib.C.byref(out[2]), _lib.C.byref(out[3]))
    if st == _lib.LDGA_ERR_NOCONV:
        warnings.warn("μ determination failed")
        return float("nan"), G
    ctx.check(st)
    return out[0].value, G


_CTX_BY_GRID: dict = {}
_HELPER_BY_GRID: dict = {}


def _current_ctx(kG: KGrid) -> Context:
    c = _CTX_BY_GRID.get(id(kG))
    if c is None:
        raise RuntimeError("pass h=lDΓAHelper so that the GPU handle of this k-grid is known")
    return c


def calc_E(G, Σ, μ: float, kG: KGrid, mP: ModelParameters, h: lDΓAHelper | None = None, νmax: int | None = None):
    """``calc_E(G, Σ, μ, kG, mP)`` (thermodynamics.jl:142-168) on the device.

    ``G`` may span fft_range (as returned by ``G_from_Σladder``); the ν_n >= 0 part over Σ's range is used.
    """
    ctx = h.ctx if h is not None else _current_ctx(kG)
    S = as_fc(Σ)
    nu = S.shape[1] if νmax is None else νmax
    Gn = np.asarray(G)
    if Gn.shape[1] == ctx.Nf:
        off = -h.sP.fft_range[0] if h is not None else (ctx.Nf - 1) // 2
        Gn = Gn[:, off:off + nu]
    Gn = as_fc(Gn[:, :nu])
    ek, ep = _lib.C.c_double(), _lib.C.c_double()
    ctx.call("ldga_calc_E", ptr(Gn), ptr(as_fc(S[:, :nu])), nu, μ, _lib.C.byref(ek), _lib.C.byref(ep))
    return ek.value, ep.value


# =============================================================================================
# λ corrections (LambdaCorrection/conditions_new.jl)
# =============================================================================================
@dataclass
class λ_result:
    """``λ_result`` (conditions_new.jl:13-46)."""
    λm: float
    λd: float
    type: str
    converged: bool
    sc_converged: bool
    EKin: float = float("nan")
    EPot_p1: float = float("nan")
    EPot_p2: float = float("nan")
    PP_p1: float = float("nan")
    PP_p2: float = float("nan")
    trace: list = field(default_factory=list)
    G_ladder: np.ndarray | None = None
    Σ_ladder: np.ndarray | None = None
    μ: float = float("nan")
    n: float = float("nan")


def λm_rhs(χ_m: χT, χ_d: χT, h: lDΓAHelper, λd: float = float("nan"), λ_rhs: str = "native",
           verbose: bool = False) -> float:
    """``λm_rhs`` (LambdaCorrection/helpers.jl:230-255)."""
    if χ_d.λ != 0 and not math.isnan(λd):
        raise RuntimeError(f"Stopping λ rhs calculation: λd = {λd} AND χ_d.λ = {χ_d.λ}.")
    χ_d_sum = sum_kω(h.kG, χ_d, λ=λd)
    if (h.sP.χ_helper is not None and λ_rhs == "native") or λ_rhs == "fixed":
        return h.mP.n * (1 - h.mP.n / 2) - χ_d_sum
    if not math.isfinite(h.imp_density):
        raise ValueError("imp_density argument is not finite! Cannot use DMFT rror compensation method")
    return 2 * h.imp_density - χ_d_sum


def λm_correction(χm: χT, rhs: float, h: lDΓAHelper, validate_threshold: float = 1e-8, verbose: bool = False):
    """``λm_correction`` (conditions_new.jl:140-172): Newton on the device -> (λm, validation)."""
    if χm._ctx is None:
        raise RuntimeError("λm_correction: χm must come from calc_χγ")
    if χm.λ != χm._dev_λ or χm._dirty:
        # the device Newton works on the device copy: hand it the current (λ-corrected) host data
        χm._ctx.call("ldga_set_chi", χm._ch, ptr(np.asfortranarray(χm._data)))
        χm._dev_λ = χm.λ
        χm._dirty = False
    out = _lib.C.c_double()
    its = _lib.C.c_int32()
    χm._ctx.call("ldga_lambda_m", rhs, _lib.C.byref(out), _lib.C.byref(its))
    λm = out.value
    c = χ_λ(χm, λm)
    check = sum_kω(h.kG, c)
    check2 = sum_ωk(h.kG, c)
    if verbose:
        print(f"CHECK for rhs = {rhs}  : {check} ?=? 0")
    validation = abs(rhs - check) <= validate_threshold and abs(rhs - check2) <= validate_threshold
    return λm, validation


def λm_correction_full(χm: χT, γm: γT, χd: χT, γd: γT, λ0, h: lDΓAHelper, νmax: int = -1,
                       validate_threshold: float = 1e-8, verbose: bool = False, fit_μ: bool = True) -> λ_result:
    """``λm_correction_full`` (conditions_new.jl:174-190)."""
    νmax = γm.shape[1] // 2 if νmax < 0 else νmax
    rhs = λm_rhs(χm, χd, h, λ_rhs="native")
    λm, validation = λm_correction(χm, rhs, h, validate_threshold=validate_threshold, verbose=verbose)
    Σ_ladder = calc_Σ(χm, γm, χd, γd, λ0, h, νmax=νmax, λm=λm)
    μnew, G_ladder = G_from_Σladder(Σ_ladder, h.Σ_loc, h.kG, h.mP, h.sP, fix_n=fit_μ, h=h)
    EKin1, EPot1 = calc_E(G_ladder, Σ_ladder, μnew, h.kG, h.mP, h=h)
    rhs_c1 = h.mP.n / 2 * (1 - h.mP.n / 2)
    χ_m_sum = sum_kω(h.kG, χm, λ=λm)
    χ_d_sum = sum_kω(h.kG, χd)
    lhs_c1 = (χ_d_sum + χ_m_sum) / 2
    EPot2 = (h.mP.U / 2) * (χ_d_sum - χ_m_sum) + h.mP.U * (h.mP.n / 2 * h.mP.n / 2)
    return λ_result(λm, χd.λ, "m", validation, True, EKin1, EPot1, EPot2, rhs_c1, lhs_c1, [], G_ladder, Σ_ladder,
                    μnew, h.mP.n)


def _λdm_sc_correction(χm, γm, χd, γd, λ0, h, νmax, λ_min_δ, λ_val_only, validate_threshold, atol, nsteps,
                       sc_max_it, sc_mixing, sc_conv, update_χ_tail):
    """``λdm_correction`` with sc_max_it > 0 (conditions_new.jl:272-283): every residual is the
    self-consistent loop run_sc! at fixed (λm, λd) on the device (ldga_run_sc from the handle's G and
    μ = mP.μ, at most sc_max_it iterations); the 2-D newton_right on the host."""
    t = "dm_tsc" if update_χ_tail else "dm_sc"
    nan = float("nan")
    if update_χ_tail:
        # residual_vals_sc λ-corrects χ before run_sc!, whose tail update then sums it with an external
        # λ: the reference raises there for every λ != 0 (the FD Jacobian's first step), its
        # newton_right call catches the error and the root is NaN (conditions_new.jl:292-300)
        print("Error: χ already λ-corrected, but external λ provided!")
        print("WARNING: No λ root was found!")
        if λ_val_only:
            return nan, nan, False
        return λ_result(nan, nan, t, True, False)
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    χm._device_λ()
    χd._device_λ()
    ctx = h.ctx
    rhs_c1 = h.mP.n / 2 * (1 - h.mP.n / 2)
    out = np.zeros(12)
    nu_auto = min(h.sP.n_iν, math.floor(3 * len(usable_ωindices(h.sP, χm, χd)) / 8))
    nu = nu_auto if νmax < 1 else min(nu_auto, νmax)
    S = _lib.cplx_out((ctx.Nq, max(nu, 1)))
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))

    def vals(lam, keep=False):
        ctx.call("ldga_run_sc", float(lam[0]), float(lam[1]), 0, float(h.mP.μ), h.χloc_m_sum, int(νmax),
                 int(sc_max_it), float(sc_mixing), float(sc_conv), 1, float(λ_min_δ), ptr(out),
                 ptr(S) if keep else None, ptr(G) if keep else None)
        return out.copy()

    def residual(lam):
        o = vals(lam)
        return np.array([o[3] - rhs_c1, o[4] - o[5]])

    lmin = np.array([get_λ_min(χm), get_λ_min(χd)])
    xmin = lmin + λ_min_δ * np.abs(lmin)
    try:
        root = _newton_right_nd(residual, np.zeros(2), xmin, nsteps=nsteps, atol=atol)
    except RuntimeError as e:
        print(f"Error: {e}")
        root = np.array([nan, nan])
    if not np.all(np.isfinite(root)):
        print("WARNING: No λ root was found!")
        if λ_val_only:
            return float(root[0]), float(root[1]), False
        return λ_result(float(root[0]), float(root[1]), t, True, False)
    o = vals(root, keep=True)
    lhs_c1, ep1, ep2, ek, n, μ = o[3], o[4], o[5], o[6], o[7], o[8]
    conv = abs(rhs_c1 - lhs_c1) <= validate_threshold and abs(ep1 - ep2) <= validate_threshold
    if λ_val_only:
        return float(root[0]), float(root[1]), conv
    return λ_result(float(root[0]), float(root[1]), t, True, conv, ek, ep1, ep2, rhs_c1, lhs_c1, [], G, S[:, :nu],
                    μ, n)


def λdm_correction(χm: χT, γm: γT, χd: χT, γd: γT, λ0, h: lDΓAHelper, νmax: int = -1, λ_min_δ: float = 1e-4,
                   λ_val_only: bool = False, validate_threshold: float = 1e-8, atol: float = 1e-8,
                   nsteps: int = 500, sc_max_it: int = 0, sc_mixing: float = 0.2, sc_conv: float = 1e-8,
                   update_χ_tail: bool = False, verbose: bool = False, par: bool = False, tc: bool = True):
    """``λdm_correction`` plain branch (conditions_new.jl:207-324); the whole root search runs in the library."""
    if χm.λ != 0 or χd.λ != 0:
        raise RuntimeError("λ parameter already set. Aborting λdm calculation")
    if sc_max_it > 0:
        return _λdm_sc_correction(χm, γm, χd, γd, λ0, h, νmax, λ_min_δ, λ_val_only, validate_threshold, atol, nsteps,
                                  sc_max_it, sc_mixing, sc_conv, update_χ_tail)
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    χm._device_λ()
    χd._device_λ()
    ctx = h.ctx
    lm, ld = _lib.C.c_double(), _lib.C.c_double()
    conv = _lib.C.c_int32()
    nu_used = _lib.C.c_int32()
    out7 = np.zeros(7)
    nu_auto = min(h.sP.n_iν, math.floor(3 * len(usable_ωindices(h.sP, χm, χd)) / 8))
    nu_alloc = nu_auto if νmax < 1 else min(nu_auto, νmax)
    S = _lib.cplx_out((ctx.Nq, max(nu_alloc, 1)))
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))
    st = ctx.lib.ldga_lambda_dm(ctx.h, h.χloc_m_sum, νmax, λ_min_δ, atol, nsteps, _lib.C.byref(lm), _lib.C.byref(ld),
                                _lib.C.byref(conv), ptr(out7), _lib.C.byref(nu_used), ptr(S), ptr(G))
    if st == _lib.LDGA_ERR_NOCONV:
        print("WARNING: No λ root was found!")
        if λ_val_only:
            return float("nan"), float("nan"), False
        return λ_result(float("nan"), float("nan"), "dm", True, False)
    ctx.check(st)
    n, μ, ek, ep1, ep2, pp1, pp2 = out7
    if λ_val_only:
        return lm.value, ld.value, bool(conv.value)
    return λ_result(lm.value, ld.value, "dm", True, bool(conv.value), ek, ep1, ep2, pp1, pp2, [], G, S, μ, n)


def λ_correction(type_, χm: χT, γm: γT, χd: χT, γd: γT, λ0, h: lDΓAHelper, νmax: int = -1,
                 λ_min_δ: float = 1e-4, λ_val_only: bool = False, verbose: bool = False,
                 validate_threshold: float = 1e-8, **kw):
    """``λ_correction`` (conditions_new.jl:60-84): :m and :dm are built; :sc / :sc_m are not."""
    t = str(type_).lstrip(":")
    if t == "m":
        return λm_correction_full(χm, γm, χd, γd, λ0, h, νmax=νmax, validate_threshold=validate_threshold,
                                  verbose=verbose)
    if t == "dm":
        return λdm_correction(χm, γm, χd, γd, λ0, h, νmax=νmax, λ_min_δ=λ_min_δ, λ_val_only=λ_val_only,
                              validate_threshold=validate_threshold, verbose=verbose)
    if t in ("sc", "sc_m"):
        # conditions_new.jl:76-79: :sc -> run_sc with its defaults (type :fix, λ = 0), :sc_m -> type :m.
        # The reference omits run_sc's positional μ there; the model's μ is used.
        μ = kw.get("μ", h.mP.μ)
        return run_sc(χm, γm, χd, γd, λ0, μ, h, type=("fix" if t == "sc" else "m"),
                      **{k: v for k, v in kw.items() if k in ("maxit", "mixing", "conv_abs", "trace")})
    raise RuntimeError(f"λ-correction type '{type_}' not recognized!")


def run_sc(χm: χT, γm: γT, χd: χT, γd: γT, λ0, μ: float, h: lDΓAHelper, par: bool = False,
           λ_min_δ: float = 0.0001, νmax: int = -1, maxit: int = 100, mixing: float = 0.2, conv_abs: float = 1e-8,
           trace: bool = False, verbose: bool = False, update_χ_tail: bool = False, fit_μ: bool = True,
           tc: bool = True, type="fix", λm: float = 0.0, λd: float = 0.0) -> λ_result:
    """``run_sc`` (conditions_new.jl:342-407) with its loop ``run_sc!`` (:409-556) on the device.

    type: ``:fix`` (the given λm, λd), ``:m`` / ``:dm`` (the given λ, then :dm re-solves λdm in every
    iteration), ``:pre_m`` / ``:pre_dm`` (λ from λm_correction / λdm_correction first).  The EoM,
    μ fit, energies and the transform of G_ladder for the next EoM all run on the GPU handle;
    the handle's own G is restored afterwards, as the reference iterates on a deepcopy.
    """
    t = str(type).lstrip(":")
    if not fit_μ:
        warnings.warn("Not fitting μ can lead to unphysical results!")
    if update_χ_tail and t == "fix" and (λm != 0 or λd != 0):
        # run_sc! sums the λ-corrected χ with the external λ = 0 of :fix after a tail update
        # (conditions_new.jl:527-528, DataTypes.jl:216)
        raise RuntimeError("χ already λ-corrected, but external λ provided!")
    if not tc:
        raise NotImplementedError("run_sc: the EoM of the loop uses the tail correction (tc = true)")
    if t not in ("fix", "m", "dm", "pre_m", "pre_dm"):
        warnings.warn(f"Unrecognized type = {type} in run_sc")
        λm, λd = 0.0, 0.0
    if t == "pre_m":
        rhs = λm_rhs(χm, χd, h)
        λm, validation = λm_correction(χm, rhs, h)
        λd = 0.0
    elif t == "pre_dm":
        λm, λd, validation = λdm_correction(χm, γm, χd, γd, λ0, h, νmax=νmax, λ_min_δ=λ_min_δ, λ_val_only=True,
                                            validate_threshold=conv_abs, verbose=verbose)
    else:
        validation = True
    if not (validation and math.isfinite(λm) and math.isfinite(λd)):
        return λ_result(float("nan"), float("nan"), t, False, False, float("nan"), float("nan"), float("nan"),
                        float("nan"), float("nan"), [], None, None, float("nan"), float("nan"))
    _prepare_eom(h, χm, γm, χd, γd, λ0)
    χm._device_λ()
    χd._device_λ()
    ctx = h.ctx
    nu_auto = min(h.sP.n_iν, math.floor(3 * len(usable_ωindices(h.sP, χm, χd)) / 8))
    nu = nu_auto if νmax < 1 else min(nu_auto, νmax)
    out = np.zeros(12)
    S = _lib.cplx_out((ctx.Nq, max(nu, 1)))
    G = _lib.cplx_out((ctx.Nq, ctx.Nf))
    flags = ((SC_REDO_DM if t in ("dm", "pre_dm") else 0) | (SC_UPDATE_CHI_TAIL if update_χ_tail else 0)
             | (SC_LAMBDA_TYPE if t in ("m", "dm", "pre_m", "pre_dm") else 0))
    ctx.call("ldga_run_sc", float(λm), float(λd), flags, float(μ), h.χloc_m_sum, int(νmax),
             int(maxit), float(mixing), float(conv_abs), int(bool(fit_μ)), float(λ_min_δ), ptr(out), ptr(S), ptr(G))
    lm, ld, rhs_c1, lhs_c1, ep1, ep2, ek, n, μr, scc = out[:10]
    if t == "fix":
        lm, ld = 0.0, 0.0   # run_sc! reports its loop-local λ, which :fix never sets (conditions_new.jl:426-446)
    sc_converged = bool(scc)
    converged = (sc_converged and math.isfinite(lhs_c1) and math.isfinite(ep2) and abs(rhs_c1 - lhs_c1) <= conv_abs
                 and abs(ep1 - ep2) <= conv_abs)
    # λ_result(λm, λd, type, sc_converged, converged, ...) in the reference's positional order (:404-405)
    return λ_result(float(lm), float(ld), t, sc_converged, converged, float(ek), float(ep1), float(ep2),
                    float(rhs_c1), float(lhs_c1), [], G, S[:, :nu], float(μr), float(n))


# =============================================================================================
# uneven parameter scans: the λm chain of many points in one call
# =============================================================================================
@dataclass
class ChainResult:
    """One point of ``λm_chain_batch``: the λm chain's outputs (Σ_ladder on ν_n = 0..Nν/2-1)."""
    λm: float
    μ: float
    EKin: float
    EPot_p1: float
    EPot_p2: float
    PP_p2: float
    newton_iterations: int
    n: float
    Σ_ladder: np.ndarray
    χ_m: np.ndarray
    χ_d: np.ndarray


def _pinned(shape, dtype) -> np.ndarray:
    """A numpy view of page-locked host memory: copies from and to it stay asynchronous, so the
    points of a batch overlap (pageable memory would make every copy wait for its stream)."""
    import torch
    t = torch.empty(int(np.prod(shape)) * np.dtype(dtype).itemsize, dtype=torch.uint8, pin_memory=True)
    return t.numpy().view(dtype).reshape(shape, order="F"), t


def _chain_host_inputs(h: lDΓAHelper, keep: list) -> dict:
    out = {}
    for k, a in (("sigma_loc", h.Σ_loc), ("gamma_m", h.Γ_m), ("gamma_d", h.Γ_d), ("chi_loc_m", h.χDMFT_m),
                 ("gimp", h.gImp)):
        src = np.asarray(a, dtype=np.complex128).reshape(-1, order="F")
        buf, t = _pinned(src.shape, np.complex128)
        buf[...] = src
        keep.append(t)
        out[k] = buf
    return out


def λm_chain_batch(hs, use_graph: bool = False) -> list:
    """bubble → BSE (m, d) → λ₀ → λm correction → EoM → μ, energies (``run_minimal.jl:7-14`` with
    λ_correction(:m)) for every helper of ``hs`` in one ``ldga_batch_chain_m`` call: all points'
    chains are in flight on the GPU together.  Each helper keeps its own handle (k-grid, box, U, β)."""
    hs = list(hs)
    n = len(hs)
    ios = (_lib.ChainIO * max(n, 1))()
    keep, outs = [], []
    for i, h in enumerate(hs):
        ctx = h.ctx
        x = _chain_host_inputs(h, keep)
        numax = ctx.Nnu // 2
        S, t1 = _pinned((ctx.Nq, numax), np.complex128)
        xm, t2 = _pinned((ctx.Nq, ctx.Nw), np.float64)
        xd, t3 = _pinned((ctx.Nq, ctx.Nw), np.float64)
        sc, t4 = _pinned((8,), np.float64)
        keep.extend([x, t1, t2, t3, t4])
        outs.append((S, xm, xd, sc))
        ios[i] = _lib.ChainIO(x["sigma_loc"].ctypes.data, len(h.Σ_loc), x["gamma_m"].ctypes.data,
                              x["gamma_d"].ctypes.data, x["chi_loc_m"].ctypes.data, x["gimp"].ctypes.data,
                              len(h.gImp), h.imp_density, h.χloc_m_sum, S.ctypes.data, xm.ctypes.data,
                              xd.ctypes.data, sc.ctypes.data)
    handles = (_lib.C.c_void_p * max(n, 1))(*[h.ctx.h.value for h in hs])
    status = (_lib.C.c_int32 * max(n, 1))()
    lib = _lib.load()
    st = lib.ldga_batch_chain_m(n, handles, ios, int(bool(use_graph)), status)
    if st != _lib.LDGA_OK:
        bad = [i for i in range(n) if status[i] != _lib.LDGA_OK]
        msgs = "; ".join(f"point {i}: {lib.ldga_last_error(hs[i].ctx.h).decode()}" for i in bad)
        raise _lib.LdgaError(st, msgs)
    res = []
    for S, xm, xd, sc in outs:
        res.append(ChainResult(float(sc[0]), float(sc[1]), float(sc[2]), float(sc[3]), float(sc[4]), float(sc[5]),
                               int(sc[6]), float(sc[7]), np.array(S, order="F"), np.array(xm, order="F"),
                               np.array(xd, order="F")))
    return res


# =============================================================================================
# parallel API (ladderDGATools.jl:46-245, parallelization_helpers.jl:197-240, 358-420)
# =============================================================================================
# The reference keeps ω blocks of χ₀, χ, γ and the EoM caches on Distributed.jl workers and
# `collect_*` gathers them.  Here the GPU handle of the k-grid is the worker pool: the arrays stay
# in its HBM and `collect_*` copies them out.  Results are identical to the single-call API.
_EOM_STATE: dict = {}


def _helper_of(h_or_kG) -> lDΓAHelper:
    if isinstance(h_or_kG, lDΓAHelper):
        return h_or_kG
    h = _HELPER_BY_GRID.get(id(h_or_kG))
    if h is None:
        raise RuntimeError("Add workers and run lDGA_setup before calling parallel functions! "
                           "(no GPU handle was set up for this k-grid)")
    return h


def calc_bubble_par(h_or_kG, mP=None, sP=None, collect_data: bool = True):
    """``calc_bubble_par(h; collect_data)`` / ``(kG, mP, sP; collect_data)`` (ladderDGATools.jl:44-57):
    χ₀ is computed on the device; with ``collect_data`` it is returned (``collect_χ0``)."""
    h = _helper_of(h_or_kG)
    h.ctx.call("ldga_bubble", None)
    return collect_χ0(h) if collect_data else None


def collect_χ0(h_or_kG, mP=None, sP=None) -> χ0T:
    """``collect_χ0`` (ladderDGATools.jl:59-90): the device χ₀ of the last ``calc_bubble_par``."""
    h = _helper_of(h_or_kG)
    ctx = h.ctx
    dev = DeviceArray(ctx, lambda: _fetch(ctx, "chi0"), (ctx.Nq, ctx.Nnu, ctx.Nw))
    return χ0T(dev, h.mP.β, range(-h.sP.n_iω, h.sP.n_iω + 1), h.sP.n_iν, h.sP.shift, ctx=ctx)


def calc_χγ_par(type_, h_or_Γ, kG=None, mP=None, sP=None, collect_data: bool = True):
    """``calc_χγ_par(type, h; collect_data)`` / ``(type, Γr, kG, mP, sP; collect_data)``
    (ladderDGATools.jl:128-145): the BSE of the device χ₀; results stay on the device unless
    ``collect_data``."""
    ch = _channel(type_)
    if isinstance(h_or_Γ, lDΓAHelper):
        h, Γ = h_or_Γ, (h_or_Γ.Γ_m if ch == CH_M else h_or_Γ.Γ_d)
    else:
        h, Γ = _helper_of(kG), h_or_Γ
    χ, γ = _bse(h.ctx, ch, Γ, h.mP)
    _log_q0_χ_check(h.ctx, χ, type_)
    h._par_χγ = getattr(h, "_par_χγ", {})
    h._par_χγ[ch] = (χ, γ)
    return (χ, γ) if collect_data else None


def collect_χ(type_, h_or_kG, mP=None, sP=None) -> χT:
    """``collect_χ`` (parallelization_helpers.jl:358-383): χ_r of the last ``calc_χγ_par``."""
    h, ch = _helper_of(h_or_kG), _channel(type_)
    if ch not in getattr(h, "_par_χγ", {}):
        raise RuntimeError(f"collect_χ: call calc_χγ_par(:{type_}, ...) first")
    return h._par_χγ[ch][0]


def collect_γ(type_, h_or_kG, mP=None, sP=None) -> γT:
    """``collect_γ`` (parallelization_helpers.jl:385-410): γ_r of the last ``calc_χγ_par``."""
    h, ch = _helper_of(h_or_kG), _channel(type_)
    if ch not in getattr(h, "_par_χγ", {}):
        raise RuntimeError(f"collect_γ: call calc_χγ_par(:{type_}, ...) first")
    return h._par_χγ[ch][1]


def initialize_EoM(h: lDΓAHelper, λ0, νGrid, force_reinit: bool = False, χ_m: χT | None = None,
                   γ_m: γT | None = None, χ_d: χT | None = None, γ_d: γT | None = None) -> None:
    """``initialize_EoM(h, λ₀, νGrid; χ_m, γ_m, χ_d, γ_d)`` (parallelization_helpers.jl:207-240):
    binds the EoM inputs (default: the last ``calc_χγ_par`` results) to the device handle."""
    νGrid = list(νGrid)
    if νGrid != list(range(νGrid[0], νGrid[0] + len(νGrid))) or νGrid[0] != 0:
        raise ValueError("νGrid must be 0:νmax-1 (the range calc_Σ_par fills)")
    χ_m = collect_χ("m", h) if χ_m is None else χ_m
    γ_m = collect_γ("m", h) if γ_m is None else γ_m
    χ_d = collect_χ("d", h) if χ_d is None else χ_d
    γ_d = collect_γ("d", h) if γ_d is None else γ_d
    _prepare_eom(h, χ_m, γ_m, χ_d, γ_d, λ0)
    _EOM_STATE.clear()
    _EOM_STATE.update(h=h, χm=χ_m, γm=γ_m, χd=χ_d, γd=γ_d, λ0=λ0, νmax=len(νGrid))


def calc_Σ_par(λm: float = 0.0, λd: float = 0.0, collect_data: bool = True, tc: bool = True):
    """``calc_Σ_par(; λm, λd, collect_data, tc)`` (ladderDGATools.jl:223-229) on the inputs bound by
    ``initialize_EoM``.  Σ_ladder[q, ν_n], ν_n = 0..νmax-1, Hartree term included."""
    if not _EOM_STATE:
        raise RuntimeError("Call initialize_EoM before calc_Σ_par in order to initialize worker caches.")
    st = _EOM_STATE
    out = calc_Σ(st["χm"], st["γm"], st["χd"], st["γd"], st["λ0"], st["h"], νmax=st["νmax"], λm=λm, λd=λd, tc=tc)
    return out if collect_data else None


def calc_Σ_par_(Σ_ladder: np.ndarray, λm: float = 0.0, λd: float = 0.0, collect_data: bool = True,
                tc: bool = True):
    """``calc_Σ_par!`` (ladderDGATools.jl:231-245): fills ``Σ_ladder`` in place."""
    res = calc_Σ_par(λm=λm, λd=λd, collect_data=True, tc=tc)
    if collect_data:
        Σ_ladder[...] = res
    return Σ_ladder if collect_data else None


def gen_ω_part(sP: SimulationParameters, N: int):
    """``gen_ω_part`` (parallelization_helpers.jl:49-53); see ``parallel``."""
    from . import parallel
    return parallel.gen_ω_part(sP, N)


def gen_ν_part(νGrid, sP: SimulationParameters, N: int):
    """``gen_ν_part`` (parallelization_helpers.jl:62-68); see ``parallel``."""
    from . import parallel
    return parallel.gen_ν_part(νGrid, sP, N)


def gen_ν_part_slices(data, index_list):
    """``gen_ν_part_slices`` (parallelization_helpers.jl:81-102); see ``parallel``."""
    from . import parallel
    return parallel.gen_ν_part_slices(data, index_list)


def par_partition(set_, N: int):
    """``par_partition`` (parallelization_helpers.jl:22-29); see ``parallel``."""
    from . import parallel
    return parallel.par_partition(set_, N)


# ASCII aliases
chi0T, chiT, gammaT = χ0T, χT, γT   # the reference's χ₀T / λ₀ are χ0T / λ0 (no subscripts in identifiers)
calc_chi_gamma = calc_χγ
calc_lambda0 = calc_λ0
calc_Sigma = calc_Σ
calc_Sigma_parts = calc_Σ_parts
sum_kw, sum_w, sum_wk = sum_kω, sum_ω, sum_ωk
chi_lambda, chi_lambda_, dchi_lambda = χ_λ, χ_λ_, dχ_λ
reset = reset_
get_lambda_min = get_λ_min
lambda_m_rhs = λm_rhs
lambda_m_correction, lambda_m_correction_full = λm_correction, λm_correction_full
lambda_dm_correction, lambda_correction = λdm_correction, λ_correction
lambda_result = λ_result
G_from_Sigma, G_from_Sigma_ladder = G_from_Σ, G_from_Σladder
find_usable_chi_interval, usable_windices = find_usable_χ_interval, usable_ωindices
LDGAHelper = lDΓAHelper
F_from_chi = F_from_χ
calc_chi_gamma_par, collect_chi0, collect_chi, collect_gamma = calc_χγ_par, collect_χ0, collect_χ, collect_γ
calc_Sigma_par, calc_Sigma_par_, gen_w_part = calc_Σ_par, calc_Σ_par_, gen_ω_part
lambda_m_chain_batch = λm_chain_batch
calc_chi_gamma_vjp, calc_Sigma_vjp, chain_vjp_Gamma = calc_χγ_vjp, calc_Σ_vjp, chain_vjp_Γ
chain_vjp_Sigma_loc = chain_vjp_Σloc
lambda_dm_vjp = λdm_vjp
chi0Asym_coeffs = χ0Asym_coeffs
gen_nu_part, gen_nu_part_slices = gen_ν_part, gen_ν_part_slices
