"""ctypes binding of libldga_b200.so (the C ABI declared in include/ldga_b200.h).

The library is built in-tree (``python ladderdga.jl_b200/build.py``).  There is no CPU fallback:
importing the GPU entry points without the built library raises ``LibraryMissing``.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libldga_b200.so"

LDGA_OK, LDGA_ERR_ARG, LDGA_ERR_CUDA, LDGA_ERR_STATE = 0, 1, 2, 3
LDGA_ERR_NUMERIC, LDGA_ERR_NOCONV, LDGA_ERR_TYPE = 4, 5, 6
PREC_FP64_INV, PREC_FP64, PREC_MIXED = 0, 1, 2
CH_M, CH_D = 0, 1
SC_REDO_DM, SC_UPDATE_CHI_TAIL, SC_LAMBDA_TYPE = 1, 2, 4     # ldga_run_sc flags

# Every symbol the header declares (checked by the CPU test suite).
EXPORTS = [
    "ldga_create", "ldga_destroy", "ldga_last_error", "ldga_status_string", "ldga_version",
    "ldga_set_model", "ldga_set_precision", "ldga_kgrid", "ldga_gloc", "ldga_set_gloc", "ldga_bubble",
    "ldga_set_chi0", "ldga_bse", "ldga_set_chi", "ldga_set_gamma", "ldga_F_from_chi", "ldga_lambda0",
    "ldga_set_lambda0", "ldga_sum_kw", "ldga_sum_wk", "ldga_lambda_min", "ldga_eom", "ldga_eom_parts",
    "ldga_lambda_m", "ldga_lambda_m_newton", "ldga_g_ladder", "ldga_set_sigma", "ldga_calc_E", "ldga_lambda_dm",
    "ldga_lambda_dm_evals", "ldga_set_stream", "ldga_profile", "ldga_stage_times", "ldga_launch_count",
    "ldga_get", "ldga_chain_m", "ldga_lambda0_noalloc", "ldga_batch_chain_m", "ldga_run_sc", "ldga_bse_vjp",
    "ldga_eom_vjp", "ldga_autotune_bse", "ldga_tune_save", "ldga_tune_load",
    "ldga_tune_reset", "ldga_bse_config_name", "ldga_gloc_vjp", "ldga_epot_vjp", "ldga_chain_vjp",
    "ldga_bse_sweeps", "ldga_profile_stages", "ldga_selftest_group_inverse", "ldga_set_omega_shard",
]
GET_CHI0, GET_CHI, GET_GAMMA, GET_LAMBDA0, GET_SIGMA, GET_GLOC = 0, 1, 2, 3, 4, 5
STAGES = ["gloc", "bubble", "bse", "bse_fallback", "lambda0", "sums", "lambda_newton", "eom_forward",
          "eom_inverse", "g_ladder"]


class LibraryMissing(RuntimeError):
    """The CUDA library has not been built; there is no CPU fallback."""


class LdgaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Lattice(C.Structure):
    _fields_ = [("dim", C.c_int32), ("ns", C.c_int32), ("t", C.c_double), ("tp", C.c_double), ("tpp", C.c_double)]


class Model(C.Structure):
    _fields_ = [("U", C.c_double), ("mu", C.c_double), ("beta", C.c_double), ("n", C.c_double),
                ("sVk", C.c_double), ("Epot_DMFT", C.c_double), ("Ekin_DMFT", C.c_double)]


class ChainIO(C.Structure):
    """``ldga_chain_io``: the arguments of ldga_chain_m for one point of ldga_batch_chain_m."""
    _fields_ = [("sigma_loc", C.c_void_p), ("n_sigma", C.c_int32), ("gamma_m", C.c_void_p), ("gamma_d", C.c_void_p),
                ("chi_loc_m", C.c_void_p), ("gimp", C.c_void_p), ("n_gimp", C.c_int32), ("imp_density", C.c_double),
                ("chiloc_m_sum", C.c_double), ("sigma_out", C.c_void_p), ("chi_m_out", C.c_void_p),
                ("chi_d_out", C.c_void_p), ("scalars_out", C.c_void_p)]


class Sim(C.Structure):
    _fields_ = [("n_iw", C.c_int32), ("n_iv", C.c_int32), ("n_iv_shell", C.c_int32), ("shift", C.c_int32),
                ("fft_lo", C.c_int32), ("fft_hi", C.c_int32), ("usable_prct_reduction", C.c_double),
                ("dbg_full_eom_omega", C.c_int32)]


_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load (once) and return the library; raise ``LibraryMissing`` if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise LibraryMissing(f"{p} not found: build it with `python ladderdga.jl_b200/build.py` (no CPU fallback)")
    lib = C.CDLL(str(p))
    P, I32, D = C.c_void_p, C.c_int32, C.c_double
    PI32, PD = C.POINTER(C.c_int32), C.POINTER(C.c_double)
    sig = {
        "ldga_create": (C.c_int, [C.POINTER(Lattice), C.POINTER(Model), C.POINTER(Sim), I32, I32, C.POINTER(P)]),
        "ldga_destroy": (C.c_int, [P]),
        "ldga_last_error": (C.c_char_p, [P]),
        "ldga_status_string": (C.c_char_p, [I32]),
        "ldga_version": (C.c_int, []),
        "ldga_set_model": (C.c_int, [P, C.POINTER(Model)]),
        "ldga_set_precision": (C.c_int, [P, I32]),
        "ldga_kgrid": (C.c_int, [P, PI32, PI32, P, P, P]),
        "ldga_gloc": (C.c_int, [P, P, I32, P]),
        "ldga_set_gloc": (C.c_int, [P, P]),
        "ldga_bubble": (C.c_int, [P, P]),
        "ldga_set_chi0": (C.c_int, [P, P]),
        "ldga_bse": (C.c_int, [P, I32, P, P, P, PI32]),
        "ldga_set_chi": (C.c_int, [P, I32, P]),
        "ldga_set_gamma": (C.c_int, [P, I32, P]),
        "ldga_F_from_chi": (C.c_int, [P, P, P, I32, P]),
        "ldga_lambda0": (C.c_int, [P, P, P]),
        "ldga_set_lambda0": (C.c_int, [P, P]),
        "ldga_sum_kw": (C.c_int, [P, I32, D, I32, PD]),
        "ldga_sum_wk": (C.c_int, [P, I32, D, PD]),
        "ldga_lambda_min": (C.c_int, [P, I32, PD]),
        "ldga_eom": (C.c_int, [P, D, D, I32, I32, D, P]),
        "ldga_eom_parts": (C.c_int, [P, D, D, I32, D, P]),
        "ldga_lambda_m": (C.c_int, [P, D, PD, PI32]),
        "ldga_lambda_m_newton": (C.c_int, [P, D, I32, D, PD, PI32, PI32]),
        "ldga_g_ladder": (C.c_int, [P, P, I32, I32, D, PD, P, PD, PD, PD]),
        "ldga_lambda_dm": (C.c_int, [P, D, I32, D, D, I32, PD, PD, PI32, P, PI32, P, P]),
        "ldga_lambda_dm_evals": (C.c_int, [P, PI32]),
        "ldga_set_stream": (C.c_int, [P, P]),
        "ldga_profile": (C.c_int, [P, I32]),
        "ldga_profile_stages": (C.c_int, [P, C.c_uint32]),
        "ldga_selftest_group_inverse": (C.c_int, [I32, P, P, I32, P, P]),
        "ldga_set_omega_shard": (C.c_int, [P, I32, I32, I32]),
        "ldga_stage_times": (C.c_int, [P, PD, PI32]),
        "ldga_launch_count": (C.c_int, [P, C.POINTER(C.c_int64)]),
        "ldga_get": (C.c_int, [P, I32, I32, P]),
        "ldga_lambda0_noalloc": (C.c_int, [P, P, I32, I32, I32, D, P, P]),
        "ldga_chain_m": (C.c_int, [P, P, I32, P, P, P, P, I32, D, D, I32, P, P, P, P]),
        "ldga_batch_chain_m": (C.c_int, [I32, P, P, I32, PI32]),
        "ldga_bse_vjp": (C.c_int, [P, I32, P, P, P, P, PI32]),
        "ldga_eom_vjp": (C.c_int, [P, D, D, I32, I32, P, P, P, P, P, P]),
        "ldga_autotune_bse": (C.c_int, [P, I32, I32, PI32, PD]),
        "ldga_tune_save": (C.c_int, [C.c_char_p]),
        "ldga_tune_load": (C.c_int, [C.c_char_p]),
        "ldga_tune_reset": (C.c_int, []),
        "ldga_bse_config_name": (C.c_char_p, [I32, I32, I32]),
        "ldga_gloc_vjp": (C.c_int, [P, P, P, P, D, D, I32, I32, P, P]),
        "ldga_epot_vjp": (C.c_int, [P, I32, D, P, P]),
        "ldga_chain_vjp": (C.c_int, [P, P, D, D, I32, I32, P, P, I32, P, P, P]),
        "ldga_bse_sweeps": (C.c_int, [P, P, P]),
        "ldga_run_sc": (C.c_int, [P, D, D, I32, D, D, I32, I32, D, D, I32, D, P, P, P]),
        "ldga_set_sigma": (C.c_int, [P, P, I32]),
        "ldga_calc_E": (C.c_int, [P, P, P, I32, D, PD, PD]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def ptr(a) -> C.c_void_p | None:
    """Address of a contiguous numpy array or a CUDA torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not (a.flags.f_contiguous or a.flags.c_contiguous):
            raise ValueError("array must be contiguous")
        v = C.c_void_p(a.ctypes.data)
        # the pointer owns a reference: `ptr(as_fc(x))` passes a temporary copy, which would
        # otherwise be freed (and its first bytes reused by the allocator) before the C call reads it
        v._owner = a
        return v
    if hasattr(a, "data_ptr"):
        v = C.c_void_p(a.data_ptr())
        v._owner = a
        return v
    raise TypeError(f"unsupported buffer type {type(a)}")


class Context:
    """Owns one ``ldga_ctx`` handle (one k-grid, frequency box and parameter point on one GPU)."""

    def __init__(self, dim: int, ns: int, t: float, tp: float, tpp: float, mp, sp, precision: int = PREC_FP64,
                 device: int = 0):
        self.lib = load()
        lat = Lattice(dim, ns, t, tp, tpp)
        self._model = Model(mp.U, mp.mu, mp.beta, mp.n, mp.sVk, mp.Epot_DMFT, mp.Ekin_DMFT)
        fr = sp.fft_range
        self._sim = Sim(sp.n_iw, sp.n_iv, sp.n_iv_shell, int(bool(sp.shift)), fr[0], fr[-1],
                        float(sp.usable_prct_reduction), int(bool(sp.dbg_full_eom_omega)))
        h = C.c_void_p()
        st = self.lib.ldga_create(C.byref(lat), C.byref(self._model), C.byref(self._sim), precision, device, C.byref(h))
        if st != LDGA_OK:
            raise LdgaError(st, self.lib.ldga_last_error(None).decode())
        self.h = h
        self.dim, self.ns, self.device, self.precision = dim, ns, device, precision
        nk, nq = C.c_int32(), C.c_int32()
        self.lib.ldga_kgrid(self.h, C.byref(nk), C.byref(nq), None, None, None)
        self.Nk, self.Nq = nk.value, nq.value
        self.kmult = np.empty(self.Nq)
        self.eps = np.empty(self.Nq)
        self.wedge = np.empty((self.Nq, dim), dtype=np.int32)
        self.lib.ldga_kgrid(self.h, None, None, ptr(self.kmult), ptr(self.eps), ptr(self.wedge))
        self.Nnu, self.Nw = 2 * sp.n_iv, 2 * sp.n_iw + 1
        self.Nf = fr[-1] - fr[0] + 1

    def check(self, st: int) -> None:
        if st != LDGA_OK:
            raise LdgaError(st, self.lib.ldga_last_error(self.h).decode())

    def call(self, name: str, *args) -> int:
        st = getattr(self.lib, name)(self.h, *args)
        self.check(st)
        return st

    def set_model(self, mp) -> None:
        self._model = Model(mp.U, mp.mu, mp.beta, mp.n, mp.sVk, mp.Epot_DMFT, mp.Ekin_DMFT)
        self.call("ldga_set_model", C.byref(self._model))

    def set_precision(self, precision: int) -> None:
        self.call("ldga_set_precision", precision)
        self.precision = precision

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ldga_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cplx_out(shape) -> np.ndarray:
    return np.empty(shape, dtype=np.complex128, order="F")


def as_fc(a, dtype=np.complex128) -> np.ndarray:
    """Fortran-ordered (Julia layout) contiguous copy/view."""
    return np.asfortranarray(np.asarray(a, dtype=dtype))
