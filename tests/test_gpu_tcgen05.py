"""The tcgen05 tensor-core group inverse of the MIXED BSE's preconditioner (ldga_selftest_group_inverse).

The preconditioned BSE solve inverts one Nν x Nν complex matrix per group of 32 q,
B_bar = Γ(ω)ᵀ + diag(mean 1/χ₀), by Newton-Schulz iterations X <- X (2I - B_bar X) on tcgen05 tensor cores
(TF32 operands, FP32 accumulators in tensor memory).  These tests pin the device product and the iteration
against a NumPy restatement with the same TF32 rounding of the operands (round to nearest, ties away).
"""
import ctypes as C

import numpy as np
import pytest

import ladderdga_b200 as L

pytestmark = pytest.mark.gpu

N = 40


def tf32(a):
    """Round FP32 values to TF32 (10-bit mantissa), ties away from zero, real and imaginary parts."""
    def r(x):
        i = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
        return ((i + 0x1000) & 0xFFFFE000).astype(np.uint32).view(np.float32)
    a = np.asarray(a, np.complex64)
    return r(a.real) + 1j * r(a.imag)


def ns_emulated(b, x0, its):
    """Newton-Schulz with both factors of every product rounded to TF32, FP32 results."""
    x = np.asarray(x0, np.complex64)
    eye = np.eye(N)
    err = 0.0
    for _ in range(its):
        y = (tf32(b).astype(np.complex128) @ tf32(x).astype(np.complex128)).astype(np.complex64)
        e = eye - y
        err = np.max(np.sum(np.abs(e.real) + np.abs(e.imag), axis=1))   # the kernel's |Re| + |Im| measure
        x = (tf32(x).astype(np.complex128) @ tf32(2 * eye - y).astype(np.complex128)).astype(np.complex64)
    return x, err


def call(b, x0, its):
    lib = L._lib.load()
    bb = np.ascontiguousarray(np.asarray(b, np.complex64))
    xx = np.ascontiguousarray(np.asarray(x0, np.complex64))
    out = np.zeros((N, N), np.complex64)
    err = np.zeros(1, np.float32)
    st = lib.ldga_selftest_group_inverse(N, bb.ctypes.data_as(C.c_void_p), xx.ctypes.data_as(C.c_void_p), its,
                                         out.ctypes.data_as(C.c_void_p), err.ctypes.data_as(C.c_void_p))
    assert st == L._lib.LDGA_OK, st
    return out, float(err[0])


def _matrices(seed):
    rng = np.random.default_rng(seed)
    g = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))) * 0.08
    d = 1.5 + rng.uniform(0, 1, N) + 0.3j * rng.standard_normal(N)
    b = g + np.diag(d)
    # the seed: the inverse of a neighbouring matrix (another diagonal), as the BSE's per-ω seed is
    b_seed = g + np.diag(d * (1 + 0.05 * rng.standard_normal(N)))
    return b.astype(np.complex64), np.linalg.inv(b_seed).astype(np.complex64)


def test_tcgen05_product_matches_tf32_matmul(require_gpu):
    rng = np.random.default_rng(5)
    b = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    x = (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))).astype(np.complex64)
    got, _ = call(b, x, -1)
    ref = tf32(b).astype(np.complex128) @ tf32(x).astype(np.complex128)
    # FP32 accumulation of 2 x 40 real products per entry
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_tcgen05_newton_schulz_converges(require_gpu):
    for seed in (1, 2, 3):
        b, x0 = _matrices(seed)
        e0 = np.max(np.sum(np.abs(np.eye(N) - b.astype(np.complex128) @ x0), axis=1))
        assert e0 < 0.6, e0
        for its in (0, 1, 3):
            got, err = call(b, x0, its)
            ref, err_ref = ns_emulated(b, x0, its)
            scale = np.max(np.abs(ref))
            assert np.max(np.abs(got - ref)) <= 2e-4 * scale, (seed, its)
            assert abs(err - err_ref) <= 1e-3 * max(err_ref, 1e-3), (seed, its, err, err_ref)
        # three iterations bring the residual to the TF32 level
        got, _ = call(b, x0, 3)
        res = np.max(np.sum(np.abs(np.eye(N) - b.astype(np.complex128) @ got.astype(np.complex128)), axis=1))
        assert res <= max(4 * e0 ** 8, 5e-3), (seed, res, e0)
