"""The allocation-free lambda_0 entry point (ldga_lambda0_noalloc) against ldga_lambda0.

Some callers cannot allocate device memory -- a host application that hands all device memory to
its own pool allocator, or code that enqueues work while a stream capture forbids cudaMalloc.  For
them ldga_lambda0_noalloc computes lambda_0 from caller-provided device buffers with its scratch in
a built-in device array.  This file is collected last (tests/test_zz_*) so that a run stopping at
the first failure has already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import ladderdga_b200 as L
from ladderdga_b200 import synthetic as S

pytestmark = pytest.mark.gpu

RTOL = 1e-10   # the tolerance every lambda_0 parity check uses


def test_lambda0_noalloc_matches_handle_path(require_gpu):
    import torch

    inp = S.make_input(dim=3, ns=8, beta=5.0, U=1.2, n_iv=4, n_iw=4, seed=91)
    h = L.setup_synthetic(inp)
    ctx = h.ctx
    chi0 = L.calc_bubble(h)
    l0_ref = np.asarray(L.calc_λ0(chi0, h))                       # existing entry point (ldga_lambda0)
    F = L.F_from_χ("m", h)                                         # F_m [Nnu, Nnu, Nw]

    dev = torch.device("cuda", ctx.device)
    chi0_d = torch.from_numpy(np.ascontiguousarray(chi0.data.reshape(-1, order="F")).view(np.float64)).to(dev)
    F_d = torch.from_numpy(np.ascontiguousarray(F.reshape(-1, order="F")).view(np.float64)).to(dev)
    lib = L._lib.load()
    for call in range(2):                                          # two calls in a row share the scratch
        out = torch.full((ctx.Nq * ctx.Nnu * ctx.Nw * 2,), float("nan"), dtype=torch.float64, device=dev)
        st = lib.ldga_lambda0_noalloc(C.c_void_p(chi0_d.data_ptr()), C.c_void_p(F_d.data_ptr()), ctx.Nq,
                                      ctx.Nnu, ctx.Nw, h.mP.β, C.c_void_p(out.data_ptr()), None)
        assert st == L._lib.LDGA_OK, lib.ldga_last_error(None).decode()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy().view(np.complex128).reshape((ctx.Nq, ctx.Nnu, ctx.Nw), order="F")
        err = np.max(np.abs(got - l0_ref)) / np.max(np.abs(l0_ref))
        assert err <= RTOL, (call, err)


def test_lambda0_noalloc_rejects_oversize(require_gpu):
    import torch

    lib = L._lib.load()
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(d.data_ptr())
    st = lib.ldga_lambda0_noalloc(p, p, 1, 200, 201, 10.0, p, None)   # 200*201 columns > 32768
    assert st == L._lib.LDGA_ERR_ARG
    assert "exceeds" in lib.ldga_last_error(None).decode()
