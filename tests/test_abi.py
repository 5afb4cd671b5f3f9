"""The C ABI boundary without a GPU: the library loads, exports every entry point the header
declares, its structs have the header's layout, and argument errors come back as status codes."""
import ctypes as C
import re
import subprocess
import sys
from pathlib import Path

import pytest

import ladderdga_b200 as L
from ladderdga_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ldga_b200.h"
PKG = ROOT / "ladderdga.jl_b200"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(ldga_\w+)\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    if not _lib.LIB_PATH.exists():                     # build in-tree (nvcc cross-compiles without a GPU)
        subprocess.run([sys.executable, str(PKG / "build.py")], check=True, cwd=ROOT)
    return _lib.load()


def test_header_declares_binding_list():
    assert header_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (ldga_\w+)$", out, flags=re.M))
    assert exported == set(header_functions())


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "ldga_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(ldga_lattice), sizeof(ldga_model),'
        ' sizeof(ldga_sim), offsetof(ldga_lattice, t), offsetof(ldga_sim, fft_lo),'
        ' offsetof(ldga_sim, usable_prct_reduction), offsetof(ldga_sim, dbg_full_eom_omega)); return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(_lib.Lattice), C.sizeof(_lib.Model), C.sizeof(_lib.Sim), _lib.Lattice.t.offset,
            _lib.Sim.fft_lo.offset, _lib.Sim.usable_prct_reduction.offset, _lib.Sim.dbg_full_eom_omega.offset]
    assert got == want


def test_header_compiles_as_cxx(tmp_path):
    src = tmp_path / "h.cpp"
    src.write_text('#include "ldga_b200.h"\nint main(){ return LDGA_OK; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o",
                    str(tmp_path / "h")], check=True)


def test_status_strings_and_version(lib):
    assert lib.ldga_version() >= 1
    names = [lib.ldga_status_string(s).decode() for s in range(7)]
    assert names[0] == "ok" and len(set(names)) == 7
    assert lib.ldga_status_string(99).decode()


def _structs(**kw):
    lat = _lib.Lattice(kw.get("dim", 2), kw.get("ns", 8), 1.0, 0.0, 0.0)
    mp = _lib.Model(1.0, 0.5, 10.0, 1.0, 0.0, 0.0, 0.5)
    n_iv, n_iw = kw.get("n_iv", 4), kw.get("n_iw", 4)
    lo, hi = kw.get("fft", (-(n_iv + n_iw) * 2 - 1, 2 * (n_iv + n_iw)))
    sp = _lib.Sim(n_iw, n_iv, kw.get("shell", 0), 0, lo, hi, 0.1, 0)
    return lat, mp, sp


@pytest.mark.parametrize("kw,code,msg", [
    ({"dim": 4}, _lib.LDGA_ERR_ARG, "dimension"),
    ({"ns": 0}, _lib.LDGA_ERR_ARG, "points per axis"),
    ({"n_iv": 0}, _lib.LDGA_ERR_ARG, "n_iv"),
    ({"shell": 2}, _lib.LDGA_ERR_ARG, "plain path"),
    ({"fft": (-2, 2)}, _lib.LDGA_ERR_ARG, "fft_range"),
])
def test_create_rejects_bad_arguments(lib, kw, code, msg):
    lat, mp, sp = _structs(**kw)
    h = C.c_void_p()
    assert lib.ldga_create(C.byref(lat), C.byref(mp), C.byref(sp), _lib.PREC_FP64, 0, C.byref(h)) == code
    assert msg in lib.ldga_last_error(None).decode()
    assert not h.value


def test_create_bad_precision(lib):
    lat, mp, sp = _structs()
    h = C.c_void_p()
    assert lib.ldga_create(C.byref(lat), C.byref(mp), C.byref(sp), 7, 0, C.byref(h)) == _lib.LDGA_ERR_ARG


def test_create_without_gpu_fails_cleanly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lat, mp, sp = _structs()
    h = C.c_void_p()
    assert lib.ldga_create(C.byref(lat), C.byref(mp), C.byref(sp), _lib.PREC_FP64, 0, C.byref(h)) == _lib.LDGA_ERR_CUDA
    assert "no CUDA device" in lib.ldga_last_error(None).decode()


def test_null_handle_is_an_argument_error(lib):
    assert lib.ldga_destroy(None) == _lib.LDGA_OK
    for name, args in [("ldga_bubble", (None,)), ("ldga_set_precision", (1,)), ("ldga_lambda_min", (0, None)),
                       ("ldga_sum_kw", (0, 0.0, 0, None))]:
        assert getattr(lib, name)(None, *args) == _lib.LDGA_ERR_ARG, name


def test_noalloc_argument_checks_need_no_gpu(lib):
    # argument validation precedes every CUDA call
    assert lib.ldga_lambda0_noalloc(None, None, 1, 1, 1, 1.0, None, None) == _lib.LDGA_ERR_ARG
    p = C.c_void_p(16)
    assert lib.ldga_lambda0_noalloc(p, p, 0, 4, 5, 1.0, p, None) == _lib.LDGA_ERR_ARG
    assert lib.ldga_lambda0_noalloc(p, p, 1, 200, 201, 1.0, p, None) == _lib.LDGA_ERR_ARG
    assert "exceeds" in lib.ldga_last_error(None).decode()


def test_missing_library_fails_loudly():
    code = ("import sys; sys.path.insert(0, %r); import ladderdga_b200 as L; from pathlib import Path;"
            "L._lib.LIB_PATH = Path('/nonexistent/libldga_b200.so');"
            "\ntry:\n    L._lib.load()\nexcept L._lib.LibraryMissing as e:\n    print('missing', e)\n" % str(ROOT))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    assert out.startswith("missing") and "no CPU fallback" in out


def test_product_never_imports_the_oracle():
    for f in list(PKG.rglob("*.py")) + list(PKG.rglob("*.cu")) + list(PKG.rglob("*.cuh")) + [ROOT / "ladderdga_b200.py"]:
        text = f.read_text()
        assert not re.search(r"^\s*(from|import)\s+oracle", text, flags=re.M), f
        assert "ldga_ref" not in text, f


def test_no_closed_copy_calls_in_sources():
    # batched memcpy entry points are closed on the target machines; keep every source free of them
    pat = re.compile(r"Memcpy(3D)?Batch")
    for f in list(PKG.rglob("*.cu")) + list(PKG.rglob("*.cuh")) + list(PKG.rglob("*.py")) + [ROOT / "bench.py"]:
        assert not pat.search(f.read_text()), f


def test_ptr_keeps_temporaries_alive():
    """ptr(as_fc(x)) of a C-ordered array makes a temporary Fortran copy; the returned pointer must
    keep it alive until the C call has read it (CPython frees unreferenced temporaries at once)."""
    import gc
    import numpy as np
    from ladderdga_b200 import _lib
    x = np.arange(24, dtype=np.complex128).reshape(2, 3, 4)       # C order: as_fc copies
    p = _lib.ptr(_lib.as_fc(x))
    gc.collect()
    junk = [np.full(24, -1.0 + 0j) for _ in range(64)]            # reuse freed blocks if any
    import ctypes as C
    got = np.ctypeslib.as_array((C.c_double * 48).from_address(p.value)).view(np.complex128)
    assert np.array_equal(got, np.asfortranarray(x).reshape(-1, order="F"))
    del junk


def test_tune_cache_roundtrip(tmp_path):
    """BSE configuration choices: a cache file is read by name (unknown lines and names ignored) and
    written back with the same entries; no GPU is needed for the registry."""
    import ladderdga_b200 as L
    src = tmp_path / "tune.txt"
    src.write_text("# comment\nbse 40 1 lu8:5\nbse 60 2 lu32x16:2\nbse 40 2 no-such-config\ngarbage line\n")
    L.tune_load(src)
    out = tmp_path / "out.txt"
    L.tune_save(out)
    lines = [l for l in out.read_text().splitlines() if not l.startswith("#")]
    assert "bse 40 1 lu8:5" in lines and "bse 60 2 lu32x16:2" in lines
    assert not any("no-such-config" in l for l in lines)
    # back to the defaults for the rest of the session
    L.tune_reset()
    L.tune_save(out)
    assert [l for l in out.read_text().splitlines() if not l.startswith("#")] == []
