"""C-ABI surface, host-side logic and input generators.  CPU only: no
compute call touches a GPU here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "powergrid_b200.h")


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pg_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from powergrid_b200 import build as B
    B.build()
    from powergrid_b200 import _lib
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = _declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from powergrid_b200 import _lib
    assert set(_declared_functions()) <= set(_lib.SIGNATURES)


def test_status_strings(lib):
    lib.pg_status_string.restype = C.c_char_p
    assert lib.pg_status_string(0) == b"PG_OK"
    assert lib.pg_status_string(8) == b"PG_REJECTED"


def test_product_kb_lut_equals_oracle(lib, oracle):
    """The product builds the same Kaiser-Bessel table as the reference (host code, no GPU)."""
    from powergrid_b200 import _lib
    out = np.zeros(40000, np.float32)
    beta = C.c_float()
    n = lib.pg_util_kb_lut(C.c_float(2.0), out.ctypes.data_as(C.c_void_p), out.size, C.byref(beta))
    ref, rbeta = oracle.kb_lut(0)
    assert n == 40000
    assert np.array_equal(out, ref)
    assert np.float32(beta.value) == np.float32(rbeta)
    _ = _lib


def test_no_cpu_fallback_without_gpu():
    """Without a GPU the operators refuse to run (no silent CPU path)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import powergrid_b200 as P
    from powergrid_b200._lib import PGError
    kx = np.zeros(4, np.float32)
    with pytest.raises(PGError):
        P.Gnufft(4, 2.0, 8, 8, 1, kx, kx, kx)


def test_synthetic_inputs_are_deterministic():
    from powergrid_b200 import synthetic as S
    a = S.config1()
    b = S.config1()
    assert np.array_equal(a.kx, b.kx) and np.array_equal(a.x_true, b.x_true)
    r = S.Rng(42)
    v = r.bits(3)
    assert v.dtype == np.uint64 and len(set(v.tolist())) == 3
    assert np.abs(a.kx).max() < 32 and np.abs(a.ky).max() < 32


def test_config_shapes():
    from powergrid_b200 import synthetic as S
    c2 = S.config2()
    assert c2.kx.size == 131072 and c2.nc == 4 and c2.L == 8 and c2.nimg == 128 * 128
    assert np.abs(c2.fm).max() <= 2 * np.pi * 100 + 1e-3
    assert abs(float(c2.t.max()) - 20e-3) < 1e-5
