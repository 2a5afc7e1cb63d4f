"""CPU tests of the C-ABI boundary: the library loads, exports every symbol the
public headers declare, and rejects illegal arguments with MAGMA's codes
without touching the GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

from magma_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)        # drop comments
        text = re.sub(r"^\s*#.*?(?<!\\)$", "", text, flags=re.M | re.S)  # drop preprocessor lines
        for m in re.finditer(r"\b(magma\w*|magmablas\w*)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert "magma_dgetrf_batched" in declared
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_bindings_cover_the_header():
    declared = header_functions()
    assert declared == set(_lib.SIGNATURES), (
        f"only in header: {sorted(declared - set(_lib.SIGNATURES))}; "
        f"only in bindings: {sorted(set(_lib.SIGNATURES) - declared)}")


@pytest.fixture(scope="module")
def q():
    """A queue around the null stream: creating it makes no CUDA call."""
    lib = _lib.load()
    h = C.c_void_p()
    lib.magma_queue_create_from_cuda_internal(0, None, None, None, C.byref(h), b"t", b"t", 0)
    yield h


def test_getrf_argument_errors(q):
    lib = _lib.load()
    # batchCount 0 keeps the call off the device; codes follow src/zgetrf_batched.cpp:96-107
    assert lib.magma_dgetrf_batched(-1, 4, None, 4, None, None, 0, q) == -1
    assert lib.magma_dgetrf_batched(4, -1, None, 4, None, None, 0, q) == -2
    assert lib.magma_dgetrf_batched(4, 4, None, 3, None, None, 0, q) == -4
    assert lib.magma_dgetrf_batched(0, 4, None, 1, None, None, 0, q) == 0


def test_getrs_gesv_argument_errors(q):
    lib = _lib.load()
    N, T_ = _lib.MagmaNoTrans, _lib.MagmaTrans
    # src/zgetrs_batched.cpp:99-113
    assert lib.magma_dgetrs_batched(7, 4, 1, None, 4, None, None, 4, 1, q) == -1
    assert lib.magma_dgetrs_batched(N, -1, 1, None, 4, None, None, 4, 1, q) == -2
    assert lib.magma_dgetrs_batched(T_, 4, -1, None, 4, None, None, 4, 1, q) == -3
    assert lib.magma_dgetrs_batched(N, 4, 1, None, 3, None, None, 4, 1, q) == -5
    assert lib.magma_dgetrs_batched(N, 4, 1, None, 4, None, None, 3, 1, q) == -8
    assert lib.magma_dgetrs_batched(N, 0, 1, None, 1, None, None, 1, 1, q) == 0
    # src/zgesv_batched.cpp:107-118
    assert lib.magma_dgesv_batched(-1, 1, None, 4, None, None, 4, None, 1, q) == -1
    assert lib.magma_dgesv_batched(4, -1, None, 4, None, None, 4, None, 1, q) == -2
    assert lib.magma_dgesv_batched(4, 1, None, 3, None, None, 4, None, 1, q) == -4
    assert lib.magma_dgesv_batched(4, 1, None, 4, None, None, 3, None, 1, q) == -6


def test_strerror_and_xerbla(capfd):
    lib = _lib.load()
    assert lib.magma_strerror(-113) == b"cannot allocate memory on GPU device"
    lib.magma_xerbla(b"magma_dgetrf_batched", 4)
    err = capfd.readouterr().err
    assert "On entry to magma_dgetrf_batched, parameter 4 had an illegal value (info = -4)" in err


def test_server_submit_argument_errors():
    """magma_b200_server_submit checks its arguments before it touches the server."""
    lib = _lib.load()
    buf = (C.c_double * 16)()
    p = C.cast(buf, C.c_void_p)
    assert lib.magma_b200_server_submit(None, 2, 4, 1, p, 4, p, 4, p, 4, 0) == -1
    assert lib.magma_b200_server_submit(None, 0, 0, 1, p, 4, p, 4, p, 4, 0) == -2
    assert lib.magma_b200_server_submit(None, 0, 4, 0, p, 4, p, 4, p, 4, 0) == -3
    assert lib.magma_b200_server_submit(None, 1, 4, 1, None, 4, p, 4, p, 4, 0) == -4
    assert lib.magma_b200_server_submit(None, 0, 4, 1, p, 3, p, 4, p, 4, 0) == -5
    assert lib.magma_b200_server_submit(None, 0, 4, 1, p, 4, p, 4, p, 2, 0) == -9
    assert lib.magma_b200_server_submit(None, 0, 2000, 1, p, 2000, p, 2000, p, 2000, 0) == _lib.MAGMA_ERR_NOT_SUPPORTED


def test_cholesky_argument_errors(q):
    lib = _lib.load()
    L, U = _lib.MagmaLower, _lib.MagmaUpper
    # potrf: uplo -1, n -2, ldda -4; batchCount 0 keeps the info reset off the device
    assert lib.magma_dpotrf_batched(7, 4, None, 4, None, 0, q) == -1
    assert lib.magma_dpotrf_batched(L, -1, None, 4, None, 0, q) == -2
    assert lib.magma_dpotrf_batched(U, 4, None, 3, None, 0, q) == -4
    assert lib.magma_dpotrf_batched(L, 0, None, 1, None, 0, q) == 0
    # potrs / posv test every argument in turn and report the last failure,
    # as src/zpotrs_batched.cpp:79-88 and src/zposv_batched.cpp:99-108 do
    for f, tail in ((lib.magma_dpotrs_batched, (1, q)), (lib.magma_dposv_batched, (None, 1, q))):
        assert f(7, 4, 1, None, 4, None, 4, *tail) == -1
        assert f(L, -1, 1, None, 4, None, 4, *tail) == -2
        assert f(L, 4, -1, None, 4, None, 4, *tail) == -3
        assert f(U, 4, 1, None, 3, None, 4, *tail) == -5
        assert f(L, 4, 1, None, 4, None, 3, *tail) == -7
        assert f(7, 4, 1, None, 3, None, 3, *tail) == -7
        assert f(L, 0, 1, None, 1, None, 1, *tail) == 0


def test_mixed_inverse_nopiv_rbt_argument_errors(q):
    lib = _lib.load()
    # magma_dsgesv_batched: n -1, nrhs -2, ldda -4, lddb -7, lddx -9
    f = lib.magma_dsgesv_batched
    assert f(-1, 1, None, 4, None, None, 4, None, 4, None, None, 1, q) == -1
    assert f(4, -1, None, 4, None, None, 4, None, 4, None, None, 1, q) == -2
    assert f(4, 1, None, 3, None, None, 4, None, 4, None, None, 1, q) == -4
    assert f(4, 1, None, 4, None, None, 3, None, 4, None, None, 1, q) == -7
    assert f(4, 1, None, 4, None, None, 4, None, 3, None, None, 1, q) == -9
    assert f(0, 1, None, 1, None, None, 1, None, 1, None, None, 1, q) == 0
    # magma_dgetri_outofplace_batched: n -1, ldda -3, lddia -6
    g = lib.magma_dgetri_outofplace_batched
    assert g(-1, None, 4, None, None, 4, None, 1, q) == -1
    assert g(4, None, 3, None, None, 4, None, 1, q) == -3
    assert g(4, None, 4, None, None, 3, None, 1, q) == -6
    assert g(0, None, 1, None, None, 1, None, 1, q) == 0
    # magma_dgesv_nopiv_batched: n -1, nrhs -2, ldda -4, lddb -6
    h = lib.magma_dgesv_nopiv_batched
    assert h(-1, 1, None, 4, None, 4, None, 1, q) == -1
    assert h(4, -1, None, 4, None, 4, None, 1, q) == -2
    assert h(4, 1, None, 3, None, 4, None, 1, q) == -4
    assert h(4, 1, None, 4, None, 3, None, 1, q) == -6
    # magma_dgerbt_batched: gen -1, n -2, nrhs -3, ldda -5, lddb -7, also written to the
    # host info argument (src/zgerbt_batched.cpp:129-142)
    info = C.c_int(123)
    r = lib.magma_dgerbt_batched
    assert r(5, 4, 1, None, 4, None, 4, None, None, C.byref(info), 1, q) == -1 and info.value == -1
    assert r(_lib.MagmaTrue, -4, 1, None, 4, None, 4, None, None, C.byref(info), 1, q) == -2 and info.value == -2
    assert r(_lib.MagmaFalse, 4, -1, None, 4, None, 4, None, None, C.byref(info), 1, q) == -3
    assert r(_lib.MagmaFalse, 4, 1, None, 3, None, 4, None, None, C.byref(info), 1, q) == -5
    assert r(_lib.MagmaFalse, 4, 1, None, 4, None, 3, None, None, C.byref(info), 1, q) == -7 and info.value == -7
    assert r(_lib.MagmaFalse, 0, 1, None, 1, None, 1, None, None, C.byref(info), 1, q) == 0 and info.value == 0


def test_ptr_array_rejects_host_tensors():
    """The Python binding builds MAGMA's device pointer arrays; a host tensor is an error."""
    import torch

    from magma_b200.api import ptr_array

    with pytest.raises(ValueError):
        ptr_array(torch.zeros((2, 3, 3), dtype=torch.float64))
