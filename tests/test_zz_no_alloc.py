"""The allocation-free GEMM entry point (uw12c_dgemm_noalloc) against the
regular one (uw12c_dgemm) through the C-ABI.

uw12c_dgemm_noalloc serves host programs that cannot let the library
allocate device memory (they reserve the device heap for their own pool, or
run where cudaMalloc/cudaFree would fail or synchronise the device); its
split-K partial tiles live in a fixed 16 MiB device array instead of a
stream-ordered allocation.  Two calls in a row must both reproduce the
regular entry point to the GEMM tolerance of tests/test_gpu_gemm.py
(1e-13 relative to sum |a||b|), including after a call that left other
partial tiles in the shared array.  This file sorts last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL = ctypes.c_longlong


def _bind(lib):
    P = ctypes.c_void_p
    args = [LL, LL, LL, ctypes.c_double, P, LL, ctypes.c_int, P, LL, ctypes.c_int,
            ctypes.c_double, P, LL, LL, LL, ctypes.POINTER(LL), LL, LL, ctypes.POINTER(LL),
            ctypes.c_int]
    for name in ("uw12c_dgemm", "uw12c_dgemm_noalloc"):
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = ctypes.c_int
    lib.uw12c_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    return lib


def _call(lib, name, m, n, k, A, lda, B, ldb, C, ldc, nbo1=1, so=(0,) * 6, split=0, beta=0.0):
    fn = getattr(lib, name)
    return fn(m, n, k, 1.0, ctypes.c_void_p(A.data_ptr()), lda, 0, ctypes.c_void_p(B.data_ptr()),
              ldb, 1, beta, ctypes.c_void_p(C.data_ptr()), ldc, nbo1, 1, (LL * 6)(*so), 1, 1,
              (LL * 4)(0, 0, 0, 0), split)


def _bound(torch, A, B, m, n, k, nbo1):
    a = A.abs().reshape(nbo1, k, m)
    b = B.abs().reshape(nbo1, k, n)
    return torch.einsum("bkm,bkn->bnm", a, b).reshape(-1)


@pytest.fixture(scope="module")
def clib(uw12lib):
    return _bind(ctypes.CDLL(str(uw12lib.library_path())))


def test_noalloc_matches_regular_entry_point_twice(clib, cuda_device):
    import torch
    g = torch.Generator(device=cuda_device)
    g.manual_seed(7)
    shapes = [
        # (m, n, k, nbo1, split): split-K partials in the fixed array
        (200, 192, 40000, 1, 0),
        (130, 70, 9000, 3, 16),
        (200, 192, 40000, 1, 12),
    ]
    for (m, n, k, nbo1, split) in shapes:
        A = torch.randn(nbo1 * m * k, dtype=torch.float64, device=cuda_device, generator=g)
        B = torch.randn(nbo1 * n * k, dtype=torch.float64, device=cuda_device, generator=g)
        so = (m * k, 0, n * k, 0, m * n, 0)
        ref = torch.zeros(nbo1 * m * n, dtype=torch.float64, device=cuda_device)
        assert _call(clib, "uw12c_dgemm", m, n, k, A, m, B, n, ref, m, nbo1, so) == 0
        bound = 1e-13 * _bound(torch, A, B, m, n, k, nbo1)
        for _ in range(2):  # two calls in a row share (and reuse) the scratch
            out = torch.full((nbo1 * m * n,), float("nan"), dtype=torch.float64,
                             device=cuda_device)
            st = _call(clib, "uw12c_dgemm_noalloc", m, n, k, A, m, B, n, out, m, nbo1, so, split)
            assert st == 0
            torch.cuda.synchronize()
            assert bool(torch.all((out - ref).abs() <= bound))


def test_noalloc_rejects_partials_beyond_the_fixed_scratch(clib, cuda_device):
    import torch
    m = n = 1024
    k = 4096
    A = torch.randn(m * k, dtype=torch.float64, device=cuda_device)
    B = torch.randn(n * k, dtype=torch.float64, device=cuda_device)
    C = torch.zeros(m * n, dtype=torch.float64, device=cuda_device)
    # 4 splits of 1024 x 1024 doubles = 4M doubles > 2M doubles of scratch
    st = _call(clib, "uw12c_dgemm_noalloc", m, n, k, A, m, B, n, C, m, split=4)
    assert st == 5
    buf = ctypes.create_string_buffer(512)
    clib.uw12c_last_error(buf, 512)
    assert b"exceeds the fixed scratch" in buf.value
    # an automatic split is reduced until the partial tiles fit
    ref = torch.zeros_like(C)
    assert _call(clib, "uw12c_dgemm", m, n, k, A, m, B, n, ref, m) == 0
    assert _call(clib, "uw12c_dgemm_noalloc", m, n, k, A, m, B, n, C, m) == 0
    torch.cuda.synchronize()
    assert bool(torch.all((C - ref).abs() <= 1e-13 * _bound(torch, A, B, m, n, k, 1)))
