"""The FP64 tensor-core GEMM engine against numpy (float64), all operand
layouts, output batches, reduction batches and split-K.  Tolerance: the
result error of an FP64 dot product of length k, 1e-13 relative to
sum |a||b|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("a_k,b_n", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (128, 128, 16), (129, 131, 33),
                                   (300, 70, 517), (64, 1000, 40)])
def test_single(uw12lib, cuda_device, a_k, b_n, m, n, k):
    import torch
    rng = np.random.default_rng(m * 1000 + n * 10 + k)
    lda = (k if a_k else m) + 3
    ldb = (n if b_n else k) + 2
    ldc = m + 1
    A = rng.standard_normal(lda * (m if a_k else k))
    B = rng.standard_normal(ldb * (k if b_n else n))
    C = rng.standard_normal(ldc * n)
    Am = A.reshape((lda, m if a_k else k), order="F")
    Am = Am[:k, :m].T if a_k else Am[:m, :k]
    Bm = B.reshape((ldb, k if b_n else n), order="F")
    Bm = Bm[:n, :k].T if b_n else Bm[:k, :n]
    Cm = C.reshape((ldc, n), order="F")[:m, :]
    ref = 1.5 * Am @ Bm - 0.5 * Cm
    dA, dB, dC = _dev(torch, A), _dev(torch, B), _dev(torch, C)
    uw12lib.dgemm(m, n, k, 1.5, dA.data_ptr(), lda, a_k, dB.data_ptr(), ldb, b_n, -0.5,
                  dC.data_ptr(), ldc)
    torch.cuda.synchronize()
    out = dC.cpu().numpy().reshape((ldc, n), order="F")[:m, :]
    scale = 1.5 * np.abs(Am) @ np.abs(Bm) + 0.5 * np.abs(Cm)
    assert np.all(np.abs(out - ref) <= 1e-13 * scale + 1e-300)
    # padding rows untouched
    assert np.array_equal(dC.cpu().numpy().reshape((ldc, n), order="F")[m:, :],
                          C.reshape((ldc, n), order="F")[m:, :])


@pytest.mark.parametrize("a_k,b_n", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", [(129, 131, 33), (255, 97, 1001), (64, 300, 65)])
def test_sixteen_byte_copies(uw12lib, cuda_device, a_k, b_n, m, n, k):
    """Even leading dimensions select the 16-byte copy path; odd extents make
    the last copy of a row partial (8 bytes copied, 8 zero-filled)."""
    import torch
    rng = np.random.default_rng(m + 7 * n + 11 * k)
    lda = (k if a_k else m) + 1
    lda += lda % 2
    ldb = (n if b_n else k) + 1
    ldb += ldb % 2
    A = rng.standard_normal(lda * (m if a_k else k))
    B = rng.standard_normal(ldb * (k if b_n else n))
    Am = A.reshape((lda, m if a_k else k), order="F")
    Am = Am[:k, :m].T if a_k else Am[:m, :k]
    Bm = B.reshape((ldb, k if b_n else n), order="F")
    Bm = Bm[:n, :k].T if b_n else Bm[:k, :n]
    dA, dB = _dev(torch, A), _dev(torch, B)
    dC = torch.zeros(m * n, dtype=torch.float64, device=cuda_device)
    uw12lib.dgemm(m, n, k, 1.0, dA.data_ptr(), lda, a_k, dB.data_ptr(), ldb, b_n, 0.0,
                  dC.data_ptr(), m)
    torch.cuda.synchronize()
    out = dC.cpu().numpy().reshape((m, n), order="F")
    assert np.all(np.abs(out - Am @ Bm) <= 1e-13 * (np.abs(Am) @ np.abs(Bm)) + 1e-300)


@pytest.mark.parametrize("split", [0, 1, 3, 7])
def test_batched_and_reduction(uw12lib, cuda_device, split):
    import torch
    rng = np.random.default_rng(5)
    m, n, k = 37, 45, 21
    nb1, nb2, nr1, nr2 = 3, 2, 4, 5
    # A[bo, r] : m x k col-major at offset bo1*sAo1 + bo2*sAo2 + r1*sAr1 + r2*sAr2
    A = rng.standard_normal((nb2, nb1, nr2, nr1, k, m))  # C-order: innermost m
    B = rng.standard_normal((nb2, nb1, nr2, nr1, n, k))
    C = np.zeros((nb2, nb1, n, m))
    sA = [m * k * nr1 * nr2, m * k * nr1 * nr2 * nb1, m * k, m * k * nr1]
    sB = [n * k * nr1 * nr2, n * k * nr1 * nr2 * nb1, n * k, n * k * nr1]
    dA, dB, dC = _dev(torch, A), _dev(torch, B), _dev(torch, C)
    uw12lib.dgemm(m, n, k, 1.0, dA.data_ptr(), m, False, dB.data_ptr(), k, False, 0.0,
                  dC.data_ptr(), m, nbo1=nb1, nbo2=nb2,
                  so=(sA[0], sA[1], sB[0], sB[1], m * n, m * n * nb1),
                  nbr1=nr1, nbr2=nr2, sr=(sA[2], sA[3], sB[2], sB[3]), split=split)
    torch.cuda.synchronize()
    out = dC.cpu().numpy()
    for b2 in range(nb2):
        for b1 in range(nb1):
            ref = np.zeros((m, n))
            for r2 in range(nr2):
                for r1 in range(nr1):
                    Am = A[b2, b1, r2, r1].T  # (m, k)
                    Bm = B[b2, b1, r2, r1].T  # (k, n)
                    ref += Am @ Bm
            got = out[b2, b1].T
            assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_empty_contraction_scales_c(uw12lib, cuda_device):
    import torch
    C = np.arange(12.0)
    dC = _dev(torch, C)
    uw12lib.dgemm(3, 4, 0, 1.0, 0, 3, False, 0, 1, False, 2.0, dC.data_ptr(), 3)
    torch.cuda.synchronize()
    assert np.array_equal(dC.cpu().numpy(), 2.0 * C)
