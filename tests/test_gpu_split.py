"""The split-precision GEMM (int8 residues on the tcgen05 tensor cores, CRT
reconstruction) on the GPU.

* Small-integer operands: every step is exact, so the result must equal the
  FP64 product bit for bit (all layouts, odd sizes, several moduli counts).
* Gaussian operands with rows / columns spread over many binades: the error is
  within the scheme's bound 2^-beta (max|a_i.| sum|b_.j| + sum|a_i.| max|b_.j|)
  plus FP64 rounding of the reference.
* Output batches (operands shared or per batch), reduction batches,
  alpha / beta, K beyond one 65536-byte accumulator chunk, and contractions
  long enough to run as several K ranges accumulated in C.
* Whole evaluations with every GEMM routed through the split path: the
  same parity tolerances as the FP64 path against the oracle at 14 moduli,
  and 1e-6 relative at 8 moduli.
"""
import numpy as np
import pytest

from tests.parity_cases import CASES, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _operands(rng, m, n, k, a_k, b_n, ints, spread=0.0):
    lda = (k if a_k else m) + 1
    ldb = (n if b_n else k) + 3
    if ints:
        A = rng.integers(-8, 9, lda * (m if a_k else k)).astype(np.float64)
        B = rng.integers(-8, 9, ldb * (k if b_n else n)).astype(np.float64)
    else:
        A = rng.standard_normal(lda * (m if a_k else k))
        B = rng.standard_normal(ldb * (k if b_n else n))
    Am = A.reshape((lda, m if a_k else k), order="F")
    Bm = B.reshape((ldb, k if b_n else n), order="F")
    if spread:
        # scale rows of A and columns of B over many binades (in place)
        if a_k:
            Am *= np.exp(rng.uniform(-spread, spread, (1, Am.shape[1])))
        else:
            Am *= np.exp(rng.uniform(-spread, spread, (Am.shape[0], 1)))
        if b_n:
            Bm *= np.exp(rng.uniform(-spread, spread, (Bm.shape[0], 1)))
        else:
            Bm *= np.exp(rng.uniform(-spread, spread, (1, Bm.shape[1])))
    Av = Am[:k, :m].T if a_k else Am[:m, :k]
    Bv = Bm[:n, :k].T if b_n else Bm[:k, :n]
    return A, lda, Av, B, ldb, Bv


def _bound(lib, L, Av, Bv, k_total):
    beta = lib.split_bits(L, k_total)
    aa, bb = np.abs(Av), np.abs(Bv)
    return 2.0 ** -beta * (aa.max(1)[:, None] * bb.sum(0)[None, :] +
                           aa.sum(1)[:, None] * bb.max(0)[None, :]) + 1e-15 * (aa @ bb)


@pytest.mark.parametrize("a_k,b_n", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (128, 256, 128), (257, 129, 1000),
                                   (300, 200, 517)])
@pytest.mark.parametrize("L", [6, 14])
def test_integer_products_are_exact(uw12lib, cuda_device, a_k, b_n, m, n, k, L):
    import torch
    rng = np.random.default_rng(m + 3 * n + 7 * k + L)
    A, lda, Av, B, ldb, Bv = _operands(rng, m, n, k, a_k, b_n, ints=True)
    ldc = m + 2
    C = np.full(ldc * n, 7.0)
    dA, dB, dC = _dev(torch, A), _dev(torch, B), _dev(torch, C)
    uw12lib.dgemm_split(m, n, k, 1.0, dA.data_ptr(), lda, a_k, dB.data_ptr(), ldb, b_n, 0.0,
                        dC.data_ptr(), ldc, n_moduli=L)
    torch.cuda.synchronize()
    out = dC.cpu().numpy().reshape((ldc, n), order="F")
    assert np.array_equal(out[:m], Av @ Bv)
    assert np.all(out[m:] == 7.0)  # rows past m untouched


@pytest.mark.parametrize("a_k,b_n", [(False, False), (True, True), (False, True)])
@pytest.mark.parametrize("m,n,k", [(300, 200, 517), (1000, 130, 1500), (64, 700, 2500)])
@pytest.mark.parametrize("L", [8, 12, 16])
def test_gaussian_within_bound(uw12lib, cuda_device, a_k, b_n, m, n, k, L):
    import torch
    rng = np.random.default_rng(m * 7 + n + k + L)
    A, lda, Av, B, ldb, Bv = _operands(rng, m, n, k, a_k, b_n, ints=False, spread=12.0)
    ldc = m
    C = rng.standard_normal(ldc * n)
    Cm = C.reshape((ldc, n), order="F")
    ref = -0.75 * (Av @ Bv) + 0.5 * Cm
    dA, dB, dC = _dev(torch, A), _dev(torch, B), _dev(torch, C)
    uw12lib.dgemm_split(m, n, k, -0.75, dA.data_ptr(), lda, a_k, dB.data_ptr(), ldb, b_n, 0.5,
                        dC.data_ptr(), ldc, n_moduli=L)
    torch.cuda.synchronize()
    out = dC.cpu().numpy().reshape((ldc, n), order="F")
    bound = 0.75 * _bound(uw12lib, L, Av, Bv, k) + 1e-15 * np.abs(Cm)
    assert np.all(np.abs(out - ref) <= bound)


def test_batches_and_reductions(uw12lib, cuda_device):
    """Output batches (A per batch, B shared in dim 1; both per batch in dim 2)
    and reduction batches (2 x 3) summed into C with beta = 1."""
    import torch
    rng = np.random.default_rng(42)
    m, n, k = 150, 90, 70
    nbo1, nbo2, nbr1, nbr2 = 3, 2, 2, 3
    # A: (m, k) blocks at A[i + m*kk + sA...], m-contiguous
    sAr1, sAr2 = m * k, 2 * m * k
    sAo1, sAo2 = 6 * m * k, 18 * m * k
    sBr1, sBr2 = k * n, 2 * k * n
    sBo1, sBo2 = 0, 6 * k * n
    sCo1, sCo2 = m * n, 3 * m * n
    A = rng.standard_normal(36 * m * k)
    B = rng.standard_normal(12 * k * n)
    C = rng.standard_normal(6 * m * n)
    ref = C.copy()
    for b1 in range(nbo1):
        for b2 in range(nbo2):
            acc = np.zeros((m, n))
            for r1 in range(nbr1):
                for r2 in range(nbr2):
                    a0 = b1 * sAo1 + b2 * sAo2 + r1 * sAr1 + r2 * sAr2
                    b0 = b1 * sBo1 + b2 * sBo2 + r1 * sBr1 + r2 * sBr2
                    acc += (A[a0:a0 + m * k].reshape((m, k), order="F") @
                            B[b0:b0 + k * n].reshape((k, n), order="F"))
            c0 = b1 * sCo1 + b2 * sCo2
            blk = ref[c0:c0 + m * n].reshape((m, n), order="F")
            ref[c0:c0 + m * n] = (2.0 * acc + blk).reshape(-1, order="F")
    dA, dB, dC = _dev(torch, A), _dev(torch, B), _dev(torch, C)
    uw12lib.dgemm_split(m, n, k, 2.0, dA.data_ptr(), m, False, dB.data_ptr(), k, False, 1.0,
                        dC.data_ptr(), m, nbo1, nbo2, (sAo1, sAo2, sBo1, sBo2, sCo1, sCo2),
                        nbr1, nbr2, (sAr1, sAr2, sBr1, sBr2), n_moduli=14)
    torch.cuda.synchronize()
    out = dC.cpu().numpy()
    scale = 2.0 * 6 * k * np.max(np.abs(A)) * np.max(np.abs(B)) + np.max(np.abs(C))
    assert np.max(np.abs(out - ref)) <= 1e-12 * scale


def test_long_contraction_uses_several_accumulator_chunks(uw12lib, cuda_device):
    """K = 140000 > 2 x 65536: three K chunks whose residues are summed mod p."""
    import torch
    rng = np.random.default_rng(3)
    m, n, k = 40, 24, 140000
    A = rng.integers(-128, 128, m * k).astype(np.float64)
    B = rng.integers(-128, 128, k * n).astype(np.float64)
    dA, dB = _dev(torch, A), _dev(torch, B)
    dC = torch.zeros(m * n, dtype=torch.float64, device="cuda")
    uw12lib.dgemm_split(m, n, k, 1.0, dA.data_ptr(), m, False, dB.data_ptr(), k, False, 0.0,
                        dC.data_ptr(), m, n_moduli=12)
    torch.cuda.synchronize()
    ref = A.reshape((m, k), order="F") @ B.reshape((k, n), order="F")
    assert np.array_equal(dC.cpu().numpy().reshape((m, n), order="F"), ref)


@pytest.mark.parametrize("nbr1,a_k,b_n", [(1, False, False), (100, True, True)])
def test_contraction_cut_into_k_ranges(uw12lib, cuda_device, nbr1, a_k, b_n):
    """K = 1.2e6 (one range, or 100 reduction batches of 12000): the operands'
    residues (14 x (128 + 256) x K bytes) exceed the temporaries budget, so
    the contraction runs as consecutive K ranges accumulated in C; small
    integers keep every range exact, so the result equals the FP64 product."""
    import torch
    rng = np.random.default_rng(17)
    m, n, k_total = 40, 24, 1_200_000
    k = k_total // nbr1
    Am = rng.integers(-8, 9, (m, k_total)).astype(np.float64)
    Bm = rng.integers(-8, 9, (k_total, n)).astype(np.float64)
    # reduction batch r holds columns [r k, (r + 1) k) of Am and rows of Bm
    if a_k:  # A(i, kk) at A[kk + k i] within each batch of k m elements
        A = np.concatenate([Am[:, r * k:(r + 1) * k].reshape(-1) for r in range(nbr1)])
        lda, sAr1 = k, k * m
    else:
        A = Am.reshape(-1, order="F")
        lda, sAr1 = m, m * k
    if b_n:  # B(kk, j) at B[j + n kk]
        B = Bm.reshape(-1)
        ldb, sBr1 = n, n * k
    else:
        B = Bm.reshape(-1, order="F")
        ldb, sBr1 = k_total, k
    dA, dB = _dev(torch, A), _dev(torch, B)
    dC = torch.full((m * n,), 3.0, dtype=torch.float64, device="cuda")
    uw12lib.dgemm_split(m, n, k, 1.0, dA.data_ptr(), lda, a_k, dB.data_ptr(), ldb, b_n, 0.5,
                        dC.data_ptr(), m, nbr1=nbr1, sr=(sAr1, 0, sBr1, 0) if nbr1 > 1
                        else (0, 0, 0, 0), n_moduli=14)
    torch.cuda.synchronize()
    ref = Am @ Bm + 1.5
    assert np.array_equal(dC.cpu().numpy().reshape((m, n), order="F"), ref)


def test_zero_rows_and_columns(uw12lib, cuda_device):
    import torch
    rng = np.random.default_rng(9)
    m, n, k = 70, 50, 33
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    A[5] = 0.0
    B[:, 7] = 0.0
    dA, dB = _dev(torch, A.reshape(-1, order="F")), _dev(torch, B.reshape(-1, order="F"))
    dC = torch.full((m * n,), 3.0, dtype=torch.float64, device="cuda")
    uw12lib.dgemm_split(m, n, k, 1.0, dA.data_ptr(), m, False, dB.data_ptr(), k, False, 0.0,
                        dC.data_ptr(), m, n_moduli=14)
    torch.cuda.synchronize()
    out = dC.cpu().numpy().reshape((m, n), order="F")
    assert np.all(out[5] == 0.0) and np.all(out[:, 7] == 0.0)
    assert np.max(np.abs(out - A @ B)) <= 1e-12 * np.max(np.abs(A) @ np.abs(B))


def test_bad_moduli_rejected(uw12lib, cuda_device):
    with pytest.raises(uw12lib.UW12Error):
        uw12lib.set_precision(17)
    with pytest.raises(uw12lib.UW12Error):
        uw12lib.dgemm_split(1, 1, 1, 1.0, 0, 1, False, 0, 1, False, 0.0, 0, 1, n_moduli=0)


def _evaluate(lib, d, case, L):
    W = lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = lib.setup_base_integrals(d.WV3, d.WV2)
    A = lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    lib.set_precision(L)
    lib.set_split_threshold(0.0)
    try:
        return lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True, 1.0, 0.5)
    finally:
        lib.set_precision(0)
        lib.set_split_threshold(2e9)


@pytest.mark.parametrize("case", [c for c in CASES if c.name in
                                  ("c0_closed", "uhf_small", "unit_open", "unit_tiles")],
                         ids=lambda c: c.name)
def test_evaluation_split_14_matches_oracle(uw12lib, cuda_device, case):
    from tests.test_gpu_parity import _cmp
    d = make_case(case)
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    e_dir, f_dir, _ = oracle_form_fock(d, False, True, 1.0, 0.5)
    f_scale = float(np.max(np.abs(np.concatenate(f_dir, axis=1))))
    e, f, _ = _evaluate(uw12lib, d, case, 14)
    _cmp(case, e_ref, f_ref, e, f, abs(e_dir), f_scale)


@pytest.mark.parametrize("case", [c for c in CASES if c.name in ("unit_open", "unit_tiles")],
                         ids=lambda c: c.name)
def test_evaluation_split_8_within_1e6(uw12lib, cuda_device, case):
    d = make_case(case)
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    e, f, _ = _evaluate(uw12lib, d, case, 8)
    assert abs(e - e_ref) <= 1e-6 * max(1.0, abs(e_ref))
    for s in range(len(f)):
        assert np.max(np.abs(f[s] - f_ref[s])) <= 1e-5 * max(1.0, np.max(np.abs(f_ref[s])))
