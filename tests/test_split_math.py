"""The arithmetic of the split-precision GEMM, restated on the CPU.

The CUDA path scales rows of A / columns of B to beta-bit integers, multiplies
their residues modulo L coprime moduli <= 256 exactly (int8 x int8 -> int32),
and rebuilds the integer product with the Chinese remainder theorem in FP64
on 36-bit chunks.  These tests replay each step with numpy / Python integers,
using the library's own beta (uw12c_split_bits), and check that
  * the moduli are pairwise coprime and their residues fit int8,
  * the chunked FP64 CRT reconstruction recovers every integer |C'| <= M/4
    (every partial sum exact, below 2^53); the error-free join returns it
    exactly when it is a double and within one ulp otherwise,
  * the K-chunk bound keeps the int32 accumulator within +-2^30,
  * the end-to-end error stays within 2^-beta of the operand scales.
"""
import math
from fractions import Fraction

import numpy as np
import pytest

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193]
MAX_CHUNK_BITS = 41  # r (< 2^8) * chunk summed over <= 16 moduli stays below 2^53
K_CHUNK = 65536


def chunking(L):
    bits = math.prod(MODULI[:L]).bit_length()
    nch = -(-bits // MAX_CHUNK_BITS)
    return nch, -(-bits // nch)


def fma(a, b, c):
    """Correctly rounded a * b + c (math.fma needs Python 3.13)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def consts(L):
    M = math.prod(MODULI[:L])
    nch, cw = chunking(L)
    mask = (1 << cw) - 1
    w = []
    for p in MODULI[:L]:
        Ml = M // p
        y = pow(Ml % p, -1, p)
        wl = Ml * y
        assert wl < M
        w.append([float((wl >> (cw * c)) & mask) for c in range(nch)])
    mc = [float((M >> (cw * c)) & mask) for c in range(nch)]
    return M, nch, cw, np.array(w), np.array(mc), 1.0 / float(M)


def crt_fp64(res, L):
    """The reconstruction kernel's arithmetic for one element: res[l] in [0, p_l)."""
    M, nch, cw, w, mc, inv_m = consts(L)
    S = [0.0] * nch
    for l in range(L):
        for c in range(nch):
            S[c] = fma(float(res[l]), w[l][c], S[c])
            assert abs(S[c]) < 2.0 ** 53
    approx = 0.0
    for c in range(nch - 1, -1, -1):
        approx = fma(approx, 2.0 ** cw, S[c])
    q = (approx * inv_m + ROUND) - ROUND  # rint: ties cannot occur (|C'| <= M/4)
    terms = []
    for c in range(nch):
        d = fma(-q, mc[c], S[c])
        assert abs(d) < 2.0 ** 53 and d == int(d)
        terms.append(d * 2.0 ** (cw * c))  # exact power-of-two scaling
    # error-free running sum (TwoSum), integer errors added at the end
    total, err = terms[-1], 0.0
    for t in reversed(terms[:-1]):
        s_ = total + t
        bb = s_ - total
        err += (total - (s_ - bb)) + (t - bb)
        total = s_
    return total + err


ROUND = 1.5 * 2.0 ** 52


def residue_byte(v, p):
    """The preparation kernel's residue: q = fma(v, 1/p, 1.5 2^52) - 1.5 2^52,
    r = v - q p (exact), then the low byte of r read as int8."""
    q = fma(v, 1.0 / p, ROUND) - ROUND
    r = int(fma(-q, float(p), v))
    assert -(p // 2) <= r <= p // 2  # q is exactly rint(v / p)
    return (r + 128) % 256 - 128


def test_moduli_pairwise_coprime_and_fit_int8():
    for a in range(16):
        for b in range(a):
            assert math.gcd(MODULI[a], MODULI[b]) == 1
    rng = np.random.default_rng(0)
    for p in MODULI:
        vals = list(rng.integers(-2 ** 50, 2 ** 50, 2000)) + [p // 2, -(p // 2), p, -p, 0]
        # values whose quotient is closest to a half-integer, at the top of the range
        vals += [2 ** 50 // p * p + p // 2 - t for t in range(3)]
        vals += [-(2 ** 50 // p * p + p // 2 - t) for t in range(3)]
        for v in vals:
            r = residue_byte(float(v), p)
            assert -128 <= r <= 127 and (r - int(v)) % p == 0


@pytest.mark.parametrize("L", [6, 8, 10, 12, 14, 16])
def test_chunked_crt_is_exact(L):
    M = math.prod(MODULI[:L])
    rng = np.random.default_rng(L)
    vals = [0, 1, -1, M // 4, -(M // 4), M // 4 - 12345, 2 ** 53 + 1, -(2 ** 60) - 3]
    # exact small-integer products scaled by large powers of two (the integer tests)
    vals += [c * 2 ** s for c in (-70, 3, 127, -4097) for s in (40, 60, 80, 97, 100)]
    vals += [int(x) for x in rng.integers(-2 ** 62, 2 ** 62, 200)]
    vals += [int(rng.integers(0, 2 ** 62)) * int(rng.integers(0, 2 ** 40)) % (M // 4) *
             (1 if i % 2 else -1) for i in range(200)]
    for x in vals:
        if abs(x) > M // 4:
            continue
        res = [x % p for p in MODULI[:L]]
        got = crt_fp64(res, L)
        if float(x) == x:  # representable: exact
            assert got == float(x), (L, x, got)
        else:  # within one unit in the last place
            assert abs(Fraction(got) - x) <= math.ulp(float(x)), (L, x, got)


def test_library_bits_match_bound(uw12lib):
    for L in (4, 8, 12, 14, 16):
        M = math.prod(MODULI[:L])
        for k_total in (1, 100, 1500, 2500, 65536, 1_600_000):
            beta = uw12lib.split_bits(L, k_total)
            assert beta <= 50  # |A'| <= 2^50 keeps the FP64 rounding tricks exact
            if beta >= 1:
                # |C'| <= k 2^(2 beta) <= M / 4
                assert k_total * 2 ** (2 * beta) <= M // 4
                assert (2 * k_total) * 2 ** (2 * (beta + 1)) > M // 4 or beta == 50


def test_accumulator_bound():
    assert K_CHUNK * 128 * 128 == 2 ** 30
    # offset trick of the epilogue: acc + off stays in uint32 for every modulus
    for p in MODULI:
        off = ((1 << 30) + p - 1) // p * p
        assert off % p == 0 and off >= 2 ** 30 and 2 ** 30 + off < 2 ** 32


@pytest.mark.parametrize("L", [8, 14])
def test_end_to_end_replay(uw12lib, L):
    """Scale, residues, exact modular products, CRT: error within 2^-beta scales."""
    rng = np.random.default_rng(5)
    m, n, k = 7, 5, 300
    A = rng.standard_normal((m, k)) * np.exp(rng.uniform(-20, 20, (m, 1)))
    B = rng.standard_normal((k, n)) * np.exp(rng.uniform(-5, 5, (1, n)))
    A[2] = 0.0
    beta = uw12lib.split_bits(L, k)
    ea = np.array([math.frexp(np.max(np.abs(r)))[1] if np.any(r) else 0 for r in A])
    eb = np.array([math.frexp(np.max(np.abs(c)))[1] if np.any(c) else 0 for c in B.T])
    sa = np.where(np.any(A, axis=1), beta - ea, 0)
    sb = np.where(np.any(B, axis=0), beta - eb, 0)
    Ai = (np.ldexp(A, sa[:, None]) + ROUND) - ROUND
    Bi = (np.ldexp(B, sb[None, :]) + ROUND) - ROUND
    C = np.zeros((m, n))
    for i in range(m):
        for j in range(n):
            res = []
            for p in MODULI[:L]:
                ra = [residue_byte(x, p) for x in Ai[i]]
                rb = [residue_byte(x, p) for x in Bi[:, j]]
                acc = sum(x * y for x, y in zip(ra, rb))
                assert abs(acc) <= 2 ** 30
                res.append(acc % p)
            C[i, j] = math.ldexp(crt_fp64(res, L), -int(sa[i] + sb[j]))
    exact = A @ B
    bound = 2.0 ** -beta * (np.max(np.abs(A), axis=1)[:, None] * np.abs(B).sum(0)[None, :] +
                            np.abs(A).sum(1)[:, None] * np.max(np.abs(B), axis=0)[None, :])
    assert np.all(np.abs(C - exact) <= bound + 1e-300)
    assert np.all(C[2] == 0.0)
