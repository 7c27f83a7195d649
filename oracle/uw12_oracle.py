"""CPU oracle for the UW12 energy + Fock path -- TEST INFRASTRUCTURE ONLY.

This module is a plain-numpy restatement of libuw12's algorithm, written
operation for operation after the reference sources (each function cites the
file:line it follows, paths relative to the libuw12 project root).  It is the
checker for the CUDA path: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.  The
product (``libuw12_b200``) never calls it and has no CPU fallback.

Parity pinning.  The oracle is pinned to libuw12 itself: ``oracle/ref.mk``
compiles libuw12's unmodified sources (over this project's Armadillo-subset
header, ``oracle/refshim/``) into ``oracle/_ref/libuw12_ref.so``, and
``tests/golden/make_golden.py`` records that build's energies, per-term
energies, Fock matrices, ABS+ projector blocks at the eigenvalue drop
threshold and exception classes/messages in ``tests/golden/`` (with the
SHA-256 of every reference source it compiled).  ``tests/test_reference_goldens.py``
checks this module against every golden (tolerances 1e-12 relative on
well-conditioned inputs and 1e-9 on the workload generators, whose metrics
have condition numbers near 1e6; observed 1e-15 and 3e-11 to 6e-11).  The oracle is also checked against the reference's own
known-answer and invariant tests (spin factors, square/lower, os+ss
linearity, open==closed shell, W<->V symmetry, zero cases, analytic Fock ==
finite-difference dE/dD) in ``tests/test_oracle.py``.  libuw12's one absolute
golden, the water fixture (``tests/test_water.cpp``), cannot run: its RI
tensors (``W3_ri.csv``/``V3_ri.csv``) are not shipped.

Layout conventions follow Armadillo: matrices are column-major, every
``reshape`` reinterprets a column-major buffer (``order='F'``), packed
symmetric vectors store the lower triangle row by row,
``idx(i, j<=i) = i(i+1)/2 + j`` (``src/utils/utils.hpp:23-48``).

Heavy loops (the reference's ``parallel_for`` / ``parallel_sum`` /
``parallel_sum_2d`` over aux functions and orbital pairs) iterate through
``Sampler.range``.  With the default sampler every iteration runs.  A timing
sampler runs a bounded subset and extrapolates the loop time; its numeric
results are then meaningless and are only used by the CPU-baseline timer.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

DBL_EPS = np.finfo(np.float64).eps


class UW12RuntimeError(RuntimeError):
    """Mirrors the reference's ``std::runtime_error`` (user-input errors)."""


class UW12LogicError(ValueError):
    """Mirrors the reference's ``std::logic_error`` (shape errors)."""


# --------------------------------------------------------------------------
# loop sampling (timing only)
# --------------------------------------------------------------------------
class Sampler:
    """Iteration source for the reference's parallel loops.

    ``max_iters=None`` runs every iteration.  Otherwise at most ``max_iters``
    evenly spaced iterations run and ``extra_seconds`` accumulates the
    extrapolated time of the skipped ones (loop time * (n/k - 1)); large
    products (``matmul``) likewise compute a leading block of rows and
    extrapolate by the row count.
    """

    def __init__(self, max_iters: Optional[int] = None, min_rows: int = 2048):
        self.max_iters = max_iters
        self.min_rows = min_rows
        self.extra_seconds = 0.0
        self.loops = 0

    def matmul(self, A: np.ndarray, B: np.ndarray) -> np.ndarray:
        if self.max_iters is None:
            return A @ B
        n = A.shape[0]
        k = min(n, max(self.min_rows, n // 64))
        if k == n:
            return A @ B
        out = np.zeros((n, B.shape[1]))
        t0 = time.perf_counter()
        out[:k] = A[:k] @ B
        self.extra_seconds += (time.perf_counter() - t0) * (n / k - 1.0)
        return out

    def range(self, n: int):
        n = int(n)
        if self.max_iters is None or n <= self.max_iters:
            yield from range(n)
            return
        k = max(1, int(self.max_iters))
        idx = np.unique(np.linspace(0, n - 1, k).astype(np.int64))
        t0 = time.perf_counter()
        for i in idx:
            yield int(i)
        dt = time.perf_counter() - t0
        self.extra_seconds += dt * (n / len(idx) - 1.0)
        self.loops += 1

    def range2d(self, n1: int, n2: int):
        for flat in self.range(n1 * n2):
            yield flat // n2 if n2 else 0, flat % n2 if n2 else 0


FULL = Sampler(None)


# --------------------------------------------------------------------------
# utils.hpp / linalg.hpp
# --------------------------------------------------------------------------
def nearly_zero(value: float, epsilon: int = 4) -> bool:
    """``utils::nearly_zero`` (src/utils/utils.hpp:186-189)."""
    return abs(value) <= epsilon * DBL_EPS


def spin_channels(obj) -> int:
    """``utils::spin_channels`` (src/utils/utils.hpp:198-205)."""
    n = len(obj)
    if n < 1 or n > 2:
        raise UW12LogicError("invalid number of spin channels")
    return n


def packed_size(n: int) -> int:
    return n * (n + 1) // 2


def n_from_packed(n1: int) -> int:
    """Inverse of n(n+1)/2 as in ``square`` (src/utils/utils.hpp:24-29)."""
    n2 = int(math.sqrt(8 * n1 - 1) / 2) if n1 > 0 else 0
    if n2 * (n2 + 1) // 2 != n1:
        raise UW12LogicError("vector must be of length n(n+1)/2")
    return n2


def square(vec: np.ndarray, factor: float = 1.0) -> np.ndarray:
    """Packed lower triangle -> symmetric matrix (src/utils/utils.hpp:23-48)."""
    vec = np.asarray(vec, dtype=np.float64).reshape(-1)
    n = n_from_packed(vec.size)
    rows, cols = np.tril_indices(n)
    out = np.zeros((n, n))
    out[rows, cols] = factor * vec
    out[cols, rows] = factor * vec
    diag = rows == cols
    out[rows[diag], cols[diag]] = vec[diag]
    return out


def is_symmetric(mat: np.ndarray, threshold: float = 1e-10) -> bool:
    """``linalg::is_symmetric`` (src/utils/linalg.hpp:309-330)."""
    if mat.ndim != 2 or mat.shape[0] != mat.shape[1]:
        return False
    if mat.size == 0:
        return True
    scale = max(1.0, float(np.max(np.abs(mat))))
    return float(np.max(np.abs(mat - mat.T))) <= threshold * scale


def lower(mat: np.ndarray, factor: float = 1.0) -> np.ndarray:
    """Symmetric matrix -> packed lower triangle (src/utils/utils.hpp:58-79)."""
    if mat.ndim != 2 or mat.shape[0] != mat.shape[1]:
        raise UW12LogicError("matrix is not square")
    if not is_symmetric(mat):
        raise UW12LogicError("matrix is not symmetric")
    n = mat.shape[0]
    rows, cols = np.tril_indices(n)
    vec = mat[rows, cols].astype(np.float64)
    vec = np.where(rows == cols, vec, factor * vec)
    return vec


def symmetrise(f: np.ndarray) -> np.ndarray:
    """``symmetrise_fock`` for one spin block (src/utils/utils.hpp:215-224)."""
    return 0.5 * (f + f.T)


def eigen_system(mat: np.ndarray):
    """``linalg::eigen_system`` -- ascending eigenpairs (linalg.hpp:1112-1146)."""
    if mat.ndim != 2 or mat.shape[0] != mat.shape[1]:
        raise UW12LogicError("matrix must be square")
    if not is_symmetric(mat):
        raise UW12LogicError("matrix must be symmetric")
    vals, vecs = np.linalg.eigh(mat)
    return vals, vecs


def eigen_decomposition(mat: np.ndarray, ld_threshold: float, eig_ld_threshold: float):
    """Eigenpairs with linear-dependency removal (linalg.hpp:1157-1197).

    Keeps ``|lambda| > max(max|lambda| * eig_ld_threshold, ld_threshold)``.
    """
    vals, vecs = eigen_system(mat)
    if ld_threshold > 0 or eig_ld_threshold > 0:
        max_eig = float(np.max(np.abs(vals))) if vals.size else 0.0
        threshold = max(max_eig * eig_ld_threshold, ld_threshold)
        keep = np.abs(vals) > threshold
        return vals[keep], vecs[:, keep]
    return vals, vecs


def p_inv_diag(vals: np.ndarray, threshold: float = 1e-10) -> np.ndarray:
    """Diagonal of ``pinv(diagmat(vals), 1e-10)`` (linalg.hpp:469-481)."""
    out = np.zeros_like(vals)
    keep = np.abs(vals) > threshold
    out[keep] = 1.0 / vals[keep]
    return out


def freeze_core(orbitals: Sequence[np.ndarray], n_active: Sequence[int]):
    """Last ``n_active`` columns per spin (src/utils/utils.hpp:235-253)."""
    n_spin = spin_channels(orbitals)
    if spin_channels(n_active) != n_spin:
        raise UW12RuntimeError("Different number of spin channels in orbitals and n_active")
    out = []
    for sigma in range(n_spin):
        c = orbitals[sigma]
        na = int(n_active[sigma])
        if na > c.shape[1]:
            raise UW12LogicError("Cannot have submatix with more columns than parent matrix")
        out.append(np.ascontiguousarray(c[:, c.shape[1] - na:]))
    return out


def construct_density(orbitals: Sequence[np.ndarray]):
    """D = (2|1) C C^T per spin (src/utils/utils.hpp:261-282)."""
    n_spin = spin_channels(orbitals)
    nao = orbitals[0].shape[0]
    out = []
    for c in orbitals:
        if c.shape[1] == 0:
            out.append(np.zeros((nao, nao)))
        else:
            out.append((2.0 if n_spin == 1 else 1.0) * (c @ c.T))
    return out


def occupation_weighted_orbitals(orb: Sequence[np.ndarray], occ: Sequence[np.ndarray]):
    """C[:, :n_occ] * sqrt(occ / (2|1)) (src/utils/utils.hpp:289-310)."""
    n_spin = len(orb)
    if len(occ) != n_spin:
        raise UW12RuntimeError("orbitals and occupations must be of equal size")
    per = 2.0 if n_spin == 1 else 1.0
    out = []
    for i in range(n_spin):
        o = np.asarray(occ[i], dtype=np.float64).reshape(-1)
        if not np.all(o > 0):
            raise UW12RuntimeError("occupations must be positive")
        n_occ = o.size
        if n_occ > orb[i].shape[1]:
            raise UW12LogicError("Cannot have submatix with more columns than parent matrix")
        out.append(orb[i][:, :n_occ] * np.sqrt(o / per)[None, :])
    return out


def get_energy_spin_factor(n_spin, sigma, sigmaprime, s_os, s_ss) -> float:
    """src/four_electron/four_electron_utils.cpp:9-30."""
    if sigma >= n_spin or sigmaprime >= n_spin:
        raise UW12RuntimeError("Invalid spin channel")
    if n_spin == 1:
        return 2.0 * (s_os + s_ss)
    if n_spin == 2:
        return s_ss if sigma == sigmaprime else s_os
    raise UW12RuntimeError("Invalid number of spin channels")


# --------------------------------------------------------------------------
# integrals
# --------------------------------------------------------------------------
class BaseIntegrals:
    """In-core ``BaseIntegrals(J3_0, J2[, J3_ri_0])``.

    Follows src/integrals/base_integrals.cpp:282-303 (ctor) and :155-166
    (eig_sym(J2) -> P2 = Q pinv(Lambda), df_vals = Lambda).
    """

    def __init__(self, J3_0: np.ndarray, J2: np.ndarray, J3_ri_0: Optional[np.ndarray] = None):
        J3_0 = np.asarray(J3_0, dtype=np.float64)
        J2 = np.asarray(J2, dtype=np.float64)
        if J3_0.shape[0] == 0:
            raise UW12RuntimeError("Number of ao orbitals is zero")
        self.n_ao = n_from_packed(J3_0.shape[0])
        self.n_df = J2.shape[0]
        if J3_0.shape[1] != self.n_df:
            raise UW12RuntimeError("Number of density-fitting basis functions inconsistent")
        self.J3_0 = J3_0
        vals, vecs = eigen_system(J2)
        self.P2 = vecs * p_inv_diag(vals)[None, :]
        self.df_vals = vals
        if J3_ri_0 is not None:
            J3_ri_0 = np.asarray(J3_ri_0, dtype=np.float64)
            self.n_ri = J3_ri_0.shape[0] // self.n_ao
            assert self.n_ri * self.n_ao == J3_ri_0.shape[0]
            self.J3_ri_0 = J3_ri_0
        else:
            self.n_ri = 0
            self.J3_ri_0 = None

    def has_J3_ri_0(self) -> bool:
        return self.J3_ri_0 is not None


@dataclass
class ABSProjectors:
    """``three_el::ri::ABSProjectors`` (src/three_electron/ri_utils.hpp:20-29)."""

    s_inv_ri_ri: np.ndarray
    s_inv_ri_ao: np.ndarray
    s_inv_ao_ri: np.ndarray
    s_inv_ao_ao: np.ndarray


def calculate_abs_projectors(S, n_ao, n_ri, eigen_ld_threshold=1e-8, linear_dependency_threshold=1e-6):
    """src/three_electron/ri_utils.hpp:45-74 (AO functions first in S)."""
    vals, vecs = eigen_decomposition(np.asarray(S, dtype=np.float64), linear_dependency_threshold,
                                     eigen_ld_threshold)
    if vecs.shape[0] != n_ao + n_ri:
        raise UW12RuntimeError("Total number of basis functions is inconsistent")
    inv = 1.0 / vals
    ri = vecs[n_ao:, :]
    ao = vecs[:n_ao, :]
    return ABSProjectors(
        (ri * inv) @ ri.T,
        (ri * inv) @ ao.T,
        (ao * inv) @ ri.T,
        (ao * inv) @ ao.T,
    )


def mo_transform_one_index_full(J3: np.ndarray, C: np.ndarray, sampler: Sampler = FULL) -> np.ndarray:
    """(mu k|A) = square(J3[:,A]) C, column A vectorised (transformations.hpp:33-54)."""
    n_ao, n_orb = C.shape
    n_df = J3.shape[1]
    if J3.shape[0] != packed_size(n_ao):
        raise UW12RuntimeError("J3 and C of incompatible sizes")
    out = np.zeros((n_ao * n_orb, n_df))
    for A in sampler.range(n_df):
        out[:, A] = (square(J3[:, A]) @ C).reshape(-1, order="F")
    return out


def transform_first_index(J3: np.ndarray, C: np.ndarray, sampler: Sampler = FULL) -> np.ndarray:
    """(i k|A) = C^T reshape(J3[:,A], n1, n2) (transformations.hpp:79-106)."""
    n1, n4 = C.shape
    n3 = J3.shape[1]
    if n1 == 0 or J3.shape[0] % n1 != 0:
        raise UW12RuntimeError("number of rows of J3 not a multiple of n_ao")
    n2 = J3.shape[0] // n1
    out = np.zeros((n4 * n2, n3))
    for A in sampler.range(n3):
        a12 = J3[:, A].reshape((n1, n2), order="F")
        out[:, A] = (C.T @ a12).reshape(-1, order="F")
    return out


def transform_second_index(J3: np.ndarray, C: np.ndarray, sampler: Sampler = FULL) -> np.ndarray:
    """(p i|A) = reshape(J3[:,A], n1, n2) C (transformations.hpp:130-158)."""
    n2, n4 = C.shape
    n3 = J3.shape[1]
    if n2 == 0 or J3.shape[0] % n2 != 0:
        raise UW12RuntimeError(
            "number of rows J3 is not a multiple of number of orbitals being transformed")
    n1 = J3.shape[0] // n2
    out = np.zeros((n1 * n4, n3))
    for A in sampler.range(n3):
        m = J3[:, A].reshape((n1, n2), order="F")
        out[:, A] = (m @ C).reshape(-1, order="F")
    return out


class Integrals:
    """MO-transformed caches (src/integrals/integrals.cpp:184-424)."""

    def __init__(self, base: BaseIntegrals, occ_orbitals, active_orbitals, sampler: Sampler = FULL):
        if len(occ_orbitals) in (1, 2):
            if len(occ_orbitals) != len(active_orbitals):
                raise UW12RuntimeError(
                    "different number of spin channels in occupied and active orbitals")
        else:
            raise UW12RuntimeError("Invalid number of spin channels")
        self.base = base
        self.occ = list(occ_orbitals)
        self.act = list(active_orbitals)
        self.sampler = sampler
        self._one = None
        self._one_ri = None
        self._two = None

    # sizes -------------------------------------------------------------
    def spin_channels(self) -> int:
        return len(self.act)

    def number_ao_orbitals(self) -> int:
        n_ao = self.act[0].shape[0]
        if self.base.n_ao != n_ao:
            raise UW12RuntimeError("Inconsistent number of atomic orbitals")
        return n_ao

    def number_occ_orbitals(self, sigma) -> int:
        return self.occ[sigma].shape[1]

    def number_active_orbitals(self, sigma) -> int:
        return self.act[sigma].shape[1]

    @property
    def df_vals(self):
        return self.base.df_vals

    @property
    def P2(self):
        return self.base.P2

    # caches ------------------------------------------------------------
    def get_X3idx_one_trans(self):
        """integrals.cpp:213-248 (in-core J3_0 branch)."""
        if self._one is None:
            self._one = [self.sampler.matmul(mo_transform_one_index_full(self.base.J3_0, c,
                                                                         self.sampler),
                                             self.base.P2)
                         for c in self.occ]
        return self._one

    def get_X3idx_one_trans_ri(self):
        """integrals.cpp:250-287 (in-core J3_ri_0 branch)."""
        if self._one_ri is None:
            if not self.base.has_J3_ri_0():
                raise UW12RuntimeError("J3_ri_0 not stored")
            self._one_ri = [self.sampler.matmul(transform_second_index(self.base.J3_ri_0, c,
                                                                       self.sampler),
                                                self.base.P2)
                            for c in self.act]
        return self._one_ri

    def get_X3idx_two_trans(self):
        """integrals.cpp:289-331 (stored one_trans branch)."""
        if self._two is None:
            one = self.get_X3idx_one_trans()
            self._two = [transform_first_index(one[s], self.act[s], self.sampler)
                         for s in range(len(self.act))]
        return self._two

    def get_X4idx_three_trans(self, sigma):
        """(rho k|j l) = B1 Lambda B2^T (integrals.cpp:333-337)."""
        return (self.get_X3idx_one_trans()[sigma] * self.df_vals[None, :]) @ self.get_X3idx_two_trans()[sigma].T

    def get_X4idx_four_trans(self, sigma):
        """(i k|j l) = B2 Lambda B2^T (integrals.cpp:339-345)."""
        b2 = self.get_X3idx_two_trans()[sigma]
        return (b2 * self.df_vals[None, :]) @ b2.T

    def get_X_D(self):
        """X_D = 0.5 s P2^T J3_0^T lower(D, 2) (integrals.cpp:347-378)."""
        n_spin = len(self.act)
        D = construct_density(self.act)
        out = []
        for s in range(n_spin):
            d = lower(D[s], 2.0)
            out.append(0.5 * n_spin * (self.base.P2.T @ (self.base.J3_0.T @ d)))
        return out


# --------------------------------------------------------------------------
# two-electron term (src/two_electron/two_electron.cpp)
# --------------------------------------------------------------------------
def two_el_direct_fock(WV: Integrals, calculate_fock, s_os, s_ss):
    """two_electron.cpp:11-81."""
    n_spin = WV.spin_channels()
    n_ao = WV.number_ao_orbitals()
    fock = [np.zeros((n_ao, n_ao)) for _ in range(n_spin)]
    energy = 0.0
    WV_D = WV.get_X_D()
    WV_tilde_D = [WV.df_vals * x for x in WV_D]
    for sigma in range(n_spin):
        for sp in range(n_spin):
            scale_factor = s_ss if sigma == sp else s_os
            f = 2 * (s_os + s_ss) if n_spin == 1 else scale_factor
            if f == 0:
                continue
            energy += 0.5 * f * float(np.dot(WV_D[sigma], WV_tilde_D[sp]))
            if calculate_fock:
                fock_spin_factor = 0.5 * n_spin * f
                fock[sigma] = fock[sigma] + fock_spin_factor * square(
                    WV.base.J3_0 @ (WV.base.P2 @ WV_tilde_D[sp]))
    return fock, energy


def two_el_indirect_fock(WV: Integrals, calculate_fock):
    """two_electron.cpp:87-132."""
    n_spin = WV.spin_channels()
    n_ao = WV.number_ao_orbitals()
    vals = WV.df_vals
    n_df = vals.size
    fock = [np.zeros((n_ao, n_ao)) for _ in range(n_spin)]
    energy = 0.0
    two = WV.get_X3idx_two_trans()
    esf = 2 if n_spin == 1 else 1
    for sigma in range(n_spin):
        n_occ = WV.number_occ_orbitals(sigma)
        if n_occ == 0:
            continue
        tmp = two[sigma] * vals[None, :]
        energy -= 0.5 * esf * float(np.sum(tmp * two[sigma]))
        if calculate_fock:
            one = WV.get_X3idx_one_trans()[sigma]
            tmp2 = one * vals[None, :]
            r_tilde = tmp2.reshape((n_ao, n_occ * n_df), order="F")
            r_one = one.reshape((n_ao, n_occ * n_df), order="F")
            fock[sigma] = -(r_one @ r_tilde.T)
    return fock, energy


def form_fock_two_el_df(WV_base, active_Co, indirect_term, calculate_fock, s_os, s_ss,
                        sampler: Sampler = FULL):
    """two_electron.cpp:134-153."""
    ints = Integrals(WV_base, active_Co, active_Co, sampler)
    fock, energy = two_el_direct_fock(ints, calculate_fock, s_os, s_ss)
    if indirect_term and s_ss != 0:
        f2, e2 = two_el_indirect_fock(ints, calculate_fock)
        fock = [a + s_ss * b for a, b in zip(fock, f2)]
        energy += s_ss * e2
    return fock, energy


# --------------------------------------------------------------------------
# four-electron term (src/four_electron)
# --------------------------------------------------------------------------
def calculate_tab(W: Integrals, V: Integrals):
    """four_electron_utils.cpp:33-49."""
    return [w.T @ v for w, v in zip(W.get_X3idx_two_trans(), V.get_X3idx_two_trans())]


def calculate_ttilde(W: Integrals, V: Integrals, tab=None):
    """four_electron_utils.cpp:51-79."""
    if tab is None:
        tab = calculate_tab(W, V)
    return [W.df_vals[:, None] * t * V.df_vals[None, :] for t in tab]


def four_el_direct_fock_contribution(W1, V1, ttilde, esf, n_ao, n_spin):
    """four_electron.cpp:11-41."""
    n_occ = W1.shape[0] // n_ao
    n_df = V1.shape[1]
    W1t = W1 @ ttilde
    fsf = (0.5 if n_spin == 1 else 1.0) * esf
    return 2 * fsf * (V1.reshape((n_ao, n_occ * n_df), order="F")
                      @ W1t.reshape((n_ao, n_occ * n_df), order="F").T)


def four_el_direct_fock_matrix(W1, V1, ttilde, esf, n_active, n_ao, n_spin):
    """four_electron.cpp:43-77."""
    n_occ = W1.shape[0] // n_ao
    fock = four_el_direct_fock_contribution(W1, V1, ttilde, esf, n_ao, n_spin)
    if n_occ == n_active or n_active == 0:
        return fock
    frozen = four_el_direct_fock_contribution(W1[W1.shape[0] - n_ao * n_active:, :],
                                              V1[V1.shape[0] - n_ao * n_active:, :],
                                              ttilde, esf, n_ao, n_spin)
    return 0.5 * (fock + frozen)


def four_el_direct_fock(W: Integrals, V: Integrals, calculate_fock, s_os, s_ss):
    """four_electron.cpp:80-137."""
    n_ao = W.number_ao_orbitals()
    n_spin = W.spin_channels()
    fock = [np.zeros((n_ao, n_ao)) for _ in range(n_spin)]
    energy = 0.0
    tab = calculate_tab(W, V)
    tt = calculate_ttilde(W, V, tab)
    for sigma in range(n_spin):
        n_active = W.number_active_orbitals(sigma)
        for sp in range(n_spin):
            esf = get_energy_spin_factor(n_spin, sigma, sp, s_os, s_ss)
            if esf == 0:
                continue
            energy += 0.5 * esf * float(np.sum(tt[sp] * tab[sigma]))
            if calculate_fock:
                fock[sigma] = fock[sigma] + four_el_direct_fock_matrix(
                    W.get_X3idx_one_trans()[sigma], V.get_X3idx_one_trans()[sigma], tt[sp], esf,
                    n_active, n_ao, n_spin)
    return [symmetrise(f) for f in fock], energy


def four_el_indirect_energy(W4, V4, n_occ, n_spin, sampler: Sampler = FULL):
    """four_electron.cpp:143-179."""
    n_active = W4.shape[0] // n_occ
    total = 0.0
    for k, l in sampler.range2d(n_occ, n_occ):
        e = float(np.sum(W4[l * n_active:(l + 1) * n_active, k * n_active:(k + 1) * n_active]
                         * V4[k * n_active:(k + 1) * n_active, l * n_active:(l + 1) * n_active]))
        total += -0.5 * (2 if n_spin == 1 else 1) * e
    return total


def four_el_indirect_fock_matrix(W43, V43, n_ao, sampler: Sampler = FULL):
    """four_electron.cpp:181-249."""
    n_occ = W43.shape[0] // n_ao
    n_active = W43.shape[1] // n_occ if n_occ else 0
    n_core = n_occ - n_active
    contrib = np.zeros((n_ao, n_ao))
    for i, k in sampler.range2d(n_active, n_occ):
        W4_ik = W43[(n_core + i) * n_ao:(n_core + i + 1) * n_ao, n_active * k:n_active * (k + 1)]
        col = V43[:, i + n_active * k]
        V4_ik = col[col.size - n_ao * n_active:].reshape((n_ao, n_active), order="F")
        contrib += -2 * (W4_ik @ V4_ik.T)
    if n_core == 0:
        return contrib
    frozen = np.zeros((n_ao, n_ao))
    for k, l in sampler.range2d(n_occ, n_occ):
        a = W43[l * n_ao:(l + 1) * n_ao, k * n_active:(k + 1) * n_active]
        b = V43[k * n_ao:(k + 1) * n_ao, l * n_active:(l + 1) * n_active]
        frozen += -2 * (a @ b.T)
    return 0.5 * (contrib + frozen)


def four_el_indirect_fock(W: Integrals, V: Integrals, calculate_fock, sampler: Sampler = FULL):
    """four_electron.cpp:253-290."""
    n_ao = W.number_ao_orbitals()
    n_spin = W.spin_channels()
    fock = [np.zeros((n_ao, n_ao)) for _ in range(n_spin)]
    energy = 0.0
    for sigma in range(n_spin):
        n_occ = W.number_occ_orbitals(sigma)
        n_active = W.number_active_orbitals(sigma)
        if n_active == 0 or n_occ == 0 or n_ao == 0:
            continue
        W4 = W.get_X4idx_four_trans(sigma)
        V4 = V.get_X4idx_four_trans(sigma)
        energy += four_el_indirect_energy(W4, V4, n_occ, n_spin, sampler)
        if calculate_fock:
            fock[sigma] = four_el_indirect_fock_matrix(W.get_X4idx_three_trans(sigma),
                                                       V.get_X4idx_three_trans(sigma), n_ao, sampler)
    return [symmetrise(f) for f in fock], energy


def form_fock_four_el_df(W, V, indirect_term, calculate_fock, s_os, s_ss, sampler: Sampler = FULL):
    """four_electron.cpp:296-312."""
    fock, energy = four_el_direct_fock(W, V, calculate_fock, s_os, s_ss)
    if indirect_term and not (s_ss == 0):
        f2, e2 = four_el_indirect_fock(W, V, calculate_fock, sampler)
        fock = [a + s_ss * b for a, b in zip(fock, f2)]
        energy += s_ss * e2
    return fock, energy


# --------------------------------------------------------------------------
# three-electron term, direct part (src/three_electron/direct_utils.cpp)
# --------------------------------------------------------------------------
def calculate_xab_component(Wm, Vm, projector, sampler: Sampler = FULL):
    """direct_utils.cpp:31-52: out[:, A] = W^T vec(P reshape(V[:,A]))."""
    n_orb = projector.shape[1]
    n_df = Vm.shape[1]
    n_active = Vm.shape[0] // n_orb if n_orb else 0
    out = np.zeros((Wm.shape[1], n_df))
    for A in sampler.range(n_df):
        v_proj = projector @ Vm[:, A].reshape((n_orb, n_active), order="F")
        out[:, A] = Wm.T @ v_proj.reshape(-1, order="F")
    return out


def calculate_xab(W: Integrals, V: Integrals, abs_p: ABSProjectors, sampler: Sampler = FULL):
    """direct_utils.cpp:62-133."""
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    n_df = V.df_vals.size
    n_spin = W.spin_channels()
    W1 = W.get_X3idx_one_trans()
    V1 = V.get_X3idx_one_trans()
    Wr = W.get_X3idx_one_trans_ri()
    Vr = V.get_X3idx_one_trans_ri()
    x = [np.zeros((n_df, n_df)) for _ in range(n_spin)]
    for s in range(n_spin):
        na = W.number_active_orbitals(s)
        x[s] = x[s] + calculate_xab_component(Wr[s], Vr[s], abs_p.s_inv_ri_ri, sampler)
        if na == 0:
            continue
        w_tail = W1[s][W1[s].shape[0] - na * n_ao:, :]
        v_tail = V1[s][V1[s].shape[0] - na * n_ao:, :]
        x[s] = x[s] + calculate_xab_component(w_tail, Vr[s], abs_p.s_inv_ao_ri, sampler)
        x[s] = x[s] + calculate_xab_component(w_tail, v_tail, abs_p.s_inv_ao_ao, sampler)
        x[s] = x[s] + calculate_xab_component(Wr[s], v_tail, abs_p.s_inv_ri_ao, sampler)
    return x


def calculate_direct_energy(x, ttilde, s_os, s_ss):
    """direct_utils.cpp:136-157."""
    n_spin = spin_channels(x)
    e = 0.0
    for s in range(n_spin):
        for sp in range(n_spin):
            f = get_energy_spin_factor(n_spin, s, sp, s_os, s_ss)
            e -= f * float(np.sum(x[s] * ttilde[sp]))
    return e


def calculate_xab_dttilde(W1, V1, xab, W_vals, V_vals, n_active, n_ao, sampler: Sampler = FULL):
    """direct_utils.cpp:164-204."""
    n_df = W_vals.size
    n_occ = W1.shape[0] // n_ao
    if W1.shape[0] != n_occ * n_ao:
        raise UW12RuntimeError("Incorrect number of rows in W3_imA")
    if V1.shape[0] != n_occ * n_ao:
        raise UW12RuntimeError("Incorrect number of rows in V3_imA")
    w = (W1 * W_vals[None, :]) @ xab
    v_tilde = V1 * V_vals[None, :]
    out = np.zeros((n_ao, n_ao))
    for A in sampler.range(n_df):
        wA = w[:, A].reshape((n_ao, n_occ), order="F")
        vA = v_tilde[:, A].reshape((n_ao, n_occ), order="F")
        f = -(wA @ vA.T)
        if n_active != 0:
            f -= wA[:, n_occ - n_active:] @ vA[:, n_occ - n_active:].T
        out += f
    return out


def calculate_ttilde_dxab_incore(W: Integrals, V: Integrals, ttilde, abs_p: ABSProjectors,
                                 sampler: Sampler = FULL):
    """s-term (direct_utils.cpp:256-286) + p-term (:302-334), in-core branch."""
    n_ri = abs_p.s_inv_ri_ri.shape[0]
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    Wb, Vb = W.base, V.base

    def W3_fn(A):  # get_X3_fn, :206-219
        return Wb.J3_0 @ Wb.P2[:, A]

    def W3_ri_fn(A):  # get_W3_ri_fn, :221-240
        return (Wb.J3_ri_0 @ Wb.P2[:, A]).reshape((n_ri, n_ao), order="F")

    # calculate_s_matrix (:242-250); Armadillo evaluates the triple product in
    # the cheaper association J3_0 (P2 t~^T), as here.
    s = sampler.matmul(Vb.J3_0, Vb.P2 @ ttilde.T)
    fock = np.zeros((n_ao, n_ao))
    for A in sampler.range(s.shape[1]):
        sA = square(s[:, A])
        fock -= square(W3_fn(A)) @ abs_p.s_inv_ao_ao @ sA
        fock -= W3_ri_fn(A).T @ abs_p.s_inv_ri_ao @ sA
    p = sampler.matmul(Vb.J3_ri_0, Vb.P2 @ ttilde.T)  # calculate_p_matrix, :288-296
    for A in sampler.range(p.shape[1]):
        pA = p[:, A].reshape((n_ri, n_ao), order="F")
        fock -= square(W3_fn(A)) @ abs_p.s_inv_ao_ri @ pA
        fock -= W3_ri_fn(A).T @ abs_p.s_inv_ri_ri @ pA
    return fock


def three_el_direct_fock_matrix(W, V, x, ttilde, abs_p, s_os, s_ss, sampler: Sampler = FULL):
    """three_electron.cpp:32-83 (note the cross-spin fock[sigma'] update)."""
    n_spin = W.spin_channels()
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    W1 = W.get_X3idx_one_trans()
    V1 = V.get_X3idx_one_trans()
    fock = [np.zeros((n_ao, n_ao)) for _ in range(n_spin)]
    for s in range(n_spin):
        na = W.number_active_orbitals(s)
        fock_sp = calculate_ttilde_dxab_incore(W, V, ttilde[s], abs_p, sampler)
        for sp in range(n_spin):
            dfs = (0.5 if n_spin == 1 else 1.0) * get_energy_spin_factor(n_spin, s, sp, s_os, s_ss)
            fock[s] = fock[s] + dfs * calculate_xab_dttilde(W1[s], V1[s], x[sp], W.df_vals, V.df_vals,
                                                            na, n_ao, sampler)
            fock[sp] = fock[sp] + dfs * fock_sp
    return fock


def three_el_direct_fock(W, V, abs_p, calculate_fock, s_os, s_ss, sampler: Sampler = FULL):
    """three_electron.cpp:86-115."""
    x = calculate_xab(W, V, abs_p, sampler)
    tt = calculate_ttilde(W, V)
    energy = calculate_direct_energy(x, tt, s_os, s_ss)
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    if calculate_fock:
        fock = three_el_direct_fock_matrix(W, V, x, tt, abs_p, s_os, s_ss, sampler)
    else:
        fock = [np.zeros((n_ao, n_ao)) for _ in range(W.spin_channels())]
    return [symmetrise(f) for f in fock], energy


# --------------------------------------------------------------------------
# three-electron term, indirect part (src/three_electron/indirect_utils.cpp)
# --------------------------------------------------------------------------
def calculate_xij(W, V, abs_p, n_core, i, j, sigma):
    """indirect_utils.cpp:19-63."""
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    n_ri = abs_p.s_inv_ri_ri.shape[0]
    W1 = W.get_X3idx_one_trans()[sigma]
    V1 = V.get_X3idx_one_trans()[sigma]
    Wr = W.get_X3idx_one_trans_ri()[sigma]
    Vr = V.get_X3idx_one_trans_ri()[sigma]
    wr = Wr[i * n_ri:(i + 1) * n_ri, :]
    vr = Vr[j * n_ri:(j + 1) * n_ri, :]
    wa = W1[(i + n_core) * n_ao:(i + n_core + 1) * n_ao, :]
    va = V1[(j + n_core) * n_ao:(j + n_core + 1) * n_ao, :]
    out = wr.T @ abs_p.s_inv_ri_ri @ vr
    out += wr.T @ abs_p.s_inv_ri_ao @ va
    out += wa.T @ abs_p.s_inv_ao_ri @ vr
    out += wa.T @ abs_p.s_inv_ao_ao @ va
    return out


def calculate_ttilde_ij(W, V, n_active, i, j, sigma):
    """indirect_utils.cpp:67-94."""
    n_occ = W.number_occ_orbitals(sigma)
    W2 = W.get_X3idx_two_trans()[sigma]
    V2 = V.get_X3idx_two_trans()[sigma]
    n_df_W = W.df_vals.size
    n_df_V = V.df_vals.size
    W_tmp = W2.reshape((n_active, n_occ * n_df_W), order="F")
    Wt = W_tmp[j, :].reshape((n_occ, n_df_W), order="F") * W.df_vals[None, :]
    V_tmp = V2.reshape((n_active, n_occ * n_df_V), order="F")
    Vt = V_tmp[i, :].reshape((n_occ, n_df_V), order="F") * V.df_vals[None, :]
    return Wt.T @ Vt


def indirect_3el_energy(W, V, abs_p, sampler: Sampler = FULL):
    """indirect_utils.cpp:101-133."""
    n_spin = W.spin_channels()
    energy = 0.0
    for s in range(n_spin):
        n_occ = W.number_occ_orbitals(s)
        na = W.number_active_orbitals(s)
        n_core = n_occ - na
        tot = 0.0
        for i, j in sampler.range2d(na, na):
            xij = calculate_xij(W, V, abs_p, n_core, i, j, s)
            tij = calculate_ttilde_ij(W, V, na, i, j, s)
            tot += (2 if n_spin == 1 else 1) * float(np.sum(xij * tij))
        energy += tot
    return energy


def _x3_fn(X: Integrals, vec):
    """get_X3_func (indirect_utils.cpp:261-277), J3_0 branch."""
    return X.base.J3_0 @ (X.base.P2 @ vec)


def _x3_ri_fn(X: Integrals, vec):
    """get_X3_ri_fn (indirect_utils.cpp:279-295), J3_ri_0 branch."""
    return X.base.J3_ri_0 @ (X.base.P2 @ vec)


def fock_i(X: Integrals, Y: Integrals, abs_p, j, k, sigma):
    """indirect_utils.cpp:139-194."""
    n_ri = abs_p.s_inv_ri_ri.shape[0]
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    n_occ = X.number_occ_orbitals(sigma)
    na = X.number_active_orbitals(sigma)
    n_core = n_occ - na
    row = X.get_X3idx_two_trans()[sigma][k * na + j, :]
    xt = row * X.df_vals
    X_jk_am = _x3_ri_fn(X, xt).reshape((n_ri, n_ao), order="F")
    Y1 = Y.get_X3idx_one_trans()[sigma]
    Yr = Y.get_X3idx_one_trans_ri()[sigma]
    Yt_k = Y.df_vals[:, None] * Y1[k * n_ao:(k + 1) * n_ao, :].T
    Y_vj_kb = Yr[n_ri * j:n_ri * (j + 1), :] @ Yt_k
    out = X_jk_am.T @ abs_p.s_inv_ri_ri @ Y_vj_kb
    Y_pj_kb = Y1[(j + n_core) * n_ao:(j + n_core + 1) * n_ao, :] @ Yt_k
    out += X_jk_am.T @ abs_p.s_inv_ri_ao @ Y_pj_kb
    X_jk_ap = square(_x3_fn(X, xt))
    out += X_jk_ap @ abs_p.s_inv_ao_ri @ Y_vj_kb
    out += X_jk_ap @ abs_p.s_inv_ao_ao @ Y_pj_kb
    return out


def fock_k(W: Integrals, V: Integrals, abs_p, i, j, sigma):
    """indirect_utils.cpp:199-259."""
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    n_ri = abs_p.s_inv_ri_ri.shape[0]
    W1 = W.get_X3idx_one_trans()[sigma]
    V1 = V.get_X3idx_one_trans()[sigma]
    Wr = W.get_X3idx_one_trans_ri()[sigma]
    Vr = V.get_X3idx_one_trans_ri()[sigma]
    n_occ = W.number_occ_orbitals(sigma)
    na = W.number_active_orbitals(sigma)
    n_core = n_occ - na
    Wt_j = W.df_vals[:, None] * W1[n_ao * (j + n_core):n_ao * (j + n_core + 1), :].T
    W_jb_im = Wr[n_ri * i:n_ri * (i + 1), :] @ Wt_j
    Vt_i = V.df_vals[:, None] * V1[n_ao * (i + n_core):n_ao * (i + n_core + 1), :].T
    V_vj_ai = Vr[n_ri * j:n_ri * (j + 1), :] @ Vt_i
    out = W_jb_im.T @ abs_p.s_inv_ri_ri @ V_vj_ai
    V_pj_ai = V1[n_ao * (j + n_core):n_ao * (j + n_core + 1), :] @ Vt_i
    out += W_jb_im.T @ abs_p.s_inv_ri_ao @ V_pj_ai
    W_jb_ip = W1[(n_core + i) * n_ao:(n_core + i + 1) * n_ao, :] @ Wt_j
    out += W_jb_ip.T @ abs_p.s_inv_ao_ri @ V_vj_ai
    out += W_jb_ip.T @ abs_p.s_inv_ao_ao @ V_pj_ai
    return out


def indirect_3el_fock_matrix(W, V, abs_p, sigma, sampler: Sampler = FULL):
    """indirect_utils.cpp:297-345: i-, j- and k-terms over orbital pairs."""
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    n_occ = W.number_occ_orbitals(sigma)
    na = W.number_active_orbitals(sigma)
    f = np.zeros((n_ao, n_ao))
    for j, k in sampler.range2d(na, n_occ):
        f += fock_i(W, V, abs_p, j, k, sigma)
    for i, k in sampler.range2d(na, n_occ):
        f += fock_i(V, W, abs_p, i, k, sigma)
    for i, j in sampler.range2d(na, na):
        f += fock_k(W, V, abs_p, i, j, sigma)
    return f


def three_el_indirect_fock(W, V, abs_p, calculate_fock, sampler: Sampler = FULL):
    """three_electron.cpp:143-166."""
    energy = indirect_3el_energy(W, V, abs_p, sampler)
    n_spin = W.spin_channels()
    n_ao = abs_p.s_inv_ao_ao.shape[0]
    if calculate_fock:
        fock = [indirect_3el_fock_matrix(W, V, abs_p, s, sampler) for s in range(n_spin)]
    else:
        fock = [np.zeros((n_ao, n_ao)) for _ in range(n_spin)]
    return [symmetrise(f) for f in fock], energy


def form_fock_three_el_term_df_ri(W, V, abs_p, indirect_term, calculate_fock, s_os, s_ss,
                                  sampler: Sampler = FULL):
    """three_electron.cpp:170-189."""
    fock, energy = three_el_direct_fock(W, V, abs_p, calculate_fock, s_os, s_ss, sampler)
    if indirect_term and s_ss != 0:
        f2, e2 = three_el_indirect_fock(W, V, abs_p, calculate_fock, sampler)
        fock = [a + s_ss * b for a, b in zip(fock, f2)]
        energy += s_ss * e2
    return fock, energy


# --------------------------------------------------------------------------
# orchestrator and public API
# --------------------------------------------------------------------------
@dataclass
class TermResults:
    fock: List[np.ndarray]
    energy: float
    terms: dict = field(default_factory=dict)


def form_fock(W: BaseIntegrals, V: BaseIntegrals, WV: BaseIntegrals, abs_p: ABSProjectors,
              orbitals, occupations, n_active, indirect_term: bool, calculate_fock: bool,
              s_os: float, s_ss: float, print_level: int = 0,
              sampler: Sampler = FULL) -> TermResults:
    """``uw12::form_fock`` (src/uw12.cpp:22-119)."""
    n_spin = spin_channels(orbitals)
    if spin_channels(occupations) != n_spin:
        raise UW12RuntimeError("Different number of spin channels for orbitals and occupations")
    if spin_channels(n_active) != n_spin:
        raise UW12RuntimeError("Different number of spin channels in n_active and orbitals")
    Co = occupation_weighted_orbitals(orbitals, occupations)
    active_Co = freeze_core(Co, n_active)

    f2, e2 = form_fock_two_el_df(WV, active_Co, indirect_term, calculate_fock, s_os, s_ss, sampler)
    W_ints = Integrals(W, Co, active_Co, sampler)
    V_ints = Integrals(V, Co, active_Co, sampler)
    f3, e3 = form_fock_three_el_term_df_ri(W_ints, V_ints, abs_p, indirect_term, calculate_fock,
                                           s_os, s_ss, sampler)
    f4, e4 = form_fock_four_el_df(W_ints, V_ints, indirect_term, calculate_fock, s_os, s_ss, sampler)
    fock = [a + b + c for a, b, c in zip(f2, f3, f4)]
    energy = e2 + e3 + e4
    if print_level > 1:
        print(f" {'Two electron energy:':<33}{e2:12.6f}")
        print(f" {'Three electron energy:':<33}{e3:12.6f}")
        print(f" {'Four electron energy:':<33}{e4:12.6f}")
    if print_level > 0:
        print(f" {'Total UW12 energy:':<33}{energy:12.6f}")
    return TermResults(fock, energy, {"two": e2, "three": e3, "four": e4})


def setup_orbitals(C: np.ndarray, n_ao: int, n_orb: int, n_spin: int):
    """libuw12.cpp:58-77 (alpha columns then beta)."""
    if n_spin not in (1, 2):
        raise UW12RuntimeError("Number of spin channels must be 1 or 2")
    C1 = np.asarray(C, dtype=np.float64).reshape((n_ao, n_orb * n_spin), order="F")
    if n_spin == 1:
        return [C1.copy()]
    return [C1[:, :n_orb].copy(), C1[:, n_orb:].copy()]


def setup_occupations(occ: np.ndarray, n_occ_alpha: int, n_occ_beta: Optional[int] = None):
    """libuw12.cpp:79-112 (closed shell when ``n_occ_beta`` is None)."""
    occ = np.asarray(occ, dtype=np.float64).reshape(-1)
    if n_occ_beta is None:
        return [occ[:n_occ_alpha].copy()]
    return [occ[:n_occ_alpha].copy(), occ[n_occ_alpha:n_occ_alpha + n_occ_beta].copy()]


def uw12_fock(W, V, WV, abs_p, orbitals, occ, n_active, s_os, s_ss, print_level=0,
              calculate_fock=True, sampler: Sampler = FULL):
    """libuw12.cpp:125-154 and :184-214; returns (energy, fock n_ao x n_ao*n_spin)."""
    indirect = not nearly_zero(s_ss)
    res = form_fock(W, V, WV, abs_p, orbitals, occ, n_active, indirect, calculate_fock, s_os, s_ss,
                    print_level, sampler)
    return res.energy, np.concatenate(res.fock, axis=1)


def uw12_energy(W, V, WV, abs_p, orbitals, occ, n_active, s_os, s_ss, print_level=0,
                sampler: Sampler = FULL):
    """libuw12.cpp:156-182."""
    return uw12_fock(W, V, WV, abs_p, orbitals, occ, n_active, s_os, s_ss, print_level, False,
                     sampler)[0]
