"""Cases pinned by golden fixtures produced by the compiled libuw12 reference.

``tests/golden/make_golden.py`` evaluates every case below with libuw12 itself
(its unmodified sources compiled by ``oracle/ref.mk``) and writes
``tests/golden/reference_goldens.npz``; the tests regenerate the same inputs
from the seeds here and compare the numpy oracle (CPU) and the CUDA path
(GPU) with the stored results.

* ``PARITY``: the parity cases of ``tests/parity_cases.py`` (c0 closed and
  frozen core, UHF variants, empty beta, one channel inactive, the reference
  unit-test shapes, a multi-tile case) at scales (1, 0.5), (1, 0), (0, 1).
* ``C1S``: the c1 workload's generators at reduced size (N=200, M=600,
  R=800, UHF 16/15, decay 30) at (1, 0.5) and (1, 0).
* ``C4_SUBSET``: molecules of the 64-molecule batch (N ~ U[20, 300],
  M = 3N, R = 4N, n_occ = round(N/10), even index closed shell, odd index UHF
  with n_beta = n_alpha - 1, decay 8, seed 2024000 + index) whose N is at
  most 60, at (1, 0.5).
* ``ABS_EDGE``: overlaps whose spectrum puts one eigenvalue just below and
  one just above the ABS+ drop threshold max(1e-6, 1e-8 lambda_max)
  (``src/three_electron/ri_utils.hpp:45-74``, ``src/utils/linalg.hpp:1157-1197``),
  once where the absolute and once where the relative threshold binds.
* ``ERRORS``: inputs libuw12 rejects, with the exception class and message
  it raises.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from tests.parity_cases import CASES, Case

SCALES = [(1.0, 0.5), (1.0, 0.0), (0.0, 1.0)]

PARITY = [(c, SCALES) for c in CASES]

C1S = Case("c1s", 200, 600, 800, (16, 15), (16, 15), "baseline", 11, 30.0)
C1S_SCALES = [(1.0, 0.5), (1.0, 0.0)]

C4_SEED = 2024
C4_MAX_N = 60


def c4_molecules(n_mol: int = 64, seed: int = C4_SEED) -> List[Tuple[int, Case]]:
    """(index, case) of every molecule of the 64-molecule batch, drawn as the
    benchmark draws them (numpy default_rng(seed).integers(20, 301) per
    molecule)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_mol):
        N = int(rng.integers(20, 301))
        o = max(1, int(round(N / 10)))
        occ = (o,) if i % 2 == 0 else (o, max(1, o - 1))
        out.append((i, Case(f"c4_{i}", N, 3 * N, 4 * N, occ, occ, "baseline",
                            seed * 1000 + i, 8.0)))
    return out


def c4_subset() -> List[Tuple[int, Case]]:
    return [(i, c) for i, c in c4_molecules() if c.n_ao <= C4_MAX_N]


@dataclass
class AbsEdge:
    name: str
    n_ao: int
    n_ri: int
    lam_max: float
    seed: int


ABS_EDGE = [AbsEdge("abs_edge_absolute", 6, 10, 1.0, 5),
            AbsEdge("abs_edge_relative", 6, 10, 1.0e3, 6)]


def abs_edge_overlap(e: AbsEdge) -> Tuple[np.ndarray, np.ndarray]:
    """Symmetric positive definite overlap Q diag(lam) Q^T with two eigenvalues
    at threshold * (1 -/+ 1e-3), the rest log-spaced in [10 threshold, lam_max]
    (lam_max included); returns (S, lam)."""
    from oracle import synth
    n = e.n_ao + e.n_ri
    thr = max(1e-6, 1e-8 * e.lam_max)
    rest = np.geomspace(10 * thr, e.lam_max, n - 2)
    lam = np.concatenate([[thr * (1 - 1e-3), thr * (1 + 1e-3)], rest])
    G = synth.gaussian_matrix(e.seed, e.name, n, n)
    Q, R = np.linalg.qr(G)
    Q = Q * np.sign(np.diag(R))[None, :]
    S = (Q * lam[None, :]) @ Q.T
    return 0.5 * (S + S.T), lam


# (name, case, mutation, expected exception class) -- the mutation is applied
# to the inputs before the evaluation; the class and message are recorded from
# libuw12 by the golden script.
ERROR_CASE = Case("err", 9, 13, 11, (4, 3), (3, 2), "baseline", 3, 4.0)
ERRORS = [
    ("n_active_spin_channels", "n_active", [3]),
    ("n_active_above_n_occ", "n_active", [5, 2]),
    ("negative_occupation", "occ_alpha_negative", None),
    ("asymmetric_metric", "W2_asymmetric", None),
]
