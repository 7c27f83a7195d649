"""Shared parity-case construction for the CPU oracle and the CUDA path.

Two input families:

* ``baseline``: the benchmark generators (three-index tensors
  N(0,1) exp(-|m-n|/L), metrics B B^T + 1e-6 I, S-orthonormal orbitals); the
  metric condition number reaches 1e4-1e6, so energies are large and the
  comparison is relative.
* ``unit``: the reference unit tests' shapes (``random_pd`` metrics with
  eigenvalues in [1, 2], U(0,1)-like three-index tensors and orbitals,
  ``tests/setup_integrals.hpp:24-152``); well conditioned, compared with
  libuw12's regression tolerances (1e-8 Eh energy, 1e-7 Eh Fock) relative to
  max(1, |value|).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from oracle import synth
from oracle import uw12_oracle as O


@dataclass
class Case:
    name: str
    n_ao: int
    n_df: int
    n_ri: int
    n_occ: Sequence[int]
    n_active: Sequence[int]
    family: str = "baseline"
    seed: int = 11
    decay: float = 8.0
    n_df_v: Optional[int] = None


@dataclass
class CaseData:
    case: Case
    W3: np.ndarray
    W2: np.ndarray
    W3_ri: np.ndarray
    V3: np.ndarray
    V2: np.ndarray
    V3_ri: np.ndarray
    WV3: np.ndarray
    WV2: np.ndarray
    S: np.ndarray
    orbitals: List[np.ndarray]
    occ: List[np.ndarray]


def make_case(c: Case) -> CaseData:
    N, M, R = c.n_ao, c.n_df, c.n_ri
    Mv = c.n_df_v or M
    np_ = N * (N + 1) // 2
    seed = c.seed
    if c.family == "baseline":
        g = synth
        W3 = g.three_index_ao(seed, "W3", N, M, c.decay)
        V3 = g.three_index_ao(seed, "V3", N, Mv, c.decay)
        WV3 = g.three_index_ao(seed, "WV3", N, M, c.decay)
        W3_ri = g.three_index_ri(seed, "W3_ri", N, R, M, c.decay)
        V3_ri = g.three_index_ri(seed, "V3_ri", N, R, Mv, c.decay)
        W2, V2, WV2 = g.metric(seed, "W2", M), g.metric(seed, "V2", Mv), g.metric(seed, "WV2", M)
        S = g.overlap(seed, N, R)
        orbitals = []
        for s, o in enumerate(c.n_occ):
            orbitals.append(g.orbitals(seed, S[:N, :N], max(o, 1), f"C{s}")[:, :max(o, 1)])
        per = 2.0 if len(c.n_occ) == 1 else 1.0
        occ = [np.full(o, per) for o in c.n_occ]
    elif c.family == "unit":
        u = synth.uniform_matrix
        W3 = u(seed, "uW3", np_, M)
        V3 = u(seed, "uV3", np_, Mv)
        WV3 = u(seed, "uWV3", np_, M)
        W3_ri = u(seed, "uW3_ri", N * R, M)
        V3_ri = u(seed, "uV3_ri", N * R, Mv)
        W2 = synth.random_pd(M, seed, "uW2")
        V2 = synth.random_pd(Mv, seed, "uV2")
        WV2 = synth.random_pd(M, seed, "uWV2")
        S = synth.random_pd(N + R, seed, "uS")
        orbitals = [u(seed, f"uC{s}", N, max(o, 1)) for s, o in enumerate(c.n_occ)]
        occ = [np.ones(o) for o in c.n_occ]
    else:
        raise ValueError(c.family)
    return CaseData(c, W3, W2, W3_ri, V3, V2, V3_ri, WV3, WV2, S, orbitals, occ)


def oracle_form_fock(d: CaseData, indirect: bool, calc: bool, s_os: float, s_ss: float):
    c = d.case
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, c.n_ao, c.n_ri)
    res = O.form_fock(W, V, WV, absp, d.orbitals, d.occ, list(c.n_active), indirect, calc, s_os,
                      s_ss)
    return res.energy, res.fock, res.terms


CASES = [
    Case("c0_closed", 24, 84, 116, (5,), (5,), "baseline", 11, 8.0),
    Case("c0_frozen", 24, 84, 116, (5,), (4,), "baseline", 11, 8.0),
    Case("uhf_small", 9, 13, 11, (4, 3), (3, 2), "baseline", 3, 4.0),
    Case("uhf_allel", 9, 13, 11, (4, 3), (4, 3), "baseline", 4, 4.0),
    Case("uhf_one_inactive", 8, 12, 10, (4, 3), (2, 0), "baseline", 5, 4.0),
    Case("uhf_no_beta", 8, 12, 10, (3, 0), (2, 0), "baseline", 6, 4.0),
    Case("unit_closed", 5, 8, 14, (3,), (2,), "unit", 11),
    Case("unit_open", 5, 8, 14, (4, 3), (3, 2), "unit", 11),
    Case("unit_tiles", 37, 150, 170, (13, 11), (12, 9), "unit", 12),
]
