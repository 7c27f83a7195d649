"""The numpy oracle against libuw12's own results (tests/golden/reference_goldens.npz,
written by tests/golden/make_golden.py from the reference's unmodified sources
compiled by oracle/ref.mk).

Tolerances: both sides are FP64 with different summation orders (and the
reference's OpenMP reductions are not order-stable); the error is relative to
the magnitude of the terms, which the metric condition number amplifies:
  * ``unit`` family (well conditioned): 1e-12 of max(1, |E|, |terms|);
  * ``baseline`` family (cond(J2) up to 1e6): 1e-9 of the same scale;
  * with same-spin scaling the same-spin direct and exchange parts cancel by up
    to 1e-8, so the scale is the magnitude of the run without the exchange
    term (as in the GPU parity tests).
Observed: 1e-15 (unit) and 3e-11..6e-11 (baseline, c0 and c1s).
"""
import json

import numpy as np
import pytest

from oracle import uw12_oracle as O
from tests import golden_cases as G
from tests.parity_cases import make_case, oracle_form_fock

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                          "reference_goldens.npz"))


def key(name, s_os, s_ss, what):
    return f"{name}|{s_os:g},{s_ss:g}|{what}"


def tol(case):
    return 1e-12 if case.family == "unit" else 1e-9


def checksum(d):
    return np.array([d.W3.sum(), d.V3.sum(), d.WV3.sum(), d.W3_ri.sum(), d.V3_ri.sum(),
                     d.W2.sum(), d.S.sum()])


def compare(case, d, s_os, s_ss, fock=True):
    indirect = s_ss != 0.0
    e, f, t = oracle_form_fock(d, indirect, fock, s_os, s_ss)
    E = float(GOLD[key(case.name, s_os, s_ss, "energy")])
    T = GOLD[key(case.name, s_os, s_ss, "terms")]
    scale = max(1.0, abs(E), float(np.max(np.abs(T))))
    f_scale = 0.0
    if indirect:
        e_dir, f_dir, t_dir = oracle_form_fock(d, False, fock, s_os, s_ss)
        scale = max(scale, abs(e_dir), max(abs(v) for v in t_dir.values()))
        if fock:
            f_scale = float(np.max(np.abs(np.concatenate(f_dir, axis=1))))
    assert abs(e - E) <= tol(case) * scale, (case.name, e, E)
    for k, nm in enumerate(("two", "three", "four")):
        assert abs(t[nm] - T[k]) <= tol(case) * scale * 10, (case.name, nm, t[nm], T[k])
    fk = key(case.name, s_os, s_ss, "fock")
    if fock and fk in GOLD:
        F = GOLD[fk]
        got = np.concatenate(f, axis=1)
        fs = max(1.0, float(np.max(np.abs(F))), f_scale)
        assert np.max(np.abs(got - F)) <= tol(case) * fs * 10, case.name


@pytest.mark.parametrize("case,scales", G.PARITY, ids=lambda x: getattr(x, "name", ""))
def test_oracle_matches_reference_parity_cases(case, scales):
    d = make_case(case)
    np.testing.assert_allclose(checksum(d), GOLD[f"{case.name}|checksum"], rtol=1e-12, atol=1e-9)
    for s_os, s_ss in scales:
        compare(case, d, s_os, s_ss)


@pytest.mark.parametrize("idx_case", G.c4_subset(), ids=lambda x: x[1].name)
def test_oracle_matches_reference_c4_subset(idx_case):
    _, case = idx_case
    d = make_case(case)
    np.testing.assert_allclose(checksum(d), GOLD[f"{case.name}|checksum"], rtol=1e-12, atol=1e-9)
    compare(case, d, 1.0, 0.5)


def test_oracle_matches_reference_c1s():
    """The c1 generators at N=200, M=600, R=800, UHF 16/15, every loop run
    (about a minute of numpy)."""
    d = make_case(G.C1S)
    np.testing.assert_allclose(checksum(d), GOLD[f"{G.C1S.name}|checksum"], rtol=1e-12)
    e, f, t = oracle_form_fock(d, True, True, 1.0, 0.5)
    E = float(GOLD[key("c1s", 1.0, 0.5, "energy")])
    F = GOLD[key("c1s", 1.0, 0.5, "fock")]
    assert abs(e - E) <= 1e-9 * abs(E)
    assert np.max(np.abs(np.concatenate(f, axis=1) - F)) <= 1e-9 * np.max(np.abs(F))


@pytest.mark.parametrize("edge", G.ABS_EDGE, ids=lambda e: e.name)
def test_oracle_abs_projectors_at_drop_threshold(edge):
    """One eigenvalue 0.1 % below and one 0.1 % above max(1e-6, 1e-8 lambda_max):
    the oracle keeps the same eigenvectors as libuw12 and gives the same blocks."""
    S, lam = G.abs_edge_overlap(edge)
    np.testing.assert_allclose(S, GOLD[f"abs|{edge.name}|S"], rtol=1e-13, atol=1e-15)
    n = edge.n_ao + edge.n_ri
    assert int(GOLD[f"abs|{edge.name}|n_kept"]) == n - 1
    p = O.calculate_abs_projectors(GOLD[f"abs|{edge.name}|S"], edge.n_ao, edge.n_ri)
    # S^-1 over the kept space has condition number lambda_max / lambda_kept_min
    # (1e6 and 1e8 here): rounding of the eigenvectors is amplified by it
    cond = lam.max() / lam[1]
    for nm, got in zip(("ri_ri", "ri_ao", "ao_ri", "ao_ao"),
                       (p.s_inv_ri_ri, p.s_inv_ri_ao, p.s_inv_ao_ri, p.s_inv_ao_ao)):
        ref = GOLD[f"abs|{edge.name}|{nm}"]
        assert np.max(np.abs(got - ref)) <= 1e-14 * cond * np.max(np.abs(ref)), nm


@pytest.mark.parametrize("err", G.ERRORS, ids=lambda e: e[0])
def test_oracle_raises_the_reference_error_class(err):
    name, what, arg = err
    cls = int(GOLD[f"error|{name}|class"])
    assert cls in (1, 2)
    d = make_case(G.ERROR_CASE)
    n_active = list(G.ERROR_CASE.n_active)
    if what == "n_active":
        n_active = arg
    elif what == "occ_alpha_negative":
        d.occ = [-d.occ[0], d.occ[1]]
    elif what == "W2_asymmetric":
        d.W2 = d.W2 + np.triu(np.ones_like(d.W2), 1)
    expected = O.UW12RuntimeError if cls == 1 else O.UW12LogicError
    with pytest.raises(expected):
        W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
        V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
        WV = O.BaseIntegrals(d.WV3, d.WV2)
        absp = O.calculate_abs_projectors(d.S, d.case.n_ao, d.case.n_ri)
        O.form_fock(W, V, WV, absp, d.orbitals, d.occ, n_active, True, True, 1.0, 0.5)


def test_goldens_record_the_reference_sources():
    srcs = json.loads(str(GOLD["meta|sources"]))
    for f in ("src/uw12.cpp", "src/three_electron/indirect_utils.cpp",
              "src/three_electron/direct_utils.cpp", "src/four_electron/four_electron.cpp",
              "src/two_electron/two_electron.cpp", "src/integrals/integrals.cpp", "libuw12.cpp"):
        assert len(srcs[f]) == 64
