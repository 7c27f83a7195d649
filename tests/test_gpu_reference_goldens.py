"""The CUDA path (through the C-ABI) against libuw12's own results
(tests/golden/reference_goldens.npz, written by tests/golden/make_golden.py from
the reference's unmodified sources).

Tolerances are the GPU parity tests' (FP64 on both sides, different summation
orders and eigensolvers): ``unit`` inputs |dE| <= 1e-8 max(1, scale) and
max|dF| <= 1e-7 max(1, scale) (libuw12's regression tolerances); ``baseline``
inputs (metric condition numbers up to 1e6) 1e-9 and 1e-8 relative. With
same-spin scaling the scale is the magnitude of the run without the exchange
term, whose cancellation against the direct part FP64 cannot resolve below
that magnitude.
"""
import re

import numpy as np
import pytest

from tests import golden_cases as G
from tests.parity_cases import make_case

pytestmark = pytest.mark.gpu

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                          "reference_goldens.npz"))


def key(name, s_os, s_ss, what):
    return f"{name}|{s_os:g},{s_ss:g}|{what}"


def tols(case):
    return (1e-8, 1e-7) if case.family == "unit" else (1e-9, 1e-8)


def handles(lib, d):
    c = d.case
    return (lib.setup_base_integrals(d.W3, d.W2, d.W3_ri),
            lib.setup_base_integrals(d.V3, d.V2, d.V3_ri),
            lib.setup_base_integrals(d.WV3, d.WV2),
            lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri))


def check(case, got, s_os, s_ss, direct=None):
    """got = (energy, fock list or None, terms); direct = the same run without
    the exchange term (scale of the cancellation) or None."""
    e, f, t = got
    te, tf = tols(case)
    E = float(GOLD[key(case.name, s_os, s_ss, "energy")])
    T = GOLD[key(case.name, s_os, s_ss, "terms")]
    scale = max(abs(E), float(np.max(np.abs(T))))
    f_scale = 0.0
    if direct is not None:
        scale = max(scale, abs(direct[0]), max(abs(x) for x in direct[2]))
        if direct[1] is not None:
            f_scale = float(np.max(np.abs(np.concatenate(direct[1], axis=1))))
    if case.family == "unit":
        scale = max(1.0, scale)
    assert abs(e - E) <= te * scale, (case.name, s_os, s_ss, e, E)
    for k in range(3):
        assert abs(t[k] - T[k]) <= te * scale * 10, (case.name, k, t[k], T[k])
    fk = key(case.name, s_os, s_ss, "fock")
    if f is not None and fk in GOLD:
        F = GOLD[fk]
        fs = max(float(np.max(np.abs(F))), f_scale)
        fs = max(1.0, fs) if case.family == "unit" else fs
        assert np.max(np.abs(np.concatenate(f, axis=1) - F)) <= tf * fs, (case.name, s_os, s_ss)


def run(lib, h, d, s_os, s_ss, indirect=None, fock=True):
    W, V, WV, A = h
    ind = (s_ss != 0.0) if indirect is None else indirect
    return lib.form_fock(W, V, WV, A, d.orbitals, d.occ, list(d.case.n_active), ind, fock,
                         s_os, s_ss)


@pytest.mark.parametrize("case,scales", G.PARITY, ids=lambda x: getattr(x, "name", ""))
def test_cuda_matches_reference_parity_cases(uw12lib, cuda_device, case, scales):
    d = make_case(case)
    h = handles(uw12lib, d)
    for s_os, s_ss in scales:
        got = run(uw12lib, h, d, s_os, s_ss)
        direct = run(uw12lib, h, d, s_os, s_ss, indirect=False) if s_ss != 0.0 else None
        check(case, got, s_os, s_ss, direct)


def test_cuda_matches_reference_c1s(uw12lib, cuda_device):
    """The c1 workload's generators at N=200, M=600, R=800, UHF 16/15."""
    d = make_case(G.C1S)
    h = handles(uw12lib, d)
    for s_os, s_ss in G.C1S_SCALES:
        got = run(uw12lib, h, d, s_os, s_ss)
        direct = run(uw12lib, h, d, s_os, s_ss, indirect=False) if s_ss != 0.0 else None
        check(G.C1S, got, s_os, s_ss, direct)


@pytest.mark.parametrize("n_streams", [1, 4])
def test_cuda_batch_matches_reference_c4_subset(uw12lib, cuda_device, n_streams):
    """Molecules of the 64-molecule batch (N <= 60) evaluated in one batched
    call, each against libuw12's result."""
    mols, cases = [], []
    for _, case in G.c4_subset():
        d = make_case(case)
        W, V, WV, A = handles(uw12lib, d)
        mols.append({"W": W, "V": V, "WV": WV, "abs": A, "orbitals": d.orbitals, "occ": d.occ,
                     "n_active": list(case.n_active)})
        cases.append((case, d))
    res = uw12lib.fock_batched(mols, True, True, 1.0, 0.5, n_streams=n_streams)
    direct = uw12lib.fock_batched(mols, False, True, 1.0, 0.5, n_streams=n_streams)
    for (case, d), got, dr in zip(cases, res, direct):
        check(case, got, 1.0, 0.5, dr)


@pytest.mark.parametrize("edge", G.ABS_EDGE, ids=lambda e: e.name)
def test_cuda_abs_projectors_at_drop_threshold(uw12lib, cuda_device, edge):
    """An eigenvalue 0.1 % below the drop threshold is dropped and one 0.1 %
    above is kept, as by libuw12 (a different kept set changes the blocks by
    ~1/threshold)."""
    S = GOLD[f"abs|{edge.name}|S"]
    A = uw12lib.setup_abs_projectors(S, edge.n_ao, edge.n_ri)
    _, lam = G.abs_edge_overlap(edge)
    cond = lam.max() / lam[1]
    for nm, got in zip(("ri_ri", "ri_ao", "ao_ri", "ao_ao"), A.blocks()):
        ref = GOLD[f"abs|{edge.name}|{nm}"]
        assert np.max(np.abs(got - ref)) <= 1e-14 * cond * np.max(np.abs(ref)), nm


@pytest.mark.parametrize("err", G.ERRORS, ids=lambda e: e[0])
def test_cuda_raises_the_reference_error(uw12lib, cuda_device, err):
    name, what, arg = err
    cls = int(GOLD[f"error|{name}|class"])
    msg = str(GOLD[f"error|{name}|message"])
    d = make_case(G.ERROR_CASE)
    n_active = list(G.ERROR_CASE.n_active)
    if what == "n_active":
        n_active = arg
    elif what == "occ_alpha_negative":
        d.occ = [-d.occ[0], d.occ[1]]
    elif what == "W2_asymmetric":
        d.W2 = d.W2 + np.triu(np.ones_like(d.W2), 1)
    expected = uw12lib.UW12RuntimeError if cls == 1 else uw12lib.UW12LogicError
    with pytest.raises(expected, match=re.escape(msg)):
        W, V, WV, A = handles(uw12lib, d)
        uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, n_active, True, True, 1.0, 0.5)
