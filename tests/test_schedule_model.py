"""The pair-loop-free schedule implemented by the CUDA engine (numpy model in
tests/schedule_model.py) equals the operation-for-operation oracle."""
import numpy as np
import pytest

from oracle import uw12_oracle as O
from tests import schedule_model as K
from tests.parity_cases import Case, make_case

CASES = [
    Case("closed", 6, 10, 9, (3,), (3,), "baseline", 3, 4.0),
    Case("frozen", 6, 10, 9, (3,), (2,), "baseline", 3, 4.0),
    Case("open", 7, 11, 9, (4, 3), (3, 2), "baseline", 3, 4.0),
    Case("open_allel", 7, 11, 9, (4, 3), (4, 3), "baseline", 4, 4.0),
    Case("one_inactive", 7, 11, 9, (4, 3), (2, 0), "baseline", 5, 4.0),
    Case("no_beta", 7, 11, 9, (3, 0), (2, 0), "baseline", 6, 4.0),
    Case("none_active", 7, 11, 9, (4, 3), (0, 0), "baseline", 7, 4.0),
    Case("unit", 5, 8, 14, (4, 3), (3, 2), "unit", 11),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.5), (1.0, 0.0), (0.0, 1.0)])
def test_schedule_equals_oracle(case, scales):
    d = make_case(case)
    s_os, s_ss = scales
    ind = not O.nearly_zero(s_ss)
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    vals, vecs = O.eigen_decomposition(d.S, 1e-6, 1e-8)
    Sinv = (vecs / vals) @ vecs.T
    r = O.form_fock(W, V, WV, absp, d.orbitals, d.occ, list(case.n_active), ind, True, s_os, s_ss)
    e, F, _ = K.form_fock(W, V, WV, Sinv, d.orbitals, d.occ, list(case.n_active), ind, True,
                          s_os, s_ss)
    scale = max(abs(r.energy), 1e-300)
    assert abs(e - r.energy) <= 1e-12 * scale + 1e-300
    fo = np.concatenate(r.fock, 1)
    fc = np.concatenate(F, 1)
    assert np.max(np.abs(fo - fc)) <= 1e-12 * max(np.max(np.abs(fo)), 1e-300)


@pytest.mark.parametrize("case", [c for c in CASES if c.name in ("closed", "frozen", "open",
                                                                   "one_inactive", "unit")],
                         ids=lambda c: c.name)
@pytest.mark.parametrize("chunk", [1, 2, 3])
def test_orbital_chunked_direct_terms(case, chunk):
    """X_AB, t and the combined direct-Fock contraction formed over chunks of
    orbitals equal the same quantities formed whole (1e-12)."""
    d = make_case(case)
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    vals, vecs = O.eigen_decomposition(d.S, 1e-6, 1e-8)
    Sinv = (vecs / vals) @ vecs.T
    Co = O.occupation_weighted_orbitals(d.orbitals, d.occ)
    Ca = O.freeze_core(Co, list(case.n_active))
    N, R, M = W.n_ao, W.n_ri, W.n_df
    Rp = N + R
    rng = np.random.default_rng(1)
    for s in range(len(Co)):
        o, a = Co[s].shape[1], Ca[s].shape[1]
        # whole, as in the schedule model
        st = {}
        for Xi, nm in ((W, "W"), (V, "V")):
            st[nm] = (K._stacked(Xi, Co[s], Ca[s], 0, a, R) if a else np.zeros((0, M)))
        svs = (Sinv @ st["V"].reshape(Rp, a * M, order="F")).reshape(Rp * a, M, order="F")
        X = st["W"].T @ svs
        t = (K.T3(K.T1(W.J3_0, Co[s], W.P2), Ca[s]).T @ K.T3(K.T1(V.J3_0, Co[s], V.P2), Ca[s]))
        Xc, tc = K.chunked_xab_t(W, V, Sinv, Co[s], Ca[s], chunk)
        for got, ref in ((Xc, X), (tc, t)):
            assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
        if o == 0:
            continue
        Y = rng.standard_normal((M, M))
        b1w, b1v = K.T1(W.J3_0, Co[s], W.P2), K.T1(V.J3_0, Co[s], V.P2)
        Z3 = (b1w @ Y).reshape((N, o, M), order="F").copy()
        if a > 0:
            Z3[:, o - a:, :] *= 2.0
        Fw = Z3.reshape(N, o * M, order="F") @ b1v.reshape(N, o * M, order="F").T
        Fc = K.chunked_direct_fock(W, V, Co[s], a, Y, chunk)
        assert np.max(np.abs(Fc - Fw)) <= 1e-12 * max(1.0, np.max(np.abs(Fw)))
