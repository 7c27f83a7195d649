"""The adjoint of the direct UW12 terms (tests/adjoint_ref.py, the checker of
the CUDA backward pass) against central finite differences of the oracle
energy: every gradient (J3_0, J3_ri_0 and J2 of W and V, J3_0 and J2 of WV)
contracted with a random direction (symmetric for the metrics), for closed-shell,
open-shell and frozen-core cases and both scale-factor settings."""
import numpy as np
import pytest

from oracle import uw12_oracle as O
from tests import adjoint_ref as AR
from tests.parity_cases import Case, make_case

CASES = [
    Case("unit_closed_small", 5, 8, 14, (3,), (2,), "unit", 11),
    Case("unit_open_small", 5, 8, 14, (4, 3), (3, 2), "unit", 13),
    Case("unit_open_allel", 6, 9, 12, (3, 2), (3, 2), "unit", 17),
]


def _energy(d, c, ints, s_os, s_ss):
    W = O.BaseIntegrals(ints["W3"], ints["W2"], ints["W3_ri"])
    V = O.BaseIntegrals(ints["V3"], ints["V2"], ints["V3_ri"])
    WV = O.BaseIntegrals(ints["WV3"], ints["WV2"])
    absp = O.calculate_abs_projectors(d.S, c.n_ao, c.n_ri)
    return AR.direct_energy(W, V, WV, absp, d.orbitals, d.occ, list(c.n_active), s_os, s_ss)


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.0), (1.0, 0.5)])
def test_adjoint_matches_finite_differences(case, scales):
    s_os, s_ss = scales
    d = make_case(case)
    ints = {"W3": d.W3, "W2": d.W2, "W3_ri": d.W3_ri, "V3": d.V3, "V2": d.V2,
            "V3_ri": d.V3_ri, "WV3": d.WV3, "WV2": d.WV2}
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    g = AR.direct_adjoint(W, V, WV, absp, d.orbitals, d.occ, list(case.n_active), s_os, s_ss)
    e0 = _energy(d, case, ints, s_os, s_ss)
    rng = np.random.default_rng(7)
    h = 1e-5
    for key in ("W3", "W3_ri", "W2", "V3", "V3_ri", "V2", "WV3", "WV2"):
        base = ints[key]
        dirn = rng.standard_normal(base.shape)
        if key.endswith("2"):
            dirn = 0.5 * (dirn + dirn.T)
        plus = dict(ints, **{key: base + h * dirn})
        minus = dict(ints, **{key: base - h * dirn})
        fd = (_energy(d, case, plus, s_os, s_ss) - _energy(d, case, minus, s_os, s_ss)) / (2 * h)
        an = float(np.sum(g[key] * dirn))
        scale = max(abs(fd), 1e-3 * max(1.0, abs(e0)))
        assert abs(an - fd) <= 1e-6 * scale, (key, an, fd)


def test_stacked_x_matches_oracle_xab():
    """The stacked form X = Wst_W^T (I (x) S^-1) Wst_V used by the adjoint is the
    oracle's four-block calculate_xab."""
    case = CASES[1]
    d = make_case(case)
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    Co = O.occupation_weighted_orbitals(d.orbitals, d.occ)
    Ca = O.freeze_core(Co, list(case.n_active))
    Wi, Vi = O.Integrals(W, Co, Ca), O.Integrals(V, Co, Ca)
    x_ref = O.calculate_xab(Wi, Vi, absp)
    N, R = case.n_ao, case.n_ri
    Rp = N + R
    Sinv = np.block([[absp.s_inv_ao_ao, absp.s_inv_ao_ri], [absp.s_inv_ri_ao, absp.s_inv_ri_ri]])
    for s in range(len(Co)):
        o, a = Co[s].shape[1], Ca[s].shape[1]
        c = o - a

        def st(X):
            B1, Bri = X.get_X3idx_one_trans()[s], X.get_X3idx_one_trans_ri()[s]
            out = np.zeros((Rp * a, B1.shape[1]))
            for j in range(a):
                out[Rp * j:Rp * j + N] = B1[N * (c + j):N * (c + j + 1)]
                out[Rp * j + N:Rp * (j + 1)] = Bri[R * j:R * (j + 1)]
            return out

        x = st(Wi).T @ np.kron(np.eye(a), Sinv) @ st(Vi)
        assert np.allclose(x, x_ref[s], rtol=1e-12, atol=1e-12 * np.abs(x_ref[s]).max())


@pytest.mark.parametrize("chunk", [1, 2])
@pytest.mark.parametrize("name", ["closed", "frozen", "open"])
def test_orbital_chunked_three_index_adjoint(name, chunk):
    """The reverse sweep over orbital chunks (the memory layout of large
    systems) equals the whole-intermediate adjoint (1e-12)."""
    case = {"closed": Case("closed", 6, 10, 9, (3,), (3,), "baseline", 3, 4.0),
            "frozen": Case("frozen", 6, 10, 9, (3,), (2,), "baseline", 3, 4.0),
            "open": Case("open", 7, 11, 9, (4, 3), (3, 2), "baseline", 3, 4.0)}[name]
    d = make_case(case)
    Wb = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    Vb = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WVb = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    ref = AR.direct_adjoint(Wb, Vb, WVb, absp, d.orbitals, d.occ, list(case.n_active), 1.0, 0.5)
    got = AR.chunked_three_index_adjoint(Wb, Vb, absp, d.orbitals, d.occ, list(case.n_active),
                                         1.0, 0.5, chunk)
    for key in ("W3", "W3_ri", "V3", "V3_ri"):
        scale = max(np.max(np.abs(ref[key])), 1e-300)
        assert np.max(np.abs(got[key] - ref[key])) <= 1e-12 * scale, key


def _full_energy(d, c, ints, s_os, s_ss):
    W = O.BaseIntegrals(ints["W3"], ints["W2"], ints["W3_ri"])
    V = O.BaseIntegrals(ints["V3"], ints["V2"], ints["V3_ri"])
    WV = O.BaseIntegrals(ints["WV3"], ints["WV2"])
    absp = O.calculate_abs_projectors(d.S, c.n_ao, c.n_ri)
    return AR.full_energy(W, V, WV, absp, d.orbitals, d.occ, list(c.n_active), s_os, s_ss)


@pytest.mark.parametrize("case", CASES + [Case("base_open_frozen", 7, 10, 9, (4, 3), (3, 2),
                                               "baseline", 21, 4.0)], ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.5), (0.0, 1.0)])
def test_same_spin_adjoint_matches_finite_differences(case, scales):
    """dE/d(integrals) of the full energy (same-spin terms included) =
    direct_adjoint + s_ss indirect_adjoint, against central differences."""
    s_os, s_ss = scales
    d = make_case(case)
    ints = {"W3": d.W3, "W2": d.W2, "W3_ri": d.W3_ri, "V3": d.V3, "V2": d.V2,
            "V3_ri": d.V3_ri, "WV3": d.WV3, "WV2": d.WV2}
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    act = list(case.n_active)
    gd = AR.direct_adjoint(W, V, WV, absp, d.orbitals, d.occ, act, s_os, s_ss)
    gi = AR.indirect_adjoint(W, V, WV, absp, d.orbitals, d.occ, act)
    e0 = _full_energy(d, case, ints, s_os, s_ss)
    rng = np.random.default_rng(11)
    for key in ("W3", "W3_ri", "W2", "V3", "V3_ri", "V2", "WV3", "WV2"):
        base = ints[key]
        dirn = rng.standard_normal(base.shape)
        # the baseline metrics have eigenvalues down to ~1e-6: their step must
        # stay well below that for the central difference to be accurate
        h = 1e-5 if (case.family == "unit" or not key.endswith("2")) else 1e-9
        if key.endswith("2"):
            dirn = 0.5 * (dirn + dirn.T)
        plus = dict(ints, **{key: base + h * dirn})
        minus = dict(ints, **{key: base - h * dirn})
        fd = (_full_energy(d, case, plus, s_os, s_ss) -
              _full_energy(d, case, minus, s_os, s_ss)) / (2 * h)
        an = float(np.sum((gd[key] + s_ss * gi[key]) * dirn))
        scale = max(abs(fd), 1e-3 * max(1.0, abs(e0)))
        assert abs(an - fd) <= 1e-6 * scale, (key, an, fd)


@pytest.mark.parametrize("case", CASES[1:] + [Case("base_frozen_b", 7, 10, 9, (4, 3), (3, 2),
                                                   "baseline", 21, 4.0)], ids=lambda c: c.name)
def test_blocked_three_index_adjoint_equals_whole(case):
    """The per-aux-block reverse sweep (no stacked intermediate) gives the whole
    sweep's three-index gradients."""
    d = make_case(case)
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    act = list(case.n_active)
    g = AR.direct_adjoint(W, V, WV, absp, d.orbitals, d.occ, act, 1.0, 0.5)
    for nb in (1, 3):
        gb = AR.blocked_three_index_adjoint(W, V, absp, d.orbitals, d.occ, act, 1.0, 0.5, nb)
        for k in ("W3", "W3_ri", "V3", "V3_ri"):
            assert np.max(np.abs(gb[k] - g[k])) <= 1e-11 * np.max(np.abs(g[k])), (k, nb)
