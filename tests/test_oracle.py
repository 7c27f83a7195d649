"""Pins the CPU oracle to libuw12's own known-answer and invariant tests.

libuw12's only absolute golden (water, tests/test_water.cpp) cannot be
evaluated because its RI tensors are not shipped, so the oracle is checked
against every known answer and invariant the reference's test-suite asserts
for this path (file:line of the reference test in each docstring), plus a
tighter finite-difference check of the analytic Fock matrix.
"""
import numpy as np
import pytest

from oracle import synth
from oracle import uw12_oracle as O
from tests.parity_cases import Case, make_case

EPS = 1e-10  # tests/catch.hpp:10-15


def test_energy_spin_factor_known_answers():
    """tests/test_four_el_utils.cpp:16-55."""
    f = O.get_energy_spin_factor
    with pytest.raises(Exception):
        f(0, 0, 0, 0, 0)
    with pytest.raises(Exception):
        f(1, 1, 0, 1, 0)
    with pytest.raises(Exception):
        f(1, 0, 1, 1, 0)
    assert f(1, 0, 0, 1, 0) == 2
    assert f(1, 0, 0, 0, 1) == 2
    assert f(1, 0, 0, 1, 0.5) == 3
    with pytest.raises(Exception):
        f(2, 2, 0, 1, 0)
    with pytest.raises(Exception):
        f(2, 0, 2, 1, 0)
    assert f(2, 0, 0, 1, 0.5) == 0.5
    assert f(2, 0, 1, 1, 0.5) == 1
    assert f(2, 1, 0, 1, 0.5) == 1
    assert f(2, 1, 1, 1, 0.5) == 0.5
    with pytest.raises(Exception):
        f(3, 0, 0, 0, 0)


def test_square_lower():
    """tests/test_utils.cpp:14-80: packed order and lower(square(v)) == v."""
    n = 6
    n2 = n * (n + 1) // 2
    vec = synth.uniform_matrix(11, "v", n2, 1).reshape(-1)
    with pytest.raises(O.UW12LogicError):
        O.square(np.ones(13))
    sq = O.square(vec)
    assert sq.shape == (n, n) and np.array_equal(sq, sq.T)
    idx = 0
    for r in range(n):
        for c in range(r + 1):
            assert sq[r, c] == vec[idx]
            idx += 1
    assert np.array_equal(O.lower(sq), vec)
    spd = synth.random_pd(n, 11, "pd")
    with pytest.raises(O.UW12LogicError):
        O.lower(np.ones((n, n + 1)))
    with pytest.raises(O.UW12LogicError):
        O.lower(np.triu(np.ones((n, n))))
    for factor in (1.0, 2.0, 3.5):
        v = O.lower(spd, factor)
        idx = 0
        for r in range(n):
            for c in range(r + 1):
                assert abs(spd[r, c] - v[idx] / (1.0 if r == c else factor)) <= EPS
                idx += 1


def test_transformations_against_explicit_products():
    """tests/test_integral_transformations.cpp:12-88."""
    n_ao, n_df, n_occ, n1 = 7, 9, 3, 5
    J3 = synth.uniform_matrix(1, "J3", n_ao * (n_ao + 1) // 2, n_df)
    C = synth.uniform_matrix(1, "C", n_ao, n_occ)
    one = O.mo_transform_one_index_full(J3, C)
    for A in range(n_df):
        ref = O.square(J3[:, A]) @ C
        assert np.allclose(one[:, A].reshape((n_ao, n_occ), order="F"), ref, atol=EPS, rtol=0)
    J = synth.uniform_matrix(2, "J", n_ao * n1, n_df)
    first = O.transform_first_index(J, C)
    second = O.transform_second_index(synth.uniform_matrix(3, "K", n1 * n_ao, n_df), C)
    K = synth.uniform_matrix(3, "K", n1 * n_ao, n_df)
    for A in range(n_df):
        ref1 = C.T @ J[:, A].reshape((n_ao, n1), order="F")
        assert np.allclose(first[:, A].reshape((n_occ, n1), order="F"), ref1, atol=EPS, rtol=0)
        ref2 = K[:, A].reshape((n1, n_ao), order="F") @ C
        assert np.allclose(second[:, A].reshape((n1, n_occ), order="F"), ref2, atol=EPS, rtol=0)


def test_abs_projector_shapes_and_errors():
    """tests/test_ri_utils.cpp:12-44."""
    n_ao, n_ri = 10, 24
    s = synth.random_pd(n_ao + n_ri, 11, "S")
    p = O.calculate_abs_projectors(s, n_ao, n_ri)
    assert p.s_inv_ao_ao.shape == (n_ao, n_ao)
    assert p.s_inv_ao_ri.shape == (n_ao, n_ri)
    assert p.s_inv_ri_ao.shape == (n_ri, n_ao)
    assert p.s_inv_ri_ri.shape == (n_ri, n_ri)
    # full-rank S: the projectors are the blocks of S^-1
    inv = np.linalg.inv(s)
    assert np.allclose(p.s_inv_ao_ao, inv[:n_ao, :n_ao], atol=1e-10)
    assert np.allclose(p.s_inv_ri_ao, inv[n_ao:, :n_ao], atol=1e-10)
    for bad in ((n_ao + 1, n_ri), (n_ao - 1, n_ri), (n_ao, n_ri + 1), (n_ao, n_ri - 1)):
        with pytest.raises(O.UW12RuntimeError):
            O.calculate_abs_projectors(s, *bad)


def test_ttilde_symmetric_when_w_equals_v():
    """tests/test_four_el_utils.cpp:101-164."""
    d = make_case(Case("t", 9, 19, 5, (4,), (3,), "unit", 11))
    base = O.BaseIntegrals(d.W3, d.W2)
    Co = O.occupation_weighted_orbitals(d.orbitals, d.occ)
    Ca = O.freeze_core(Co, [3])
    ints = O.Integrals(base, Co, Ca)
    t = O.calculate_tab(ints, ints)[0]
    tt = O.calculate_ttilde(ints, ints)[0]
    assert np.allclose(t, t.T, atol=1e-10 * np.max(np.abs(t)))
    assert np.allclose(tt, tt.T, atol=1e-10 * np.max(np.abs(tt)))


def _ff(d, s_os, s_ss, indirect=True, calc=True, act=None):
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, d.case.n_ao, d.case.n_ri)
    r = O.form_fock(W, V, WV, absp, d.orbitals, d.occ, list(act or d.case.n_active), indirect,
                    calc, s_os, s_ss)
    return r


UNIT_OPEN = Case("o", 5, 8, 14, (4, 3), (3, 2), "unit", 11)
UNIT_CLOSED = Case("c", 5, 8, 14, (3,), (2,), "unit", 11)


@pytest.mark.parametrize("case", [UNIT_CLOSED, UNIT_OPEN], ids=["closed", "open"])
def test_uw12_linearity(case):
    """tests/test_uw12.cpp:42-95: E(1,0) + 0.5 E(0,1) == E(1,0.5), same for F."""
    d = make_case(case)
    a = _ff(d, 1.0, 0.0)
    b = _ff(d, 0.0, 1.0)
    c = _ff(d, 1.0, 0.5)
    assert abs(a.energy + 0.5 * b.energy - c.energy) <= EPS * abs(c.energy)
    for s in range(len(case.n_occ)):
        assert np.allclose(a.fock[s] + 0.5 * b.fock[s], c.fock[s], atol=EPS, rtol=EPS)


def test_uw12_error_handling():
    """tests/test_uw12.cpp:97-113."""
    d = make_case(UNIT_OPEN)
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, 5, 14)
    ff = lambda orb, occ, act: O.form_fock(W, V, WV, absp, orb, occ, act, True, True, 1.0, 0.5)
    with pytest.raises(Exception):
        ff(d.orbitals, d.occ, [3])
    with pytest.raises(Exception):
        ff(d.orbitals, [d.occ[0]], [3, 2])
    with pytest.raises(Exception):
        ff([d.orbitals[0]], d.occ, [3, 2])
    act_orb = [o[:, 1:] for o in d.orbitals]
    with pytest.raises(Exception):
        ff(act_orb, [np.ones(3), np.ones(2)], [4, 3])


def test_energy_unchanged_without_fock_or_indirect():
    """tests/multi_el_test_utils.hpp:39-60."""
    d = make_case(UNIT_OPEN)
    full = _ff(d, 1.0, 0.0, True, True)
    no_ind = _ff(d, 1.0, 0.0, False, True)
    no_fock = _ff(d, 1.0, 0.0, False, False)
    assert abs(full.energy - no_ind.energy) <= EPS * abs(full.energy)
    assert abs(full.energy - no_fock.energy) <= EPS * abs(full.energy)
    for s in range(2):
        assert np.allclose(full.fock[s], no_ind.fock[s], rtol=EPS, atol=EPS)
        assert np.array_equal(no_fock.fock[s], np.zeros_like(no_fock.fock[s]))


def test_scale_zero_and_scale_factor():
    """tests/multi_el_test_utils.hpp:62-83, 137-152."""
    d = make_case(UNIT_OPEN)
    z = _ff(d, 0.0, 0.0)
    assert z.energy == 0.0 and all(np.all(f == 0) for f in z.fock)
    a = _ff(d, 1.0, 0.0)
    b = _ff(d, 1.5, 0.0)
    assert abs(b.energy - 1.5 * a.energy) <= EPS * abs(b.energy)
    a = _ff(d, 0.0, 1.0)
    b = _ff(d, 0.0, 1.5)
    assert abs(b.energy - 1.5 * a.energy) <= 10 * EPS * abs(b.energy)
    for s in range(2):
        assert np.allclose(b.fock[s], 1.5 * a.fock[s], rtol=10 * EPS, atol=10 * EPS)


def test_w_v_symmetry_of_opposite_spin_terms():
    """tests/multi_el_test_utils.hpp:85-94 (three- and four-electron terms,
    opposite spin): swapping W and V leaves energy and Fock unchanged."""
    d = make_case(UNIT_OPEN)
    Wb = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    Vb = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    absp = O.calculate_abs_projectors(d.S, 5, 14)
    Co = O.occupation_weighted_orbitals(d.orbitals, d.occ)
    Ca = O.freeze_core(Co, [3, 2])
    for fn in (lambda W, V: O.form_fock_four_el_df(W, V, False, True, 1.0, 0.0),
               lambda W, V: O.form_fock_three_el_term_df_ri(W, V, absp, False, True, 1.0, 0.0)):
        f1, e1 = fn(O.Integrals(Wb, Co, Ca), O.Integrals(Vb, Co, Ca))
        f2, e2 = fn(O.Integrals(Vb, Co, Ca), O.Integrals(Wb, Co, Ca))
        assert abs(e1 - e2) <= EPS * abs(e1)
        for s in range(2):
            assert np.allclose(f1[s], f2[s], rtol=1e-9, atol=1e-9 * np.max(np.abs(f1[s])))


def test_open_shell_equals_closed_shell():
    """tests/multi_el_test_utils.hpp:183-215."""
    d = make_case(UNIT_CLOSED)
    c = _ff(d, 1.0, 0.5)
    d2 = make_case(UNIT_CLOSED)
    d2.orbitals = [d.orbitals[0], d.orbitals[0]]
    # same occupation-weighted orbitals in both channels: occ/2 per spin
    d2.occ = [d.occ[0] / 2, d.occ[0] / 2]
    o = _ff(d2, 1.0, 0.5, act=[2, 2])
    assert abs(c.energy - o.energy) <= EPS * abs(c.energy)
    for s in range(2):
        assert np.allclose(o.fock[s], c.fock[0], rtol=EPS, atol=EPS * np.max(np.abs(c.fock[0])))


def test_zero_active_and_zero_occupied():
    """tests/multi_el_test_utils.hpp:217-311."""
    d = make_case(Case("z", 6, 9, 8, (5,), (0,), "unit", 12))
    r = _ff(d, 1.0, 0.5)
    assert abs(r.energy) <= EPS and np.all(np.abs(r.fock[0]) <= EPS)
    d = make_case(Case("z2", 6, 9, 8, (0,), (0,), "unit", 12))
    r = _ff(d, 1.0, 0.5)
    assert r.energy == 0.0 and np.all(r.fock[0] == 0.0)
    # open shell, one channel without active orbitals: zero energy for os,
    # zero Fock in that channel for the opposite-spin term of the other one
    d = make_case(Case("z3", 6, 9, 8, (5, 4), (2, 0), "unit", 12))
    r = _ff(d, 1.0, 0.0)
    assert abs(r.energy) <= 1e-8


@pytest.mark.parametrize("n_occ", [(3,), (3, 2)], ids=["closed", "open"])
@pytest.mark.parametrize("s_ss", [0.0, 0.5])
def test_analytic_fock_is_derivative_of_energy(n_occ, s_ss):
    """tests/numerical_fock.hpp:22-141 and multi_el_test_utils.hpp:313-367,
    tightened: the directional derivative of E along D(t) = per (C+tX)(C+tX)^T
    (all-electron, occupations fixed) equals <F, dD/dt> to 1e-6 relative
    (central differences, h = 1e-5; the reference bound is 0.5)."""
    case = Case("fd", 6, 11, 9, n_occ, n_occ, "unit", 21)
    d = make_case(case)
    ns = len(n_occ)
    per = 2.0 if ns == 1 else 1.0
    d.occ = [np.full(o, per) for o in n_occ]
    X = [synth.gaussian_matrix(5, f"X{s}", 6, o) for s, o in enumerate(n_occ)]
    base = [o.copy() for o in d.orbitals]

    def energy(t):
        d.orbitals = [b + t * x for b, x in zip(base, X)]
        return _ff(d, 1.0, s_ss, calc=False).energy

    d.orbitals = base
    r = _ff(d, 1.0, s_ss)
    h = 1e-5
    num = (energy(h) - energy(-h)) / (2 * h)
    ana = 0.0
    for s in range(ns):
        dD = per * (X[s] @ base[s].T + base[s] @ X[s].T)
        ana += float(np.sum(r.fock[s] * dD))
    assert abs(num - ana) <= 1e-6 * max(abs(ana), 1e-12 * abs(r.energy))
