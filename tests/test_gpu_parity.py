"""CUDA path vs the CPU oracle on identical seeded inputs (through the C-ABI).

Tolerances (FP64 on both sides, different summation orders and different
eigensolvers for the metrics):
  * well-conditioned ``unit`` inputs: |dE| <= 1e-8 max(1,|E|) and
    max|dF| <= 1e-7 max(1, max|F|) -- libuw12's regression tolerances;
  * ``baseline`` inputs (metric condition numbers up to ~1e6):
    |dE| <= 1e-9 |E| and max|dF| <= 1e-8 max|F|.
With same-spin scaling the same-spin direct and exchange contributions cancel
(by up to 1e-7 for the all-positive ``unit`` tensors), so |E| and max|F| above
are replaced by the larger magnitude of the same run without the exchange
(indirect) term: FP64 rounding is relative to the terms, not their difference.
"""
import numpy as np
import pytest

from tests.parity_cases import CASES, Case, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu


def _tols(case):
    return (1e-8, 1e-7) if case.family == "unit" else (1e-9, 1e-8)


def _gpu_objects(lib, d):
    c = d.case
    W = lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = lib.setup_base_integrals(d.WV3, d.WV2)
    A = lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    return W, V, WV, A


def _cmp(case, e_ref, f_ref, e_gpu, f_gpu, e_scale=0.0, f_scale=0.0):
    """e_scale / f_scale: magnitude of the same-spin direct part when the
    same-spin direct and exchange terms cancel (the error of FP64 evaluation is
    relative to the terms, not to their difference)."""
    te, tf = _tols(case)
    scale_e = max(abs(e_ref), e_scale)
    scale_e = max(1.0, scale_e) if case.family == "unit" else scale_e
    assert abs(e_gpu - e_ref) <= te * max(scale_e, 1e-300), (e_gpu, e_ref)
    if f_ref is not None:
        fr = np.concatenate(f_ref, axis=1)
        fg = np.concatenate(f_gpu, axis=1)
        scale_f = max(np.max(np.abs(fr)) if fr.size else 0.0, f_scale)
        scale_f = max(1.0, scale_f) if case.family == "unit" else max(scale_f, 1e-300)
        assert np.max(np.abs(fg - fr)) <= tf * scale_f


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.5), (1.0, 0.0), (0.0, 1.0)])
def test_form_fock_matches_oracle(uw12lib, cuda_device, case, scales):
    d = make_case(case)
    s_os, s_ss = scales
    indirect = s_ss != 0.0
    e_ref, f_ref, t_ref = oracle_form_fock(d, indirect, True, s_os, s_ss)
    e_dir, f_dir, t_dir = oracle_form_fock(d, False, True, s_os, s_ss)
    f_scale = float(np.max(np.abs(np.concatenate(f_dir, axis=1))))
    W, V, WV, A = _gpu_objects(uw12lib, d)
    e, f, terms = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, indirect, True,
                                    s_os, s_ss)
    _cmp(case, e_ref, f_ref, e, f, abs(e_dir), f_scale)
    for k, name in enumerate(("two", "three", "four")):
        te, _ = _tols(case)
        scale = max(1.0, abs(e_ref), abs(t_ref[name]), abs(t_dir[name]))
        assert abs(terms[k] - t_ref[name]) <= te * scale * 10


@pytest.mark.parametrize("case", [c for c in CASES if c.name in ("c0_closed", "uhf_small")],
                         ids=lambda c: c.name)
def test_energy_only_and_public_api(uw12lib, cuda_device, case):
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d)
    e_full, f_full = uw12lib.uw12_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0, 0.5)
    e_only = uw12lib.uw12_energy(W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0, 0.5)
    assert abs(e_full - e_only) <= 1e-12 * abs(e_full)
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    _cmp(case, e_ref, f_ref, e_full,
         [f_full[:, s * case.n_ao:(s + 1) * case.n_ao] for s in range(len(case.n_occ))])


def test_linearity_in_scale_factors(uw12lib, cuda_device):
    """os + 0.5 ss == full (tests/test_uw12.cpp:42-72)."""
    case = CASES[2]
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d)
    run = lambda a, b: uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True,
                                         True, a, b)
    e_os, f_os, _ = run(1.0, 0.0)
    e_ss, f_ss, _ = run(0.0, 1.0)
    e, f, _ = run(1.0, 0.5)
    assert abs(e_os + 0.5 * e_ss - e) <= 1e-10 * abs(e)
    for s in range(2):
        assert np.max(np.abs(f_os[s] + 0.5 * f_ss[s] - f[s])) <= 1e-10 * np.max(np.abs(f[s]))


def test_open_equals_closed(uw12lib, cuda_device):
    """Closed shell == open shell with duplicated orbitals
    (tests/multi_el_test_utils.hpp:183-215)."""
    case = Case("c", 9, 13, 11, (4,), (3,), "baseline", 8, 4.0)
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d)
    e1, f1, _ = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, [3], True, True, 1.0, 0.5)
    orb2 = [d.orbitals[0], d.orbitals[0]]
    occ2 = [d.occ[0] / 2.0, d.occ[0] / 2.0]
    e2, f2, _ = uw12lib.form_fock(W, V, WV, A, orb2, occ2, [3, 3], True, True, 1.0, 0.5)
    assert abs(e1 - e2) <= 1e-10 * abs(e1)
    for s in range(2):
        assert np.max(np.abs(f2[s] - f1[0])) <= 1e-10 * np.max(np.abs(f1[0]))


def test_error_handling(uw12lib, cuda_device):
    """tests/test_uw12.cpp:97-113: mismatched spin channels and n_active > n_occ."""
    case = CASES[2]
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d)
    ff = lambda orb, occ, act: uw12lib.form_fock(W, V, WV, A, orb, occ, act, True, True, 1.0, 0.5)
    with pytest.raises(uw12lib.UW12Error):
        ff(d.orbitals, d.occ, [3])
    with pytest.raises(uw12lib.UW12Error):
        ff(d.orbitals, [d.occ[0]], [3, 2])
    with pytest.raises(uw12lib.UW12Error):
        ff([d.orbitals[0]], d.occ, [3, 2])
    with pytest.raises(uw12lib.UW12LogicError):
        ff(d.orbitals, d.occ, [5, 2])
    with pytest.raises(uw12lib.UW12RuntimeError):
        ff(d.orbitals, [-d.occ[0], d.occ[1]], [3, 2])
    with pytest.raises(uw12lib.UW12LogicError):
        uw12lib.setup_base_integrals(d.W3, d.W2 + np.triu(np.ones_like(d.W2), 1), d.W3_ri)
    # the library stays usable after errors
    e, _, _ = ff(d.orbitals, d.occ, [3, 2])
    assert np.isfinite(e)


def test_unequal_df_sizes_rejected(uw12lib, cuda_device):
    """libuw12's calculate_xab sums (M_W x M_V) blocks into an n_df(V)^2 matrix
    (src/three_electron/direct_utils.cpp:75-111), so unequal df sizes throw."""
    c1 = make_case(Case("a", 8, 12, 10, (3,), (3,), "baseline", 9, 4.0))
    c2 = make_case(Case("b", 8, 13, 10, (3,), (3,), "baseline", 9, 4.0))
    W = uw12lib.setup_base_integrals(c1.W3, c1.W2, c1.W3_ri)
    V = uw12lib.setup_base_integrals(c2.V3, c2.V2, c2.V3_ri)
    WV = uw12lib.setup_base_integrals(c1.WV3, c1.WV2)
    A = uw12lib.setup_abs_projectors(c1.S, 8, 10)
    with pytest.raises(uw12lib.UW12LogicError):
        uw12lib.form_fock(W, V, WV, A, c1.orbitals, c1.occ, [3], True, True, 1.0, 0.5)


def test_eigenbasis_integrals_constructor(uw12lib, cuda_device):
    """BaseIntegrals(J3, df_vals) (base_integrals.hpp:104) with J3 = J3_0 P2 gives the
    same result as BaseIntegrals(J3_0, J2) (the metric enters only through P2 Λ P2^T)."""
    from oracle import uw12_oracle as O
    case = CASES[2]
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d)
    ob = O.BaseIntegrals(d.WV3, d.WV2)
    WV_eig = uw12lib.base_integrals_eigenbasis(d.WV3 @ ob.P2, ob.df_vals)
    e1, f1, _ = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True,
                                  1.0, 0.5)
    e2, f2, _ = uw12lib.form_fock(W, V, WV_eig, A, d.orbitals, d.occ, case.n_active, True, True,
                                  1.0, 0.5)
    assert abs(e1 - e2) <= 1e-9 * abs(e1)
    for s in range(2):
        assert np.max(np.abs(f1[s] - f2[s])) <= 1e-8 * np.max(np.abs(f1[s]))


def test_abs_projectors_match_oracle(uw12lib, cuda_device):
    from oracle import uw12_oracle as O
    d = make_case(CASES[0])
    c = d.case
    ref = O.calculate_abs_projectors(d.S, c.n_ao, c.n_ri)
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    got = A.blocks()
    for g, r in zip(got, (ref.s_inv_ri_ri, ref.s_inv_ri_ao, ref.s_inv_ao_ri, ref.s_inv_ao_ao)):
        assert np.max(np.abs(g - r)) <= 1e-10 * max(1.0, np.max(np.abs(r)))
