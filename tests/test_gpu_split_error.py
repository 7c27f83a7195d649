"""A split-precision evaluation states its error against FP64 in Hartree
(``form_fock_split``).

Every GEMM is routed through the split path (threshold 0).  The stated errors
are the differences from the FP64 evaluation of the same handles; at 14 moduli
the split result meets the FP64 parity tolerances against the oracle, and at 8
moduli the 1e-6 / 1e-5 relative tolerances of split precision.
"""
import numpy as np
import pytest

from tests.parity_cases import CASES, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_moduli,tol_e,tol_f", [(14, 1e-8, 1e-7), (8, 1e-6, 1e-5)])
def test_split_result_states_its_error(uw12lib, cuda_device, n_moduli, tol_e, tol_f):
    L = uw12lib
    case = [c for c in CASES if c.name == "unit_tiles"][0]
    d = make_case(case)
    W = L.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = L.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = L.setup_base_integrals(d.WV3, d.WV2)
    A = L.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    L.set_split_threshold(0.0)
    try:
        e, f, t, err = L.form_fock_split(W, V, WV, A, d.orbitals, d.occ, case.n_active, True,
                                         True, 1.0, 0.5, n_moduli=n_moduli)
    finally:
        L.set_split_threshold(2e9)
    e64, f64, t64 = L.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True, 1.0,
                                0.5)
    assert err["n_moduli"] == n_moduli
    assert err["energy_Eh"] == abs(e - e64)
    assert err["terms_Eh"] == tuple(abs(a - b) for a, b in zip(t, t64))
    assert err["fock_max_Eh"] == max(float(np.max(np.abs(a - b))) for a, b in zip(f, f64))
    # against the oracle (the same-spin terms cancel: scale by the run without them)
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    e_dir, f_dir, _ = oracle_form_fock(d, False, True, 1.0, 0.5)
    scale_e = max(1.0, abs(e_ref), abs(e_dir))
    scale_f = max(1.0, max(float(np.max(np.abs(x))) for x in f_ref + f_dir))
    assert abs(e - e_ref) <= tol_e * scale_e
    assert err["energy_Eh"] <= tol_e * scale_e
    assert err["fock_max_Eh"] <= tol_f * scale_f
    for s in range(len(f)):
        assert np.max(np.abs(f[s] - f_ref[s])) <= tol_f * scale_f
