"""Batched evaluation (uw12c_fock_batched): molecules of different sizes and
spin states evaluated concurrently on several streams give the results of
one-at-a-time form_fock calls (1e-12 relative: each worker's chunk budget is a
share of the free memory, so the summation order of chunked terms may differ),
match the oracle, and a failing molecule is reported without stopping the
others."""
import numpy as np
import pytest

from tests.parity_cases import Case, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu

BATCH = [
    Case("b0", 12, 30, 26, (4,), (3,), "baseline", 31, 6.0),
    Case("b1", 9, 13, 11, (4, 3), (3, 2), "baseline", 32, 4.0),
    Case("b2", 24, 84, 116, (5,), (5,), "baseline", 33, 8.0),
    Case("b3", 7, 10, 15, (4, 3), (3, 3), "unit", 34),
    Case("b4", 30, 90, 120, (3, 2), (3, 2), "baseline", 35, 8.0),
    Case("b5", 5, 8, 14, (3,), (2,), "unit", 36),
]


def _molecule(lib, c):
    d = make_case(c)
    return d, {"W": lib.setup_base_integrals(d.W3, d.W2, d.W3_ri),
               "V": lib.setup_base_integrals(d.V3, d.V2, d.V3_ri),
               "WV": lib.setup_base_integrals(d.WV3, d.WV2),
               "abs": lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri),
               "orbitals": d.orbitals, "occ": d.occ, "n_active": list(c.n_active)}


@pytest.mark.parametrize("n_streams", [1, 3, 8])
def test_batched_equals_single_calls_and_oracle(uw12lib, cuda_device, n_streams):
    mols = [_molecule(uw12lib, c) for c in BATCH]
    res = uw12lib.fock_batched([m for _, m in mols], True, True, 1.0, 0.5, n_streams=n_streams)
    for (d, m), (e, f, t) in zip(mols, res):
        e1, f1, t1 = uw12lib.form_fock(m["W"], m["V"], m["WV"], m["abs"], m["orbitals"], m["occ"],
                                       m["n_active"], True, True, 1.0, 0.5)
        assert abs(e - e1) <= 1e-12 * abs(e1)
        for s in range(len(f)):
            assert np.max(np.abs(f[s] - f1[s])) <= 1e-12 * np.max(np.abs(f1[s]))
        e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
        assert abs(e - e_ref) <= 1e-8 * max(1.0, abs(e_ref))


def test_failing_molecule_is_reported(uw12lib, cuda_device):
    mols = [_molecule(uw12lib, c)[1] for c in BATCH[:3]]
    bad = dict(mols[1])
    bad["occ"] = [np.full(4, -1.0), np.full(3, 1.0)]  # occupations must be positive
    with pytest.raises(uw12lib.UW12RuntimeError, match="molecule 1"):
        uw12lib.fock_batched([mols[0], bad, mols[2]], True, True, 1.0, 0.5, n_streams=2)
    # the same handles still work afterwards
    res = uw12lib.fock_batched([mols[0], mols[2]], True, False, 1.0, 0.5, n_streams=2)
    assert len(res) == 2 and res[0][1] is None
