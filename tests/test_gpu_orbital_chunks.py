"""Direct-term evaluations formed over chunks of orbitals.

Without same-spin terms the stacked transforms serve only X_AB, t and the
direct Fock; when the whole intermediates exceed the chunk budget they are
formed for a chunk of orbitals at a time.  A 64 KiB budget forces one-orbital
chunks on these cases; energies, terms and Fock matrices must equal the
whole-intermediate evaluation (default budget) to 1e-12, with and without a
same-spin scale on the direct pairs.
"""
import numpy as np
import pytest

from tests.parity_cases import CASES, Case, make_case

pytestmark = pytest.mark.gpu

CHUNK_CASES = [c for c in CASES if c.name in ("c0_closed", "c0_frozen", "unit_tiles")] + [
    Case("uhf_chunk", 20, 40, 30, (6, 5), (5, 3), "baseline", 9, 4.0),
    Case("uhf_chunk_no_beta_active", 20, 40, 30, (6, 5), (5, 0), "baseline", 10, 4.0),
]


@pytest.mark.parametrize("case", CHUNK_CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.0), (0.8, 0.5)])
def test_orbital_chunked_equals_whole(uw12lib, cuda_device, case, scales):
    d = make_case(case)
    W = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    A = uw12lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    s_os, s_ss = scales
    ref = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, False, True, s_os, s_ss)
    uw12lib.set_memory_budget(64 << 10)
    try:
        got = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, False, True, s_os,
                                s_ss)
        e_only = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, False, False,
                                   s_os, s_ss)[0]
    finally:
        uw12lib.set_memory_budget(0)
    scale = max(1.0, abs(ref[0]))
    assert abs(got[0] - ref[0]) <= 1e-12 * scale
    assert abs(e_only - ref[0]) <= 1e-12 * scale
    for a, b in zip(got[2], ref[2]):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b))
    for s in range(len(ref[1])):
        fs = max(1.0, np.max(np.abs(ref[1][s])))
        assert np.max(np.abs(got[1][s] - ref[1][s])) <= 1e-12 * fs
