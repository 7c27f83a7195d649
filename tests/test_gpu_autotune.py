"""The split-K autotuner of the FP64 GEMM engine on the GPU.

* One GEMM with few output tiles and a long contraction: tuning records its
  class and leaves the product of the fastest split (1e-13 relative to
  sum |a||b|, as tests/test_gpu_gemm.py); "use" mode reproduces that result bit
  for bit, and the rule's result agrees to rounding.
* Whole evaluations tuned, then run from the table and from a saved and
  reloaded table: energy, terms and Fock agree with the rule's evaluation to
  1e-12 (relative to the magnitude of the run without the exchange term,
  which the same-spin terms cancel against) and with the oracle at the parity
  tolerances; "use" runs from the same table are identical.
"""
import numpy as np
import pytest

from tests.parity_cases import CASES, make_case, oracle_form_fock

pytestmark = pytest.mark.gpu


@pytest.fixture
def tuner(uw12lib):
    uw12lib.autotune_clear()
    uw12lib.autotune(uw12lib.AUTOTUNE_OFF)
    yield uw12lib
    uw12lib.autotune_clear()
    uw12lib.autotune(uw12lib.AUTOTUNE_OFF)


def test_tuned_gemm_matches_rule(tuner, cuda_device):
    import torch
    L = tuner
    m, n, k = 200, 300, 6000  # 6 output tiles, 375 k tiles
    rng = np.random.default_rng(11)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    dA = torch.from_numpy(np.asfortranarray(A).reshape(-1, order="F")).cuda()
    dB = torch.from_numpy(np.asfortranarray(B).reshape(-1, order="F")).cuda()

    def run():
        dC = torch.full((m * n,), np.nan, dtype=torch.float64, device="cuda")
        L.dgemm(m, n, k, 1.0, dA.data_ptr(), m, False, dB.data_ptr(), k, False, 0.0,
                dC.data_ptr(), m)
        torch.cuda.synchronize()
        return dC.cpu().numpy().reshape((m, n), order="F")

    rule = run()
    L.autotune(L.AUTOTUNE_TUNE)
    tuned = run()
    assert L.autotune_size() == 1
    split = L.autotune_lookup(m, n, k)
    assert 1 <= split <= 64
    L.autotune(L.AUTOTUNE_USE)
    used = run()
    assert np.array_equal(used, tuned)
    scale = np.abs(A) @ np.abs(B)
    ref = A @ B
    assert np.all(np.abs(tuned - ref) <= 1e-13 * scale)
    assert np.all(np.abs(rule - tuned) <= 2e-13 * scale)


def test_tuned_evaluations_match_rule_and_oracle(tuner, cuda_device, tmp_path):
    L = tuner
    case = [c for c in CASES if c.name == "unit_tiles"][0]
    d = make_case(case)
    W = L.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = L.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = L.setup_base_integrals(d.WV3, d.WV2)
    A = L.setup_abs_projectors(d.S, case.n_ao, case.n_ri)

    def evaluate():
        return L.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True, 1.0, 0.5)

    rule = evaluate()
    L.autotune(L.AUTOTUNE_TUNE)
    tuned = evaluate()
    n_classes = L.autotune_size()
    assert n_classes >= 1
    L.autotune(L.AUTOTUNE_USE)
    used = evaluate()
    path = tmp_path / "splits.txt"
    L.autotune_save(str(path))
    L.autotune_clear()
    L.autotune(L.AUTOTUNE_USE, str(path))
    assert L.autotune_size() == n_classes
    reloaded = evaluate()
    assert reloaded[0] == used[0] and reloaded[2] == used[2]
    for s in range(len(used[1])):
        assert np.array_equal(reloaded[1][s], used[1][s])
    e_ref, f_ref, _ = oracle_form_fock(d, True, True, 1.0, 0.5)
    # the parity tolerances; the same-spin direct and exchange terms cancel, so
    # the scale is the larger magnitude of the run without the exchange term
    e_dir, f_dir, _ = oracle_form_fock(d, False, True, 1.0, 0.5)
    te, tf = (1e-8, 1e-7) if case.family == "unit" else (1e-9, 1e-8)
    scale_e = max(1.0, abs(e_ref), abs(e_dir))
    scale_f = max(1.0, max(np.max(np.abs(f)) for f in f_ref + f_dir))
    for got in (tuned, used):
        assert abs(got[0] - rule[0]) <= 1e-12 * scale_e
        for a, b in zip(got[2], rule[2]):
            assert abs(a - b) <= 1e-12 * max(scale_e, abs(b))
        for s in range(len(rule[1])):
            assert np.max(np.abs(got[1][s] - rule[1][s])) <= 1e-12 * scale_f
        assert abs(got[0] - e_ref) <= te * scale_e
        for s in range(len(f_ref)):
            assert np.max(np.abs(got[1][s] - f_ref[s])) <= tf * scale_f
