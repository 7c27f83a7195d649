"""Sharded evaluation: the partial energies and Fock matrices of n shards sum to
the unsharded result (shards run one after another on one GPU; on several GPUs
they run concurrently and are summed by an all-reduce)."""
import numpy as np
import pytest

from tests.parity_cases import CASES, make_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[-1]], ids=lambda c: c.name)
@pytest.mark.parametrize("n_shards", [2, 3])
def test_shards_sum_to_full_evaluation(uw12lib, cuda_device, case, n_shards):
    d = make_case(case)
    W = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    A = uw12lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    # a small budget forces several chunks per loop, so every shard gets work
    uw12lib.set_memory_budget(64 << 10)
    try:
        run = lambda: uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True,
                                        1.0, 0.5)
        e_full, f_full, t_full = run()
        e_sum, f_sum, t_sum = 0.0, [np.zeros_like(f) for f in f_full], np.zeros(3)
        for sh in range(n_shards):
            uw12lib.set_shard(sh, n_shards)
            e, f, t = run()
            e_sum += e
            t_sum += np.array(t)
            for s in range(len(f)):
                f_sum[s] += f[s]
    finally:
        uw12lib.set_shard(0, 1)
        uw12lib.set_memory_budget(0)
    assert abs(e_sum - e_full) <= 1e-11 * abs(e_full)
    assert np.max(np.abs(t_sum - np.array(t_full))) <= 1e-11 * abs(e_full) * 10
    for s in range(len(f_full)):
        assert np.max(np.abs(f_sum[s] - f_full[s])) <= 1e-11 * np.max(np.abs(f_full[s]))

