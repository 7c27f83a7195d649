"""The benchmark's input generator (libuw12_b200/workload.py) produces exactly
the oracle's seeded inputs (oracle/synth.py, tests/parity_cases.py), so the
CUDA arm and the reference arm of bench.py evaluate identical bytes, and the
64-molecule batch is the one the golden fixtures pin."""
import numpy as np

from libuw12_b200 import workload as WL
from oracle import synth
from tests import golden_cases as G
from tests.parity_cases import Case, make_case


def test_three_index_tensors_bitwise_equal_to_the_oracle_generator():
    w = WL.Workload("t", 11, 7, 13, (3, 2), 4.0)
    for nm in ("W3", "V3", "WV3"):
        assert np.array_equal(WL.make_three_index(w, nm, 5),
                              synth.three_index_ao(5, nm, 11, 7, 4.0))
    for nm in ("W3_ri", "V3_ri"):
        assert np.array_equal(WL.make_three_index(w, nm, 5),
                              synth.three_index_ri(5, nm, 11, 13, 7, 4.0))


def test_in_place_fill_equals_fresh_array():
    w = WL.Workload("t", 9, 5, 6, (2,), 3.0)
    buf = np.full(9 * 10 // 2 * 5, np.nan)
    WL.make_three_index(w, "W3", 3, out=buf)
    assert np.array_equal(buf.reshape((45, 5), order="F"), WL.make_three_index(w, "W3", 3))


def test_small_inputs_equal_the_parity_case_generator():
    case = Case("x", 8, 12, 10, (4, 3), (4, 3), "baseline", 6, 4.0)
    d = make_case(case)
    w = WL.Workload("x", 8, 12, 10, (4, 3), 4.0)
    s = WL.make_small(w, 6)
    for nm in ("W2", "V2", "WV2", "S"):
        assert np.array_equal(s[nm], getattr(d, nm)), nm
    for a, b in zip(s["orbitals"], d.orbitals):
        assert np.array_equal(a, b)
    for a, b in zip(s["occ"], d.occ):
        assert np.array_equal(a, b)


def test_batch_is_the_pinned_c4_batch():
    mols = WL.batch_molecules()
    ref = G.c4_molecules()
    assert len(mols) == len(ref) == 64
    for (w, seed), (_, c) in zip(mols, ref):
        assert (w.n_ao, w.n_df, w.n_ri, tuple(w.n_occ), w.decay, seed) == \
            (c.n_ao, c.n_df, c.n_ri, tuple(c.n_occ), c.decay, c.seed)


def test_bench_arms_generate_identical_bytes():
    """bench.py's GPU arm (libuw12_b200.workload) and reference arm (oracle
    generators) see the same inputs, element for element."""
    import bench
    w = WL.Workload("t", 12, 20, 15, (4, 3), 8.0)
    a = bench.host_inputs(w, pinned=False)
    b = bench.reference_inputs(w)
    for nm in ("W3", "V3", "WV3", "W3_ri", "V3_ri", "W2", "V2", "WV2", "S"):
        assert np.array_equal(a[nm], b[nm]), nm
    for x, y in zip(a["orbitals"], b["orbitals"]):
        assert np.array_equal(x, y)
    for x, y in zip(a["occ"], b["occ"]):
        assert np.array_equal(x, y)
