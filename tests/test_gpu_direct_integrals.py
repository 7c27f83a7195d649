"""BaseIntegrals from producers (uw12c_integrals_create_callback), stored and
integral-direct.

* Host producers with storage: the handle holds exactly the stored tensors,
  so energies and Fock matrices are bit-identical to setup_base_integrals.
* Integral-direct (nothing stored) under a 64 KiB memory budget, so that every
  loop over aux functions runs in many blocks that the producer regenerates:
  results equal the stored evaluation to 1e-12 relative (the contractions over
  aux functions are summed block by block), forward and adjoint.
* The library's native device producer (synthetic tensors) against the same
  tensors stored.
* Host producers are read ahead on a background thread.
* A failing producer is reported as a runtime error.
"""
import ctypes

import numpy as np
import pytest

from tests.parity_cases import CASES, make_case

pytestmark = pytest.mark.gpu


def _host_producer(T, calls=None):
    """Columns [first, first + count) of the column-major array T into host memory."""
    T = np.asfortranarray(T)

    def f(first, count, out, ld, stream):
        if calls is not None:
            calls.append((first, count))
        view = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_double)),
                                     shape=(ld * count,)).reshape((ld, count), order="F")
        view[:T.shape[0], :] = T[:, first:first + count]
    return f


def _handles(lib, d, c, store):
    n_ao, n_df, n_ri = c.n_ao, d.W2.shape[0], c.n_ri
    mk = lambda X3, X2, X3_ri: lib.setup_base_integrals_callback(  # noqa: E731
        X2, _host_producer(X3), _host_producer(X3_ri) if X3_ri is not None else None,
        n_ao=n_ao, n_df=n_df, n_ri=n_ri if X3_ri is not None else 0, store_ao=store,
        store_ri=store)
    return mk(d.W3, d.W2, d.W3_ri), mk(d.V3, d.V2, d.V3_ri), mk(d.WV3, d.WV2, None)


def _stored(lib, d):
    return (lib.setup_base_integrals(d.W3, d.W2, d.W3_ri),
            lib.setup_base_integrals(d.V3, d.V2, d.V3_ri),
            lib.setup_base_integrals(d.WV3, d.WV2))


@pytest.mark.parametrize("name", ["unit_open", "unit_tiles", "c0_frozen"])
def test_stored_producers_are_bit_identical(uw12lib, cuda_device, name):
    c = [x for x in CASES if x.name == name][0]
    d = make_case(c)
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    ref = uw12lib.form_fock(*_stored(uw12lib, d), A, d.orbitals, d.occ, c.n_active, True, True,
                            1.0, 0.5)
    got = uw12lib.form_fock(*_handles(uw12lib, d, c, True), A, d.orbitals, d.occ, c.n_active,
                            True, True, 1.0, 0.5)
    assert got[0] == ref[0]
    for s in range(len(ref[1])):
        assert np.array_equal(got[1][s], ref[1][s])


@pytest.mark.parametrize("name", ["unit_open", "unit_tiles", "unit_closed"])
def test_integral_direct_matches_stored(uw12lib, cuda_device, name):
    c = [x for x in CASES if x.name == name][0]
    d = make_case(c)
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    uw12lib.set_memory_budget(64 << 10)
    try:
        ref = uw12lib.form_fock(*_stored(uw12lib, d), A, d.orbitals, d.occ, c.n_active, True,
                                True, 1.0, 0.5)
        got = uw12lib.form_fock(*_handles(uw12lib, d, c, False), A, d.orbitals, d.occ,
                                c.n_active, True, True, 1.0, 0.5)
        g_ref = uw12lib.fock_backward(*_stored(uw12lib, d), A, d.orbitals, d.occ, c.n_active,
                                      1.0, 0.0)[3]
        g_got = uw12lib.fock_backward(*_handles(uw12lib, d, c, False), A, d.orbitals, d.occ,
                                      c.n_active, 1.0, 0.0)[3]
    finally:
        uw12lib.set_memory_budget(0)
    assert abs(got[0] - ref[0]) <= 1e-12 * max(1.0, abs(ref[0]))
    for s in range(len(ref[1])):
        assert np.max(np.abs(got[1][s] - ref[1][s])) <= 1e-12 * max(1.0, np.max(np.abs(ref[1][s])))
    for k, v in g_ref.items():
        assert np.max(np.abs(g_got[k] - v)) <= 1e-12 * max(1e-300, np.max(np.abs(v))), k


def test_producer_is_called_in_blocks(uw12lib, cuda_device):
    c = [x for x in CASES if x.name == "unit_tiles"][0]
    d = make_case(c)
    calls = []
    W = uw12lib.setup_base_integrals_callback(d.W2, _host_producer(d.W3, calls),
                                              _host_producer(d.W3_ri), n_ao=c.n_ao,
                                              n_df=d.W2.shape[0], n_ri=c.n_ri, store_ao=False,
                                              store_ri=False)
    assert calls == []  # nothing produced until it is used
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    V, WV = _stored(uw12lib, d)[1:]
    uw12lib.set_memory_budget(64 << 10)
    try:
        uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, c.n_active, False, False, 1.0, 0.0)
    finally:
        uw12lib.set_memory_budget(0)
    M = d.W2.shape[0]
    assert len(calls) > 1 and all(0 <= f and f + n <= M for f, n in calls)


def test_host_producer_reads_ahead(uw12lib, cuda_device):
    """Host producers are read ahead: after a block is staged, the next range
    is produced on a background thread while the GPU works, and the request
    for it takes the staged copy.  Results equal the stored evaluation."""
    import threading
    c = [x for x in CASES if x.name == "unit_tiles"][0]
    d = make_case(c)
    main = threading.get_ident()
    threads, calls = [], []

    def traced(T):
        inner = _host_producer(T, calls)

        def f(first, count, out, ld, stream):
            threads.append(threading.get_ident())
            inner(first, count, out, ld, stream)
        return f

    M = d.W2.shape[0]
    W = uw12lib.setup_base_integrals_callback(d.W2, traced(d.W3), traced(d.W3_ri), n_ao=c.n_ao,
                                              n_df=M, n_ri=c.n_ri, store_ao=False,
                                              store_ri=False)
    V, WV = _stored(uw12lib, d)[1:]
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    uw12lib.set_memory_budget(64 << 10)
    try:
        got = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, c.n_active, True, True, 1.0, 0.5)
        ref = uw12lib.form_fock(*_stored(uw12lib, d), A, d.orbitals, d.occ, c.n_active, True,
                                True, 1.0, 0.5)
    finally:
        uw12lib.set_memory_budget(0)
    assert abs(got[0] - ref[0]) <= 1e-12 * max(1.0, abs(ref[0]))
    for s in range(len(ref[1])):
        assert np.max(np.abs(got[1][s] - ref[1][s])) <= 1e-12 * max(1.0, np.max(np.abs(ref[1][s])))
    assert any(t != main for t in threads)  # some blocks were produced ahead
    assert all(0 <= f and f + n <= M for f, n in calls)


def test_native_device_producer_matches_stored_synthetic(uw12lib, cuda_device):
    """uw12c_synth_block as the device producer of unstored W, V and WV tensors
    against the same synthetic tensors stored (evaluated under a small budget,
    so the producer runs in many blocks)."""
    import torch
    N, M, R, decay = 24, 84, 116, 8.0
    np_ = N * (N + 1) // 2
    specs, dev = {}, {}
    for tag, (nm, kind, rows) in enumerate((("W3", 0, np_), ("W3_ri", 1, R * N), ("V3", 0, np_),
                                            ("V3_ri", 1, R * N), ("WV3", 0, np_))):
        specs[nm] = uw12lib.SynthSpec(kind, N, R, 7, 1000 + tag, decay)
        t = torch.empty(rows * M, dtype=torch.float64, device="cuda")
        uw12lib.synth_three_index(t.data_ptr(), kind, N, R, M, 7, 1000 + tag, decay)
        dev[nm] = t
    rng = np.random.default_rng(1)
    mets = {}
    for nm in ("W2", "V2", "WV2"):
        B = rng.standard_normal((M, M)) / np.sqrt(M)
        mets[nm] = np.ascontiguousarray(B @ B.T + 1e-3 * np.eye(M))
    torch.cuda.synchronize()
    d = make_case([x for x in CASES if x.name == "c0_frozen"][0])
    A = uw12lib.setup_abs_projectors(d.S, N, R)
    stored = (
        uw12lib.setup_base_integrals(dev["W3"].cpu().numpy().reshape((np_, M), order="F"),
                                     mets["W2"],
                                     dev["W3_ri"].cpu().numpy().reshape((R * N, M), order="F")),
        uw12lib.setup_base_integrals(dev["V3"].cpu().numpy().reshape((np_, M), order="F"),
                                     mets["V2"],
                                     dev["V3_ri"].cpu().numpy().reshape((R * N, M), order="F")),
        uw12lib.setup_base_integrals(dev["WV3"].cpu().numpy().reshape((np_, M), order="F"),
                                     mets["WV2"]))
    fp = uw12lib.synth_producer()

    def direct(ao, ri, met):
        return uw12lib.setup_base_integrals_callback(
            mets[met], fp, fp if ri else None, n_ao=N, n_df=M, n_ri=R if ri else 0,
            store_ao=False, store_ri=False, device=True, user=ctypes.addressof(specs[ao]),
            user_ri=ctypes.addressof(specs[ri]) if ri else 0)

    produced = (direct("W3", "W3_ri", "W2"), direct("V3", "V3_ri", "V2"),
                direct("WV3", None, "WV2"))
    uw12lib.set_memory_budget(64 << 10)
    try:
        ref = uw12lib.form_fock(*stored, A, d.orbitals, d.occ, [5], True, True, 1.0, 0.5)
        got = uw12lib.form_fock(*produced, A, d.orbitals, d.occ, [5], True, True, 1.0, 0.5)
    finally:
        uw12lib.set_memory_budget(0)
    assert abs(got[0] - ref[0]) <= 1e-11 * abs(ref[0])
    assert np.max(np.abs(got[1][0] - ref[1][0])) <= 1e-11 * np.max(np.abs(ref[1][0]))


def test_failing_producer_is_reported(uw12lib, cuda_device):
    c = [x for x in CASES if x.name == "unit_open"][0]
    d = make_case(c)

    def bad(first, count, out, ld, stream):
        raise RuntimeError("no integrals today")

    with pytest.raises(uw12lib.UW12RuntimeError, match="callback returned"):
        uw12lib.setup_base_integrals_callback(d.W2, bad, None, n_ao=c.n_ao, n_df=d.W2.shape[0])
    W = uw12lib.setup_base_integrals_callback(d.W2, bad, _host_producer(d.W3_ri), n_ao=c.n_ao,
                                              n_df=d.W2.shape[0], n_ri=c.n_ri, store_ao=False)
    V, WV = _stored(uw12lib, d)[1:]
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    with pytest.raises(uw12lib.UW12RuntimeError, match="callback returned"):
        uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, c.n_active, True, True, 1.0, 0.5)
