"""Three-index gradients delivered in aux blocks (uw12c_fock_backward_blocks).

* Host sinks under a 64 KiB memory budget (many blocks): every aux function of
  every requested gradient arrives once, in increasing order, and the blocks
  put together equal the whole gradients of uw12c_fock_backward (1e-12
  relative); energy, terms, Fock and metric gradients are identical.
* Device sinks (the library's squared-norm sink) on integral-direct handles:
  the squared norms equal those of the whole gradients of stored handles.
* A failing sink is reported as a runtime error.
"""
import ctypes

import numpy as np
import pytest

from tests.parity_cases import CASES, make_case

pytestmark = pytest.mark.gpu

NAMES = ("W3", "V3", "WV3", "W3_ri", "V3_ri")


def _objects(lib, d, c):
    W = lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = lib.setup_base_integrals(d.WV3, d.WV2)
    A = lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    return W, V, WV, A


@pytest.mark.parametrize("name", ["unit_tiles", "c0_frozen", "uhf_small"])
def test_host_blocks_equal_whole_gradients(uw12lib, cuda_device, name):
    c = [x for x in CASES if x.name == name][0]
    d = make_case(c)
    W, V, WV, A = _objects(uw12lib, d, c)
    uw12lib.set_memory_budget(64 << 10)
    try:
        e, f, terms, whole = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, c.n_active,
                                                   1.0, 0.5)
        parts = {n: [] for n in NAMES}

        def sink(n):
            return lambda first, count, block: parts[n].append((first, block.copy()))
        e2, f2, terms2, metric = uw12lib.fock_backward_blocks(
            W, V, WV, A, d.orbitals, d.occ, c.n_active, 1.0, 0.5, {n: sink(n) for n in NAMES})
    finally:
        uw12lib.set_memory_budget(0)
    assert e2 == e and terms2 == terms
    for s in range(len(f)):
        assert np.array_equal(f2[s], f[s])
    for n in ("W2", "V2", "WV2"):
        assert np.array_equal(metric[n], whole[n])
    for n in NAMES:
        ref = whole[n]
        firsts = [p[0] for p in parts[n]]
        assert firsts == sorted(firsts) and firsts[0] == 0
        got = np.concatenate([p[1] for p in parts[n]], axis=1)
        assert got.shape == ref.shape, n
        if name != "uhf_small" and n != "WV3":  # several blocks under the small budget
            assert len(parts[n]) > 1, n
        scale = max(np.max(np.abs(ref)), 1e-300)
        assert np.max(np.abs(got - ref)) <= 1e-12 * scale, n


def _host_producer(T):
    T = np.asfortranarray(T)

    def f(first, count, out, ld, stream):
        view = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_double)),
                                     shape=(ld * count,)).reshape((ld, count), order="F")
        view[:T.shape[0], :] = T[:, first:first + count]
    return f


def test_device_norm_sinks_on_integral_direct_handles(uw12lib, cuda_device):
    import torch
    c = [x for x in CASES if x.name == "unit_tiles"][0]
    d = make_case(c)
    W, V, WV, A = _objects(uw12lib, d, c)
    _, _, _, whole = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, c.n_active, 1.0, 0.0)
    M = d.W2.shape[0]

    def direct(X3, X2, X3_ri):
        return uw12lib.setup_base_integrals_callback(
            X2, _host_producer(X3), _host_producer(X3_ri) if X3_ri is not None else None,
            n_ao=c.n_ao, n_df=M, n_ri=c.n_ri if X3_ri is not None else 0, store_ao=False,
            store_ri=False)
    Wd, Vd, WVd = direct(d.W3, d.W2, d.W3_ri), direct(d.V3, d.V2, d.V3_ri), direct(d.WV3, d.WV2,
                                                                                  None)
    acc = torch.zeros(len(NAMES), dtype=torch.float64, device="cuda")
    users = {n: acc.data_ptr() + 8 * i for i, n in enumerate(NAMES)}
    fn = uw12lib.sink_norm2()
    uw12lib.set_memory_budget(64 << 10)
    try:
        uw12lib.fock_backward_blocks(Wd, Vd, WVd, A, d.orbitals, d.occ, c.n_active, 1.0, 0.0,
                                     {n: fn for n in NAMES}, calculate_fock=False, device=True,
                                     users=users)
    finally:
        uw12lib.set_memory_budget(0)
    torch.cuda.synchronize()
    got = acc.cpu().numpy()
    for i, n in enumerate(NAMES):
        ref = float(np.sum(whole[n] ** 2))
        assert abs(got[i] - ref) <= 1e-10 * ref, (n, got[i], ref)


def test_failing_sink_is_reported(uw12lib, cuda_device):
    c = [x for x in CASES if x.name == "unit_open"][0]
    d = make_case(c)
    W, V, WV, A = _objects(uw12lib, d, c)

    def bad(first, count, block):
        raise RuntimeError("no room for gradients")

    with pytest.raises(uw12lib.UW12RuntimeError, match="sink returned"):
        uw12lib.fock_backward_blocks(W, V, WV, A, d.orbitals, d.occ, c.n_active, 1.0, 0.0,
                                     {"V3_ri": bad})
