"""Reverse mode of the direct terms over chunks of orbitals.

Without same-spin terms the backward pass needs the recomputed intermediates
(B2, Wst and S^-1 Wst of W and V) only through sums over orbitals, so when
they do not fit the chunk budget it forms them for a chunk of orbitals at a
time (the reverse sweep of tests/adjoint_ref.py
``chunked_three_index_adjoint``).  A 64 KiB budget forces one-orbital chunks
on these cases; energy, terms, Fock and every gradient must equal the
whole-intermediate backward pass (default budget) to 1e-12.  The chunked
pass on integral-direct handles, with the three-index gradients handed to
host sinks in aux blocks (with and without the RI gradients, the form of
the largest configuration, whose RI gradients are not asked for), must
equal the whole gradients of stored handles.
"""
import ctypes

import numpy as np
import pytest

from tests.parity_cases import CASES, Case, make_case

pytestmark = pytest.mark.gpu

CHUNK_CASES = [c for c in CASES if c.name in ("c0_closed", "c0_frozen", "unit_tiles")] + [
    Case("uhf_chunk", 20, 40, 30, (6, 5), (5, 3), "baseline", 9, 4.0),
    Case("uhf_chunk_no_beta_active", 20, 40, 30, (6, 5), (5, 0), "baseline", 10, 4.0),
]
SMALL = 64 << 10


def _objects(lib, d, c):
    W = lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = lib.setup_base_integrals(d.WV3, d.WV2)
    A = lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    return W, V, WV, A


def _close(got, ref, tol=1e-12):
    scale = max(np.max(np.abs(ref)), 1e-300)
    return np.max(np.abs(got - ref)) <= tol * scale


@pytest.mark.parametrize("case", CHUNK_CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.0), (0.8, 0.5)])
def test_chunked_backward_equals_whole(uw12lib, cuda_device, case, scales):
    s_os, s_ss = scales
    d = make_case(case)
    W, V, WV, A = _objects(uw12lib, d, case)
    e, f, terms, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, s_os,
                                           s_ss)
    uw12lib.set_memory_budget(SMALL)
    try:
        e2, f2, terms2, g2 = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ,
                                                   case.n_active, s_os, s_ss)
    finally:
        uw12lib.set_memory_budget(0)
    scale = max(1.0, abs(e))
    assert abs(e2 - e) <= 1e-12 * scale
    for a, b in zip(terms2, terms):
        assert abs(a - b) <= 1e-12 * max(1.0, abs(b))
    for s in range(len(f)):
        assert _close(f2[s], f[s])
    for key in uw12lib.GRADIENT_NAMES:
        assert g2[key].shape == g[key].shape, key
        assert _close(g2[key], g[key]), (key, np.max(np.abs(g2[key] - g[key])))


def test_chunked_backward_subset_of_gradients(uw12lib, cuda_device):
    """Only the AO three-index and metric gradients (no RI gradients): the
    chunked pass holds no RI-row factor and gives the same values."""
    c = [x for x in CHUNK_CASES if x.name == "uhf_chunk"][0]
    d = make_case(c)
    W, V, WV, A = _objects(uw12lib, d, c)
    names = ("W3", "V3", "WV3", "W2", "V2", "WV2")
    _, _, _, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, c.n_active, 1.0, 0.5)
    uw12lib.set_memory_budget(SMALL)
    try:
        _, _, _, g2 = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, c.n_active, 1.0, 0.5,
                                            gradients=names)
    finally:
        uw12lib.set_memory_budget(0)
    for key in names:
        assert _close(g2[key], g[key]), key


def _host_producer(T):
    T = np.asfortranarray(T)

    def f(first, count, out, ld, stream):
        view = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_double)),
                                     shape=(ld * count,)).reshape((ld, count), order="F")
        view[:T.shape[0], :] = T[:, first:first + count]
    return f


@pytest.mark.parametrize("with_ri", [True, False], ids=["all", "no_ri"])
def test_chunked_backward_on_integral_direct_handles(uw12lib, cuda_device, with_ri):
    c = [x for x in CHUNK_CASES if x.name == "uhf_chunk"][0]
    d = make_case(c)
    W, V, WV, A = _objects(uw12lib, d, c)
    e, f, terms, whole = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, c.n_active, 1.0,
                                               0.5)
    M = d.W2.shape[0]

    def direct(X3, X2, X3_ri):
        return uw12lib.setup_base_integrals_callback(
            X2, _host_producer(X3), _host_producer(X3_ri) if X3_ri is not None else None,
            n_ao=c.n_ao, n_df=M, n_ri=c.n_ri if X3_ri is not None else 0, store_ao=False,
            store_ri=False)
    Wd, Vd, WVd = direct(d.W3, d.W2, d.W3_ri), direct(d.V3, d.V2, d.V3_ri), direct(d.WV3, d.WV2,
                                                                                  None)
    names = ("W3", "V3", "WV3") + (("W3_ri", "V3_ri") if with_ri else ())
    parts = {n: [] for n in names}

    def sink(n):
        return lambda first, count, block: parts[n].append((first, block.copy()))
    uw12lib.set_memory_budget(SMALL)
    try:
        e2, f2, terms2, metric = uw12lib.fock_backward_blocks(
            Wd, Vd, WVd, A, d.orbitals, d.occ, c.n_active, 1.0, 0.5, {n: sink(n) for n in names})
    finally:
        uw12lib.set_memory_budget(0)
    assert abs(e2 - e) <= 1e-12 * max(1.0, abs(e))
    for s in range(len(f)):
        assert _close(f2[s], f[s])
    for n in ("W2", "V2", "WV2"):
        assert _close(metric[n], whole[n]), n
    for n in names:
        firsts = [p[0] for p in parts[n]]
        assert firsts == sorted(firsts) and firsts[0] == 0, n
        got = np.concatenate([p[1] for p in parts[n]], axis=1)
        assert got.shape == whole[n].shape, n
        assert _close(got, whole[n]), n
