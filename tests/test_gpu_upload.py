"""Host-to-device copies of the integrals.

Three-index tensors of more than 32 MiB in pageable host memory are copied
through pinned chunks filled by several host threads (while the metric is
diagonalised); pinned and device sources are copied directly.  Every route
gives bit-identical handles: the evaluations agree exactly.
"""
import numpy as np
import pytest

from tests.parity_cases import Case, make_case

pytestmark = pytest.mark.gpu

# X3 5050 x 900 (36 MB) and X3_ri 15000 x 900 (108 MB): both above the threshold
BIG = Case("upload_big", 100, 900, 150, (6,), (6,), "baseline", 7, 8.0)


def _evaluate(lib, W, V, WV, A, d, c):
    return lib.form_fock(W, V, WV, A, d.orbitals, d.occ, c.n_active, True, True, 1.0, 0.5)


def test_pageable_pinned_and_device_sources_agree(uw12lib, cuda_device):
    import torch
    c = BIG
    d = make_case(c)
    assert d.W3.nbytes > 32 << 20 and d.W3_ri.nbytes > 32 << 20
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)

    # pageable numpy arrays (staged route)
    W_page = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    ref = _evaluate(uw12lib, W_page, V, WV, A, d, c)

    # pinned host buffers (direct route)
    def pinned(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = np.asfortranarray(a).reshape(-1, order="F")
        return t
    p3, p3r = pinned(d.W3), pinned(d.W3_ri)
    W_pin = uw12lib.setup_base_integrals(p3.numpy().reshape(d.W3.shape, order="F"), d.W2,
                                         p3r.numpy().reshape(d.W3_ri.shape, order="F"))
    got_pin = _evaluate(uw12lib, W_pin, V, WV, A, d, c)

    # device buffers
    g3, g3r = p3.cuda(), p3r.cuda()
    g2 = torch.from_numpy(np.ascontiguousarray(d.W2)).cuda()
    torch.cuda.synchronize()
    W_dev = uw12lib.setup_base_integrals(g3.data_ptr(), g2.data_ptr(), g3r.data_ptr(),
                                         n_ao=c.n_ao, n_df=c.n_df, n_ri=c.n_ri, device=True)
    got_dev = _evaluate(uw12lib, W_dev, V, WV, A, d, c)

    for got in (got_pin, got_dev):
        assert got[0] == ref[0]
        assert np.array_equal(got[1][0], ref[1][0])
    np.testing.assert_array_equal(W_page.get_df_vals(), W_dev.get_df_vals())


def test_pageable_strided_view_is_copied_correctly(uw12lib, cuda_device):
    """A C-ordered (row-major) array is reordered by the Python layer into a
    column-major copy before the staged upload; results match the F-ordered
    input exactly."""
    c = BIG
    d = make_case(c)
    A = uw12lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    W_f = uw12lib.setup_base_integrals(np.asfortranarray(d.W3), d.W2, np.asfortranarray(d.W3_ri))
    W_c = uw12lib.setup_base_integrals(np.ascontiguousarray(d.W3), d.W2,
                                       np.ascontiguousarray(d.W3_ri))
    a = _evaluate(uw12lib, W_f, V, WV, A, d, c)
    b = _evaluate(uw12lib, W_c, V, WV, A, d, c)
    assert a[0] == b[0] and np.array_equal(a[1][0], b[1][0])
