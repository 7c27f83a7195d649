"""Reverse mode of the direct terms on the GPU (uw12c_fock_backward).

* Every gradient (J3_0, J3_ri_0, J2 of W and V; J3_0, J2 of WV) against the CPU
  adjoint of tests/adjoint_ref.py (itself checked against finite differences
  of the oracle energy), 1e-10 relative to the largest gradient entry.
* Central finite differences of the GPU energy along random directions.
* Energy, terms and Fock of the backward call equal form_fock with
  indirect_term = False; device outputs equal host outputs.
"""
import numpy as np
import pytest

from oracle import uw12_oracle as O
from tests import adjoint_ref as AR
from tests.parity_cases import CASES, Case, make_case

pytestmark = pytest.mark.gpu

ADJ_CASES = [c for c in CASES if c.name in ("c0_closed", "c0_frozen", "uhf_small", "unit_open",
                                            "unit_tiles")] + [
    Case("unit_no_beta_active", 6, 9, 12, (3, 2), (3, 0), "unit", 19)]


def _gpu_objects(lib, d, c):
    W = lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = lib.setup_base_integrals(d.WV3, d.WV2)
    A = lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    return W, V, WV, A


@pytest.mark.parametrize("case", ADJ_CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.0), (0.8, 0.5)])
def test_gradients_match_cpu_adjoint(uw12lib, cuda_device, case, scales):
    s_os, s_ss = scales
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d, case)
    e, f, terms, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, s_os,
                                           s_ss)
    e_fwd, f_fwd, t_fwd = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, False,
                                            True, s_os, s_ss)
    assert e == e_fwd and terms == t_fwd
    for s in range(len(f)):
        assert np.array_equal(f[s], f_fwd[s])
    Wo = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    Vo = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WVo = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    ref = AR.direct_adjoint(Wo, Vo, WVo, absp, d.orbitals, d.occ, list(case.n_active), s_os, s_ss)
    for key, r in ref.items():
        scale = max(np.max(np.abs(r)), 1e-300)
        err = np.max(np.abs(g[key] - r)) / scale
        assert err <= 1e-9, (key, err)


def test_finite_differences_of_gpu_energy(uw12lib, cuda_device):
    case = Case("unit_open_fd", 7, 10, 15, (4, 3), (3, 3), "unit", 23)
    d = make_case(case)
    s_os, s_ss = 1.0, 0.5
    W, V, WV, A = _gpu_objects(uw12lib, d, case)
    _, _, _, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, s_os, s_ss,
                                       calculate_fock=False)
    ints = {"W3": d.W3, "W2": d.W2, "W3_ri": d.W3_ri, "V3": d.V3, "V2": d.V2, "V3_ri": d.V3_ri,
            "WV3": d.WV3, "WV2": d.WV2}

    def energy(x):
        Wx = uw12lib.setup_base_integrals(x["W3"], x["W2"], x["W3_ri"])
        Vx = uw12lib.setup_base_integrals(x["V3"], x["V2"], x["V3_ri"])
        WVx = uw12lib.setup_base_integrals(x["WV3"], x["WV2"])
        return uw12lib.form_fock(Wx, Vx, WVx, A, d.orbitals, d.occ, case.n_active, False, False,
                                 s_os, s_ss)[0]

    rng = np.random.default_rng(3)
    h = 1e-5
    for key in uw12lib.GRADIENT_NAMES:
        dirn = rng.standard_normal(ints[key].shape)
        if key.endswith("2"):
            dirn = 0.5 * (dirn + dirn.T)
        fd = (energy(dict(ints, **{key: ints[key] + h * dirn})) -
              energy(dict(ints, **{key: ints[key] - h * dirn}))) / (2 * h)
        an = float(np.sum(g[key] * dirn))
        assert abs(an - fd) <= 1e-6 * max(abs(fd), 1e-3), (key, an, fd)


def test_device_outputs_and_partial_requests(uw12lib, cuda_device):
    import torch
    case = [c for c in CASES if c.name == "uhf_small"][0]
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d, case)
    _, _, _, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0, 0.0)
    bufs = {k: torch.zeros(v.size, dtype=torch.float64, device="cuda") for k, v in g.items()
            if k in ("W3", "V3_ri", "WV2")}
    e, _, _, empty = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0,
                                           0.0, calculate_fock=False,
                                           device_out={k: b.data_ptr() for k, b in bufs.items()})
    torch.cuda.synchronize()
    assert empty == {}
    for k, b in bufs.items():
        assert np.array_equal(b.cpu().numpy(), g[k].reshape(-1, order="F")), k
    # only the requested host gradients are computed and returned
    _, _, _, some = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0,
                                          0.0, gradients=("V2",))
    assert set(some) == {"V2"} and np.array_equal(some["V2"], g["V2"])
