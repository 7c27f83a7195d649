"""Reverse mode with the same-spin terms on the GPU (uw12c_fock_backward with
indirect_term = 1): the gradient of the energy uw12_energy returns.

* Every gradient against the CPU reverse sweep of tests/adjoint_ref.py
  (direct_adjoint + s_ss * indirect_adjoint, itself checked against central
  finite differences of the oracle energy in tests/test_adjoint_math.py),
  1e-9 relative to the largest gradient entry.
* Central finite differences (h = 1e-5) of the GPU energy with the same-spin
  terms along random directions, every gradient.
* Energy, terms and Fock of the backward call equal form_fock with
  indirect_term = True; the blocked form equals the whole gradients.
"""
import numpy as np
import pytest

from oracle import uw12_oracle as O
from tests import adjoint_ref as AR
from tests.parity_cases import CASES, Case, make_case

pytestmark = pytest.mark.gpu

SS_CASES = [c for c in CASES if c.name in ("c0_closed", "c0_frozen", "uhf_small", "unit_open",
                                           "unit_tiles")] + [
    Case("unit_no_beta_active", 6, 9, 12, (3, 2), (3, 0), "unit", 19)]


def _gpu_objects(lib, d, c):
    W = lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = lib.setup_base_integrals(d.WV3, d.WV2)
    A = lib.setup_abs_projectors(d.S, c.n_ao, c.n_ri)
    return W, V, WV, A


@pytest.mark.parametrize("case", SS_CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("scales", [(1.0, 0.5), (0.0, 1.0)])
def test_same_spin_gradients_match_cpu_adjoint(uw12lib, cuda_device, case, scales):
    s_os, s_ss = scales
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d, case)
    act = list(case.n_active)
    e, f, terms, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, act, s_os, s_ss,
                                           indirect_term=True)
    e_fwd, f_fwd, t_fwd = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, act, True, True,
                                            s_os, s_ss)
    assert e == e_fwd and terms == t_fwd
    for s in range(len(f)):
        assert np.array_equal(f[s], f_fwd[s])
    Wo = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    Vo = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WVo = O.BaseIntegrals(d.WV3, d.WV2)
    absp = O.calculate_abs_projectors(d.S, case.n_ao, case.n_ri)
    gd = AR.direct_adjoint(Wo, Vo, WVo, absp, d.orbitals, d.occ, act, s_os, s_ss)
    gi = AR.indirect_adjoint(Wo, Vo, WVo, absp, d.orbitals, d.occ, act)
    for key in gd:
        r = gd[key] + s_ss * gi[key]
        # the same-spin and direct parts cancel partly: scale by the larger part
        scale = max(np.max(np.abs(r)), np.max(np.abs(gd[key])),
                    abs(s_ss) * np.max(np.abs(gi[key])), 1e-300)
        err = np.max(np.abs(g[key] - r)) / scale
        assert err <= 1e-9, (key, err)


def test_same_spin_finite_differences_of_gpu_energy(uw12lib, cuda_device):
    case = Case("unit_open_fd_ss", 7, 10, 15, (4, 3), (3, 3), "unit", 29)
    d = make_case(case)
    s_os, s_ss = 1.0, 0.5
    W, V, WV, A = _gpu_objects(uw12lib, d, case)
    _, _, _, g = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, s_os, s_ss,
                                       calculate_fock=False, indirect_term=True)
    ints = {"W3": d.W3, "W2": d.W2, "W3_ri": d.W3_ri, "V3": d.V3, "V2": d.V2, "V3_ri": d.V3_ri,
            "WV3": d.WV3, "WV2": d.WV2}

    def energy(x):
        Wx = uw12lib.setup_base_integrals(x["W3"], x["W2"], x["W3_ri"])
        Vx = uw12lib.setup_base_integrals(x["V3"], x["V2"], x["V3_ri"])
        WVx = uw12lib.setup_base_integrals(x["WV3"], x["WV2"])
        return uw12lib.uw12_energy(Wx, Vx, WVx, A, d.orbitals, d.occ, case.n_active, s_os, s_ss)

    rng = np.random.default_rng(5)
    h = 1e-5
    for key in uw12lib.GRADIENT_NAMES:
        dirn = rng.standard_normal(ints[key].shape)
        if key.endswith("2"):
            dirn = 0.5 * (dirn + dirn.T)
        fd = (energy(dict(ints, **{key: ints[key] + h * dirn})) -
              energy(dict(ints, **{key: ints[key] - h * dirn}))) / (2 * h)
        an = float(np.sum(g[key] * dirn))
        assert abs(an - fd) <= 1e-6 * max(abs(fd), 1e-3), (key, an, fd)


def test_same_spin_blocks_equal_whole(uw12lib, cuda_device):
    """Host blocks of the three-index gradients, put together, equal the whole
    gradients with the same-spin terms (small memory budget: many blocks)."""
    case = [c for c in CASES if c.name == "uhf_small"][0]
    d = make_case(case)
    W, V, WV, A = _gpu_objects(uw12lib, d, case)
    _, _, _, whole = uw12lib.fock_backward(W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0,
                                           0.5, indirect_term=True)
    got = {k: np.zeros_like(whole[k]) for k in uw12lib.BLOCK_GRADIENT_NAMES}

    def sink(name):
        def f(first, count, block):
            got[name][:, first:first + count] = block
        return f

    uw12lib.set_memory_budget(1 << 16)
    try:
        _, _, _, metric = uw12lib.fock_backward_blocks(
            W, V, WV, A, d.orbitals, d.occ, case.n_active, 1.0, 0.5,
            {k: sink(k) for k in uw12lib.BLOCK_GRADIENT_NAMES}, indirect_term=True)
    finally:
        uw12lib.set_memory_budget(0)
    for k in uw12lib.BLOCK_GRADIENT_NAMES:
        assert np.max(np.abs(got[k] - whole[k])) <= 1e-12 * np.max(np.abs(whole[k])), k
    for k in ("W2", "V2", "WV2"):
        assert np.max(np.abs(metric[k] - whole[k])) <= 1e-12 * np.max(np.abs(whole[k])), k
