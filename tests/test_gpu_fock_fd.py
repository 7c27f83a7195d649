"""The Fock matrix of the GPU path is the derivative of the GPU energy with
respect to the density (tests/numerical_fock.hpp:22-141 and
multi_el_test_utils.hpp:313-367 in libuw12, tightened).

Along 50 random directions per case, D(t) = per (C + tX)(C + tX)^T
(all-electron, occupations fixed), the central difference (h = 1e-5) of the
energy that form_fock computes on the device equals <F, dD/dt> with the Fock
matrix of the backward pass (uw12c_fock_backward), to 1e-6 relative; libuw12
itself accepts 0.5.  The backward pass runs with whole intermediates and, for
the direct terms, over one-orbital chunks (64 KiB budget).
"""
import numpy as np
import pytest

from oracle import synth
from tests.parity_cases import Case, make_case

pytestmark = pytest.mark.gpu

N_DIRECTIONS = 50


@pytest.mark.parametrize("n_occ", [(3,), (3, 2)], ids=["closed", "open"])
@pytest.mark.parametrize("s_ss,indirect", [(0.0, False), (0.5, False), (0.5, True)],
                         ids=["os", "ss_direct", "ss_indirect"])
@pytest.mark.parametrize("budget", [0, 64 << 10], ids=["whole", "chunked"])
def test_fock_is_derivative_of_gpu_energy(uw12lib, cuda_device, n_occ, s_ss, indirect, budget):
    case = Case("fd", 6, 11, 9, n_occ, n_occ, "unit", 21)
    d = make_case(case)
    ns = len(n_occ)
    per = 2.0 if ns == 1 else 1.0
    occ = [np.full(o, per) for o in n_occ]
    W = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    A = uw12lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    base = [np.asfortranarray(o) for o in d.orbitals]
    act = list(n_occ)

    def energy(orbs):
        return uw12lib.form_fock(W, V, WV, A, orbs, occ, act, indirect, False, 1.0, s_ss)[0]

    uw12lib.set_memory_budget(budget)
    try:
        e, fock, _, _ = uw12lib.fock_backward(W, V, WV, A, base, occ, act, 1.0, s_ss,
                                              gradients=(), indirect_term=indirect)
    finally:
        uw12lib.set_memory_budget(0)
    assert abs(e - energy(base)) <= 1e-12 * max(1.0, abs(e))
    h = 1e-5
    worst = 0.0
    for r in range(N_DIRECTIONS):
        X = [synth.gaussian_matrix(100 + r, f"X{s}", case.n_ao, o) for s, o in enumerate(n_occ)]
        num = (energy([b + h * x for b, x in zip(base, X)]) -
               energy([b - h * x for b, x in zip(base, X)])) / (2 * h)
        ana = 0.0
        for s in range(ns):
            dD = per * (X[s] @ base[s].T + base[s] @ X[s].T)
            ana += float(np.sum(fock[s] * dD))
        err = abs(num - ana) / max(abs(ana), 1e-12 * abs(e))
        worst = max(worst, err)
    assert worst <= 1e-6, worst
