"""Sharded evaluation through the C-ABI: n shards, each on its own host thread
and CUDA stream of one GPU, their in-evaluation sums done by an all-reduce
hook that synchronises the shards' streams on the host (no kernel waits on
another shard), and the partial energies and Fock matrices of the shards add
up to the unsharded evaluation.  On several GPUs the same hook is
torch.distributed.all_reduce (libuw12_b200.distributed)."""
import threading

import numpy as np
import pytest
import torch

from tests.parity_cases import CASES, make_case

pytestmark = pytest.mark.gpu


class _StreamGroup:
    """All-reduce among n host threads on one device: each shard's stream is
    synchronised, shard 0 sums the buffers in shard order and writes the sum
    back into every buffer, then all continue."""

    def __init__(self, n, device):
        self.n = n
        self.device = device
        self.barrier = threading.Barrier(n, timeout=120)
        self.bufs = [None] * n
        self.calls = [0] * n

    def hook(self, rank):
        from libuw12_b200.distributed import device_view

        def fn(ptr, count, stream):
            torch.cuda.ExternalStream(stream, device=self.device).synchronize()
            self.bufs[rank] = device_view(ptr, count, self.device)
            self.calls[rank] += 1
            self.barrier.wait()
            if rank == 0:
                total = torch.zeros(count, dtype=torch.float64, device=self.device)
                for b in self.bufs:
                    total += b
                for b in self.bufs:
                    b.copy_(total)
                torch.cuda.synchronize(self.device)
            self.barrier.wait()
        return fn


def _sharded(uw12lib, handles, d, case, n, scales, budget):
    W, V, WV, A = handles
    dev = torch.device("cuda", 0)
    g = _StreamGroup(n, dev)
    out = [None] * n
    errs = []

    def work(rank):
        try:
            torch.cuda.set_device(dev)
            st = torch.cuda.Stream(dev)
            uw12lib.set_stream(st.cuda_stream)
            uw12lib.set_memory_budget(budget)
            uw12lib.set_shard(rank, n)
            uw12lib.set_allreduce(g.hook(rank))
            try:
                out[rank] = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True,
                                              True, *scales)
            finally:
                uw12lib.set_allreduce(None)
                uw12lib.set_shard(0, 1)
                uw12lib.set_memory_budget(0)
                uw12lib.set_stream(0)
        except Exception as exc:  # reported below
            errs.append(exc)
            g.barrier.abort()

    ts = [threading.Thread(target=work, args=(r,)) for r in range(n)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs
    assert len(set(g.calls)) == 1 and g.calls[0] > 0  # every shard took the same steps
    return out


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[4], CASES[-1]], ids=lambda c: c.name)
@pytest.mark.parametrize("n_shards", [2, 3])
@pytest.mark.parametrize("scales", [(1.0, 0.5), (1.0, 0.0)])
def test_shards_sum_to_full_evaluation(uw12lib, cuda_device, case, n_shards, scales):
    d = make_case(case)
    W = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    A = uw12lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    e_full, f_full, t_full = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active,
                                               True, True, *scales)
    # a small budget forces several chunks per loop (and the orbital-chunked
    # transforms when the same-spin terms are off)
    for budget in (0, 64 << 10):
        out = _sharded(uw12lib, (W, V, WV, A), d, case, n_shards, scales, budget)
        e_sum = sum(o[0] for o in out)
        t_sum = np.sum([np.array(o[2]) for o in out], axis=0)
        assert abs(e_sum - e_full) <= 1e-11 * abs(e_full)
        assert np.max(np.abs(t_sum - np.array(t_full))) <= 1e-10 * abs(e_full)
        for s in range(len(f_full)):
            f_sum = sum(o[1][s] for o in out)
            assert np.max(np.abs(f_sum - f_full[s])) <= 1e-11 * np.max(np.abs(f_full[s]))


def test_sharded_evaluation_needs_an_allreduce(uw12lib, cuda_device):
    case = CASES[2]
    d = make_case(case)
    W = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    A = uw12lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)
    uw12lib.set_shard(1, 2)
    try:
        with pytest.raises(uw12lib.UW12Error, match="all-reduce"):
            uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True, 1.0, 0.5)
    finally:
        uw12lib.set_shard(0, 1)


def test_failing_allreduce_fails_the_evaluation(uw12lib, cuda_device):
    """An exception in the hook (a rank that left, a collective that timed
    out) ends the evaluation with an error instead of a wrong result."""
    case = CASES[2]
    d = make_case(case)
    W = uw12lib.setup_base_integrals(d.W3, d.W2, d.W3_ri)
    V = uw12lib.setup_base_integrals(d.V3, d.V2, d.V3_ri)
    WV = uw12lib.setup_base_integrals(d.WV3, d.WV2)
    A = uw12lib.setup_abs_projectors(d.S, case.n_ao, case.n_ri)

    def broken(ptr, count, stream):
        raise RuntimeError("peer rank gone")

    uw12lib.set_shard(0, 2)
    uw12lib.set_allreduce(broken)
    try:
        with pytest.raises(uw12lib.UW12Error, match="all-reduce"):
            uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True, 1.0, 0.5)
    finally:
        uw12lib.set_allreduce(None)
        uw12lib.set_shard(0, 1)
    # the thread is usable again: an unsharded evaluation succeeds
    e, _, _ = uw12lib.form_fock(W, V, WV, A, d.orbitals, d.occ, case.n_active, True, True,
                                1.0, 0.5)
    assert np.isfinite(e)
