"""The sharded evaluation's partition (tests/sharded_model.py, the numpy model
of engine.cu's shard / all-reduce schedule) run as real ranks on CPU: the
partial energies and Fock matrices of the shards, with their intermediates
summed by the collective inside the evaluation, add up to the whole
evaluation.  Two gloo ranks (torch.distributed, world size 2) and, in one
process, 2-4 shards on threads.  The package's form_fock_sharded plumbing
(shard and all-reduce hook set for the call and removed afterwards, final
all-reduce of Fock and energies) is checked with the library call faked."""
import os
import socket
import threading

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import uw12_oracle as O
from tests import schedule_model as K
from tests import sharded_model as SM
from tests.parity_cases import Case, make_case

CASES = [
    Case("closed", 6, 10, 9, (3,), (3,), "baseline", 3, 4.0),
    Case("frozen", 6, 10, 9, (3,), (2,), "baseline", 3, 4.0),
    Case("open", 7, 11, 9, (4, 3), (3, 2), "baseline", 3, 4.0),
    Case("one_inactive", 7, 11, 9, (4, 3), (2, 0), "baseline", 5, 4.0),
    Case("unit", 5, 8, 14, (4, 3), (3, 2), "unit", 11),
]


def _inputs(case):
    d = make_case(case)
    W = O.BaseIntegrals(d.W3, d.W2, d.W3_ri)
    V = O.BaseIntegrals(d.V3, d.V2, d.V3_ri)
    WV = O.BaseIntegrals(d.WV3, d.WV2)
    vals, vecs = O.eigen_decomposition(d.S, 1e-6, 1e-8)
    Sinv = (vecs / vals) @ vecs.T
    return d, W, V, WV, Sinv


def _whole(case, s_os, s_ss):
    d, W, V, WV, Sinv = _inputs(case)
    ind = not O.nearly_zero(s_ss)
    return K.form_fock(W, V, WV, Sinv, d.orbitals, d.occ, list(case.n_active), ind, True,
                       s_os, s_ss)


def _check_sum(case, s_os, s_ss, e_sum, F_sum):
    e, F, _ = _whole(case, s_os, s_ss)
    scale = max(abs(e), 1e-300)
    assert abs(e_sum - e) <= 1e-12 * scale
    for s in range(len(F)):
        fs = O.symmetrise(F_sum[s])
        assert np.max(np.abs(fs - F[s])) <= 1e-12 * max(np.max(np.abs(F[s])), 1e-300)


class _ThreadGroup:
    """An in-process all-reduce among n threads (sum in rank order)."""

    def __init__(self, n):
        self.n = n
        self.barrier = threading.Barrier(n, timeout=60)
        self.slots = [None] * n
        self.total = None

    def allreduce(self, rank):
        def fn(arr):
            self.slots[rank] = arr
            self.barrier.wait()
            if rank == 0:
                self.total = sum(np.array(x) for x in self.slots)
            self.barrier.wait()
            arr[...] = self.total
            self.barrier.wait()
        return fn


def _run_threads(case, s_os, s_ss, n):
    d, W, V, WV, Sinv = _inputs(case)
    ind = not O.nearly_zero(s_ss)
    g = _ThreadGroup(n)
    out = [None] * n
    errs = []

    def work(rank):
        try:
            out[rank] = SM.form_fock_shard(W, V, WV, Sinv, d.orbitals, d.occ,
                                           list(case.n_active), ind, s_os, s_ss, rank, n,
                                           g.allreduce(rank))
        except Exception as exc:  # reported below
            errs.append(exc)
            g.barrier.abort()

    ts = [threading.Thread(target=work, args=(r,)) for r in range(n)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errs, errs
    return out


@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
@pytest.mark.parametrize("n", [1, 2, 3])
@pytest.mark.parametrize("scales", [(1.0, 0.5), (1.0, 0.0)])
def test_shards_on_threads_sum_to_whole(case, n, scales):
    out = _run_threads(case, *scales, n)
    e_sum = sum(sum(E.values()) for E, _ in out)
    F_sum = [sum(F[s] for _, F in out) for s in range(len(out[0][1]))]
    _check_sum(case, *scales, e_sum, F_sum)


def test_every_shard_gets_work_with_more_shards_than_orbitals():
    # 4 shards, 3 occupied alpha orbitals: one shard has no orbitals, all
    # still take every collective step
    case = CASES[2]
    out = _run_threads(case, 1.0, 0.5, 4)
    e_sum = sum(sum(E.values()) for E, _ in out)
    F_sum = [sum(F[s] for _, F in out) for s in range(2)]
    _check_sum(case, 1.0, 0.5, e_sum, F_sum)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gloo_rank(rank, world, port, case, scales, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        d, W, V, WV, Sinv = _inputs(case)
        s_os, s_ss = scales
        ind = not O.nearly_zero(s_ss)

        def allreduce(arr):
            t = torch.from_numpy(np.ascontiguousarray(arr))
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            arr[...] = t.numpy()

        E, F = SM.form_fock_shard(W, V, WV, Sinv, d.orbitals, d.occ, list(case.n_active), ind,
                                  s_os, s_ss, rank, world, allreduce)
        part = torch.tensor([sum(E.values())], dtype=torch.float64)
        fock = torch.from_numpy(np.concatenate([f.reshape(-1) for f in F]))
        dist.all_reduce(part)
        dist.all_reduce(fock)
        out_q.put((rank, float(part[0]), fock.numpy().copy(), sum(E.values())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [CASES[1], CASES[2]], ids=lambda c: c.name)
def test_partition_on_two_gloo_ranks(case):
    scales = (1.0, 0.5)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, case, scales, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    N = case.n_ao
    ns = len(case.n_occ)
    for rank, e_sum, fock, e_part in results:
        F_sum = [fock[N * N * s:N * N * (s + 1)].reshape(N, N) for s in range(ns)]
        _check_sum(case, *scales, e_sum, F_sum)
    # both ranks did part of the work
    assert all(abs(r[3]) > 0 for r in results)


def _plumbing_rank(rank, world, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import libuw12_b200.distributed as D
        calls = []
        fock = torch.zeros(6, dtype=torch.float64)

        def fake_set_shard(shard, n):
            calls.append(("shard", shard, n))

        def fake_set_allreduce(fn):
            calls.append(("allreduce", fn is not None))

        def fake_form_fock(*args, fock_out=None):
            assert fock_out == fock.data_ptr()
            shard = [c for c in calls if c[0] == "shard"][-1][1]
            fock.fill_(float(shard + 1))
            return float(10 * (shard + 1)), None, (1.0 * shard, 2.0 * shard, 3.0 * shard)

        D.set_shard = fake_set_shard
        D.set_allreduce = fake_set_allreduce
        D.nccl_allreduce = lambda group=None, device=None: (lambda p, c, s: None)
        D.form_fock = fake_form_fock
        e, terms = D.form_fock_sharded(None, None, None, None, [], [], [], True, True, 1.0, 0.5,
                                       fock)
        out_q.put((rank, calls, e, terms, fock.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharded_plumbing_two_cpu_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_plumbing_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, calls, e, terms, fock in results:
        # own shard and the hook for the call, then full evaluations again
        assert calls == [("shard", rank, 2), ("allreduce", True), ("allreduce", False),
                         ("shard", 0, 1)]
        assert e == 10.0 + 20.0
        assert terms == (1.0, 2.0, 3.0)
        assert fock == [3.0] * 6
