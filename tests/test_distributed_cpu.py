"""Host-side plumbing of the sharded evaluation on CPU ranks (gloo,
world_size 2): form_fock_sharded sets shard = rank of n_shards = world size,
restores the full-evaluation setting afterwards, and sums the partial Fock
matrices (in place) and energies over the ranks.  The CUDA evaluation is
replaced by a fake that writes a rank-dependent partial result."""
import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import libuw12_b200.distributed as D
        calls = []
        fock = torch.zeros(6, dtype=torch.float64)

        def fake_set_shard(shard, n):
            calls.append((shard, n))

        def fake_form_fock(*args, fock_out=None):
            shard, n = calls[-1]
            assert fock_out == fock.data_ptr()
            fock.fill_(float(shard + 1))
            return float(10 * (shard + 1)), None, (1.0 * shard, 2.0 * shard, 3.0 * shard)

        D.set_shard = fake_set_shard
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
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, calls, e, terms, fock in results:
        assert calls == [(rank, 2), (0, 1)]   # own shard, then full evaluations again
        assert e == 10.0 + 20.0               # partial energies summed
        assert terms == (1.0, 2.0, 3.0)       # (0 + 1, 0 + 2, 0 + 3)
        assert fock == [3.0] * 6              # 1 + 2, summed in place
