"""Several GPUs as independent replicas: the range split and the host-side collectives, run as two
gloo ranks on CPU (no GPU, no data-path collective)."""
import os
import socket

import pytest


def _primes(hi):
    from mersenneprime_python_cpp_gmp_benchmark_b200.llgpu import _primes as pr
    return pr(2, hi)


def test_shard_partitions_and_balances():
    from mersenneprime_python_cpp_gmp_benchmark_b200 import replicas
    ps = _primes(100001)
    for world in (1, 2, 3, 4, 8):
        parts = [replicas.shard(ps, r, world) for r in range(world)]
        flat = sorted(p for part in parts for p in part)
        assert flat == ps
        loads = [sum(replicas.squaring_cost(p) for p in part) for part in parts]
        assert max(loads) <= 1.01 * min(loads), (world, loads)
    with pytest.raises(ValueError):
        replicas.shard(ps, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, ps, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from mersenneprime_python_cpp_gmp_benchmark_b200 import replicas
    from oracle import oracle
    mine = replicas.shard(ps, rank, world)
    # each rank "tests" its share (the oracle stands in for the GPU here) and times itself
    res = [{"p": p, "is_zero": oracle.ll_gmp(p)[0], "rank": rank} for p in mine]
    t_max = replicas.reduce_max(float(rank + 1))
    n_all = replicas.reduce_sum(float(len(mine)))
    allres = replicas.gather(res)
    out.put((rank, t_max, n_all, [(r["p"], r["is_zero"], r["rank"]) for r in allres]))
    dist.destroy_process_group()


def test_two_gloo_ranks_split_and_gather():
    import torch.multiprocessing as mp
    from conftest import KNOWN
    ps = _primes(4423)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, ps, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=120) for _ in procs]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, t_max, n_all, allres in got:
        assert t_max == 2.0 and n_all == len(ps)
        assert [p for p, _, _ in allres] == ps
        assert [p for p, z, _ in allres if z] == KNOWN
        assert {r for _, _, r in allres} == {0, 1}
