"""The N > 1 replica path on CPU: two gloo ranks shard independent commits,
each rank's results equal a single-process run of the same jobs, and the
reported whole-job throughput is all units over the slowest rank's time."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _oracle_commit_root(seed):
    import oracle_lib as O
    coeffs = O.sample_fr(seed, 1 << 10)
    rc, cw = O.rs_interleaved_encode(coeffs.reshape(8, 128, 4), np.zeros((0, 4), np.uint64), 512)
    assert rc == 0
    O.lib().pko_from_mont_many(O.p64(cw), cw.shape[0])
    return O.merkle_tree(cw.tobytes(), 32 * 8, 512)[-32:]


def _rank_main(rank, world, port, jobs, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    import torch.distributed as dist
    from provekit_b200.replicas import job_throughput, max_over_ranks, shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    mine = shard(jobs, rank, world)
    roots = {j: _oracle_commit_root(j) for j in mine}
    seconds = 1.0 + rank  # stand-in per-rank time
    tput = job_throughput(len(mine), seconds)
    slowest = max_over_ranks(seconds)
    out.put((rank, roots, tput, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_partitions_jobs():
    from provekit_b200.replicas import shard
    jobs = list(range(11))
    parts = [shard(jobs, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == jobs
    assert all(len(p) in (3, 4) for p in parts)
    with pytest.raises(ValueError):
        shard(jobs, 3, 3)


def test_two_gloo_ranks_replicas_match_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    jobs = [101, 102, 103, 104, 105]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, jobs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    roots = {}
    for rank, r, tput, slowest in res:
        roots.update(r)
        assert slowest == 2.0                       # max over the two ranks
        assert tput == pytest.approx(len(jobs) / 2.0)  # all units / slowest rank
    assert sorted(roots) == jobs
    for j in jobs:                                   # same bytes as a single-process run
        assert roots[j] == _oracle_commit_root(j)
