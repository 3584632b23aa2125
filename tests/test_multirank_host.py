"""The N-rank host logic of bench.py on two gloo ranks (CPU, no GPU): the
ensemble is split by member index with no exchange (every member on exactly
one rank, the per-rank meshes summing to the whole), and the max / sum
reductions the timing and the counters use agree with a single process."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COUNT = 48


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    from fast_b200 import decks
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mine = bench.ensemble_members(rank, world, count=COUNT)
        idx = [k for k, _ in mine]
        gathered = [None] * world
        dist.all_gather_object(gathered, idx)
        d, noff, _ = decks.concat_decks([m for _, m in mine])
        neq_sum, ne_sum = bench.reduce_over_ranks([d.num_eq(), d.num_elems], "sum", world, "cpu")
        tmax = bench.reduce_over_ranks([0.25 + rank], "max", world, "cpu")[0]
        # the same members as a single process draws them
        solo = dict(bench.ensemble_members(0, 1, count=COUNT))
        same = all(np.array_equal(solo[k].E, m.E) and np.array_equal(solo[k].conn, m.conn) for k, m in mine)
        q.put((rank, gathered, neq_sum, ne_sum, tmax, same, len(noff) - 1))
    finally:
        dist.destroy_process_group()


def test_ensemble_split_and_reductions_on_two_gloo_ranks():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, ROOT)
    import bench
    from fast_b200 import decks
    full, _, _ = decks.concat_decks([m for _, m in bench.ensemble_members(0, 1, count=COUNT)])
    for rank, gathered, neq_sum, ne_sum, tmax, same, nprob in res:
        assert sorted(gathered[0] + gathered[1]) == list(range(COUNT))
        assert not set(gathered[0]) & set(gathered[1])
        assert gathered[rank] == list(range(rank, COUNT, 2))
        assert nprob == len(gathered[rank])
        assert int(neq_sum) == full.num_eq() and int(ne_sum) == full.num_elems
        assert tmax == 1.25
        assert same
