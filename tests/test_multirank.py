"""The N>1 host logic of bench.py on CPU: two gloo ranks, each owning its
own shard; the job time is the max over ranks, the row count the sum, and
the per-rank shards are disjoint (distinct seeds).  Each rank runs the
oracle on its shard; the ranks' kds_final buffers are gathered on rank 0
(the input of the device merge that follows at N>1) and their states add up
to the union's."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    for sub in ("pg-strom_b200", os.path.join("pg-strom_b200", "producer"), "oracle", ""):
        sys.path.insert(0, os.path.join(ROOT, sub))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import numpy as np
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        import xb_configs as C
        import xb_final as F
        import xb_oracle as O
        fact, sess, km, expect, meta = C.join_groupby(nfact=40_000, ndim1=2000, ndim2=300,
                                                      seed_config=bench.shard_seed(rank))
        o = O.Oracle(sess, km)
        for ch in fact.block_chunks(pages_per_chunk=100):
            o.exec(ch)
        o_final = o.final()
        got = F.decode_kds_final(o_final, sess)
        o.close()
        truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
        ok = F.compare_groups(got, truth) == []
        t = bench.max_over_ranks(float(rank + 1), world)
        n = bench.sum_over_ranks(1000.0, world)
        objs = [None] * world
        dist.all_gather_object(objs, (rank, ok, sorted(got.items())[:3]))
        # per-rank kds_final collected on rank 0 (the input of the device
        # merge); the union's groups are the sum of the ranks' states
        fin = o_final
        finals = bench.gather_finals(fin, rank, world)
        union = None
        if rank == 0:
            union = {}
            for f in finals:
                for k, v in F.decode_kds_final(f, sess).items():
                    u = union.setdefault(k, [(0, 0), 0])
                    union[k] = [(u[0][0] + v[0][0], u[0][1] + v[0][1]), u[1] + v[1]]
            assert all(isinstance(f, np.ndarray) for f in finals)
        else:
            assert finals is None
        q.put((rank, ok, t, n, objs, union, sum(v[1] for v in got.values())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda x: x[0])
    for rank, ok, t, n, objs, union, nrows in res:
        assert ok
        assert t == 2.0          # max over ranks
        assert n == 2000.0       # sum over ranks
    union = res[0][5]
    assert sum(v[1] for v in union.values()) == sum(r[6] for r in res)
    # shards differ: the first groups' states are not identical across ranks
    objs = res[0][4]
    assert objs[0][2] != objs[1][2]


def _a2a_worker(rank, world, port, q):
    for sub in ("pg-strom_b200", os.path.join("pg-strom_b200", "producer"), "oracle", ""):
        sys.path.insert(0, os.path.join(ROOT, sub))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import numpy as np
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import xb_exchange as X
        # part r of rank s: (s, r) repeated s + r + 1 times; rank 1 sends nothing to rank 0
        parts = []
        for r in range(world):
            if rank == 1 and r == 0:
                parts.append(None)
            else:
                parts.append(np.full(7 * (rank + r + 1), 16 * rank + r, dtype=np.uint8))
        got = X.alltoall_bytes(parts, rank, world)
        q.put((rank, [None if g is None else (len(g), int(g[0]), bool((g == g[0]).all())) for g in got]))
    finally:
        dist.destroy_process_group()


def test_alltoall_of_final_parts_over_gloo():
    """The byte exchange of the hash-partitioned final merge: every rank
    receives, in rank order, exactly the part each rank addressed to it."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 3
    procs = [ctx.Process(target=_a2a_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        for s_, g in enumerate(res[r]):
            if s_ == 1 and r == 0:
                assert g is None
            else:
                assert g == (7 * (s_ + r + 1), 16 * s_ + r, True)


def _exchange_worker(rank, world, port, q):
    for sub in ("pg-strom_b200", os.path.join("pg-strom_b200", "producer"), "oracle", ""):
        sys.path.insert(0, os.path.join(ROOT, sub))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        import xb_configs as C
        import xb_exchange as X
        import xb_final as F
        import xb_oracle as O
        import xb_split as S
        # every rank's shard through the oracle, its kds_final split by hash
        # % world, the parts exchanged, the received parts merged
        fact, sess, km, expect, meta = C.join_groupby(nfact=30_000, ndim1=2000, ndim2=300,
                                                      regions=C.long_strings(200, lo=8, hi=40),
                                                      seed_config=bench.shard_seed(rank))
        o = O.Oracle(sess, km)
        for ch in fact.block_chunks(pages_per_chunk=100):
            o.exec(ch)
        parts = S.split_kds_final(o.final(), world)
        o.close()
        got = X.alltoall_bytes(parts, rank, world)
        actions = [a for a, _, _ in F.session_aggs(sess) if a != 101]
        mine, hashes_ok = {}, True
        for p in got:
            if p is None:
                continue
            hashes_ok &= all(h % world == rank for h in S.tuple_hashes(p))
            for k, v in F.decode_kds_final(p, sess).items():
                mine[k] = S.merge_states(actions, mine[k], v) if k in mine else v
        # the truth of every shard, for the union
        truth = {}
        for r in range(world):
            _, _, _, ex, _ = C.join_groupby(nfact=30_000, ndim1=2000, ndim2=300,
                                            regions=C.long_strings(200, lo=8, hi=40),
                                            seed_config=bench.shard_seed(r))
            for k, v in ex.items():
                t = truth.setdefault(k, [(0, 0), 0])
                truth[k] = [(t[0][0] + v["sum_amount"][0], t[0][1] + v["sum_amount"][1]), t[1] + v["nrows"]]
        q.put((rank, hashes_ok, {k: v for k, v in mine.items()}, truth))
    finally:
        dist.destroy_process_group()


def test_exchange_split_merge_through_the_oracle():
    """The whole exchange step on two gloo ranks: each rank's oracle
    kds_final split by hash % 2 (the host restatement of FinalParts), the
    parts exchanged all-to-all, the received parts merged.  Every group
    ends on the rank its hash names, on exactly one rank, and the ranks'
    merged groups are the union of both shards."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict((r[0], r[1:]) for r in (q.get(timeout=180) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import xb_final as F
    union = {}
    for r in range(world):
        ok, mine, truth = res[r]
        assert ok
        assert not (set(mine) & set(union))
        union.update(mine)
    assert F.compare_groups(union, res[0][2], rtol=0.0) == []
