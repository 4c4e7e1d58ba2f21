"""CPU: the multi-GPU sharding path with world_size 2 over gloo.

Each rank takes its query range from shard_ranges, computes its shard (here
with the oracle, which stands in for the GPU join on a CPU-only host), and
gather_pairs reassembles the full result on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from new_fgssjoin_b200 import datagen
from new_fgssjoin_b200.shard import agreed_ranges, gather_pairs, shard_ranges
from oracle import oracle as O


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _cost_on_rank0_only(rank, mlen):
    """A per-query cost only rank 0 may compute (as the library's cost model
    runs on rank 0): any other rank calling it fails the test."""
    def f():
        assert rank == 0, "costs computed on a rank other than 0"
        return np.asarray(mlen, dtype=np.float64) ** 3
    return f


def _worker(rank, world, port, data, t, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        mid, mpos, mlen, mtok, nt = data
        # the cost partition: rank 0's cuts, broadcast (each rank's join stands in for the GPU's)
        ranges = agreed_ranges(mlen, world, _cost_on_rank0_only(rank, mlen))
        assert ranges == shard_ranges(mlen, world, np.asarray(mlen, dtype=np.float64) ** 3)
        qb, qe = ranges[rank]
        pairs, st = O.join(mpos, mlen, mtok, nt, t, query_range=(qb, qe))
        local = {"q": pairs["q"], "s": pairs["s"], "id_q": mid[pairs["q"]], "id_s": mid[pairs["s"]],
                 "overlap": pairs["overlap"], "sim": pairs["sim"]}
        full = gather_pairs(local)
        import torch
        tot = torch.tensor([st["candidates"], st["results"]], dtype=torch.int64)
        dist.all_reduce(tot)
        q.put((rank, {k: v.tolist() for k, v in full.items()}, tot.tolist(), (qb, qe)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("t", [0.6, 0.8])
def test_two_ranks_reassemble_the_full_join(t):
    text = datagen.titles(3000, seed=17)
    ids, lens, tok, loc, nt = O.tokenize(text, **datagen.TITLE_TOK)
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    ref, st = O.join(mpos, mlen, mtok, nt, t)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, (mid, mpos, mlen, mtok, nt), t, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ranges = sorted(g[3] for g in got)
    assert ranges[0][0] == 0 and ranges[0][1] == ranges[1][0] and ranges[1][1] == len(mlen)
    for rank, full, tot, _ in got:
        assert full["q"] == ref["q"].tolist() and full["s"] == ref["s"].tolist()
        assert full["overlap"] == ref["overlap"].tolist()
        assert tot == [st["candidates"], st["results"]]


def test_shard_ranges_cover_and_balance():
    rng = np.random.default_rng(0)
    lens = np.sort(rng.integers(1, 300, 10000))[::-1]
    for world in (1, 2, 3, 8):
        r = shard_ranges(lens, world)
        assert r[0][0] == 0 and r[-1][1] == len(lens)
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        if world > 1:
            c = [(lens[b:e].astype(float) ** 2).sum() for b, e in r]
            assert max(c) < 1.2 * (sum(c) / world) + lens.max() ** 2
