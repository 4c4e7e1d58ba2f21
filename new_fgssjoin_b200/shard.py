"""One self-join sharded over ranks (one process per GPU).

Every rank holds the whole record set and builds the same inverted index
(read-only, replicated); the queries -- the first record of each pair -- are
split into contiguous memory-index ranges of equal work, each rank joins its
range (``Context.selfjoin(..., query_range=...)``), and the only exchange is
a final gather of the pair buffers: counts first, then the padded payloads.
Ranges are ascending, so concatenating the gathered shards in rank order
keeps the pairs sorted by (q, s).

Work per query: by default the batched method's own estimate
(``Context.query_costs``: exact window entries + 4 x the learned model's
predicted candidates + size), computed on rank 0, whose cuts are broadcast so
every rank agrees; without a context, a size-squared proxy.
"""
import numpy as np


def query_costs(lens):
    """Work estimate per query: candidates grow with prefix length x list length ~ size^2."""
    lens = np.asarray(lens, dtype=np.float64)
    return lens * lens + 1.0


def shard_ranges(lens, world, costs=None):
    """Contiguous query ranges [b, e) of about equal estimated work, one per
    rank; ``costs`` (per query) overrides the size-squared proxy."""
    n = len(lens)
    if world <= 1 or n == 0:
        return [(0, n)] * max(1, world)
    c = np.cumsum(np.asarray(costs, dtype=np.float64) if costs is not None else query_costs(lens))
    total = c[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(c, total * r / world, side="left")))
    cuts.append(n)
    for i in range(1, len(cuts)):
        cuts[i] = max(cuts[i], cuts[i - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


FIELDS = ("q", "s", "id_q", "id_s", "overlap", "sim")


def gather_pairs(local, group=None):
    """All-gather of per-rank pair columns (dict of equal-length numpy arrays
    for FIELDS) over torch.distributed; returns the concatenation in rank order."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    n_local = len(local["q"])
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, torch.tensor([n_local], dtype=torch.int64, device=dev), group=group)
    counts = [int(x.item()) for x in counts]
    cap = max(max(counts), 1)
    out = {}
    for f in FIELDS:
        a = np.asarray(local[f])
        buf = np.zeros(cap, dtype=a.dtype)
        buf[:n_local] = a
        t = torch.from_numpy(buf.view(np.int32)).to(dev)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        out[f] = np.concatenate([p.cpu().numpy().view(a.dtype)[:k] for p, k in zip(parts, counts)])
    return out


def agreed_ranges(lens, world, costs_fn=None, group=None):
    """Query ranges every rank agrees on: rank 0 computes them (from
    ``costs_fn()`` when given, else the size proxy) and broadcasts the cuts."""
    import torch
    import torch.distributed as dist
    if world <= 1:
        return [(0, len(lens))]
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    cuts = torch.zeros(world + 1, dtype=torch.int64, device=dev)
    if dist.get_rank(group) == 0:
        r = shard_ranges(lens, world, costs_fn() if costs_fn else None)
        cuts.copy_(torch.tensor([b for b, _ in r] + [r[-1][1]], dtype=torch.int64))
    dist.broadcast(cuts, src=0, group=group)
    c = cuts.tolist()
    return [(c[i], c[i + 1]) for i in range(world)]


def sharded_selfjoin(ctx, sets, threshold, rank, world, group=None, method="batched", gather=True, use_model=True,
                     ranges=None):
    """This rank's shard of the join, its queries split by the batched method's
    cost estimate; with ``gather`` every rank gets the full, sorted result.
    ``ranges``: query ranges agreed earlier (agreed_ranges), to reuse."""
    if ranges is None:
        ranges = agreed_ranges(sets.len, world, lambda: ctx.query_costs(sets, threshold, use_model=use_model), group)
    qb, qe = ranges[rank]
    local = ctx.selfjoin(sets, threshold, method=method, query_range=(qb, qe), use_model=use_model)
    if not gather:
        return local
    cols = {f: getattr(local, f) for f in FIELDS}
    return gather_pairs(cols, group)
