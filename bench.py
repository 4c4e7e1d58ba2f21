"""Benchmark of the set-similarity self-join (one JSON line on stdout).

Workload (default, "heavy1m"): 1,000,000 heavy-tailed records (lognormal word
counts, mu 2.5, sigma 1.0, 2-600 words drawn Zipf(1.1) from a seeded 50,000-word
vocabulary, 5 % near-duplicate clusters of 2-20 perturbed copies), padded
lower-case 3-grams with distinct ids by ascending frequency, self-joined at
t = 0.7.  One step = that join.
Other workloads:
  titles100k 100,000 title records (5-15 words, 10 % perturbed copies) self-joined
             at every t in {0.5, 0.6, 0.7, 0.8, 0.9} (one step = the five joins);
  reads500k  500,000 150-base reads from a seeded 5 Mbp genome (0.5 % substitutions),
             canonical 16-mer sets, t = 0.8;
  batch256   256 independent joins of title records, log-uniform sizes 1,000-200,000,
             each with its own t from {0.6, 0.7, 0.8, 0.9, 0.95}; one step = the 256
             joins, batched in one call against 256 sequential plain calls, with the
             per-join latency p50/p99 of both forms;
  rs200k     R-S join: 200,000 title records dealt alternately into R and S (one
             vocabulary), t in {0.6, 0.8} (no counterpart in the reference);
  titles18k, heavy300k  smaller cases (the 18k-title join at t = 0.9; a profiling size).

Metric: candidates per second (candidates = the reference's "# Candidates"
counter, identical for every method) of the batched + learned form; the plain
per-stage form (same filters, per-stage launches, exact two-pass counts) and
the batched form without the learned model are timed on the same step and
reported beside it, device-resident and end to end, with checks that every
pair set is identical and equal to the CPU oracle's.

  python bench.py [--gpus N] [--steps K] [--warmup W]
                  [--workload heavy1m|titles100k|reads500k|batch256|rs200k|titles18k|heavy300k]
                  [--thresholds 0.7,0.9] [--no-model] [--no-tune] [--no-cpu-baseline]
  python bench.py --impl reference ...   # the CPU restatement of the reference algorithm
  torchrun ... bench.py --gpus N --shard  # one join split over N GPUs by the cost model (strong scaling)
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "titles100k": dict(kind="titles", n=100_000, seed=2, thresholds=[0.5, 0.6, 0.7, 0.8, 0.9]),
    # ref_step: the reference arm times every ref_step-th query per step (a strided sample)
    "heavy1m": dict(kind="heavy", n=1_000_000, seed=3, thresholds=[0.7], ref_step=4),
    "reads500k": dict(kind="reads", n=500_000, seed=5, thresholds=[0.8]),
    "batch256": dict(kind="batch", joins=256, lo=1000, hi=200_000, seed=6),
    "rs200k": dict(kind="rs", n=200_000, seed=8, thresholds=[0.6, 0.8]),
    "titles18k": dict(kind="titles", n=18_000, seed=1, thresholds=[0.9]),
    "heavy300k": dict(kind="heavy", n=300_000, seed=4, thresholds=[0.7]),  # profiling size: > L2, a few GB
}
GENOME_LEN = 5_000_000


def make_text(w, seed_offset=0, n=None):
    """One record file of a single-file workload (``n`` overrides its size; a
    smaller read sample keeps the genome's coverage by shrinking the genome)."""
    from new_fgssjoin_b200 import datagen
    n = n or w["n"]
    if w["kind"] in ("titles", "rs"):
        return datagen.titles(n, seed=w["seed"] + seed_offset)
    if w["kind"] == "reads":
        return datagen.reads(n, seed=w["seed"] + seed_offset, genome_len=max(10_000, GENOME_LEN * n // w["n"]))
    return datagen.heavy(n, seed=w["seed"] + seed_offset)


def _titles_job(args):
    from new_fgssjoin_b200 import datagen
    n, seed = args
    return datagen.titles(int(n), seed=int(seed))


def workload_jobs(w, seed_offset=0, n=None, only=None):
    """-> (texts, jobs): the record files of one step and its joins as
    (text index, threshold).  The 256-join batch draws log-uniform sizes and a
    threshold per join (datagen.batch_sizes); its files are generated in a
    spawned process pool before the first GPU call.  ``only``: the file
    indices to generate (the others are None)."""
    if w["kind"] == "rs":  # one title file dealt alternately into R and S
        lines = make_text(w, seed_offset, n).split(b"\n")[:-1]
        return [b"\n".join(lines[0::2]) + b"\n", b"\n".join(lines[1::2]) + b"\n"], [(0, t) for t in w["thresholds"]]
    if w["kind"] != "batch":
        return [make_text(w, seed_offset, n)], [(0, t) for t in w["thresholds"]]
    from new_fgssjoin_b200 import datagen
    sizes, ts = datagen.batch_sizes(w["joins"], w["lo"], w["hi"], seed=w["seed"] + seed_offset)
    if n:
        sizes = np.minimum(sizes, n)
    keep = range(len(sizes)) if only is None else sorted(only)
    work = [(int(sizes[i]), (w["seed"] + seed_offset) * 100_003 + i) for i in keep]
    import concurrent.futures as cf
    import multiprocessing as mp
    made = []
    if work:
        with cf.ProcessPoolExecutor(max_workers=max(1, min(32, os.cpu_count() or 1, len(work))),
                                    mp_context=mp.get_context("spawn")) as ex:
            made = list(ex.map(_titles_job, work, chunksize=2))
    texts = [None] * len(sizes)
    for i, t in zip(keep, made):
        texts[i] = t
    return texts, [(i, float(t)) for i, t in enumerate(ts)]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.p = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), "fgss_bench_clocks_%d.csv" % os.getpid())
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic(workload):
    """DRAM bytes (read + write) of one k_fused launch from the committed ncu
    summary of this workload (profiles/k_fused_<workload>.md), or None."""
    import re
    path = os.path.join(ROOT, "profiles", "k_fused_%s.md" % workload)
    if not os.path.exists(path):
        return None
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    tot = 0.0
    found = 0
    for line in open(path):
        m = re.match(r"\| dram__bytes_(read|write)\.sum \| ([0-9.]+) (\w+) \|", line)
        if m:
            tot += float(m.group(2)) * scale.get(m.group(3), 1.0)
            found += 1
    return tot if found == 2 else None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_sample(w, jobs):
    """The bounded CPU sample of one step, as job indices: every join of a
    single-file workload; every 8th join of the 256-join batch (32 joins, about
    1/8 of its records)."""
    if w["kind"] == "batch":
        return [k for k in range(len(jobs)) if k % 8 == 0]
    return list(range(len(jobs)))


def oracle_sets(w, texts, sample, jobs):
    """Memory-order records of the sampled files, tokenized by the oracle."""
    from oracle import oracle as O
    if w["kind"] == "rs":
        (_, rp, rl, rt), (_, sp, sl, stk), nt = O.tokenize_dual(texts[0], texts[1], **tok_opts(w))
        return {0: (rp, rl, rt, nt), 1: (sp, sl, stk, nt)}
    mem = {}
    for k in sample:
        ti = jobs[k][0]
        if ti not in mem:
            ids, lens, tok, loc, nt = O.tokenize(texts[ti], **tok_opts(w))
            _, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
            mem[ti] = (mpos, mlen, mtok, nt)
    return mem


def cpu_reference(w, jobs, mem, steps, warmup, q_step=1, keep_pairs=False):
    """The reference algorithm on the host cores (oracle restatement, OpenMP)
    over the bounded sample of one step; ``mem`` maps a file index to its
    memory-order (pos, len, tokens, n_terms).  With q_step > 1 a step joins
    every q_step-th query only (phase = step number mod q_step), against the
    whole index.  -> (candidates/s, ms per step, threads, note, {job index:
    pairs} of the last step when keep_pairs)."""
    from oracle import oracle as O
    sample = cpu_sample(w, jobs)
    threads = O.lib().orc_num_threads()
    times, cands, pairs = [], [], {}
    for it in range(warmup + steps):
        phase = it % q_step
        t0 = time.perf_counter()
        c = 0
        for k in sample:
            ti, t = jobs[k]
            if w["kind"] == "rs":  # R-S join of file 0 (R) with file 1 (S)
                p, st = O.rsjoin(mem[0][:3], mem[1][:3], mem[0][3], t, threads=threads)
            else:
                mpos, mlen, mtok, nt = mem[ti]
                p, st = O.join(mpos, mlen, mtok, nt, t, threads=threads, query_step=q_step, query_phase=phase)
            c += st["candidates"]
            if keep_pairs:
                pairs[k] = p
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
            cands.append(c)
    recs = sum(len(m[1]) for m in mem.values())
    note = ("%d of %d joins (%d records)%s, oracle restatement, OpenMP, %d threads"
            % (len(sample), len(jobs), recs,
               ", every %dth query per step" % q_step if q_step > 1 else "", threads))
    return float(np.sum(cands) / np.sum(times)), float(np.mean(times) * 1000.0), threads, note, pairs


def bench_config(args, w, jobs, ws):
    """The config dict of the JSON line; both arms print the same one."""
    return {"workload": args.workload, "joins_per_step": len(jobs),
            "thresholds": sorted({float(t) for _, t in jobs}),
            "l2": "flushed between steps (256 MB write)", "parallelism": "replicas x%d" % ws}


def tok_opts(w):
    from new_fgssjoin_b200 import datagen
    return dict(datagen.READ_TOK if w["kind"] == "reads" else datagen.TITLE_TOK)


METRIC = "self-join candidates/s (batched+learned vs plain GPU, identical pair set)"


def run_reference(args, w):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    _, jobs = workload_jobs(w, only=())
    sample = cpu_sample(w, jobs)
    texts, _ = workload_jobs(w, only={jobs[k][0] for k in sample})
    mem = oracle_sets(w, texts, sample, jobs)
    v, ms, threads, note, _ = cpu_reference(w, jobs, mem, args.steps, args.warmup, q_step=w.get("ref_step", 1))
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "candidates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator, see bench.py docstring)",
            "config": bench_config(args, w, jobs, ws),
            "cpu_baseline": {"value": v, "unit": "candidates/s", "cores": threads, "kind": "port", "sample": note},
            "e2e": {"value": v, "unit": "candidates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_sharded(args, w):
    """--shard: ONE join of the workload split over the ranks by query ranges of
    equal estimated work (the batched method's cost estimates, computed on rank
    0 and broadcast), each rank joining its range against the replicated index,
    then an all-gather of the pair buffers over NCCL (the one exchange).  Every
    rank holds the same records (the same seed).  Timed: the local joins and the
    gather, max over ranks; strong scaling (total work fixed)."""
    import datetime
    import torch
    import torch.distributed as dist
    import new_fgssjoin_b200 as F
    from new_fgssjoin_b200.binding import _View
    from new_fgssjoin_b200.shard import agreed_ranges, gather_pairs, FIELDS
    ws, rank, local = dist_env()
    if w["kind"] not in ("titles", "heavy", "reads"):
        raise SystemExit("--shard takes a single-file workload")
    text = make_text(w)  # every rank: the same records
    t = w["thresholds"][0]
    train = [make_text(w, seed_offset=7919 + k, n=max(1000, w["n"] // d)) for k, d in enumerate((27, 9, 3))]
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ctx = F.Context(device=local, stream=stream.cuda_stream)
    to = tok_opts(w)
    sets = ctx.tokenize(text, **to)
    del text
    ctx.model_train([ctx.tokenize(x, **to) for x in train], [t] * len(train), epochs=300, lr=0.01, seed=1)
    d = [torch.from_numpy(a.view(np.int32)).to(dev) for a in (sets.id, sets.pos, sets.len, sets.tokens)]
    v = _View()
    v.id, v.pos, v.len, v.tokens = [x.data_ptr() for x in d]
    v.n_sets, v.n_tokens, v.n_terms, v.on_device = sets.n_sets, sets.n_tokens, sets.n_terms, 1
    if ws > 1:
        ranges = agreed_ranges(sets.len, ws, lambda: ctx.query_costs(v, t, use_model=True))
    else:
        ranges = [(0, int(sets.n_sets))]
    qr = ranges[rank]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        p = ctx.selfjoin(v, t, method="batched", use_model=True, query_range=qr)
        cols = {f: getattr(p, f) for f in FIELDS}
        return p, (gather_pairs(cols) if ws > 1 else cols)

    def barrier():
        torch.cuda.synchronize(dev)
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step()
    barrier()
    clocks = Clocks(local)
    tot = 0.0
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        p, full = step()
        e1.record(stream)
        e1.synchronize()
        tot += e0.elapsed_time(e1)
    clk = clocks.stop()
    barrier()
    mine = torch.tensor([float(p.stats["candidates"]), float(p.stats["window_entries"])], dtype=torch.float64,
                        device=dev)
    if ws > 1:
        mx = torch.tensor([tot], dtype=torch.float64, device=dev)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        tot = mx.item()
        parts = [torch.zeros_like(mine) for _ in range(ws)]
        dist.all_gather(parts, mine)
        per_rank = [x.tolist() for x in parts]
    else:
        per_rank = [mine.tolist()]
    if rank == 0:
        per_step = tot / args.steps
        cands_all = int(sum(x[0] for x in per_rank))
        line = {"metric": METRIC, "value": cands_all / (per_step * 1e-3), "unit": "candidates/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "int32",
                "data": "synthetic (seeded generator, see bench.py docstring)",
                "config": {"workload": args.workload, "joins_per_step": 1, "thresholds": [t],
                           "l2": "flushed between steps (256 MB write)",
                           "parallelism": "query-range shards x%d (cost-model balanced), all-gather of pairs" % ws},
                "results_per_step": len(full["q"]), "candidates_per_step": cands_all,
                "shard_ranges": ranges, "shard_window_entries": [x[1] for x in per_rank], "clocks": clk}
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        dist.destroy_process_group()


def model_report(used, loss, first, timed, n_joins):
    """The learned model's error against the exact counts of the same joins, and
    how often its presized result buffers overflowed (an exact re-run each)."""
    rep = {"used": used, "train_loss": loss}
    if not used:
        return rep

    def err(key, pkey):
        p = np.array([s[pkey] for s in first], np.float64)
        a = np.array([s[key] for s in first], np.float64)
        rel = np.abs(p - a) / np.maximum(a, 1.0)
        return {"predicted": float(p.sum()), "actual": float(a.sum()),
                "total_rel_err": float(abs(p.sum() - a.sum()) / max(a.sum(), 1.0)),
                "per_join_rel_err_p50": float(np.median(rel)), "per_join_rel_err_p90": float(np.percentile(rel, 90))}
    rep["candidates"] = err("candidates", "predicted_candidates")
    rep["results"] = err("results", "predicted_results")
    rep["overflow_first_call"] = "%d of %d joins" % (sum(s["overflow_retries"] for s in first), n_joins)
    rep["overflow_timed_steps"] = "%d of %d joins" % (sum(s["overflow_retries"] for st in timed for s in st),
                                                       n_joins * len(timed))
    return rep


def _pct(xs):
    xs = np.asarray(xs, dtype=np.float64)
    return {"p50": float(np.percentile(xs, 50)), "p99": float(np.percentile(xs, 99)), "max": float(xs.max())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="heavy1m", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-model", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--shard", action="store_true", help="one join split over the GPUs (strong scaling)")
    ap.add_argument("--thresholds", type=str, default=None, help="comma-separated, overrides the workload's")
    args = ap.parse_args()
    w = dict(WORKLOADS[args.workload])
    if args.thresholds and w["kind"] != "batch":
        w["thresholds"] = [float(x) for x in args.thresholds.split(",")]
    if args.impl == "reference":
        return run_reference(args, w)
    if args.shard:
        return run_sharded(args, w)

    ws, rank, local = dist_env()
    # record files (untimed) are generated before the first GPU call
    texts, jobs = workload_jobs(w, seed_offset=rank * 1000)
    train_texts = []
    if not args.no_model:
        if w["kind"] == "batch":  # 8 joins of another batch draw
            train_texts, _ = workload_jobs(w, seed_offset=7919 + rank, only=range(8))
            train_texts = [x for x in train_texts if x is not None]
        else:  # other samples of the workload at 1/27, 1/9 and 1/3 of its size
            train_texts = [make_text(w, seed_offset=7919 + rank + k, n=max(1000, w["n"] // d))
                           for k, d in enumerate((27, 9, 3))]

    import torch
    import new_fgssjoin_b200 as F
    from new_fgssjoin_b200.binding import _View
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ctx = F.Context(device=local, stream=stream.cuda_stream)
    to = tok_opts(w)

    # ---- inputs (untimed): text -> GPU tokenizer -> device-resident sets + pinned host copies
    sets, d_arrays, host_sets = [], [], []
    tokenized = list(ctx.tokenize_dual(texts[0], texts[1], **to)) if w["kind"] == "rs" else \
        [ctx.tokenize(text, **to) for text in texts]
    tune_union = ctx.tokenize(texts[0] + texts[1], **to) if w["kind"] == "rs" and not args.no_tune else None
    for s in tokenized:
        sets.append(s)
        d_arrays.append([torch.from_numpy(a.view(np.int32)).to(dev) for a in (s.id, s.pos, s.len, s.tokens)])
        pinned = [torch.from_numpy(a.view(np.int32)).pin_memory() for a in (s.id, s.pos, s.len, s.tokens)]
        host_sets.append(F.Sets(*(p.numpy().view(np.uint32) for p in pinned), n_terms=s.n_terms))
    del tokenized  # (the texts stay for the text-to-pairs leg)

    def dev_view(ti):
        v = _View()
        v.id, v.pos, v.len, v.tokens = [t.data_ptr() for t in d_arrays[ti]]
        s = sets[ti]
        v.n_sets, v.n_tokens, v.n_terms, v.on_device = s.n_sets, s.n_tokens, s.n_terms, 1
        return v

    def host_view(ti):
        return host_sets[ti].view()

    ts = [t for _, t in jobs]
    t_list = sorted(set(ts))

    # ---- learned cost model: trained (untimed) on a different sample of the workload
    use_model = not args.no_model
    model_loss = None
    if use_model:
        tr = [ctx.tokenize(x, **to) for x in train_texts]
        if w["kind"] == "batch":
            pairs = [(tr[k], t_list[k % len(t_list)]) for k in range(len(tr))]
        else:
            pairs = [(x, t) for x in tr for t in t_list]
        model_loss = ctx.model_train([x for x, _ in pairs], [t for _, t in pairs], epochs=300, lr=0.01, seed=1)
        del tr, pairs

    # autotuner (untimed): fastest fused-kernel shape per threshold on its largest join, cached in the context
    tuned = {}
    if not args.no_tune:
        for t in t_list:
            if w["kind"] == "rs":  # the R-S join runs on the union of R and S: tune on a self-join that size
                tuned[str(t)] = ctx.autotune(tune_union, t, reps=1)
                continue
            ti = max((j for j in jobs if j[1] == t), key=lambda j: sets[j[0]].n_tokens)[0]
            tuned[str(t)] = ctx.autotune(dev_view(ti), t, reps=1)
    tune_union = None

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def step_batched(view_fn, model=None):
        um = use_model if model is None else model
        if w["kind"] == "rs":
            return [ctx.rsjoin(view_fn(0), view_fn(1), t, method="batched", use_model=um) for t in ts]
        return ctx.selfjoin_batch([view_fn(ti) for ti, _ in jobs], ts, method="batched", use_model=um)

    def step_plain(view_fn, per_join_ms=None):
        """The plain form: the joins one after another, one call each."""
        outs = []
        for ti, t in jobs:
            if per_join_ms is not None:
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            if w["kind"] == "rs":
                outs.append(ctx.rsjoin(view_fn(0), view_fn(1), t, method="plain"))
            else:
                outs += ctx.selfjoin_batch([view_fn(ti)], [t], method="plain")
            if per_join_ms is not None:
                b.record(stream)
                b.synchronize()
                per_join_ms.append(a.elapsed_time(b))
        return outs

    def barrier():
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    first_stats = []

    def timed(fn, k, wu, name):
        for i in range(wu):
            outs = fn()
            if i == 0:
                first_stats.append([o.stats for o in outs])
        barrier()
        tot_ms, outs, stats = 0.0, None, []
        for _ in range(k):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push(name)  # lets a profiler select the timed steps (ncu --nvtx-include)
            e0.record(stream)
            outs = fn()
            e1.record(stream)
            e1.synchronize()
            torch.cuda.nvtx.range_pop()
            tot_ms += e0.elapsed_time(e1)
            stats.append([o.stats for o in outs])
        barrier()
        return tot_ms, outs, stats

    def same_pairs(xs, ys):
        return all(np.array_equal(a.q, b.q) and np.array_equal(a.s, b.s) and np.array_equal(a.overlap, b.overlap)
                   for a, b in zip(xs, ys))

    clocks = Clocks(local)
    bat_ms, bat_out, bat_stats = timed(lambda: step_batched(dev_view), args.steps, args.warmup, "batched_step")
    clk = clocks.stop()
    # the batched form without the learned model (model-free presizing and work items)
    nom_ms, nom_out = None, None
    if use_model:
        nom_ms, nom_out, _ = timed(lambda: step_batched(dev_view, False), args.steps, args.warmup, "no_model_step")
    plain_steps = max(1, args.steps // 2)
    plain_join_ms = []
    plain_ms, plain_out, _ = timed(lambda: step_plain(dev_view, plain_join_ms), plain_steps, 1, "plain_step")
    cands = sum(o.stats["candidates"] for o in bat_out)
    # e2e: host (pinned) inputs, H2D + join + D2H of the pairs inside the timed region
    e2e_ms, e2e_out, _ = timed(lambda: step_batched(host_view), args.steps, 1, "e2e_step")
    plain_e2e_ms, plain_e2e_out, _ = timed(lambda: step_plain(host_view), plain_steps, 1, "plain_e2e_step")

    def step_text():
        """Text in host memory to pairs in host memory: GPU tokenizer, then the
        batched join of the tokenized records (the user's whole path)."""
        if w["kind"] == "rs":
            r, s_ = ctx.tokenize_dual(texts[0], texts[1], **to)
            return [ctx.rsjoin(r, s_, t, method="batched", use_model=use_model) for t in ts]
        tok = [ctx.tokenize(x, **to) for x in texts]
        return ctx.selfjoin_batch([tok[ti] for ti, _ in jobs], ts, method="batched", use_model=use_model)

    text_steps = max(1, args.steps // 2)
    text_ms, text_out, _ = timed(step_text, text_steps, 1, "text_e2e_step")
    text_bytes = sum(len(x) for x in texts)
    same = same_pairs(bat_out, plain_out) and same_pairs(e2e_out, plain_out) and \
        same_pairs(plain_e2e_out, plain_out) and (nom_out is None or same_pairs(nom_out, plain_out)) and \
        same_pairs(text_out, plain_out)
    # bytes copied to the device per step: an R-S join copies both files per call; the joins of one
    # batched call that share host arrays copy them once
    def set_bytes(k):
        return sum(a.nbytes for a in (sets[k].id, sets[k].pos, sets[k].len, sets[k].tokens))
    if w["kind"] == "rs":
        h2d = len(jobs) * (set_bytes(0) + set_bytes(1))
    else:
        h2d = sum(set_bytes(k) for k in {ti for ti, _ in jobs})
    d2h = sum(len(o) * 24 for o in e2e_out)

    # per-join latency (the 256-join batch): every join of the batch finishes when the batched call
    # returns; the plain joins finish one after another.  "alone": each join run by itself.
    per_join = None
    if w["kind"] == "batch":
        nj = len(jobs)
        pj = np.asarray(plain_join_ms[-nj:], dtype=np.float64)
        alone_b = []
        for ti, t in jobs:
            ctx.selfjoin_batch([dev_view(ti)], [t], method="batched", use_model=use_model)  # records + captures
            flush.fill_(1.0)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ctx.selfjoin_batch([dev_view(ti)], [t], method="batched", use_model=use_model)
            b.record(stream)
            b.synchronize()
            alone_b.append(a.elapsed_time(b))
        per_step = bat_ms / args.steps
        per_join = {"unit": "ms",
                    "batched_completion": _pct([per_step] * nj),
                    "plain_sequential_completion": _pct(np.cumsum(pj)),
                    "batched_alone": _pct(alone_b),
                    "plain_alone": _pct(pj),
                    "sizes_records": _pct([sets[ti].n_sets for ti, _ in jobs])}

    # max over ranks
    vals = torch.tensor([bat_ms, plain_ms, e2e_ms, plain_e2e_ms, nom_ms or 0.0, text_ms], dtype=torch.float64,
                        device=dev)
    if ws > 1:
        torch.distributed.all_reduce(vals, op=torch.distributed.ReduceOp.MAX)
    bat_ms, plain_ms, e2e_ms, plain_e2e_ms, nom_ms_m, text_ms = vals.tolist()
    if nom_ms is not None:
        nom_ms = nom_ms_m

    # roofline of the fused filter+verify kernel (one launch per step covers every join of the step)
    last = bat_stats[-1]
    # (an R-S step is one call per threshold; a batched self-join step is one call for all its joins)
    kern_ms = float(np.mean([sum(x["ms_probe"] for x in s) if w["kind"] == "rs" else s[0]["ms_probe"]
                             for s in bat_stats]))
    # the global-memory accumulator's launch (queries too long for the fused kernel's tables)
    heavy_ms = float(np.mean([sum(x["ms_heavy"] for x in s) if w["kind"] == "rs" else s[0]["ms_heavy"]
                              for s in bat_stats]))
    P = sum(s["probe_tokens"] for s in last)
    W = sum(s["window_entries"] for s in last)
    M = sum(s["merged_tokens"] for s in last)
    R = sum(s["results"] for s in last)
    Q = sum(s["query_tokens"] for s in last)
    # probe tokens + their list bounds, window entries (source, size|position), merged source
    # tokens, results, and the query records' tokens staged in shared memory
    alg_bytes = 12 * P + 8 * W + 4 * M + 12 * R + 4 * Q
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9 if kern_ms > 0 else 0.0
    launches = int(np.mean([sum(x["launches"] for x in s) if w["kind"] == "rs" else s[0]["launches"]
                            for s in bat_stats]))

    cpu, oracle_eq = None, None
    if rank == 0 and not args.no_cpu_baseline:
        # the same records the GPU joined (the GPU tokenizer's output equals the oracle's), the
        # whole join once: its rate is the CPU baseline and its pairs are compared with the GPU's
        sample = cpu_sample(w, jobs)
        mem = {ti: (sets[ti].pos, sets[ti].len, sets[ti].tokens, sets[ti].n_terms)
               for ti in (range(len(sets)) if w["kind"] == "rs" else {jobs[k][0] for k in sample})}
        v, ms, threads, note, opairs = cpu_reference(w, jobs, mem, 1, 0, keep_pairs=True)
        cpu = {"value": v, "unit": "candidates/s", "cores": threads, "kind": "port", "sample": note}
        # R-S pairs carry (r, s): the GPU result's q column is the index in R
        eq = all(np.array_equal(bat_out[k].q, p["r" if w["kind"] == "rs" else "q"]) and
                 np.array_equal(bat_out[k].s, p["s"]) and
                 np.array_equal(bat_out[k].overlap, p["overlap"]) and np.array_equal(bat_out[k].sim, p["sim"])
                 for k, p in opairs.items())
        oracle_eq = {"equal": bool(eq), "joins_compared": len(opairs), "joins": len(jobs),
                     "compared": "q, s, overlap, float similarity (bit-exact)"}

    if rank == 0:
        per_step = bat_ms / args.steps
        plain_step = plain_ms / plain_steps
        uniq = range(len(sets)) if w["kind"] == "rs" else sorted({ti for ti, _ in jobs})
        line = {
            "metric": METRIC,
            "value": ws * cands / (per_step * 1e-3), "unit": "candidates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, see bench.py docstring)",
            "config": bench_config(args, w, jobs, ws),
            "workload_size": {"records": sum(sets[ti].n_sets for ti in uniq),
                              "tokens": sum(sets[ti].n_tokens for ti in uniq)},
            "plain_ms_per_step": plain_step,
            "plain_e2e_ms_per_step": plain_e2e_ms / plain_steps,
            "speedup_vs_plain": plain_step / per_step,
            "speedup_vs_plain_e2e": (plain_e2e_ms / plain_steps) / (e2e_ms / args.steps),
            "no_model_ms_per_step": nom_ms / args.steps if nom_ms is not None else None,
            "speedup_vs_plain_no_model": plain_step / (nom_ms / args.steps) if nom_ms is not None else None,
            "model_speedup": (nom_ms / args.steps) / per_step if nom_ms is not None else None,
            "plain_method": "same filters as batched (bitmap bound included), per-stage launches, exact two-pass counts",
            "pair_sets_identical": bool(same),
            "pairs_equal_oracle": oracle_eq,
            "candidates_per_step": cands, "results_per_step": R,
            "counters": {"probe_tokens": P, "window_entries": W, "merged_tokens": M, "query_tokens": Q,
                         "verified": sum(s["verified"] for s in last), "results": R,
                         "heavy_queries": sum(s["heavy_queries"] for s in last)},
            "autotune": {t: "%s %dx%d/rt%d" % (v["filter"], v["threads"], v["hash_log2"], v["regs_rt"])
                         for t, v in tuned.items()},
            "model": model_report(use_model, model_loss, first_stats[0], bat_stats, len(jobs)),
            "e2e": {"value": ws * cands / (e2e_ms / args.steps * 1e-3), "unit": "candidates/s",
                    "ms_per_step": e2e_ms / args.steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "e2e_text": {"value": ws * cands / (text_ms / text_steps * 1e-3), "unit": "candidates/s",
                         "ms_per_step": text_ms / text_steps, "text_bytes_per_step": text_bytes,
                         "path": "text in host memory -> GPU tokenizer -> batched join -> pairs in host memory"},
            "roofline": {"bound": "hbm", "kernel": "k_fused", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profiled_traffic(args.workload), "traffic_source": "profiles/k_fused_%s.md"
                         % args.workload, "alg_bytes": alg_bytes,
                         "alg_bytes_formula": "12 probe_tokens + 8 window_entries + 4 merged_tokens + 12 results"
                                              " + 4 query_tokens", "kernel_ms": kern_ms, "heavy_kernel_ms": heavy_ms},
            "gpu_launches": launches * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        if per_join:
            line["per_join_latency"] = per_join
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
