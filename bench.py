"""Benchmark of the set-similarity self-join (one JSON line on stdout).

Workload (default, "titles100k"): 100,000 synthetic title records (5-15 words,
Zipf(1.1) over a seeded 50,000-word vocabulary, 10 % perturbed copies),
padded lower-case 3-grams with distinct ids by ascending frequency, self-joined
at every threshold t in {0.5, 0.6, 0.7, 0.8, 0.9}.  One step = the five joins.
"heavy1m" is the 1M heavy-tailed-record workload at t = 0.7.

Metric: candidates per second (candidates = the reference's "# Candidates"
counter, identical for every method) of the batched + learned form; the plain
per-stage form is timed on the same step and reported beside it, with a check
that both pair sets are identical.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload titles100k|heavy1m|titles18k|heavy300k]
                 [--thresholds 0.7,0.9] [--no-model] [--no-tune] [--no-cpu-baseline]
  python bench.py --impl reference ...   # the CPU restatement of the reference algorithm
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
    "heavy1m": dict(kind="heavy", n=1_000_000, seed=3, thresholds=[0.7]),
    "titles18k": dict(kind="titles", n=18_000, seed=1, thresholds=[0.9]),
    "heavy300k": dict(kind="heavy", n=300_000, seed=4, thresholds=[0.7]),  # profiling size: > L2, a few GB
}


def make_text(w, seed_offset=0, n=None):
    from new_fgssjoin_b200 import datagen
    n = n or w["n"]
    if w["kind"] == "titles":
        return datagen.titles(n, seed=w["seed"] + seed_offset)
    return datagen.heavy(n, seed=w["seed"] + seed_offset)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.p = None
        self.path = os.path.join(ROOT, "gpurun_out", "bench_clocks_%d.csv" % os.getpid())
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


def cpu_reference(w, steps, warmup, sample_note):
    """The reference algorithm on the host cores (oracle restatement, OpenMP)."""
    from oracle import oracle as O
    text = make_text(w)
    ids, lens, tok, loc, nt = O.tokenize(text, **tok_opts(w))
    mid, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    threads = O.lib().orc_num_threads()
    times, cands = [], []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        c = 0
        for t in w["thresholds"]:
            _, st = O.join(mpos, mlen, mtok, nt, t, threads=threads)
            c += st["candidates"]
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
            cands.append(c)
    return float(np.sum(cands) / np.sum(times)), float(np.mean(times) * 1000.0), threads


def tok_opts(w):
    from new_fgssjoin_b200 import datagen
    return dict(datagen.TITLE_TOK)


def run_reference(args, w):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    v, ms, threads = cpu_reference(w, args.steps, args.warmup, "")
    sample = "full step: %d records x thresholds %s (oracle restatement, OpenMP)" % (w["n"], w["thresholds"])
    line = {"metric": "self-join candidates/s (batched+learned vs plain GPU, identical pair set)",
            "impl": "reference", "value": v, "unit": "candidates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, see bench.py docstring)",
            "config": {"workload": args.workload, "records": w["n"], "thresholds": w["thresholds"]},
            "cpu_baseline": {"value": v, "unit": "candidates/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "candidates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="titles100k", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-model", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--thresholds", type=str, default=None, help="comma-separated, overrides the workload's")
    args = ap.parse_args()
    w = dict(WORKLOADS[args.workload])
    if args.thresholds:
        w["thresholds"] = [float(x) for x in args.thresholds.split(",")]
    if args.impl == "reference":
        return run_reference(args, w)

    import torch
    import new_fgssjoin_b200 as F
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ctx = F.Context(device=local, stream=stream.cuda_stream)

    # ---- inputs (untimed): text -> GPU tokenizer -> device-resident sets
    text = make_text(w, seed_offset=rank * 1000)
    sets = ctx.tokenize(text, **tok_opts(w))
    d_arrays = [torch.from_numpy(a.view(np.int32)).to(dev) for a in (sets.id, sets.pos, sets.len, sets.tokens)]

    def dev_view():
        from new_fgssjoin_b200.binding import _View
        v = _View()
        v.id, v.pos, v.len, v.tokens = [t.data_ptr() for t in d_arrays]
        v.n_sets, v.n_tokens, v.n_terms, v.on_device = sets.n_sets, sets.n_tokens, sets.n_terms, 1
        return v

    ts = w["thresholds"]
    # pinned host copies for the end-to-end leg
    pinned = [torch.from_numpy(a.view(np.int32)).pin_memory() for a in (sets.id, sets.pos, sets.len, sets.tokens)]
    host_sets = F.Sets(*(p.numpy().view(np.uint32) for p in pinned), n_terms=sets.n_terms)

    # ---- learned cost model: trained (untimed) on a different sample of the workload
    use_model = not args.no_model
    model_loss = None
    if use_model:
        train_text = make_text(w, seed_offset=7919 + rank, n=min(w["n"], 30000))
        train_sets = ctx.tokenize(train_text, **tok_opts(w))
        model_loss = ctx.model_train([train_sets] * len(ts), ts, epochs=300, lr=0.01, seed=1)

    # autotuner (untimed): fastest fused-kernel shape per threshold, cached in the context
    tuned = {}
    if not args.no_tune:
        for t in ts:
            tuned[str(t)] = ctx.autotune(dev_view(), t, reps=1)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def step(method, view_fn, model):
        return ctx.selfjoin_batch([view_fn()] * len(ts), ts, method=method, use_model=model)

    def timed(method, view_fn, model, k, wu):
        for _ in range(wu):
            step(method, view_fn, model)
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
        tot_ms, outs = 0.0, None
        stats = []
        for _ in range(k):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            outs = step(method, view_fn, model)
            e1.record(stream)
            e1.synchronize()
            tot_ms += e0.elapsed_time(e1)
            stats.append([o.stats for o in outs])
        torch.cuda.synchronize(dev)
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)
        return tot_ms, outs, stats

    clocks = Clocks(local)
    bat_ms, bat_out, bat_stats = timed("batched", dev_view, use_model, args.steps, args.warmup)
    clk = clocks.stop()
    plain_ms, plain_out, _ = timed("plain", dev_view, False, max(1, args.steps // 2), 1)
    plain_steps = max(1, args.steps // 2)
    same = all(np.array_equal(a.q, b.q) and np.array_equal(a.s, b.s) and np.array_equal(a.overlap, b.overlap)
               for a, b in zip(bat_out, plain_out))
    cands = sum(o.stats["candidates"] for o in bat_out)
    # e2e: host (pinned) inputs, H2D + join + D2H of the pairs inside the timed region
    e2e_ms, e2e_out, _ = timed("batched", host_sets.view, use_model, args.steps, 1)
    h2d = sum(a.nbytes for a in (sets.id, sets.pos, sets.len, sets.tokens)) * len(ts)
    d2h = sum(len(o) * 24 for o in e2e_out)

    # max over ranks
    vals = torch.tensor([bat_ms, plain_ms, e2e_ms], dtype=torch.float64, device=dev)
    if ws > 1:
        torch.distributed.all_reduce(vals, op=torch.distributed.ReduceOp.MAX)
    bat_ms, plain_ms, e2e_ms = vals.tolist()

    # roofline of the fused filter+verify kernel (per launch = one step's five joins)
    last = bat_stats[-1]
    kern_ms = float(np.mean([s[0]["ms_probe"] for s in bat_stats]))
    P = sum(s["probe_tokens"] for s in last)
    W = sum(s["window_entries"] for s in last)
    M = sum(s["merged_tokens"] for s in last)
    R = sum(s["results"] for s in last)
    alg_bytes = 12 * P + 8 * W + 4 * M + 12 * R
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9 if kern_ms > 0 else 0.0
    launches = int(np.mean([s[0]["launches"] for s in bat_stats]))

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, ms, threads = cpu_reference(w, 1, 0, "")
        cpu = {"value": v, "unit": "candidates/s", "cores": threads, "kind": "port",
               "sample": "one full step (%d records x %d thresholds), oracle restatement, OpenMP" % (w["n"], len(ts))}

    if rank == 0:
        per_step = bat_ms / args.steps
        line = {
            "metric": "self-join candidates/s (batched+learned vs plain GPU, identical pair set)",
            "value": ws * cands / (per_step * 1e-3), "unit": "candidates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator, see bench.py docstring)",
            "config": {"workload": args.workload, "records": sets.n_sets, "tokens": sets.n_tokens,
                       "thresholds": ts, "joins_per_step": len(ts), "l2": "flushed between steps (256 MB write)",
                       "parallelism": "replicas x%d" % ws},
            "plain_ms_per_step": plain_ms / plain_steps,
            "speedup_vs_plain": (plain_ms / plain_steps) / per_step,
            "pair_sets_identical": bool(same),
            "candidates_per_step": cands, "results_per_step": R,
            "autotune": {t: "%dx%d/rt%d" % (v["threads"], v["hash_log2"], v["regs_rt"]) for t, v in tuned.items()},
            "model": {"used": use_model, "train_loss": model_loss,
                      "overflow_retries": sum(s["overflow_retries"] for s in last)},
            "e2e": {"value": ws * cands / (e2e_ms / args.steps * 1e-3), "unit": "candidates/s",
                    "ms_per_step": e2e_ms / args.steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": "k_fused", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profiled_traffic(args.workload), "traffic_source": "profiles/k_fused_%s.md"
                         % args.workload, "alg_bytes": alg_bytes, "kernel_ms": kern_ms},
            "gpu_launches": launches * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
