"""The benchmark's reference arm (the CPU restatement) runs without a GPU and
prints one JSON line with the keys the benchmark contract asks for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_json_line():
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "titles18k", "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr
    lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "impl", "cpu_baseline", "e2e", "config"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


def test_rs_workload_split():
    sys.path.insert(0, ROOT)
    import bench
    texts, jobs = bench.workload_jobs(dict(kind="rs", n=1000, seed=3, thresholds=[0.7, 0.9]))
    assert len(texts) == 2 and jobs == [(0, 0.7), (0, 0.9)]
    assert texts[0].count(b"\n") == 500 and texts[1].count(b"\n") == 500


def test_reference_arm_config_is_the_gpu_arms():
    """Both arms print the config of bench_config, so their lines compare."""
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "titles18k", "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    d = json.loads([x for x in p.stdout.splitlines() if x.startswith("{")][0])
    w = bench.WORKLOADS["titles18k"]
    jobs = [(0, t) for t in w["thresholds"]]
    assert d["config"] == bench.bench_config(argparse.Namespace(workload="titles18k"), w, jobs, 1)


def test_strided_query_sample_covers_the_join():
    """The reference arm's strided sample: the q_step phases partition the queries."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from new_fgssjoin_b200 import datagen
    from oracle import oracle as O
    ids, lens, tok, loc, nt = O.tokenize(datagen.heavy(3000, seed=9), **datagen.TITLE_TOK)
    _, mpos, mlen, mtok = O.file_to_memory(ids, lens, tok)
    full, st = O.join(mpos, mlen, mtok, nt, 0.7)
    parts = [O.join(mpos, mlen, mtok, nt, 0.7, query_step=4, query_phase=k) for k in range(4)]
    assert sum(p[1]["candidates"] for p in parts) == st["candidates"]
    got = np.sort(np.concatenate([p[0] for p in parts]), order=("q", "s"))
    assert np.array_equal(got["q"], full["q"]) and np.array_equal(got["s"], full["s"])


def test_every_workload_has_a_profiled_dram_traffic():
    """The roofline's `traffic` of every bench workload comes from its committed
    ncu summary (profiles/k_fused_<workload>.md): both DRAM lines parse."""
    import bench
    for wl in ("heavy1m", "titles100k", "reads500k", "batch256", "rs200k", "titles18k", "heavy300k"):
        t = bench.profiled_traffic(wl)
        assert t is not None and t > 0, wl
