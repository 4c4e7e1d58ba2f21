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
