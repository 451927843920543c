"""The benchmark's reference arm (the CPU restatement of the reference
algorithm, timed on host cores) keeps the JSON contract the driver reads; it
needs no GPU, so it runs here on a small workload."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "plain2d",
       "--steps", "2", "--warmup", "1", "--cpu-seconds", "0.5"]


def _run(env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run(CMD, capture_output=True, text=True, env=env, timeout=300)


def test_reference_arm_line():
    r = _run()
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "nnz(L+U)/s" and d["unit"] == "nnz/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["workload"] == "grid2d_64x64_5pt_natural"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    # the sample keeps every thread busy, and the serial run and the max-id
    # restatement of the reference's algorithm are reported beside it
    assert cb["sample_sources"] >= min(d["config"]["n"], 8 * cb["cores"])
    assert "omp_num_threads" in cb and cb["host_cores"] >= 1
    assert cb["serial"]["value"] > 0 and cb["serial"]["cores"] == 1
    assert cb["maxid"]["value"] > 0
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
