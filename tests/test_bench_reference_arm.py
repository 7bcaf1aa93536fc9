"""bench.py's reference arm on the host (no GPU): rank 0 prints one JSON
line carrying the bench's keys, with the reference's kernels (or the oracle
port) timed on a bounded sample of the 64-shot 500 x 1000 survey; other
ranks of a multi-process launch print nothing and exit 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1", "--cpu-seconds", "0.3"]


def _run(**env):
    e = dict(os.environ, OMP_NUM_THREADS="4", **env)
    return subprocess.run(CMD, cwd=ROOT, env=e, capture_output=True, text=True, timeout=600)


def test_rank0_prints_one_line_with_the_contract_keys():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["unit"] == "Gcell-updates/s" and d["n_gpus"] == 1
    assert "64 shots" in d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "1 shot x first" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_other_ranks_print_nothing():
    p = _run(WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
