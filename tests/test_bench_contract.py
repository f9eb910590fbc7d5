"""The bench script's reference arm (CPU): one JSON line with the contract's
keys, printed by rank 0 only.  The GPU arm's line is checked by running
bench.py on a B200."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
ARGS = ["--impl", "reference", "--nx", "128", "--nz", "64", "--nt", "40", "--steps", "2",
        "--warmup", "1"]


def _run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="2", **env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py")] + ARGS, cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "Gpt/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["nx"] == 128 and d["config"]["nz"] == 64
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
