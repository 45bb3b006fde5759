"""bench.py's reference arm on the CPU: `--impl reference` times the oracle (the
port of the reference's FP64 path) on the host cores and prints one JSON line
with the same metric and unit as the GPU arm, a cpu_baseline describing the run
and an e2e object without host-device traffic.  The small 32-rod 64^3 workload
keeps it to seconds."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*extra, env=None):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "rods32_L64_g64", "--steps", "1", "--warmup", "1", *extra],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = _run()
    assert len(lines) == 1
    d = lines[0]
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["config"]["workload"] == "rods32_L64_g64"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # whole oracle steps are timed (no scaling of a sample), the single-thread figure is labelled as derived
    assert "whole EM step" in cb["sample"] and d["gmres_iters"] > 0
    assert abs(d["ms_per_step"] - 1e3 * d["config"]["bodies"] / d["value"]) < 1e-6 * d["ms_per_step"]
    st = d["single_thread"]
    assert st["cores"] == 1 and 0 < st["value"] <= d["value"] * 1.5 and "derived" in st


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs the reference arm; the others exit 0
    without a line."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert _run(env=env) == []
