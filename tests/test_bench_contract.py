"""The bench script's workload table and its reference arm's JSON line (CPU only).

The reference arm times the oracle port on the host cores on the workload
itself; one step of the 128^3-particle / 256^3-mesh workload runs here in a few
seconds, so the line the driver parses is checked end to end without a GPU.
"""
import json
import os
import runpy
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench_globals():
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        return runpy.run_path(os.path.join(ROOT, "bench.py"), run_name="bench_contract")
    finally:
        sys.argv = argv


def test_workloads_name_a_model_and_a_metric():
    g = bench_globals()
    for name, w in g["WORKLOADS"].items():
        assert w["model"] in g["MODELS"], name
        assert {"nrow", "ngrid", "box", "seed", "nsteps"} <= set(w), name
        assert w["ngrid"] >= 2 * w["nrow"], name
        metric = g["metric_of"](name)
        assert metric.endswith("PM particle-steps/s"), metric
    # the default workload carries the headline metric
    assert g["metric_of"]("fr5_512_1024") == g["METRIC"]


def test_reference_arm_prints_one_json_line():
    env = dict(os.environ, OMP_NUM_THREADS=str(min(8, os.cpu_count() or 1)))
    # the CPU-runnable workload (128^3 particles, 256^3 mesh): its full-size step takes seconds here
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--workload", "fr5_128_256"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "f(R) PM particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "fr5_128_256" and d["config"]["same_config"] is True
