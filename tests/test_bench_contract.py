"""CPU checks of bench.py's output contract: the reference arm (the oracle
restatement of the same MG-PCG on the host cores) prints one JSON line with
the keys the contract names, and ranks other than 0 exit without output; the
percentile helper of the serving measurements uses the nearest-rank rule."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def run_bench(*args, env_extra=None):
    env = dict(os.environ)
    env.pop("RANK", None)
    if env_extra:
        env.update(env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          env=env, timeout=600, cwd=ROOT)


def test_reference_arm_prints_one_contract_line():
    p = run_bench("--impl", "reference", "--steps", "2", "--warmup", "1", "--n", "33")
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["higher_is_better"] is True and line["unit"] == "solves/s"
    assert line["config"]["grid"] == [33, 33, 33]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = run_bench("--impl", "reference", "--steps", "1", "--warmup", "1", "--n", "33", env_extra={"RANK": "1"})
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_nearest_rank_percentile():
    import bench

    assert bench._pct([], 50) is None
    assert bench._pct([3.0, 1.0, 2.0, 4.0], 50) == 2.0
    xs = list(range(1, 101))
    assert bench._pct(xs, 99) == 99 and bench._pct(xs, 100) == 100 and bench._pct(xs, 1) == 1
    assert bench._pct(list(range(1, 65)), 50) == 32


def test_reference_arm_steps_are_whole_solves():
    # each step is one whole converged solve: K steps take K x ms_per_step,
    # which fits inside the process's own wall time
    import time

    t0 = time.perf_counter()
    p = run_bench("--impl", "reference", "--steps", "3", "--warmup", "1", "--n", "33")
    wall = time.perf_counter() - t0
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["steps"] * line["ms_per_step"] / 1e3 <= wall
    assert "whole converged solve" in line["cpu_baseline"]["sample"]
    lat = line["latency_ms"]
    assert 0 < lat["p50"] <= lat["p99"]


def test_summary_picks_form_figures():
    import bench

    line = {"latency_ms": {"p50": 23.0, "p99": 24.0}, "cpu_baseline": {"value": 0.1},
            "forms": {"batched": {"solves_per_s": 7000.0, "speedup_vs_plain_fp64": 19.0},
                      "convdiff": {"mixed": {"rel_l2_vs_fp64": 3.41e-09}},
                      "serving_stream": {"points": [{"rate_hz": 50.0, "fp64": {"poisson_p50_ms": 5.0, "p99_ms": 9.0}}]}}}
    s = bench.summarize(line)
    assert s["fp64_solve_p50_ms"] == 23.0 and s["batched_vs_plain_fp64"] == 19.0
    assert s["stream_50hz_fp64_poisson_p50_ms"] == 5.0 and s["serving_host_inputs_mixed_solves_per_s"] is None
    assert s["convdiff513_mixed_rel_l2_vs_gpu_fp64"] == 3.41e-09  # small values keep their digits
