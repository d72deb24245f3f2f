"""bench.py's reference arm on the CPU: one JSON line with the keys the
benchmark contract asks for, from rank 0 only, on the q2D workload (the 256^3
default takes minutes of oracle time per step on a small host); and both
arms of the default workload build the same config and initial state."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="4", **env_extra)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "q2d", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    lines = _run({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["metric"] == d["unit"] == "grid-pt*steps/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] >= 3
    assert d["value"] > 0 and d["config"]["workload"] == "q2d-spin2-SO-realtime-512x512-quench"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_print_nothing():
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_both_arms_share_config_and_state():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    w = b.D3
    assert b.bench_config(w, "fp64", 1) == b.bench_config(w, "fp64", 1, impl="reference")
    assert b.bench_config(w)["workload"] == "3d-spin1-SO-imag-256^3"
    assert b.bench_config(w)["grid"] == [256, 256, 256]
    # the seeded start is reproducible (both arms build it the same way)
    n, d = (16, 16, 16), (1.6, 1.6, 1.6)
    a, c = b.initial_state(w, n, d), b.initial_state(w, n, d)
    assert a.shape == (16, 16, 16, 3) and (a == c).all()
