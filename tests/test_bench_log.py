"""bench.py's JSON-lines run log: one record per run with the result line,
the scene seed and the host (and, on a GPU box, the GPU) it ran on."""
import importlib.util
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_run_log_appends_one_record_per_run(tmp_path):
    bench = load_bench()
    path = str(tmp_path / "runs.jsonl")
    bench.append_run_log(path, {"metric": "m", "value": 1.5}, 2)
    bench.append_run_log(path, {"metric": "m", "value": 2.5}, 3)
    rows = [json.loads(r) for r in open(path)]
    assert [r["result"]["value"] for r in rows] == [1.5, 2.5]
    assert [r["scene_seed"] for r in rows] == [2, 3]
    for r in rows:
        assert r["host"]["cores"] >= 1 and isinstance(r["host"]["cpu"], str)
        assert "time" in r and "torch" in r and "gpu" in r
