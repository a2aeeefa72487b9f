"""bench.py on the host (no GPU): the reference arm prints one JSON line with
the keys the benchmark contract asks for, and the tuning strings parse.
The GPU arm's line is checked where a B200 runs it."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "sw_image", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]
    assert "workload" in d["config"]


def test_parse_tuning():
    import bench
    from htrdr_kmin_b200 import api
    t = bench.parse_tuning(api, "96,4,16")
    assert (t.block_size, t.queue_chunk, t.regroup_period) == (96, 4, 16)
    assert t.engine == api.ENGINE_PERSISTENT
    t = bench.parse_tuning(api, "256,1,16,2,128,4096,5000")
    assert (t.engine, t.trace_budget, t.wave_slots, t.wave_tail) == (api.ENGINE_WAVEFRONT, 128, 4096, 5000)
    with pytest.raises(Exception):
        bench.parse_tuning(api, "abc")
