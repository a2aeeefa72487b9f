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


def test_same_workload_string_on_both_arms():
    """The reference arm prints the workload string the GPU arm prints (the
    engine and tuning go under config.tuning)."""
    import bench
    for name in ("mix_full", "lw_flux", "sw_image", "cie_full", "mix"):
        args = bench.parse.__globals__["argparse"].Namespace(mix_side="16,96", mix_spp="16,128")
        assert bench.workload(name, args)[2] == bench.workload(name, args)[2]
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "sw_image", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    d = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    assert d["config"]["workload"] == bench.workload("sw_image")[2]


def test_agreement_and_samples():
    """The agreement of two maps drawn from the same distribution is about
    0.27 % |z| > 3 with mean z ~ 0; the bounded sample takes middle rows of
    every request."""
    import numpy as np
    import bench
    from htrdr_kmin_b200 import api
    from htrdr_kmin_b200 import scene as S
    reqs = [(0, S.Request(mode=S.MODE_XWAVE_SW, width=40, height=30, spp=64)),
            (0, S.Request(mode=S.MODE_IMAGE_CIE, width=20, height=20, spp=16))]
    smp = bench.sample_rows(reqs, 4)
    assert [(i, b, e) for i, b, e in smp] == [(0, 13 * 40, 17 * 40), (1, 8 * 20, 12 * 20)]
    assert bench.sample_realisations(reqs, smp) == 160 * 64 + 80 * 48
    rng = np.random.default_rng(1)

    def fake(mode, h, w):
        b = np.zeros((h, w), dtype=api.pixel_dtype(mode))
        keys = [("L", "L_se")] if mode == S.MODE_XWAVE_SW else [(c, c + "_se") for c in "XYZ"]
        for e, se in keys:
            b[e] = 1.0 + 0.1 * rng.standard_normal((h, w))
            b[se] = 0.1
        return b
    gpu = [fake(r.mode, r.height, r.width) for _, r in reqs]
    cpu = [fake(r.mode, r.height, r.width) for _, r in reqs]
    a = bench.agreement(reqs, smp, cpu, gpu)
    assert a["n"] == 160 + 3 * 80 and a["pixels"] == 240
    assert a["frac_abs_z_gt_3"] < 0.03 and abs(a["mean_z"]) < 0.3


def test_algorithmic_bytes_and_traffic_scaling():
    """The roofline's byte model: 16 B per node fetch, the grid bytes the
    device counted, 8 B per tentative collision, 32 B per realisation; the
    recorded DRAM traffic of each engine scales with those bytes."""
    import types
    import bench
    st = types.SimpleNamespace(nodes=3, grid_bytes=90, collisions=5, realisations=2)
    assert bench.alg_bytes_of(st) == 16 * 3 + 90 + 8 * 5 + 32 * 2
    for key in ("wavefront", "wavefront_lw"):
        t1, src = bench.traffic_per_launch(key, 1000)
        t2, _ = bench.traffic_per_launch(key, 2000)
        assert src and t1 > 1000 and abs(t2 - 2 * t1) < 1e-6 * t2
    assert bench.traffic_per_launch("no_such_kernel", 1000) == (None, None)
