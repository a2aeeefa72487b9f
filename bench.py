"""Benchmark of the B200 atmosphere path tracer (one JSON line on rank 0).

Workload: the longwave flux map -- 128 x 128 ground probes x 256
realisations, 16 bands x 8 correlated-k points, 50 gas layers with
per-layer k log-uniform in [1e-6, 1e2] 1/m, 64 x 64 x 32 lognormal cloud
repeated along X and Y, emissivity-0.95 ground (synthetic, seeded).  A step
is one htrdr_draw_map of that map.

* value: Mrealisations/s of the batched persistent kernel, output kept in
  HBM, scene (octrees) resident; device time from CUDA events recorded on the
  library's stream, max over ranks.
* e2e: the same through the C ABI with a pinned host buffer
  (htrdr_gpu_draw_map: request in, pixel buffer copied back), wall clock.
* --impl reference: the CPU restatement of the reference path (oracle,
  OpenMP over all host cores) on a bounded sample of the same map.

Multi-GPU (torchrun): every rank renders the whole map with its own random
streams (weak scaling) and the per-probe FP64 accumulators are summed on rank
0 with NCCL.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from htrdr_kmin_b200 import scene as S  # noqa: E402

METRIC = "Mrealisations/s at 3-sigma agreement, batched+served vs plain GPU; p50/p99 latency"
UNIT = "Mrealisations/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-sample-s", type=float, default=10.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload():
    return S.config_c2()


def cpu_baseline(scene, req, seconds: float):
    """The oracle (CPU restatement of the reference path, OpenMP over all host
    cores) on a bounded sample of the map: probe rows are added until the
    sample takes about `seconds`."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    os_ = O.OracleScene(scene, O.props_for_mode(req.mode))
    npix = req.width * req.height
    rows = 1
    done_real, spent = 0, 0.0
    begin = 0
    while spent < seconds and begin < npix:
        end = min(npix, begin + rows * req.width)
        t0 = time.perf_counter()
        _, cnt = os_.draw_map(req, begin, end, nthreads=cores)
        dt = time.perf_counter() - t0
        done_real += cnt["nreal"]
        spent += dt
        begin = end
        rows *= 2
    if begin >= npix and spent < seconds:
        pass
    os_.close()
    return {"value": done_real / spent / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done_real} realisations = the first {begin} of {npix} probes x {req.spp} "
                      f"in {spent:.1f} s (oracle, FP64, OpenMP)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    scene, req = workload()
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    os_ = O.OracleScene(scene, O.props_for_mode(req.mode))
    npix = req.width * req.height
    # each step: a bounded sample of probe rows sized to about 2 s
    t0 = time.perf_counter()
    _, cnt = os_.draw_map(req, 0, 8 * req.width, nthreads=cores)
    probe = time.perf_counter() - t0
    rows = max(1, min(req.height, int(8 * 2.0 / max(probe, 1e-3))))
    end = rows * req.width
    for _ in range(args.warmup):
        os_.draw_map(req, 0, min(end, 8 * req.width), nthreads=cores)
    times, reals = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, cnt = os_.draw_map(req, 0, end, nthreads=cores)
        times.append(time.perf_counter() - t0)
        reals += cnt["nreal"]
    total = sum(times)
    value = reals / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": "LW flux map 128x128 probes x 256 realisations, 16 bands x 8 quad, "
                               "cloud 64x64x32 repeated", "sample_probes": end},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"first {end} of {npix} probes x {req.spp} realisations per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from htrdr_kmin_b200 import api, build
    build.build()
    scene, req = workload()
    req.seed = 1000 + rank  # independent streams per rank (weak scaling)
    gs = api.GpuScene(scene, api.props_for_mode(req.mode), device=local)
    npix = req.width * req.height
    dt = api.pixel_dtype(req.mode)
    dev_out = torch.empty(npix * dt.itemsize, dtype=torch.uint8, device=f"cuda:{local}")
    host_out = torch.empty(npix * dt.itemsize, dtype=torch.uint8, pin_memory=True)

    r = api.to_request(req)
    lay = api.layout_for(req)
    L = api.lib()
    import ctypes as C

    def step_batched():
        """The batched persistent kernel, output left in HBM."""
        item = (api.BatchItem * 1)()
        item[0].scene = gs.handle.value
        item[0].req = r
        item[0].layout = lay
        item[0].buffer = dev_out.data_ptr()
        st = api.Stats()
        res = L.htrdr_gpu_draw_maps_batched_device(item, 1, None, C.byref(st))
        if res != 0:
            raise api.HtrdrError("draw_maps_batched_device", res)
        return st

    def step_device():
        st = api.Stats()
        res = L.htrdr_gpu_draw_map_device(gs.handle, C.byref(r), C.byref(lay),
                                          C.c_void_p(dev_out.data_ptr()), C.byref(st))
        if res != 0:
            raise api.HtrdrError("draw_map_device", res)
        return st

    def step_host():
        st = api.Stats()
        res = L.htrdr_gpu_draw_map(gs.handle, C.byref(r), C.byref(lay),
                                   C.c_void_p(host_out.data_ptr()), C.byref(st))
        if res != 0:
            raise api.HtrdrError("draw_map", res)
        return st

    def reduce_accumulators():
        if dist is None:
            return 0.0
        words = dev_out.view(torch.float64).view(npix, 8)
        f = words[:, [0, 1, 4, 5]].contiguous()
        u = dev_out.view(torch.int64).view(npix, 8)[:, [2, 3, 6, 7]].contiguous()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dist.reduce(f, dst=0, op=dist.ReduceOp.SUM)
        dist.reduce(u, dst=0, op=dist.ReduceOp.SUM)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # the plain drop-in kernel on the same map (reported beside the batched one)
    for _ in range(args.warmup):
        step_batched()
        step_device()
        reduce_accumulators()
    barrier()
    ms_plain = [step_device().kernel_ms for _ in range(max(1, args.steps))]

    barrier()
    kernel_ms, total_ms, stats = [], [], []
    with ClockSampler(local) as clk:
        barrier()
        for _ in range(args.steps):
            st = step_batched()
            red = reduce_accumulators()
            kernel_ms.append(st.kernel_ms)
            total_ms.append(st.total_ms + red)
            stats.append(st)
        barrier()
    clocks = clk.summary()

    # end-to-end through the C ABI with a pinned host buffer (wall clock)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_host()
    barrier()
    e2e_ms = 1e3 * (time.perf_counter() - t0) / args.steps

    step_ms = float(np.sum(total_ms)) / args.steps
    if dist is not None:
        t = torch.tensor([step_ms, e2e_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms, e2e_ms = float(t[0]), float(t[1])

    reals = stats[-1].realisations
    value = world * reals / (step_ms * 1e-3) / 1e6
    e2e_value = world * reals / (e2e_ms * 1e-3) / 1e6
    last = stats[-1]
    kms = float(np.mean(kernel_ms))
    alg_bytes = 16 * last.nodes + 8 * last.collisions + 32 * last.realisations
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kms * 1e-3) / 1e9
    plain_value = reals / (np.mean(ms_plain) * 1e-3) / 1e6

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(scene, req, args.cpu_sample_s)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene and probes)",
            "config": {"workload": "LW flux map 128x128 probes x 256 realisations/probe, 16 bands x 8 "
                                   "quad, 50 layers, cloud 64x64x32 repeated, batched persistent kernel",
                       "realisations_per_step_per_gpu": int(reals),
                       "l2": f"inputs larger than L2: scene {gs.device_bytes / 1e6:.0f} MB resident",
                       "parallelism": f"replicated scene, ranks render independent streams, NCCL sum of "
                                      f"FP64 accumulators" if world > 1 else "single GPU"},
            "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(C.sizeof(r) + C.sizeof(lay)),
                    "d2h_bytes_per_step": int(npix * dt.itemsize)},
            "gpu_launches": 2 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_kind": peak_kind, "kernel": "k_persistent",
                         "alg_bytes_per_launch": int(alg_bytes), "kernel_ms": kms},
            "cpu_baseline": cpu,
            "plain_gpu": {"value": plain_value, "unit": UNIT, "kernel": "k_plain",
                          "kernel_ms": float(np.mean(ms_plain))},
            "segments_per_s": last.segments / (kms * 1e-3),
            "counters": {"segments": last.segments, "nodes": last.nodes,
                         "collisions": last.collisions, "realisations": last.realisations,
                         "failures": last.failures},
        }
        print(json.dumps(line), flush=True)
    gs.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
