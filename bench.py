"""Benchmark of the B200 atmosphere path tracer (one JSON line on rank 0).

Default workload (``--workload lw_flux``): the longwave flux map -- 128 x 128
ground probes x 256 realisations, 16 bands x 8 correlated-k points, 50 gas
layers with per-layer k log-uniform in [1e-6, 1e2] 1/m, 64 x 64 x 32
lognormal cloud repeated along X and Y, emissivity-0.95 ground (synthetic,
seeded).  A step is one htrdr_draw_map of that map.

* value: Mrealisations/s of the work-queue engine the autotuner picks
  (persistent megakernel or wavefront), output kept in HBM, scene (octrees)
  resident; device time from CUDA events recorded on the library's stream,
  max over ranks.
* e2e: the same through the C ABI with a pinned host buffer
  (htrdr_gpu_draw_map with the same engine and tuning; request in, pixel
  buffer copied back), wall clock.
* plain_gpu: the plain one-thread-per-realisation engine of the drop-in
  (htrdr_gpu_draw_map_device with HTRDR_GPU_ENGINE_PLAIN) on the same work.
* --impl reference: the CPU restatement of the reference path (oracle,
  OpenMP over all host cores) on a bounded sample of the same map.

Other workloads (development and profiling): ``sw_image`` (SW image 64x64 x 32
spp, one band at 550 nm, 32x32x16 cloud), ``cie_image`` (CIE image 256x256 x
16 spp x 3 channels, 30 bands x 16 points, 128x128x32 power-law cloud) and
``mix`` (64 uneven SW/LW image requests on three scenes in one launch, against
the same requests one at a time on the plain kernel).

Multi-GPU (torchrun): every rank renders the whole map with its own random
streams (weak scaling) and, for flux maps, the per-probe FP64 accumulators are
summed on rank 0 with NCCL.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
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
    p.add_argument("--workload", default="lw_flux",
                   choices=["lw_flux", "sw_image", "sw_large", "cie_image", "cie_full", "mix", "serve"])
    p.add_argument("--rates", default="", help="serve: comma-separated arrival rates (requests/s)")
    p.add_argument("--tuning", default="",
                   help="block,chunk,period[,engine[,budget[,slots[,tail]]]] instead of the autotuner "
                        "(engine 0 persistent, 2 wavefront)")
    p.add_argument("--cpu-sample-s", type=float, default=10.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def parse_tuning(api, text: str):
    """block,chunk,period[,engine[,budget[,slots[,tail]]]] -> Tuning"""
    t = api.default_tuning()
    v = [int(x) for x in text.split(",")]
    t.block_size, t.queue_chunk, t.regroup_period = v[:3]
    if len(v) > 3:
        t.engine = v[3]
    if len(v) > 4:
        t.trace_budget = v[4]
    if len(v) > 5:
        t.wave_slots = v[5]
    if len(v) > 6:
        t.wave_tail = v[6]
    return t


def tuning_dict(t, source: str) -> dict:
    d = {"engine": {0: "persistent", 2: "wavefront"}.get(t.engine, str(t.engine)),
         "block_size": t.block_size}
    if t.engine == 2:
        d.update(trace_budget=t.trace_budget or 256, wave_slots=t.wave_slots or "auto",
                 wave_tail=t.wave_tail or "auto", tail_regroup_period=t.regroup_period)
    else:
        d.update(queue_chunk=t.queue_chunk, regroup_period=t.regroup_period)
    d["from"] = source
    return d


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
    """SM clocks and throttle reasons sampled during the timed region: a
    thread reading NVML every 5 ms (the timed region of a few steps lasts tens
    of milliseconds) and nvidia-smi every 100 ms.  Read-only queries; nothing
    about the GPU's settings is changed.  `window_ms' is the wall time the
    samples cover."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None
        self.nvml = None          # (module, handle) when NVML answers
        self.nvml_samples = []    # (sm MHz, reasons bitmask)
        self.nvml_max = None
        self._stop = threading.Event()
        self._thread = None
        self.window = [0.0, 0.0]

    def _nvml_open(self):
        try:
            import pynvml as N
            import torch
            N.nvmlInit()
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            try:
                h = N.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                h = N.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml_max = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            self.nvml = (N, h)
        except Exception:
            self.nvml = None

    def _nvml_loop(self):
        N, h = self.nvml
        reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(N, "nvmlDeviceGetCurrentClocksThrottleReasons")
        while not self._stop.is_set():
            try:
                self.nvml_samples.append((float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)),
                                          int(reasons(h))))
            except Exception:
                return
            time.sleep(0.005)

    def __enter__(self):
        self._nvml_open()
        self.window[0] = time.perf_counter()
        if self.nvml is not None:
            self._thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self._thread.start()
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
        self.window[1] = time.perf_counter()
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=5)
        if self.nvml is not None:
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def _nvml_reason_names(self, mask: int):
        N = self.nvml[0]
        bits = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
                "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
                "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
                "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}
        return {nm for nm, attr in bits.items() if mask & int(getattr(N, attr, 0))}

    def summary(self):
        sm, smax, reasons = [], None, set()
        if self.nvml is not None:
            for mhz, mask in self.nvml_samples:
                sm.append(mhz)
                reasons |= self._nvml_reason_names(mask)
            smax = self.nvml_max
        if self.proc is not None and self.path:
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
                    for nm, v in zip(self.REASONS, parts[5:9]):
                        if v.lower().startswith("active"):
                            reasons.add(nm)
            os.unlink(self.path)
        if not sm and smax is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "window_ms": 1e3 * (self.window[1] - self.window[0])}


def workload(name: str):
    """List of (scene index, request) and the scenes, plus a description."""
    if name == "lw_flux":
        sc, rq = S.config_c2()
        return [sc], [(0, rq)], ("LW flux map 128x128 probes x 256 realisations/probe, 16 bands x 8 "
                                 "quad, 50 layers, cloud 64x64x32 repeated")
    if name == "sw_image":
        sc, rq = S.config_c1()
        return [sc], [(0, rq)], ("SW image 64x64 x 32 spp, 1 band at 550 nm, 50 layers, cloud "
                                 "32x32x16 lognormal")
    if name == "sw_large":
        sc, rq = S.config_c1(scale=192 / 64)
        return [sc], [(0, rq)], ("SW image 192x192 x 32 spp, 1 band at 550 nm, 50 layers, cloud "
                                 "32x32x16 lognormal (SW config at 3x side: throughput-bound)")
    if name == "cie_image":
        sc, rq = S.config_c3(scale=256 / 512, spp=16, cloud_def=(128, 128, 32))
        return [sc], [(0, rq)], ("CIE image 256x256 x 16 spp x 3 channels, 30 bands x 16 quad, cloud "
                                 "128x128x32 power-law (CIE config at 1/2 side, 1/4 spp, 1/8 cloud)")
    if name == "cie_full":
        sc, rq = S.config_c3()
        return [sc], [(0, rq)], ("CIE image 512x512 x 64 spp x 3 channels, 30 bands x 16 quad, cloud "
                                 "256x256x64 power-law of 50 m cells")
    scenes = S.batched_scenes(scale=0.25)
    reqs = S.batched_requests(n=64, side_range=(16, 96), spp_range=(16, 128))
    return scenes, reqs, ("64 uneven requests (side log-U[16,96], spp log-U[16,128], 50% SW / 50% LW "
                          "images) on 3 cloud scenes (32^3, 64x64x16, 128x128x32) in one launch")


def cpu_baseline(scenes, reqs, seconds: float):
    """The oracle (CPU restatement of the reference path, OpenMP over all host
    cores) on a bounded sample of the workload: pixel rows of the first request
    are added until the sample takes about `seconds`."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    isc, req = reqs[0]
    os_ = O.OracleScene(scenes[isc], O.props_for_mode(req.mode))
    npix = req.width * req.height
    rows, begin, done_real, spent, rounds = 1, 0, 0, 0.0, 0
    while spent < seconds and rounds < 64:
        end = min(npix, begin + rows * req.width)
        t0 = time.perf_counter()
        _, cnt = os_.draw_map(req, begin, end, nthreads=cores)
        spent += time.perf_counter() - t0
        done_real += cnt["nreal"]
        begin = 0 if end >= npix else end
        rows *= 2
        rounds += 1
    os_.close()
    return {"value": done_real / spent / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{done_real} realisations of the first request's pixels, in {spent:.1f} s "
                      f"(oracle, FP64 transport, OpenMP)"}


def run_reference(args):
    rank, _, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    scenes, reqs, desc = workload(args.workload)
    isc, req = reqs[0]
    cores = os.cpu_count() or 1
    os_ = O.OracleScene(scenes[isc], O.props_for_mode(req.mode))
    npix = req.width * req.height
    t0 = time.perf_counter()
    os_.draw_map(req, 0, min(npix, 8 * req.width), nthreads=cores)
    probe = max(time.perf_counter() - t0, 1e-3)
    rows = max(1, min(req.height, int(8 * 2.0 / probe)))  # each step ~2 s of CPU work
    end = min(npix, rows * req.width)
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
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": desc, "sample_pixels_per_step": end},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"first {end} of {npix} pixels x {req.realisations_per_pixel} "
                                   f"realisations per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def _percentile(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(round(q * (len(v) - 1))))] if v else None


def run_serve(args):
    """Serving: Poisson arrivals of the uneven request mix at swept rates.

    For each rate the same arrival trace is served (a) by the request loop
    with continuous batching (htrdr_gpu_server_*) and (b) one request at a
    time, in arrival order, by the plain engine of the drop-in
    (htrdr_gpu_draw_map with HTRDR_GPU_ENGINE_PLAIN).
    Latency = arrival -> map in the host buffer.  Throughput = realisations /
    (first arrival -> last completion)."""
    import threading
    import torch
    from htrdr_kmin_b200 import api, build
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    build.build()
    scenes, reqs, desc = workload("mix")
    need = [0] * len(scenes)
    for isc, r in reqs:
        need[isc] |= api.props_for_mode(r.mode)
    gss = [api.GpuScene(s, need[i], device=local) for i, s in enumerate(scenes)]
    items = [(gss[isc], r) for isc, r in reqs]
    total_real = sum(r.realisations for _, r in reqs)
    # warm-up: samplers, kernels
    for gs, r in items:
        gs.draw_map(S.Request(**{**r.__dict__, "spp": 1}))
    # tuning of the batched kernel on the whole mix (untimed)
    dev = [torch.empty(r.width * r.height * api.pixel_dtype(r.mode).itemsize, dtype=torch.uint8,
                       device=f"cuda:{local}") for _, r in items]
    arr = (api.BatchItem * len(items))()
    for i, (gs, r) in enumerate(items):
        arr[i].scene, arr[i].req, arr[i].layout = gs.handle.value, api.to_request(r), api.layout_for(r)
        arr[i].buffer = dev[i].data_ptr()
    tuning, batched_ms = api.autotune(arr)  # the server runs the engine that wins
    for g in gss:  # the one-at-a-time arm runs the plain engine of the drop-in
        g.set_engine(api.ENGINE_PLAIN)
    plain_one = []
    for gs, r in items:
        _, st = gs.draw_map(r)
        plain_one.append(st["total_ms"])
    rates = [float(x) for x in args.rates.split(",")] if args.rates else None
    if not rates:
        capacity = len(items) / (sum(plain_one) * 1e-3)  # plain, one at a time, requests/s
        # from below the plain path's capacity to well above the batched engine's
        rates = [f * capacity for f in (0.5, 1.0, 2.0, 4.0, 8.0, 16.0)]
    rng = np.random.default_rng(5)
    sweep = []
    for rate in rates:
        gaps = rng.exponential(1.0 / rate, size=len(items))
        arrivals = np.cumsum(gaps) - gaps[0]
        # (a) continuous batching server
        srv = api.Server(device=local, hbm_budget_bytes=150 << 30, round_target_ms=30.0,
                         tuning=tuning)
        tickets, t_sub = [None] * len(items), [0.0] * len(items)
        t0 = time.perf_counter()

        def submitter():
            for i, (gs, r) in enumerate(items):
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                t_sub[i] = time.perf_counter()
                tickets[i] = srv.submit(gs, r)

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
        srv.close()
        # (b) one at a time on the plain kernel, same arrivals
        lat, t0 = [], time.perf_counter()
        t_free = 0.0
        for i, (gs, r) in enumerate(items):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            gs.draw_map(r)
            lat.append(1e3 * (time.perf_counter() - (t0 + arrivals[i])))
        fifo_wall = time.perf_counter() - t0
        sweep.append({
            "rate_req_s": rate,
            "served": {"Mreal_s": total_real / (st["wall_ms"] * 1e-3) / 1e6, "p50_ms": st["p50_ms"],
                       "p99_ms": st["p99_ms"], "rounds": st["rounds"], "busy_ms": st["busy_ms"],
                       "wall_ms": st["wall_ms"], "hbm_peak_MB": st["hbm_peak_bytes"] / 1e6},
            "plain_one_at_a_time": {"Mreal_s": total_real / fifo_wall / 1e6,
                                    "p50_ms": _percentile(lat, 0.5), "p99_ms": _percentile(lat, 0.99)},
        })
    best = max(sweep, key=lambda s: s["served"]["Mreal_s"])
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": best["served"]["Mreal_s"], "unit": UNIT, "n_gpus": 1,
            "steps": len(rates), "warmup": 1, "ms_per_step": best["served"]["wall_ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes and sensors), Poisson arrivals",
            "config": {"workload": "serving: " + desc, "rates_req_s": rates,
                       "hbm_budget_GB": 150, "tuning": tuning_dict(tuning, "autotuner / mode default")},
            "serving": sweep,
            "batched_one_launch_Mreal_s": total_real / (batched_ms * 1e-3) / 1e6,
            "plain_sequential_Mreal_s": total_real / (sum(plain_one) * 1e-3) / 1e6,
        }), flush=True)
    for g in gss:
        g.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "serve":
        run_serve(args)
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
    L = api.lib()
    scenes, reqs, desc = workload(args.workload)
    from htrdr_kmin_b200 import multigpu as M
    for _, r in reqs:
        r.seed = M.rank_seed(r.seed, rank)  # independent streams per rank (weak scaling)
    need = [0] * len(scenes)
    for isc, r in reqs:
        need[isc] |= api.props_for_mode(r.mode)
    gss = [api.GpuScene(s, need[i], device=local) for i, s in enumerate(scenes)]
    n = len(reqs)
    dev = [torch.empty(r.width * r.height * api.pixel_dtype(r.mode).itemsize, dtype=torch.uint8,
                       device=f"cuda:{local}") for _, r in reqs]
    host = [torch.empty(d.numel(), dtype=torch.uint8, pin_memory=True) for d in dev]
    creq = [api.to_request(r) for _, r in reqs]
    clay = [api.layout_for(r) for _, r in reqs]
    items_dev = (api.BatchItem * n)()
    items_host = (api.BatchItem * n)()
    for i, (isc, _) in enumerate(reqs):
        for arr, buf in ((items_dev, dev[i].data_ptr()), (items_host, host[i].data_ptr())):
            arr[i].scene = gss[isc].handle.value
            arr[i].req = creq[i]
            arr[i].layout = clay[i]
            arr[i].buffer = buf
    total_real = sum(r.realisations for _, r in reqs)

    def check(res, what):
        if res != 0:
            raise api.HtrdrError(what, res, L.htrdr_gpu_last_error().decode())

    # engine, block size, queue chunk, regroup period, step budget from the
    # autotuner (untimed)
    if args.tuning:
        tuning = parse_tuning(api, args.tuning)
    else:
        tuning, _ = api.autotune(items_dev)
    for g in gss:  # the drop-in draw_map (e2e) runs the same engine and tuning
        g.set_engine(tuning.engine, tuning)

    def step_batched():
        """all requests in one launch of the work-queue engine, outputs left in HBM"""
        st = api.Stats()
        check(L.htrdr_gpu_draw_maps_batched_device(items_dev, n, C.byref(tuning), C.byref(st)),
              "batched_device")
        return st

    def step_plain():
        """the plain engine of the drop-in, one launch per request"""
        k = 0.0
        for isc, _ in reqs:
            gss[isc].set_engine(api.ENGINE_PLAIN)
        for i, (isc, _) in enumerate(reqs):
            st = api.Stats()
            check(L.htrdr_gpu_draw_map_device(gss[isc].handle, C.byref(creq[i]), C.byref(clay[i]),
                                              C.c_void_p(dev[i].data_ptr()), C.byref(st)), "draw_map_device")
            k += st.kernel_ms
        for isc, _ in reqs:
            gss[isc].set_engine(tuning.engine, tuning)
        return k

    def step_e2e():
        """through the C ABI into pinned host buffers"""
        if n == 1:
            st = api.Stats()
            check(L.htrdr_gpu_draw_map(gss[reqs[0][0]].handle, C.byref(creq[0]), C.byref(clay[0]),
                                       C.c_void_p(host[0].data_ptr()), C.byref(st)), "draw_map")
        else:
            st = api.Stats()
            check(L.htrdr_gpu_draw_maps_batched(items_host, n, C.byref(tuning), C.byref(st)), "batched")

    flux = [i for i, (_, r) in enumerate(reqs) if r.mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW)]

    def reduce_accumulators():
        """NCCL sum of the flux maps' FP64 accumulators on rank 0"""
        if dist is None or not flux:
            return 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in flux:
            M.reduce_flux_map(dev[i], dist, dst=0)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step_batched()
        reduce_accumulators()
    step_plain()
    barrier()
    plain_ms = step_plain()

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

    step_e2e()  # untimed: the first host-buffer call sizes the library's staging buffer
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    barrier()
    e2e_ms = 1e3 * (time.perf_counter() - t0) / args.steps

    step_ms = float(np.sum(total_ms)) / args.steps
    if dist is not None:
        t = torch.tensor([step_ms, e2e_ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms, e2e_ms = float(t[0]), float(t[1])

    last = stats[-1]
    wave = tuning.engine == api.ENGINE_WAVEFRONT
    reals = last.realisations
    value = world * reals / (step_ms * 1e-3) / 1e6
    kms = float(np.mean(kernel_ms))
    alg_bytes = 16 * last.nodes + 8 * last.collisions + 32 * last.realisations
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kms * 1e-3) / 1e9
    out_bytes = sum(d.numel() for d in dev)

    if rank == 0:
        cpu = None if args.no_cpu_baseline else cpu_baseline(scenes, reqs, args.cpu_sample_s)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes and sensors)",
            "config": {"workload": desc + (", wavefront engine" if wave else ", batched persistent kernel"),
                       "realisations_per_step_per_gpu": int(total_real),
                       "tuning": tuning_dict(tuning, "command line" if args.tuning else "autotuner"),
                       "l2": "inputs larger than L2: scenes of "
                             f"{sum(g.device_bytes for g in gss) / 1e6:.0f} MB resident",
                       "parallelism": ("replicated scene, independent streams per rank, NCCL sum of FP64 "
                                       "accumulators") if world > 1 else "single GPU"},
            "clocks": clocks,
            "e2e": {"value": world * reals / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": int(n * (C.sizeof(api.Request) + C.sizeof(api.BufferLayout))),
                    "d2h_bytes_per_step": int(out_bytes)},
            "gpu_launches": int(sum(s.launches for s in stats)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "k_wave_event + k_wave_trace" if wave else "k_persistent",
                         "alg_bytes_per_launch": int(alg_bytes), "kernel_ms": kms},
            "cpu_baseline": cpu,
            "plain_gpu": {"value": reals / (plain_ms * 1e-3) / 1e6, "unit": UNIT, "kernel": "k_plain",
                          "kernel_ms": plain_ms, "launches": n},
            "batched_vs_plain": plain_ms / kms,
            "segments_per_s": last.segments / (kms * 1e-3),
            "counters": {"segments": last.segments, "nodes": last.nodes,
                         "collisions": last.collisions, "realisations": last.realisations,
                         "failures": last.failures},
        }
        print(json.dumps(line), flush=True)
    for g in gss:
        g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
