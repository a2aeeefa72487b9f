"""Benchmark of the B200 atmosphere path tracer (one JSON line on rank 0).

Default workload (``--workload mix_full``), the batched configuration the
metric names: 64 uneven image requests -- side log-uniform in [16, 64] px,
16 to 64 realisations per pixel log-uniform, 50 % shortwave / 50 % longwave
-- each on one of three full-size seeded cloud scenes (128^3, 256x256x64 and
512x512x128 cells of 50 m, 8 bands x 4 quadrature points, 50 gas layers);
the request sizes are reduced from log-U[32,1024] px and [16,1024]
realisations so that one step takes seconds (at full ranges one request holds
up to 10^9 realisations).  A step renders the whole mix.

* value: Mrealisations/s of the mix rendered in one launch of the work-queue
  engine the autotuner picks (its wavefront tail threshold timed on the full
  mix), outputs in HBM, scenes resident; the K steps timed between two CUDA
  events that bracket them (the host's share of each call included), max
  over ranks.
* plain_gpu / batched_vs_plain: the same requests one at a time through the
  plain engine of the drop-in (one thread per realisation).
* serving: the same requests arriving as a Poisson process at a rate that
  saturates the GPU, served by the request loop with continuous batching
  (htrdr_gpu_server_*), against the same arrivals rendered one at a time by
  the plain drop-in: throughput and p50/p99 latency (arrival -> map in the
  host buffer).
* e2e: the batched call through the C ABI with pinned host buffers
  (htrdr_gpu_draw_maps_batched), wall clock.
* agreement: the oracle's estimates of a sample of pixels against the GPU's
  estimates of the same pixels in the timed step (independent streams): the
  fraction of |z| > 3 and the mean z.
* lw_flux: the longwave flux map (128 x 128 probes x 256 realisations,
  16 bands x 8 points, 64 x 64 x 32 repeated cloud) on its default engine,
  with its plain arm.
* --impl reference: the reference's own CPU code for the path (its hot-path C
  files compiled unmodified, oracle/_ref; the oracle port where that library
  is absent), OpenMP over all host cores, on a bounded sample of the same
  workload.

Other workloads (development and profiling): ``lw_flux``, ``sw_image``,
``sw_large``, ``cie_image``, ``cie_full``, ``mix`` (the mix on scenes at 1/4
scale) and ``serve`` (a sweep of arrival rates on that mix).

Multi-GPU (torchrun): every rank renders the whole workload with its own
random streams (weak scaling); every map's FP64 accumulators are summed on
rank 0 with NCCL and finalized there.
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
    p.add_argument("--workload", default="mix_full",
                   choices=["mix_full", "lw_flux", "sw_image", "sw_large", "cie_image", "cie_full",
                            "mix", "serve"])
    p.add_argument("--mix-side", default="16,64", help="mix_full: request side range (px)")
    p.add_argument("--mix-spp", default="16,64", help="mix_full: realisations per pixel range")
    p.add_argument("--no-secondary", action="store_true", help="mix_full: skip the LW flux map")
    p.add_argument("--profile-once", action="store_true",
                   help="one batched launch of the workload with --tuning, then its counters (for ncu)")
    p.add_argument("--rates", default="", help="serve: comma-separated arrival rates (requests/s)")
    p.add_argument("--tuning", default="",
                   help="block,chunk,period[,engine[,budget[,slots[,tail]]]] instead of the autotuner "
                        "(engine 0 persistent, 2 wavefront, 3 sorted)")
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
    d = {"engine": {0: "persistent", 2: "wavefront", 3: "sorted"}.get(t.engine, str(t.engine)),
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


def _range(text: str):
    a, b = (int(x) for x in text.split(","))
    return a, b


def workload(name: str, args=None):
    """Scenes, list of (scene index, request) and a description."""
    if name == "mix_full":
        side = _range(args.mix_side) if args is not None else (16, 64)
        spp = _range(args.mix_spp) if args is not None else (16, 64)
        scenes = S.batched_scenes(scale=1.0)
        reqs = S.batched_requests(n=64, side_range=side, spp_range=spp)
        return scenes, reqs, (
            f"64 uneven requests (side log-U[{side[0]},{side[1]}] px, spp log-U[{spp[0]},{spp[1]}], "
            "50% SW / 50% LW images; sizes reduced from log-U[32,1024] px and [16,1024] spp) on 3 "
            "full-size cloud scenes (128^3, 256x256x64, 512x512x128 cells of 50 m; 8 bands x 4 quad, "
            "50 layers)")
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


def sample_rows(reqs, nrows: int):
    """Bounded sample of a workload: `nrows' pixel rows from the middle of
    every request, as (request index, first pixel, end pixel)."""
    out = []
    for i, (_, r) in enumerate(reqs):
        y0 = max(0, r.height // 2 - nrows // 2)
        y1 = min(r.height, y0 + nrows)
        out.append((i, y0 * r.width, y1 * r.width))
    return out


def sample_realisations(reqs, sample) -> int:
    return sum((e - b) * reqs[i][1].realisations_per_pixel for i, b, e in sample)


class CpuPath:
    """The CPU implementation timed beside the GPU: the reference's own
    hot-path files compiled unmodified (oracle/_ref) when built, else the
    oracle port; OpenMP over all host cores.  Only the reference arm and the
    CPU baseline leg use it."""

    def __init__(self, scenes, reqs, prefer_reference: bool = True):
        from oracle import oracle as O
        self.kind = "port"
        R = None
        if prefer_reference:
            try:
                from oracle import reference as R
                if R.build() is None:
                    R = None
            except Exception:
                R = None
        need = [0] * len(scenes)
        for isc, r in reqs:
            need[isc] |= O.props_for_mode(r.mode)
        if R is not None:
            self.kind = "reference"
            self.objs = [R.RefScene(s, need[i]) for i, s in enumerate(scenes)]
        else:
            self.objs = [O.OracleScene(s, need[i]) for i, s in enumerate(scenes)]
        self.reqs = reqs
        self.cores = os.cpu_count() or 1

    def draw(self, i: int, begin: int, end: int, seed_offset: int = 0):
        isc, r = self.reqs[i]
        if seed_offset:
            r = S.Request(**{**r.__dict__, "seed": (r.seed + seed_offset) & 0xFFFFFFFF})
        out = self.objs[isc].draw_map(r, begin, end, nthreads=self.cores)
        return out[0] if isinstance(out, tuple) else out

    def run(self, sample, seed_offset: int = 0):
        return [self.draw(i, b, e, seed_offset) for i, b, e in sample]

    def close(self):
        for o in self.objs:
            o.close()


def estimates(buf, mode):
    """[(E, SE)] per channel of a pixel buffer (htrdr_accum_get_estimation)."""
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        n = buf["n"].astype(np.float64)
        E = buf["sum"] / np.maximum(n, 1)
        return [(E, np.sqrt(np.maximum(buf["sum2"] / np.maximum(n, 1) - E * E, 0) / np.maximum(n, 1)))]
    if mode == S.MODE_IMAGE_CIE:
        return [(buf[c], buf[c + "_se"]) for c in ("X", "Y", "Z")]
    return [(buf["L"], buf["L_se"])]


def agreement(reqs, sample, cpu_bufs, gpu_bufs) -> dict:
    """Per-pixel z = (E_gpu - E_cpu) / sqrt(SE_gpu^2 + SE_cpu^2) over the
    sampled pixels (independent streams on the two sides)."""
    zs = []
    for (i, b, e), cb in zip(sample, cpu_bufs):
        r = reqs[i][1]
        g = gpu_bufs[i].reshape(-1)[b:e]
        c = cb.reshape(-1)[b:e]
        for (Eg, SEg), (Ec, SEc) in zip(estimates(g, r.mode), estimates(c, r.mode)):
            s = np.sqrt(SEg ** 2 + SEc ** 2)
            m = s > 0
            zs.append((Eg[m] - Ec[m]) / s[m])
    z = np.concatenate(zs) if zs else np.zeros(0)
    return {"n": int(z.size), "frac_abs_z_gt_3": float(np.mean(np.abs(z) > 3)) if z.size else None,
            "mean_z": float(z.mean()) if z.size else None,
            "expected_frac": 0.0027, "pixels": int(sum(e - b for _, b, e in sample))}


def cpu_leg(scenes, reqs, seconds: float, gpu_bufs=None):
    """CPU baseline of the timed workload (rank 0, N=1) and, when the GPU
    maps are given, the per-pixel agreement of the GPU with the CPU path on
    the sampled pixels.  The sample grows (rows per request doubling) until
    the CPU work takes about `seconds'."""
    cpu = CpuPath(scenes, reqs)
    rows, spent, reals, sample, bufs = 1, 0.0, 0, [], []
    while True:
        smp = sample_rows(reqs, rows)
        t0 = time.perf_counter()
        bufs = cpu.run(smp, seed_offset=7919)  # streams independent of the GPU's
        dt = time.perf_counter() - t0
        spent, reals, sample = dt, sample_realisations(reqs, smp), smp
        if dt >= seconds * 0.4 or rows >= max(r.height for _, r in reqs):
            break
        rows *= 2
    out = {"value": reals / spent / 1e6, "unit": UNIT, "cores": cpu.cores, "kind": cpu.kind,
           "sample": f"{reals} realisations: {rows} middle pixel row(s) of each of the {len(reqs)} "
                     f"request(s), in {spent:.1f} s ("
                     + ("the reference's hot-path C files compiled unmodified" if cpu.kind == "reference"
                        else "the oracle port") + ", FP64 transport, OpenMP)"}
    agr = agreement(reqs, sample, bufs, gpu_bufs) if gpu_bufs is not None else None
    cpu.close()
    return out, agr


def run_reference(args):
    """The reference's CPU implementation of the path on a bounded sample of
    the workload per step (rank 0 only under torchrun)."""
    rank, _, _ = dist_env()
    if rank != 0:
        return
    scenes, reqs, desc = workload(args.workload, args)
    cpu = CpuPath(scenes, reqs)
    rows = 1
    t0 = time.perf_counter()
    cpu.run(sample_rows(reqs, rows))
    probe = max(time.perf_counter() - t0, 1e-3)
    # each step ~2 s of CPU work
    rows = max(1, min(max(r.height for _, r in reqs), int(rows * 2.0 / probe)))
    smp = sample_rows(reqs, rows)
    per_step = sample_realisations(reqs, smp)
    for _ in range(args.warmup):
        cpu.run(sample_rows(reqs, 1))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cpu.run(smp)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = per_step * args.steps / total / 1e6
    what = ("the reference's hot-path C files compiled unmodified" if cpu.kind == "reference"
            else "the oracle port")
    cpu.close()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded scenes and sensors)",
        "config": {"workload": desc, "sample_realisations_per_step": per_step},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cpu.cores, "kind": cpu.kind,
                         "sample": f"{rows} middle pixel row(s) of each of the {len(reqs)} request(s) "
                                   f"per step, {per_step} realisations ({what}, OpenMP)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def _percentile(v, q):
    v = sorted(v)
    return v[min(len(v) - 1, int(round(q * (len(v) - 1))))] if v else None


def serve_arrivals(api, items, tuning, arrivals, local: int) -> dict:
    """The request loop with continuous batching fed the requests at the
    given arrival times (s from the first); latency = submit -> map in the
    host buffer."""
    srv = api.Server(device=local, hbm_budget_bytes=150 << 30, round_target_ms=30.0, tuning=tuning)
    tickets = [None] * len(items)
    t0 = time.perf_counter()

    def submitter():
        for i, (gs, r) in enumerate(items):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = srv.submit(gs, r)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    srv.close()
    total = sum(r.realisations for _, r in items)
    return {"Mreal_s": total / (st["wall_ms"] * 1e-3) / 1e6, "p50_ms": st["p50_ms"],
            "p99_ms": st["p99_ms"], "rounds": st["rounds"], "wall_ms": st["wall_ms"],
            "hbm_peak_MB": st["hbm_peak_bytes"] / 1e6}


def plain_arrivals(api, items, arrivals) -> dict:
    """The same arrivals rendered one at a time, in arrival order, by the
    plain engine of the drop-in (htrdr_gpu_draw_map, host buffers)."""
    for gs, _ in items:
        gs.set_engine(api.ENGINE_PLAIN)
    lat, t0 = [], time.perf_counter()
    for i, (gs, r) in enumerate(items):
        d = t0 + arrivals[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        gs.draw_map(r)
        lat.append(1e3 * (time.perf_counter() - (t0 + arrivals[i])))
    wall = time.perf_counter() - t0
    total = sum(r.realisations for _, r in items)
    return {"Mreal_s": total / wall / 1e6, "p50_ms": _percentile(lat, 0.5),
            "p99_ms": _percentile(lat, 0.99), "wall_ms": 1e3 * wall}


def run_serve(args):
    """Serving sweep: Poisson arrivals of the uneven request mix at swept
    rates, each served (a) by the request loop with continuous batching and
    (b) one request at a time by the plain engine of the drop-in."""
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
    for gs, r in items:  # warm-up: samplers, kernels
        gs.draw_map(S.Request(**{**r.__dict__, "spp": 1}))
    dev = [torch.empty(r.width * r.height * api.pixel_dtype(r.mode).itemsize, dtype=torch.uint8,
                       device=f"cuda:{local}") for _, r in items]
    arr = (api.BatchItem * len(items))()
    for i, (gs, r) in enumerate(items):
        arr[i].scene, arr[i].req, arr[i].layout = gs.handle.value, api.to_request(r), api.layout_for(r)
        arr[i].buffer = dev[i].data_ptr()
    tuning, batched_ms = api.autotune(arr)  # the server runs the engine that wins
    for g in gss:
        g.set_engine(api.ENGINE_PLAIN)
    plain_one = [gs.draw_map(r)[1]["total_ms"] for gs, r in items]
    rates = [float(x) for x in args.rates.split(",")] if args.rates else None
    if not rates:
        capacity = len(items) / (sum(plain_one) * 1e-3)  # plain, one at a time, requests/s
        rates = [f * capacity for f in (0.5, 1.0, 2.0, 4.0, 8.0, 16.0)]
    rng = np.random.default_rng(5)
    sweep = []
    for rate in rates:
        gaps = rng.exponential(1.0 / rate, size=len(items))
        arrivals = np.cumsum(gaps) - gaps[0]
        served = serve_arrivals(api, items, tuning, arrivals, local)
        sweep.append({"rate_req_s": rate, "served": served,
                      "plain_one_at_a_time": plain_arrivals(api, items, arrivals)})
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


def alg_bytes_of(st) -> int:
    """Algorithmic bytes of a launch from its counters: 16 per majorant node
    fetched, the leaf-grid bytes read (9 per majorant-grid lookup, 4 per
    node-grid lookup), 8 per tentative collision (its raw-property gather:
    cloud cell and gas layer) and 32 per realisation (the read-modify-write
    of its FP64 sums and count)."""
    return 16 * st.nodes + st.grid_bytes + 8 * st.collisions + 32 * st.realisations


def traffic_per_launch(kernel: str, alg_bytes: int):
    """DRAM bytes of one launch of `kernel', from the ncu capture summarised
    in profiles/traffic.json: dram__bytes_read.sum + dram__bytes_write.sum of
    a smaller case of the same engine, scaled to this launch by the ratio of
    algorithmic bytes.  (None, None) when no capture of it is recorded."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f).get(kernel)
    except Exception:
        return None, None
    if not d or not d.get("alg_bytes"):
        return None, None
    return float(d["dram_bytes"]) / float(d["alg_bytes"]) * alg_bytes, d.get("source")


class Setup:
    """Scenes resident on one device, the requests' device and pinned host
    output buffers and their C descriptions."""

    def __init__(self, api, scenes, reqs, local: int):
        import torch
        self.api, self.reqs, self.local = api, reqs, local
        need = [0] * len(scenes)
        for isc, r in reqs:
            need[isc] |= api.props_for_mode(r.mode)
        t0 = time.perf_counter()
        self.gss = [api.GpuScene(s, need[i], device=local) for i, s in enumerate(scenes)]
        torch.cuda.synchronize()
        self.build_s = time.perf_counter() - t0
        n = self.n = len(reqs)
        self.dev = [torch.empty(r.width * r.height * api.pixel_dtype(r.mode).itemsize, dtype=torch.uint8,
                                device=f"cuda:{local}") for _, r in reqs]
        self.host = [torch.empty(d.numel(), dtype=torch.uint8, pin_memory=True) for d in self.dev]
        self.creq = [api.to_request(r) for _, r in reqs]
        self.clay = [api.layout_for(r) for _, r in reqs]
        self.items_dev = (api.BatchItem * n)()
        self.items_host = (api.BatchItem * n)()
        for i, (isc, _) in enumerate(reqs):
            for arr, buf in ((self.items_dev, self.dev[i].data_ptr()), (self.items_host, self.host[i].data_ptr())):
                arr[i].scene = self.gss[isc].handle.value
                arr[i].req = self.creq[i]
                arr[i].layout = self.clay[i]
                arr[i].buffer = buf
        self.total_real = sum(r.realisations for _, r in reqs)
        self.items = [(self.gss[isc], r) for isc, r in reqs]
        # FP64 accumulators of every request in one device buffer, for the
        # multi-GPU combination (sum over ranks, finalize once)
        sizes = [api.accum_records(r) * 32 for _, r in reqs]
        self.acc_off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.acc = None
        self.items_acc = None
        self._acc_sizes = sizes

    def enable_accumulators(self):
        import torch
        api = self.api
        self.acc = torch.zeros(int(self.acc_off[-1]), dtype=torch.uint8, device=f"cuda:{self.local}")
        self.items_acc = (api.BatchItem * self.n)()
        for i, (isc, _) in enumerate(self.reqs):
            self.items_acc[i].scene = self.gss[isc].handle.value
            self.items_acc[i].req = self.creq[i]
            self.items_acc[i].layout = self.clay[i]
            self.items_acc[i].buffer = self.acc.data_ptr() + int(self.acc_off[i])

    def reduced_items(self, factor: int):
        """The same requests with 1/factor of the realisations per pixel
        (for the autotuner), on the same device buffers."""
        api = self.api
        arr = (api.BatchItem * self.n)()
        for i, (isc, r) in enumerate(self.reqs):
            q = S.Request(**{**r.__dict__, "spp": max(1, r.spp // factor)})
            arr[i].scene = self.gss[isc].handle.value
            arr[i].req = api.to_request(q)
            arr[i].layout = self.clay[i]
            arr[i].buffer = self.dev[i].data_ptr()
        return arr

    def host_maps(self):
        """The device outputs of the last launch as pixel buffers."""
        api = self.api
        out = []
        for d, (_, r) in zip(self.dev, self.reqs):
            out.append(np.frombuffer(d.cpu().numpy().tobytes(), dtype=api.pixel_dtype(r.mode))
                       .reshape(r.height, r.width))
        return out

    def close(self):
        for g in self.gss:
            g.close()


def measure(args, api, su: "Setup", desc: str, tuning, tuning_src: str, rank: int, world: int,
            dist, clocks: bool = True, traffic_key: str = "") -> dict:
    """Batched launches of the whole workload (warm-up, then `steps' timed
    launches), the plain drop-in one request at a time, and the e2e call with
    host buffers.  Returns the JSON fields of the workload."""
    import torch
    from htrdr_kmin_b200 import multigpu as M
    L = api.lib()
    n = su.n

    def check(res, what):
        if res != 0:
            raise api.HtrdrError(what, res, L.htrdr_gpu_last_error().decode())

    for g in su.gss:  # the drop-in draw_map (e2e) runs the same engine and tuning
        g.set_engine(tuning.engine, tuning)

    def step_batched():
        """one launch of the work-queue engine over all requests, outputs in
        HBM; on several ranks the requests' FP64 accumulators instead, summed
        on rank 0 over NCCL and finalized there (combine_ms)"""
        st = api.Stats()
        if dist is None:
            check(L.htrdr_gpu_draw_maps_batched_device(su.items_dev, n, C.byref(tuning), C.byref(st)),
                  "batched_device")
            return st, 0.0
        check(L.htrdr_gpu_draw_maps_batched_accum_device(su.items_acc, n, C.byref(tuning), C.byref(st)),
              "batched_accum_device")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        M.reduce_accumulators(su.acc, dist, dst=0)
        if rank == 0:
            for i, (isc, _) in enumerate(su.reqs):
                check(L.htrdr_gpu_finalize_device(su.gss[isc].handle, C.byref(su.creq[i]),
                                                  C.c_void_p(su.acc.data_ptr() + int(su.acc_off[i])),
                                                  C.byref(su.clay[i]), C.c_void_p(su.dev[i].data_ptr())),
                      "finalize_device")
        e1.record()
        torch.cuda.synchronize()
        return st, e0.elapsed_time(e1)

    def step_plain():
        k = 0.0
        for g in su.gss:
            g.set_engine(api.ENGINE_PLAIN)
        for i, (isc, _) in enumerate(su.reqs):
            st = api.Stats()
            check(L.htrdr_gpu_draw_map_device(su.gss[isc].handle, C.byref(su.creq[i]), C.byref(su.clay[i]),
                                              C.c_void_p(su.dev[i].data_ptr()), C.byref(st)), "draw_map_device")
            k += st.kernel_ms
        for g in su.gss:
            g.set_engine(tuning.engine, tuning)
        return k

    def step_e2e():
        st = api.Stats()
        if n == 1:
            check(L.htrdr_gpu_draw_map(su.gss[su.reqs[0][0]].handle, C.byref(su.creq[0]), C.byref(su.clay[0]),
                                       C.c_void_p(su.host[0].data_ptr()), C.byref(st)), "draw_map")
        else:
            check(L.htrdr_gpu_draw_maps_batched(su.items_host, n, C.byref(tuning), C.byref(st)), "batched")

    if dist is not None and su.acc is None:
        su.enable_accumulators()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step_batched()
    # plain arm: kernels loaded and samplers built by a 1-realisation pass
    for g in su.gss:
        g.set_engine(api.ENGINE_PLAIN)
    for gs, r in su.items:
        gs.draw_map(S.Request(**{**r.__dict__, "spp": 1}))
    barrier()
    plain_ms = step_plain()

    barrier()
    kernel_ms, total_ms, stats = [], [], []
    sampler = ClockSampler(su.local) if clocks else None
    if sampler:
        sampler.__enter__()
    barrier()
    # the K steps between two events on the device: each call returns after
    # its work is done, so the span also holds the host's share of every call
    # (plan building, launches, waits) and the gaps between calls
    span0, span1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    span0.record()
    for _ in range(args.steps):
        st, red = step_batched()
        kernel_ms.append(st.kernel_ms)
        total_ms.append(st.total_ms + red)
        stats.append(st)
    span1.record()
    barrier()
    span_ms = span0.elapsed_time(span1)
    if sampler:
        sampler.__exit__(None, None, None)
    gpu_maps = su.host_maps() if rank == 0 else None

    step_e2e()  # untimed: the first host-buffer call sizes the library's staging buffer
    barrier()
    e2e_steps = min(args.steps, 5)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        step_e2e()
    barrier()
    e2e_ms = 1e3 * (time.perf_counter() - t0) / e2e_steps

    step_ms = span_ms / args.steps
    if dist is not None:
        t = torch.tensor([step_ms, e2e_ms], device=f"cuda:{su.local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms, e2e_ms = float(t[0]), float(t[1])

    last = stats[-1]
    wave = tuning.engine == api.ENGINE_WAVEFRONT
    reals = last.realisations
    kms = float(np.mean(kernel_ms))
    alg_bytes = alg_bytes_of(last)
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kms * 1e-3) / 1e9
    kernel = "wavefront" if wave else ("k_sorted" if tuning.engine == api.ENGINE_SORTED else "k_persistent")
    traffic, traffic_src = traffic_per_launch(traffic_key or kernel, alg_bytes)
    out_bytes = sum(d.numel() for d in su.dev)
    line = {
        "value": world * reals / (step_ms * 1e-3) / 1e6, "ms_per_step": step_ms,
        "call_device_ms_per_step": float(np.mean(total_ms)),
        "config": {"workload": desc, "realisations_per_step_per_gpu": int(su.total_real),
                   "tuning": tuning_dict(tuning, tuning_src),
                   "l2": "inputs larger than L2: scenes of "
                         f"{sum(g.device_bytes for g in su.gss) / 1e6:.0f} MB resident",
                   "parallelism": ("replicated scenes, independent streams per rank, NCCL sum of "
                                   "every map's FP64 accumulators on rank 0, finalized there")
                                  if world > 1 else "single GPU",
                   "scene_build_s": su.build_s},
        "e2e": {"value": world * reals / (e2e_ms * 1e-3) / 1e6, "unit": UNIT, "steps": e2e_steps,
                "h2d_bytes_per_step": int(n * (C.sizeof(api.Request) + C.sizeof(api.BufferLayout))),
                "d2h_bytes_per_step": int(out_bytes)},
        "gpu_launches": int(sum(s.launches for s in stats)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                     "peak_kind": peak_kind,
                     "kernel": "k_wave_event + k_wave_trace + k_wave_finish" if wave else kernel,
                     "alg_bytes_per_launch": int(alg_bytes), "kernel_ms": kms},
        "plain_gpu": {"value": reals / (plain_ms * 1e-3) / 1e6, "unit": UNIT, "kernel": "k_plain",
                      "kernel_ms": plain_ms, "launches": n},
        "batched_vs_plain": plain_ms / kms,
        "segments_per_s": last.segments / (kms * 1e-3),
        "counters": {"segments": last.segments, "nodes": last.nodes,
                     "grid_bytes": last.grid_bytes, "collisions": last.collisions,
                     "realisations": last.realisations, "failures": last.failures},
    }
    if sampler:
        line["clocks"] = sampler.summary()
    return line, gpu_maps, stats


TAILS = (25000, 50000, 100000, 200000)


def pick_tuning(args, api, su: "Setup", name: str):
    """Tuning of the batched engine: the command line's, else the autotuner's
    (on the mix at 1/8 of its realisations per pixel for mix_full, so that its
    28 candidate runs stay short).  The tail threshold of a wavefront pick is
    then timed on the full mix: at 1/8 of the work the longest walks, which
    the threshold is about, weigh eight times as much."""
    if args.tuning:
        return parse_tuning(api, args.tuning), "command line"
    if name != "mix_full":
        tuning, _ = api.autotune(su.items_dev)
        return tuning, "autotuner"
    tuning, _ = api.autotune(su.reduced_items(8))
    src = "autotuner (on the same mix at 1/8 of the realisations per pixel)"
    if tuning.engine != api.ENGINE_WAVEFRONT:
        return tuning, src
    L = api.lib()
    best = None
    for tail in TAILS:
        t = api.Tuning(*[getattr(tuning, f) for f, _ in api.Tuning._fields_])
        t.wave_tail = tail
        st = api.Stats()
        res = L.htrdr_gpu_draw_maps_batched_device(su.items_dev, su.n, C.byref(t), C.byref(st))
        if res != 0:
            raise api.HtrdrError("batched_device", res, L.htrdr_gpu_last_error().decode())
        if best is None or st.kernel_ms < best[0]:
            best = (st.kernel_ms, t)
    return best[1], src + f", tail threshold timed on the full mix ({', '.join(map(str, TAILS))})"


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
    from htrdr_kmin_b200 import multigpu as M
    build.build()
    scenes, reqs, desc = workload(args.workload, args)
    for _, r in reqs:
        r.seed = M.rank_seed(r.seed, rank)  # independent streams per rank (weak scaling)
    su = Setup(api, scenes, reqs, local)
    if args.profile_once:
        # the launches of one step and nothing else, so that a profiler's
        # launch list holds exactly one step
        if not args.tuning:
            raise SystemExit("--profile-once needs --tuning")
        tuning = parse_tuning(api, args.tuning)
        st = api.Stats()
        res = api.lib().htrdr_gpu_draw_maps_batched_device(su.items_dev, su.n, C.byref(tuning), C.byref(st))
        if res != 0:
            raise api.HtrdrError("batched_device", res, api.lib().htrdr_gpu_last_error().decode())
        alg = alg_bytes_of(st)
        print(json.dumps({"workload": desc, "tuning": tuning_dict(tuning, "command line"),
                          "kernel_ms": st.kernel_ms, "launches": st.launches, "alg_bytes": alg,
                          "counters": {"segments": st.segments, "nodes": st.nodes,
                                       "grid_bytes": st.grid_bytes,
                                       "collisions": st.collisions, "realisations": st.realisations}}),
              flush=True)
        su.close()
        return
    tuning, src = pick_tuning(args, api, su, args.workload)
    fields, gpu_maps, _ = measure(args, api, su, desc, tuning, src, rank, world, dist,
                                  traffic_key="wavefront_lw" if (args.workload == "lw_flux"
                                                                 and tuning.engine == api.ENGINE_WAVEFRONT) else "")

    line = {"metric": METRIC, "value": fields.pop("value"), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": fields.pop("ms_per_step"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes and sensors)"}
    line.update(fields)

    if args.workload == "mix_full":
        # serving: Poisson arrivals at a rate that saturates the GPU (all
        # requests arrive within a quarter of the batched engine's time for
        # the mix), against the same arrivals on the plain drop-in
        batched_s = line["ms_per_step"] * 1e-3
        rate = su.n / (0.25 * batched_s)
        rng = np.random.default_rng(5)
        gaps = rng.exponential(1.0 / rate, size=su.n)
        arrivals = np.cumsum(gaps) - gaps[0]
        served = serve_arrivals(api, su.items, tuning, arrivals, local)
        plain = plain_arrivals(api, su.items, arrivals)
        line["serving"] = {
            "rate_req_s": rate, "arrivals": "Poisson, seeded; all requests within ~1/4 of the "
                                            "batched engine's time for the mix (saturating)",
            "hbm_budget_GB": 150, "served": served, "plain_one_at_a_time": plain,
            "served_vs_plain": served["Mreal_s"] / plain["Mreal_s"],
            "p99_plain_over_served": plain["p99_ms"] / served["p99_ms"] if served["p99_ms"] else None}
        line["target_3x"] = {"batched_vs_plain": line["batched_vs_plain"] >= 3.0,
                             "served_vs_plain": line["serving"]["served_vs_plain"] >= 3.0}

    cpu = agr = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, agr = cpu_leg(scenes, su.reqs, args.cpu_sample_s, gpu_maps)
    line["cpu_baseline"] = cpu
    line["agreement"] = agr
    su.close()

    if args.workload == "mix_full" and not args.no_secondary:
        sc2, rq2 = S.config_c2()
        rq2.seed = M.rank_seed(rq2.seed, rank)
        _, _, desc2 = workload("lw_flux")
        su2 = Setup(api, [sc2], [(0, rq2)], local)
        t2, src2 = pick_tuning(args, api, su2, "lw_flux") if not args.tuning else (
            api.mode_tuning(S.MODE_FLUX_LW), "mode default")
        f2, _, _ = measure(args, api, su2, desc2, t2, src2, rank, world, dist, clocks=False,
                           traffic_key="wavefront_lw" if t2.engine == api.ENGINE_WAVEFRONT else "")
        line["lw_flux"] = {k: f2[k] for k in ("value", "ms_per_step", "e2e", "plain_gpu",
                                              "batched_vs_plain", "roofline", "segments_per_s")}
        line["lw_flux"]["unit"] = UNIT
        line["lw_flux"]["config"] = {"workload": desc2, "tuning": f2["config"]["tuning"]}
        su2.close()

    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
