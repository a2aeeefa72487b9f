"""Serving loop (continuous batching) and graph-captured batches.

A request gives the same map alone and in a mix served by the loop: every
realisation has the same weight whatever the rounds it falls in, so per-pixel
sums agree to the FP64 summation order (1e-9 relative)."""
import random
import threading
import time

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def _cmp(a, b, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        np.testing.assert_array_equal(a["n"], b["n"])
        np.testing.assert_allclose(a["sum"], b["sum"], rtol=RTOL, atol=0)
    elif mode == S.MODE_IMAGE_CIE:
        for c in ("X", "Y", "Z"):
            np.testing.assert_allclose(a[c], b[c], rtol=RTOL, atol=0)
    else:
        np.testing.assert_allclose(a["L"], b["L"], rtol=RTOL, atol=0)
    np.testing.assert_array_equal(a["t_n"], b["t_n"])


@pytest.fixture(scope="module")
def mix(gpu_lib):
    api = gpu_lib
    s1, r1 = S.config_c1(scale=16 / 64, spp=16)
    s2, r2 = S.config_c2(scale=32 / 128, spp=16, cloud_def=(16, 16, 8))
    s3, r3 = S.config_c3(scale=12 / 512, spp=4, cloud_def=(32, 32, 8), nbands=6, nquad=3)
    g1, g2, g3 = api.GpuScene(s1), api.GpuScene(s2, 0b100), api.GpuScene(s3)
    reqs = [(g1, r1), (g2, r2), (g3, r3)]
    rng = random.Random(4)
    for i in range(9):
        g, r = reqs[i % 3]
        side = rng.choice([5, 8, 13, 20])
        reqs.append((g, S.Request(**{**r.__dict__, "width": side, "height": side + 1,
                                     "spp": rng.choice([2, 4, 8]), "seed": 100 + i})))
    return reqs


def _tuning(api, engine, slots=0, tail=0):
    """Server tuning: the persistent rounds, or the wavefront slot pool (few
    slots: regeneration, revival of free slots and queue refills all occur)"""
    t = api.default_tuning()
    t.engine = engine
    if engine == api.ENGINE_WAVEFRONT:
        t.block_size, t.regroup_period, t.wave_slots, t.wave_tail = 128, 4, slots, tail
    return t


# (name, slots, tail): the wavefront pool finishes its tail in the megakernel
# (tail 0: default threshold) or runs the stages to the end (tail 1)
ENGINES = [("persistent", 0, 0), ("wavefront", 3000, 0), ("wavefront_no_tail", 2000, 1)]
WAIT_S = 120.0


def _engine(api, name):
    return api.ENGINE_PERSISTENT if name == "persistent" else api.ENGINE_WAVEFRONT


@pytest.mark.parametrize("name,slots,tail", ENGINES)
def test_server_results_equal_alone(gpu_lib, mix, name, slots, tail):
    api = gpu_lib
    alone = [gs.draw_map(r)[0] for gs, r in mix]
    srv = api.Server(round_target_ms=2.0, round_realisations=4096,
                     tuning=_tuning(api, _engine(api, name), slots, tail))
    tickets = [None] * len(mix)

    def submitter(idx):
        rng = random.Random(idx[0])
        for i in idx:
            time.sleep(rng.uniform(0, 0.01))
            tickets[i] = srv.submit(*mix[i])

    ts = [threading.Thread(target=submitter, args=(list(range(k, len(mix), 2)),)) for k in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    out = [srv.wait(t, WAIT_S) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(mix) and st["failed"] == 0
    assert st["rounds"] > 1
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (gs, r), a, b in zip(mix, out, alone):
        _cmp(a, b, r.mode)


@pytest.mark.parametrize("name,slots,tail", ENGINES[:2])
def test_server_admission_by_budget(gpu_lib, mix, name, slots, tail):
    api = gpu_lib
    sizes = []
    for gs, r in mix:
        nch = 3 if r.mode == S.MODE_IMAGE_CIE else 1
        sizes.append(r.width * r.height * (nch + 1) * 32 + r.width * r.height * r.pixel_size)
    budget = max(sizes) + 16
    srv = api.Server(hbm_budget_bytes=budget, round_target_ms=2.0, round_realisations=2048,
                     tuning=_tuning(api, _engine(api, name), slots, tail))
    tickets = [srv.submit(gs, r) for gs, r in mix]
    out = [srv.wait(t, WAIT_S) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["hbm_peak_bytes"] <= budget
    for (gs, r), a in zip(mix, out):
        _cmp(a, gs.draw_map(r)[0], r.mode)


def test_wavefront_server_after_idle(gpu_lib, mix):
    """Two bursts with an idle gap: the pool drains, the queue restarts from
    zero, free slots are revived for the second burst, and every map equals
    its rendering alone."""
    api = gpu_lib
    srv = api.Server(tuning=_tuning(api, api.ENGINE_WAVEFRONT, 1500, 0))
    first = [srv.submit(gs, r) for gs, r in mix[:5]]
    out1 = [srv.wait(t, WAIT_S) for t in first]
    time.sleep(0.2)
    second = [srv.submit(gs, r) for gs, r in mix[5:]]
    out2 = [srv.wait(t, WAIT_S) for t in second]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(mix) and st["failed"] == 0
    for (gs, r), a in zip(mix, out1 + out2):
        _cmp(a, gs.draw_map(r)[0], r.mode)


def test_server_rejects_request_above_budget(gpu_lib, mix):
    api = gpu_lib
    srv = api.Server(hbm_budget_bytes=1024)
    t = srv.submit(*mix[0])
    with pytest.raises(api.HtrdrError) as e:
        srv.wait(t)
    assert e.value.code == api.RES_MEM_ERR
    srv.close()


def test_graph_batch_replay(gpu_lib, mix):
    import ctypes as C
    import torch
    api = gpu_lib
    sub = mix[:4]
    bufs = [torch.zeros(r.width * r.height * api.pixel_dtype(r.mode).itemsize, dtype=torch.uint8,
                        device="cuda:0") for _, r in sub]
    items = (api.BatchItem * len(sub))()
    for i, (gs, r) in enumerate(sub):
        items[i].scene = gs.handle.value
        items[i].req = api.to_request(r)
        items[i].layout = api.layout_for(r)
        items[i].buffer = bufs[i].data_ptr()
    h = C.c_void_p()
    assert api.lib().htrdr_gpu_batch_create(items, len(sub), None, C.byref(h)) == 0
    for _ in range(2):
        st = api.Stats()
        assert api.lib().htrdr_gpu_batch_run(h, C.byref(st)) == 0
        assert st.kernel_ms > 0 and st.failures == 0
        for (gs, r), b in zip(sub, bufs):
            got = np.frombuffer(b.cpu().numpy().tobytes(), dtype=api.pixel_dtype(r.mode)).reshape(r.height, r.width)
            _cmp(got, gs.draw_map(r)[0], r.mode)
    api.lib().htrdr_gpu_batch_release(h)


@pytest.mark.parametrize("name,slots,tail", ENGINES[:2])
def test_server_kinds_change(gpu_lib, mix, name, slots, tail):
    """A server that has seen only longwave requests (LW-only kernel variants;
    on the persistent engine, the variant with its paths in shared memory)
    then admits shortwave and CIE ones: every map still equals its map drawn
    alone."""
    api = gpu_lib
    lw = [(gs, r) for gs, r in mix if r.mode == S.MODE_FLUX_LW]
    sw = [(gs, r) for gs, r in mix if r.mode != S.MODE_FLUX_LW]
    assert lw and sw
    srv = api.Server(round_target_ms=2.0, round_realisations=4096,
                     tuning=_tuning(api, _engine(api, name), slots, tail))
    first = [srv.submit(gs, r) for gs, r in lw]
    out1 = [srv.wait(t, WAIT_S) for t in first]
    second = [srv.submit(gs, r) for gs, r in sw + lw[:1]]
    out2 = [srv.wait(t, WAIT_S) for t in second]
    srv.close()
    for (gs, r), got in zip(lw + sw + lw[:1], out1 + out2):
        _cmp(got, gs.draw_map(r)[0], r.mode)


@pytest.mark.parametrize("name,slots,tail", ENGINES[:2])
def test_request_admitted_mid_run_shares_launches(gpu_lib, mix, name, slots, tail):
    """Continuous batching: a request submitted while another is on the GPU
    gets its realisations into a launch that still carries the first one's
    (their launch ranges intersect), and its map is the same as alone."""
    api = gpu_lib
    gs_a, r_a = mix[0]
    big = S.Request(**{**r_a.__dict__, "width": 48, "height": 48, "spp": 64, "seed": 77})
    gs_b, r_b = mix[4]
    srv = api.Server(round_target_ms=2.0, round_realisations=4096,
                     tuning=_tuning(api, _engine(api, name), slots, tail))
    ta = srv.submit(gs_a, big)
    t0 = time.perf_counter()
    while srv.stats()["rounds"] < 2 and time.perf_counter() - t0 < 30:
        time.sleep(0.001)  # the first request is on the device
    tb = srv.submit(gs_b, r_b)
    out_b = srv.wait(tb, WAIT_S)
    srv.wait(ta, WAIT_S)
    fa, la = srv.launches(ta)
    fb, lb = srv.launches(tb)
    srv.close()
    print(f"{name}: first request launches {fa}..{la}, second {fb}..{lb}")
    assert fb > fa, "the second request reached the device after the first"
    assert fb <= la, "and shared a launch with it"
    _cmp(out_b, gs_b.draw_map(r_b)[0], r_b.mode)
