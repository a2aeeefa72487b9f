"""Batched persistent kernel vs the plain one-thread-per-realisation kernel.

Both run the same per-realisation state machine on the same Philox stream,
so every pixel sums the same weights; only the FP64 summation order differs
(tolerance 1e-9 relative).  A request gives the same result alone and in a
mix of other requests, scenes and modes."""
import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def _cmp(a, b, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        np.testing.assert_array_equal(a["n"], b["n"])
        np.testing.assert_allclose(a["sum"], b["sum"], rtol=RTOL, atol=0)
        np.testing.assert_allclose(a["sum2"], b["sum2"], rtol=RTOL, atol=0)
    elif mode == S.MODE_IMAGE_CIE:
        for c in ("X", "Y", "Z"):
            np.testing.assert_allclose(a[c], b[c], rtol=RTOL, atol=0)
            np.testing.assert_allclose(a[c + "_se"], b[c + "_se"], rtol=1e-6, atol=1e-300)
    else:
        np.testing.assert_allclose(a["L"], b["L"], rtol=RTOL, atol=0)
        np.testing.assert_allclose(a["L_se"], b["L_se"], rtol=1e-6, atol=1e-300)
        np.testing.assert_allclose(a["Tb"], b["Tb"], rtol=1e-6, atol=0)
    np.testing.assert_array_equal(a["t_n"], b["t_n"])


def _mix(gpu_lib):
    s1, r1 = S.config_c1(scale=20 / 64, spp=16)
    s2, r2 = S.config_c2(scale=24 / 128, spp=24, cloud_def=(16, 16, 8))
    s3, r3 = S.config_c3(scale=13 / 512, spp=6, cloud_def=(32, 32, 8), nbands=6, nquad=3)
    g1, g2, g3 = gpu_lib.GpuScene(s1), gpu_lib.GpuScene(s2, 0b100), gpu_lib.GpuScene(s3)
    r4 = S.Request(**{**r2.__dict__, "mode": S.MODE_XWAVE_LW, "width": 9, "height": 7,
                      "cam_pos": (800, 800, 10), "cam_tgt": (900, 900, 1500), "cam_up": (0, 1, 0),
                      "seed": 77})
    return [(g1, r1), (g2, r2), (g3, r3), (g2, r4)]


def test_batched_equals_plain(gpu_lib):
    items = _mix(gpu_lib)
    bufs, st = gpu_lib.draw_maps_batched(items)
    assert st["failures"] == 0
    for (gs, req), b in zip(items, bufs):
        gs.set_engine(gpu_lib.ENGINE_PLAIN)
        p, _ = gs.draw_map(req)
        gs.set_engine(gpu_lib.ENGINE_PERSISTENT)
        _cmp(b, p, req.mode)


@pytest.mark.parametrize("slots,budget,bs,tail", [
    (0, 0, 256, 0),         # defaults: this small mix is all tail (finishing megakernel only)
    (37, 3, 128, 1),        # stages to the end, few slots: heavy regeneration
    (1000, 1, 64, 1),       # one voxel per trace-stage visit
    (5000, 64, 256, 2000),  # stages, then the megakernel takes the live paths mid-run
])
def test_wavefront_equals_plain(gpu_lib, slots, budget, bs, tail):
    """The wavefront engine (event and trace stages over path slots, the tail
    finished by a megakernel that resumes the saved paths) gives the plain
    kernel's estimates."""
    items = _mix(gpu_lib)
    t = gpu_lib.default_tuning()
    t.engine, t.wave_slots, t.trace_budget, t.block_size = gpu_lib.ENGINE_WAVEFRONT, slots, budget, bs
    t.wave_tail = tail
    bufs, st = gpu_lib.draw_maps_batched(items, t)
    assert st["failures"] == 0
    ref, sref = gpu_lib.draw_maps_batched(items, gpu_lib.default_tuning())
    assert st["realisations"] == sref["realisations"]
    assert st["segments"] == sref["segments"] and st["collisions"] == sref["collisions"]
    assert st["nodes"] == sref["nodes"] and st["grid_bytes"] == sref["grid_bytes"]
    for (gs, req), b, r in zip(items, bufs, ref):
        gs.set_engine(gpu_lib.ENGINE_PLAIN)
        p, _ = gs.draw_map(req)
        gs.set_engine(gpu_lib.ENGINE_PERSISTENT)
        _cmp(b, p, req.mode)
        _cmp(b, r, req.mode)


def test_wavefront_refused_where_the_host_cannot_drive_it(gpu_lib):
    import ctypes as C
    items = _mix(gpu_lib)[:1]
    arr = (gpu_lib.BatchItem * 1)()
    gs, req = items[0]
    import torch
    dev = torch.empty(req.width * req.height * gpu_lib.pixel_dtype(req.mode).itemsize,
                      dtype=torch.uint8, device="cuda:0")
    arr[0].scene, arr[0].req, arr[0].layout = gs.handle.value, gpu_lib.to_request(req), gpu_lib.layout_for(req)
    arr[0].buffer = dev.data_ptr()
    t = gpu_lib.default_tuning()
    t.engine = gpu_lib.ENGINE_WAVEFRONT
    h = C.c_void_p()
    L = gpu_lib.lib()
    assert L.htrdr_gpu_batch_create(arr, 1, C.byref(t), C.byref(h)) == gpu_lib.RES_BAD_ARG
    assert b"persistent" in L.htrdr_gpu_last_error()


def test_draw_map_engines_agree(gpu_lib):
    """htrdr_gpu_draw_map on the persistent engine (default, by-mode or given
    tuning) equals the plain engine, on host and device outputs."""
    import torch
    grid_bytes = 0
    for gs, req in _mix(gpu_lib):
        gs.set_engine(gpu_lib.ENGINE_PLAIN)
        plain, sp = gs.draw_map(req)
        gs.set_engine(gpu_lib.ENGINE_PERSISTENT)
        pers, spp = gs.draw_map(req)
        _cmp(pers, plain, req.mode)
        assert sp["realisations"] == spp["realisations"] and sp["segments"] == spp["segments"]
        t = gpu_lib.default_tuning()
        t.block_size, t.queue_chunk, t.regroup_period = 64, 2, 4
        gs.set_engine(gpu_lib.ENGINE_PERSISTENT, t)
        tuned, _ = gs.draw_map(req)
        _cmp(tuned, plain, req.mode)
        gs.set_engine(gpu_lib.ENGINE_WAVEFRONT)
        wave, sw = gs.draw_map(req)
        _cmp(wave, plain, req.mode)
        assert sw["segments"] == sp["segments"]
        # every path takes the same voxel steps on every engine, so it reads
        # the same leaf-grid entries and majorant nodes
        assert sp["grid_bytes"] == spp["grid_bytes"] == sw["grid_bytes"]
        assert sp["nodes"] == spp["nodes"] == sw["nodes"]
        grid_bytes += sp["grid_bytes"]
        t.trace_budget, t.wave_slots, t.wave_tail = 5, 333, 100
        gs.set_engine(gpu_lib.ENGINE_WAVEFRONT, t)
        wave2, _ = gs.draw_map(req)
        _cmp(wave2, plain, req.mode)
        dev = torch.empty(pers.nbytes, dtype=torch.uint8, device="cuda:0")
        gs.draw_map(req, device_out=dev.data_ptr())
        torch.cuda.synchronize()
        got = np.frombuffer(dev.cpu().numpy().tobytes(), dtype=pers.dtype).reshape(pers.shape)
        _cmp(got, plain, req.mode)
        gs.set_engine(gpu_lib.ENGINE_PERSISTENT)
    assert grid_bytes > 0
    gs, req = _mix(gpu_lib)[0]
    bad = gpu_lib.default_tuning()
    bad.block_size = 48  # not a multiple of a warp
    with pytest.raises(gpu_lib.HtrdrError):
        gs.set_engine(gpu_lib.ENGINE_PERSISTENT, bad)
    with pytest.raises(gpu_lib.HtrdrError):
        gs.set_engine(7)


def test_alone_equals_in_mix(gpu_lib):
    items = _mix(gpu_lib)
    mixed, _ = gpu_lib.draw_maps_batched(items)
    for i, it in enumerate(items):
        alone, _ = gpu_lib.draw_maps_batched([it])
        _cmp(alone[0], mixed[i], it[1].mode)


@pytest.mark.parametrize("chunk,bs", [(1, 32), (3, 64), (16, 256)])
def test_tuning_does_not_change_results(gpu_lib, chunk, bs):
    items = _mix(gpu_lib)[:2]
    ref, _ = gpu_lib.draw_maps_batched(items)
    t = gpu_lib.default_tuning()
    t.queue_chunk, t.block_size = chunk, bs
    out, _ = gpu_lib.draw_maps_batched(items, t)
    for (gs, req), a, b in zip(items, out, ref):
        _cmp(a, b, req.mode)


def test_edge_cases(gpu_lib):
    sc, rq = S.config_c1(scale=1 / 64, spp=1)   # 1x1 image, one realisation
    gs = gpu_lib.GpuScene(sc)
    buf, st = gs.draw_map(rq)
    assert buf.shape == (1, 1) and buf["t_n"][0, 0] == 1
    rq2 = S.Request(**{**rq.__dict__, "width": 13, "height": 3, "spp": 2})  # ragged tiles
    buf, st = gs.draw_map(rq2)
    assert np.all(buf["t_n"] == 2)
    bad = S.Request(**{**rq.__dict__, "spp": 0})
    with pytest.raises(gpu_lib.HtrdrError) as e:
        gs.draw_map(bad)
    assert e.value.code == gpu_lib.RES_BAD_ARG
    # an LW-only scene cannot serve SW requests (missing majorants)
    s2, r2 = S.config_c2(scale=1 / 64, spp=1, cloud_def=(4, 4, 2))
    g2 = gpu_lib.GpuScene(s2, 0b100)
    with pytest.raises(gpu_lib.HtrdrError):
        g2.draw_map(S.Request(**{**r2.__dict__, "mode": S.MODE_FLUX_SW}))
    # clear sky and no ground
    slab = S.homogeneous_slab(k_abs=1e-5, k_sca=1e-5, has_ground=False)
    gsl = gpu_lib.GpuScene(slab)
    r3 = S.Request(mode=S.MODE_XWAVE_SW, width=4, height=4, spp=8, wlen_range=(550.0, 550.0),
                   cam_pos=(0, 0, 500), cam_tgt=(0, 1000, 500), cam_up=(0, 0, 1))
    buf, st = gsl.draw_map(r3)
    assert np.all(np.isfinite(buf["L"])) and st["failures"] == 0


@pytest.mark.parametrize("bs,period", [(32, 1), (64, 4), (128, 1), (256, 16)])
def test_sorted_engine_equals_plain(gpu_lib, bs, period):
    """The block-sorted persistent kernel (paths in shared memory regrouped by
    stage over the whole block) on a mix of SW, LW and CIE requests and on an
    LW-only pair (its LW-only variant): the plain kernel's sums."""
    items = _mix(gpu_lib)
    t = gpu_lib.default_tuning()
    t.engine, t.block_size, t.regroup_period, t.queue_chunk = gpu_lib.ENGINE_SORTED, bs, period, 1
    for group in (items, [items[1], items[3]]):
        bufs, st = gpu_lib.draw_maps_batched(group, t)
        assert st["failures"] == 0
        for (gs, req), b in zip(group, bufs):
            gs.set_engine(gpu_lib.ENGINE_PLAIN)
            p, _ = gs.draw_map(req)
            gs.set_engine(gpu_lib.ENGINE_PERSISTENT)
            _cmp(b, p, req.mode)
