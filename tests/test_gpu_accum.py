"""The accumulator entry points that let several GPUs combine their maps
(htrdr_gpu_draw_map_accum_device, htrdr_gpu_draw_maps_batched_accum_device,
htrdr_gpu_finalize_device), through the C ABI:

* accumulators then finalize == the map drawn directly (every mode; the
  summation order of the FP64 atomics is the only difference);
* the batched launch leaves each request's accumulators in its buffer, the
  same as each request drawn alone;
* the sum of two seeds' accumulators, finalized on the device, equals the
  host-side estimate of the summed records (the multi-GPU combination), LW
  brightness temperature included.
"""
import numpy as np
import pytest

from htrdr_kmin_b200 import multigpu as M
from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def _cases():
    s1, r1 = S.config_c1(scale=12 / 64, spp=8)
    s2, r2 = S.config_c2(scale=16 / 128, spp=16, cloud_def=(16, 16, 8))
    s3, r3 = S.config_c3(scale=8 / 512, spp=4, cloud_def=(32, 32, 8), nbands=6, nquad=3)
    s4, r4 = S.config_c2(scale=8 / 128, spp=16, cloud_def=(16, 16, 8))
    r4.mode = S.MODE_XWAVE_LW
    r4.cam_pos, r4.cam_tgt, r4.cam_up = (800, 800, 10), (900, 900, 1500), (0, 1, 0)
    return [("xwave_sw", s1, r1, 0b111), ("flux_lw", s2, r2, 0b100), ("image_cie", s3, r3, 0b111),
            ("xwave_lw", s4, r4, 0b100)]


def _ids(v):
    return v if isinstance(v, str) else ""


def _dev(nbytes):
    import torch
    return torch.zeros(nbytes, dtype=torch.uint8, device="cuda:0")


def _host(t, dtype, shape=None):
    a = np.frombuffer(t.cpu().numpy().tobytes(), dtype=dtype)
    return a.reshape(shape) if shape else a


def _same_map(a, b, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        np.testing.assert_array_equal(a["n"], b["n"])
        np.testing.assert_allclose(a["sum"], b["sum"], rtol=RTOL)
    elif mode == S.MODE_IMAGE_CIE:
        for c in ("X", "Y", "Z"):
            np.testing.assert_allclose(a[c], b[c], rtol=RTOL)
    else:
        np.testing.assert_allclose(a["L"], b["L"], rtol=RTOL)
        np.testing.assert_allclose(a["Tb"], b["Tb"], rtol=1e-7)
    np.testing.assert_array_equal(a["t_n"], b["t_n"])


@pytest.mark.parametrize("name,scene,req,props", _cases(), ids=_ids)
def test_accumulate_then_finalize_equals_draw_map(gpu_lib, name, scene, req, props):
    api = gpu_lib
    gs = api.GpuScene(scene, props)
    dt = api.pixel_dtype(req.mode)
    direct = _dev(req.width * req.height * dt.itemsize)
    gs.draw_map(req, device_out=direct.data_ptr())
    acc = _dev(api.accum_records(req) * 32)
    st = gs.draw_map_accum(req, acc.data_ptr())
    assert st["realisations"] > 0
    out = _dev(req.width * req.height * dt.itemsize)
    gs.finalize(req, acc.data_ptr(), out.data_ptr())
    shape = (req.height, req.width)
    _same_map(_host(out, dt, shape), _host(direct, dt, shape), req.mode)
    gs.close()


def test_batched_accumulators_equal_each_request_alone(gpu_lib):
    import ctypes as C
    api = gpu_lib
    cases = _cases()
    gss = [api.GpuScene(sc, props) for _, sc, _, props in cases]
    accs = [_dev(api.accum_records(r) * 32) for _, _, r, _ in cases]
    arr = (api.BatchItem * len(cases))()
    for i, ((_, _, r, _), gs) in enumerate(zip(cases, gss)):
        arr[i].scene, arr[i].req, arr[i].layout = gs.handle.value, api.to_request(r), api.layout_for(r)
        arr[i].buffer = accs[i].data_ptr()
    st = api.Stats()
    assert api.lib().htrdr_gpu_draw_maps_batched_accum_device(arr, len(cases), None, C.byref(st)) == 0
    for (name, _, r, _), gs, acc in zip(cases, gss, accs):
        alone = _dev(api.accum_records(r) * 32)
        gs.draw_map_accum(r, alone.data_ptr())
        a, b = _host(acc, M.ACCUM_DTYPE), _host(alone, M.ACCUM_DTYPE)
        nch = 3 if r.mode == S.MODE_IMAGE_CIE else 1
        k = r.width * r.height * nch  # the time records differ
        np.testing.assert_array_equal(a["n"][:k], b["n"][:k])
        np.testing.assert_allclose(a["s"][:k], b["s"][:k], rtol=RTOL)
        np.testing.assert_allclose(a["s2"][:k], b["s2"][:k], rtol=RTOL)
    for gs in gss:
        gs.close()


@pytest.mark.parametrize("name,scene,req,props", _cases(), ids=_ids)
def test_summed_accumulators_finalize_like_the_host_estimate(gpu_lib, name, scene, req, props):
    """What rank 0 does after the NCCL sum: two seeds' accumulators added and
    finalized once."""
    api = gpu_lib
    gs = api.GpuScene(scene, props)
    nrec = api.accum_records(req)
    parts = []
    for rank in range(2):
        acc = _dev(nrec * 32)
        gs.draw_map_accum(S.Request(**{**req.__dict__, "seed": M.rank_seed(req.seed, rank)}),
                          acc.data_ptr())
        parts.append(_host(acc, M.ACCUM_DTYPE))
    total = M.combine_accumulators(parts)
    import torch
    dev = torch.from_numpy(np.frombuffer(total.tobytes(), dtype=np.uint8).copy()).to("cuda:0")
    dt = api.pixel_dtype(req.mode)
    out = _dev(req.width * req.height * dt.itemsize)
    gs.finalize(req, dev.data_ptr(), out.data_ptr())
    buf = _host(out, dt, (req.height, req.width))
    nch = 3 if req.mode == S.MODE_IMAGE_CIE else 1
    npix = req.width * req.height
    E, SE = M.estimate(total[:npix * nch])
    if req.mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        np.testing.assert_array_equal(buf["n"].ravel(), total["n"][:npix])
        np.testing.assert_allclose(buf["sum"].ravel(), total["s"][:npix], rtol=1e-15)
    elif nch == 3:
        for c, ch in zip(("X", "Y", "Z"), range(3)):
            np.testing.assert_allclose(buf[c].ravel(), E[ch::3], rtol=1e-12)
            np.testing.assert_allclose(buf[c + "_se"].ravel(), SE[ch::3], rtol=1e-9, atol=1e-300)
    else:
        np.testing.assert_allclose(buf["L"].ravel(), E, rtol=1e-12)
        np.testing.assert_allclose(buf["L_se"].ravel(), SE, rtol=1e-9, atol=1e-300)
        if req.mode == S.MODE_XWAVE_LW:
            assert np.all(buf["Tb"] > 0)
    assert np.all(buf["t_n"].ravel() == total["n"][npix * nch:])
    gs.close()
