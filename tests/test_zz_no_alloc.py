"""htrdr_gpu_draw_map_noalloc: the draw_map variant for callers that cannot
allocate device memory while rendering (their HBM belongs to an application
pool, or their loop must not pay for cudaFree's device synchronisation).

Called through the C ABI on a scene and an output buffer allocated up front,
twice in a row, and compared with htrdr_gpu_draw_map_device on the same
request: both run the same kernel on the same random streams, so the pixels
agree up to the FP64 summation order (1e-9 relative), and the second call
does not see the first call's sums left in the shared static scratch."""
import ctypes as C

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def _noalloc(api, gs, req, dev_ptr):
    L = api.lib()
    fn = L.htrdr_gpu_draw_map_noalloc
    fn.argtypes = [C.c_void_p, C.POINTER(api.Request), C.POINTER(api.BufferLayout), C.c_void_p]
    r = api.to_request(req)
    lay = api.layout_for(req)
    return fn(gs.handle, C.byref(r), C.byref(lay), C.c_void_p(dev_ptr))


def _device_buffer(req, api):
    import torch
    nbytes = req.width * req.height * api.pixel_dtype(req.mode).itemsize
    return torch.zeros(nbytes, dtype=torch.uint8, device="cuda:0")


def _to_host(buf, req, api):
    return np.frombuffer(buf.cpu().numpy().tobytes(), dtype=api.pixel_dtype(req.mode)).reshape(
        req.height, req.width)


def _compare(a, b, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        np.testing.assert_array_equal(a["n"], b["n"])
        np.testing.assert_allclose(a["sum"], b["sum"], rtol=RTOL, atol=0)
        np.testing.assert_allclose(a["sum2"], b["sum2"], rtol=RTOL, atol=0)
    elif mode == S.MODE_IMAGE_CIE:
        for c in ("X", "Y", "Z"):
            np.testing.assert_allclose(a[c], b[c], rtol=RTOL, atol=0)
    else:
        np.testing.assert_allclose(a["L"], b["L"], rtol=RTOL, atol=0)
        np.testing.assert_allclose(a["Tb"], b["Tb"], rtol=1e-6, atol=0)
    np.testing.assert_array_equal(a["t_n"], b["t_n"])


def _cases():
    s2, r2 = S.config_c2(scale=32 / 128, spp=16, cloud_def=(16, 16, 8))
    s1, r1 = S.config_c1(scale=16 / 64, spp=8)
    s3, r3 = S.config_c3(scale=12 / 512, spp=4, cloud_def=(32, 32, 8), nbands=6, nquad=3)
    return [("flux_lw", s2, r2, 0b100), ("xwave_sw", s1, r1, 0b111), ("image_cie", s3, r3, 0b111)]


@pytest.mark.parametrize("name,scene,req,props", _cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_noalloc_matches_device_entry_point(gpu_lib, name, scene, req, props):
    api = gpu_lib
    gs = api.GpuScene(scene, props)
    ref_dev = _device_buffer(req, api)
    gs.draw_map(req, device_out=ref_dev.data_ptr())
    ref = _to_host(ref_dev, req, api)
    out = _device_buffer(req, api)
    for call in range(2):  # two calls in a row share the static scratch
        out.zero_()
        assert _noalloc(api, gs, req, out.data_ptr()) == api.RES_OK, api.lib().htrdr_gpu_last_error()
        _compare(_to_host(out, req, api), ref, req.mode)
    gs.close()


def test_noalloc_rejects_oversize_requests(gpu_lib):
    api = gpu_lib
    scene, req = S.config_c2(scale=1 / 128, spp=1, cloud_def=(4, 4, 2))
    gs = api.GpuScene(scene, 0b100)
    big = S.Request(**{**req.__dict__, "width": 256, "height": 256})  # 65536 px x 2 accumulators
    out = _device_buffer(S.Request(**{**req.__dict__, "width": 1, "height": 1}), api)
    assert _noalloc(api, gs, big, out.data_ptr()) == api.RES_BAD_ARG
    assert b"65536" in api.lib().htrdr_gpu_last_error()
    gs.close()


def test_noalloc_takes_no_device_memory(gpu_lib):
    """The entry point's contract: after the first call on a device (which
    looks up the static arrays and may load the kernels), further calls leave
    the device's free memory unchanged."""
    import torch
    api = gpu_lib
    scene, req = S.config_c2(scale=32 / 128, spp=4, cloud_def=(16, 16, 8))
    gs = api.GpuScene(scene, 0b100)
    out = _device_buffer(req, api)
    assert _noalloc(api, gs, req, out.data_ptr()) == api.RES_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(3):
        assert _noalloc(api, gs, req, out.data_ptr()) == api.RES_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    gs.close()


def test_noalloc_rejects_the_layouts_draw_map_device_rejects(gpu_lib):
    api = gpu_lib
    scene, req = S.config_c2(scale=4 / 128, spp=1, cloud_def=(4, 4, 2))
    gs = api.GpuScene(scene, 0b100)
    out = _device_buffer(req, api)
    L = api.lib()
    fn = L.htrdr_gpu_draw_map_noalloc
    fn.argtypes = [C.c_void_p, C.POINTER(api.Request), C.POINTER(api.BufferLayout), C.c_void_p]
    r = api.to_request(req)
    for alignment in (3, 32):  # not a power of two; above 16
        lay = api.layout_for(req)
        lay.alignment = alignment
        assert fn(gs.handle, C.byref(r), C.byref(lay), C.c_void_p(out.data_ptr())) == api.RES_BAD_ARG
        st = api.Stats()
        assert L.htrdr_gpu_draw_map_device(gs.handle, C.byref(r), C.byref(lay),
                                           C.c_void_p(out.data_ptr()), C.byref(st)) == api.RES_BAD_ARG
    gs.close()
