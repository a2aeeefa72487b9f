"""Ground geometry on the GPU against the CPU oracle.

* ray queries through the BVH (htrdr_gpu_ground_trace) are bit-exact with
  the oracle's brute-force loop: same primitive, same FP32 distance, with
  and without the repeated bounding box, from scratch and from a previous
  hit (self-hit rule);
* transport over a terrain mesh with a Lambertian soil (spectral BRDF
  table) and a specular water group: matched-stream realisations and
  independent-stream 3-sigma agreement, shortwave image, longwave image,
  and longwave and shortwave flux maps whose probes partly lie under the
  terrain (rejected on both sides alike).
"""
import math

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu

MATCH_RTOL = 2e-3
FLT_MAX = np.float32(3.4028235e38)


def _rays(n, seed, size=3200.0, amp=150.0):
    rng = np.random.default_rng(seed)
    o = np.stack([rng.uniform(-800.0, size + 800.0, n), rng.uniform(-800.0, size + 800.0, n),
                  rng.uniform(-60.0, amp + 400.0, n)], axis=1)
    d = rng.normal(size=(n, 3))
    d[: n // 2, 2] = -np.abs(d[: n // 2, 2])  # half of them downward
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.full(n, FLT_MAX, np.float32)
    tmax[n // 4: n // 2] = rng.uniform(10.0, 800.0, n // 2 - n // 4)
    return np.concatenate([o, d], axis=1).astype(np.float32), tmax


@pytest.mark.parametrize("repeat", [False, True], ids=["single", "repeated"])
def test_ground_trace_bitexact(gpu_lib, oracle_lib, repeat):
    sc = S.with_terrain(S.config_c1(scale=8 / 64, spp=1)[0], n=24, repeat=repeat)
    gs = gpu_lib.GpuScene(sc, 0b111)
    os_ = oracle_lib.OracleScene(sc, 0b111)
    n = 40000
    rays, tmax = _rays(n, 11 + int(repeat))
    none = np.full(n, S.NO_ID, np.uint32)
    zero = np.zeros(n, np.uint8)
    pg, dg = gs.ground_trace(rays, tmax, none, zero)
    pc, dc = os_.ground_trace(rays, tmax, none, zero)
    hit = pc != S.NO_ID
    print(f"repeat={repeat}: {hit.mean():.3f} of {n} rays hit")
    assert 0.2 < hit.mean() < 0.9
    np.testing.assert_array_equal(pg, pc)
    np.testing.assert_array_equal(dg.view(np.uint32), dc.view(np.uint32))
    # second bounce: leave each hit point in a new direction, from its primitive
    rng = np.random.default_rng(5)
    idx = np.nonzero(hit)[0]
    o2 = rays[idx, :3] + rays[idx, 3:] * dc[idx, None]
    d2 = rng.normal(size=(idx.size, 3))
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    r2 = np.concatenate([o2, d2], axis=1).astype(np.float32)
    t2 = np.full(idx.size, FLT_MAX, np.float32)
    e2 = rng.integers(0, 2, idx.size).astype(np.uint8)
    pg2, dg2 = gs.ground_trace(r2, t2, pc[idx], e2)
    pc2, dc2 = os_.ground_trace(r2, t2, pc[idx], e2)
    np.testing.assert_array_equal(pg2, pc2)
    np.testing.assert_array_equal(dg2.view(np.uint32), dc2.view(np.uint32))
    assert not np.any(pc2 == pc[idx])  # never the primitive it leaves


def terrain_requests():
    out = []
    sc, rq = S.config_c1(scale=10 / 64, spp=8)
    sc = S.with_terrain(sc)
    rq.cam_pos, rq.cam_tgt, rq.cam_up = (1600.0, -600.0, 700.0), (1600.0, 1600.0, 0.0), (0, 0, 1)
    out.append(("terrain_xwave_sw", sc, rq, 0b111))
    sc, rq = S.config_c2(scale=8 / 128, spp=16, cloud_def=(16, 16, 8))
    sc = S.with_terrain(sc)
    rq.mode = S.MODE_XWAVE_LW
    rq.cam_pos, rq.cam_tgt, rq.cam_up = (800.0, -400.0, 500.0), (800.0, 800.0, 0.0), (0, 0, 1)
    out.append(("terrain_xwave_lw", sc, rq, 0b100))
    sc, rq = S.config_c2(scale=8 / 128, spp=16, cloud_def=(16, 16, 8))
    sc = S.with_terrain(sc)
    rq.rect_pos, rq.rect_tgt = (800.0, 800.0, 75.0), (800.0, 800.0, 76.0)
    out.append(("terrain_flux_lw", sc, rq, 0b100))
    sc, rq = S.config_c1(scale=8 / 64, spp=8)
    sc = S.with_terrain(sc)
    rq.mode = S.MODE_FLUX_SW
    rq.rect_pos, rq.rect_tgt, rq.rect_up, rq.rect_size = (1600, 1600, 75), (1600, 1600, 76), (0, 1, 0), (3200, 3200)
    out.append(("terrain_flux_sw", sc, rq, 0b111))
    return out


@pytest.mark.parametrize("name,scene,req,props", terrain_requests(),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_terrain_matched_streams(gpu_lib, oracle_lib, name, scene, req, props):
    gs = gpu_lib.GpuScene(scene, props)
    os_ = oracle_lib.OracleScene(scene, props)
    npix = req.width * req.height
    wg = gs.realisation_weights(req, 0, npix)
    wc = os_.realisation_weights(req, 0, npix)
    np.testing.assert_array_equal(np.isnan(wg), np.isnan(wc))
    ok = ~np.isnan(wc)
    if req.mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        assert 0.05 < 1.0 - ok.mean() < 0.95  # some probes lie under the terrain
    g, c = wg[ok], wc[ok]
    scale = max(np.abs(c).mean(), 1e-300)
    close = np.abs(g - c) <= MATCH_RTOL * np.maximum(np.abs(c), 1e-6 * scale)
    print(f"{name}: {close.mean():.4f} of {close.size} realisations match within {MATCH_RTOL}")
    assert close.mean() >= 0.9


def _estimates(buf, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        n = buf["n"].astype(np.float64)
        E = buf["sum"] / np.maximum(n, 1)
        V = np.maximum(buf["sum2"] / np.maximum(n, 1) - E * E, 0)
        return [(E.ravel(), np.sqrt(V / np.maximum(n, 1)).ravel())]
    return [(buf["L"].ravel(), buf["L_se"].ravel())]


@pytest.mark.parametrize("name,scene,req,props", terrain_requests(),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_terrain_three_sigma(gpu_lib, oracle_lib, name, scene, req, props):
    req.spp = 128
    gs = gpu_lib.GpuScene(scene, props)
    os_ = oracle_lib.OracleScene(scene, props)
    bg, _ = gs.draw_map(S.Request(**{**req.__dict__, "seed": 1001}))
    bc, _ = os_.draw_map(S.Request(**{**req.__dict__, "seed": 2002}))
    zs = []
    for (Eg, SEg), (Ec, SEc) in zip(_estimates(bg, req.mode), _estimates(bc, req.mode)):
        s = np.sqrt(SEg ** 2 + SEc ** 2)
        m = s > 0
        zs.append((Eg[m] - Ec[m]) / s[m])
    z = np.concatenate(zs)
    n = z.size
    assert n > 0
    fail = np.mean(np.abs(z) > 3)
    print(f"{name}: {n} estimates, |z|>3 fraction {fail:.4f}, mean z {z.mean():+.3f}")
    assert fail <= 3 * 0.0027 + 3 * math.sqrt(0.0027 / n) + 1.0 / n
    assert abs(z.mean()) < 5.0 / math.sqrt(n) + 0.05


def test_terrain_engines_agree(gpu_lib):
    """Plain, persistent and wavefront engines give the same map over the
    terrain (same streams, same kernels' transport)."""
    sc, rq = S.config_c1(scale=12 / 64, spp=8)
    sc = S.with_terrain(sc)
    rq.cam_pos, rq.cam_tgt, rq.cam_up = (1600.0, -600.0, 700.0), (1600.0, 1600.0, 0.0), (0, 0, 1)
    gs = gpu_lib.GpuScene(sc, 0b111)
    out = {}
    for eng in (gpu_lib.ENGINE_PLAIN, gpu_lib.ENGINE_PERSISTENT, gpu_lib.ENGINE_WAVEFRONT):
        gs.set_engine(eng)
        out[eng], _ = gs.draw_map(rq)
    a = out[gpu_lib.ENGINE_PLAIN]["L"]
    for eng in (gpu_lib.ENGINE_PERSISTENT, gpu_lib.ENGINE_WAVEFRONT):
        np.testing.assert_allclose(out[eng]["L"], a, rtol=1e-9, atol=0)


def test_terrain_in_batches(gpu_lib):
    """A batch that mixes a terrain scene with plane-ground scenes runs the
    mesh variant of the batched kernels and equals each map drawn alone on
    the plain engine, on the persistent and on the wavefront engine."""
    sc1, rq1 = S.config_c1(scale=10 / 64, spp=8)
    sc1 = S.with_terrain(sc1)
    rq1.cam_pos, rq1.cam_tgt, rq1.cam_up = (1600.0, -600.0, 700.0), (1600.0, 1600.0, 0.0), (0, 0, 1)
    sc2, rq2 = S.config_c1(scale=8 / 64, spp=8)
    sc3, rq3 = S.config_c2(scale=8 / 128, spp=16, cloud_def=(16, 16, 8))
    sc3 = S.with_terrain(sc3)
    rq3.rect_pos, rq3.rect_tgt = (800.0, 800.0, 75.0), (800.0, 800.0, 76.0)
    items = [(gpu_lib.GpuScene(sc1, 0b111), rq1), (gpu_lib.GpuScene(sc2, 0b111), rq2),
             (gpu_lib.GpuScene(sc3, 0b100), rq3)]
    alone = []
    for gs, rq in items:
        gs.set_engine(gpu_lib.ENGINE_PLAIN)
        alone.append(gs.draw_map(rq)[0])
    for eng in (gpu_lib.ENGINE_PERSISTENT, gpu_lib.ENGINE_WAVEFRONT):
        t = gpu_lib.default_tuning()
        t.engine = eng
        if eng == gpu_lib.ENGINE_WAVEFRONT:
            t.wave_tail, t.regroup_period, t.trace_budget = 100, 16, 64
        bufs, st = gpu_lib.draw_maps_batched(items, t)
        for b, a, (_, rq) in zip(bufs, alone, items):
            if rq.mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
                np.testing.assert_array_equal(b["n"], a["n"])
                np.testing.assert_allclose(b["sum"], a["sum"], rtol=1e-9, atol=0)
            else:
                np.testing.assert_allclose(b["L"], a["L"], rtol=1e-9, atol=0)
