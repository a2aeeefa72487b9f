"""The CUDA path against the reference's own outputs (golden vectors).

tests/golden/reference_realisations.npz holds what the reference's atmosphere
hot-path C files, compiled unmodified over the oracle's scenes, compute for
the parity cases (tests/golden/make_ref_golden.py): every realisation weight
of a map on the streams {pixel, seed} x realisation, and a map of
``MAP_SPP`` realisations per pixel at seed ``MAP_SEED``.

* matched streams: the GPU consumes the same streams in the same order, so
  most realisations give the reference's weight up to FP32 transport
  rounding (MATCH_RTOL); a realisation whose branch flips on a rounding
  difference diverges.  Rejected flux probes (NaN) are the same on both;
* independent streams: every per-pixel estimate of the GPU at another seed
  agrees with the reference's within 3 combined standard errors;
* brightness temperature: the GPU's per-pixel Tb (FP64 bisection after the
  map, htrdr_brightness_temperature, src/core/htrdr_spectral.c:31-89) is that
  of its radiance, and on the reference's own streams the reference's Tb.
"""
import math
import os
import sys

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_ref_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu

MATCH_RTOL = 2e-3
GOLDEN = np.load(G.OUT)


def _ids(v):
    return v if isinstance(v, str) else ""


@pytest.mark.parametrize("name,scene,req,props", G.reference_cases(), ids=_ids)
def test_gpu_realisations_match_the_reference(gpu_lib, name, scene, req, props):
    gs = gpu_lib.GpuScene(scene, props)
    npix = req.width * req.height
    wg = gs.realisation_weights(req, 0, npix)
    wr = GOLDEN[f"{name}/weights"]
    np.testing.assert_array_equal(np.isnan(wg), np.isnan(wr))
    ok = ~np.isnan(wr)
    g, r = wg[ok], wr[ok]
    scale = max(np.abs(r).mean(), 1e-300)
    close = np.abs(g - r) <= MATCH_RTOL * np.maximum(np.abs(r), 1e-6 * scale)
    print(f"{name}: {close.mean():.4f} of {close.size} realisations match the reference "
          f"within {MATCH_RTOL}")
    assert close.mean() >= 0.9
    gs.close()


def _gpu_fields(buf, mode):
    return G.map_fields(buf, mode)


def _pairs(mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW) or mode in (S.MODE_XWAVE_SW, S.MODE_XWAVE_LW):
        return [("E", "SE")]
    return [("X", "X_se"), ("Y", "Y_se"), ("Z", "Z_se")]


@pytest.mark.parametrize("name,scene,req,props", G.reference_cases(), ids=_ids)
def test_gpu_maps_agree_with_the_reference(gpu_lib, name, scene, req, props):
    gs = gpu_lib.GpuScene(scene, props)
    rq = S.Request(**{**req.__dict__, "seed": G.MAP_SEED + 1, "spp": G.MAP_SPP[name]})
    buf, _ = gs.draw_map(rq)
    fg = _gpu_fields(buf, req.mode)
    zs = []
    for e, se in _pairs(req.mode):
        Er, SEr = GOLDEN[f"{name}/map_{e}"], GOLDEN[f"{name}/map_{se}"]
        s = np.sqrt(fg[se] ** 2 + SEr ** 2)
        m = s > 0
        zs.append(((fg[e] - Er)[m] / s[m]).ravel())
    z = np.concatenate(zs)
    n = z.size
    fail = float(np.mean(np.abs(z) > 3))
    print(f"{name}: {n} estimates, |z|>3 fraction {fail:.4f}, mean z {z.mean():+.3f}")
    assert n > 0
    assert fail <= 3 * 0.0027 + 3 * math.sqrt(0.0027 / n) + 1.0 / n
    assert abs(z.mean()) < 5.0 / math.sqrt(n) + 0.05
    gs.close()


def test_gpu_brightness_temperature_equals_the_reference(gpu_lib, oracle_lib):
    """LW image on the reference's own streams: the radiance agrees with the
    reference's pixel by pixel (most realisations are the same; a branch
    flipped by FP32 rounding moves a pixel within its standard error), and
    the brightness temperature the GPU derives from its radiance by its FP64
    bisection is htrdr_brightness_temperature of that radiance (the oracle's
    restatement, itself equal to the compiled reference's), and the
    reference's own Tb wherever the radiance is the same."""
    name, scene, req, props = [c for c in G.reference_cases() if c[0] == "xwave_lw"][0]
    gs = gpu_lib.GpuScene(scene, props)
    rq = S.Request(**{**req.__dict__, "seed": G.MAP_SEED, "spp": G.MAP_SPP[name]})
    buf, _ = gs.draw_map(rq)
    L_ref, SE_ref = GOLDEN[f"{name}/map_E"], GOLDEN[f"{name}/map_SE"]
    Tb_ref = GOLDEN[f"{name}/map_Tb"]
    assert np.all(Tb_ref > 150) and np.all(Tb_ref < 330)
    L, SE, Tb, Tb_se = buf["L"], buf["L_se"], buf["Tb"], buf["Tb_se"]
    assert np.all(np.abs(L - L_ref) <= 3 * np.sqrt(SE ** 2 + SE_ref ** 2))
    same = np.abs(L / L_ref - 1) <= 1e-4
    print(f"Tb: {same.mean():.3f} of the pixels have the reference's radiance to 1e-4")
    assert same.sum() >= 8  # long LW walks in the cloud: a quarter of the pixels measured
    # dTb/Tb = (lambda T / c2) dL/L at most, about 0.2 dL/L here
    np.testing.assert_allclose(Tb[same], Tb_ref[same], rtol=3e-5)
    lo, hi = rq.wlen_range[0] * 1e-9, rq.wlen_range[1] * 1e-9
    T = oracle_lib.lib().ora_radiance_temperature
    expect = np.array([T(lo, hi, float(x)) for x in L.ravel()]).reshape(L.shape)
    np.testing.assert_allclose(Tb, expect, rtol=1e-7)
    e_se = np.array([T(lo, hi, float(a + b)) - T(lo, hi, float(a - b))
                     for a, b in zip(L.ravel(), SE.ravel())]).reshape(L.shape)
    np.testing.assert_allclose(Tb_se, e_se, rtol=1e-5, atol=1e-7)
    gs.close()
