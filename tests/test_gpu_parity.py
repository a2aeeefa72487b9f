"""Parity of the CUDA path with the CPU oracle (FP32 transport vs FP64).

* matched streams: both sides consume the same Philox stream per (pixel,
  realisation), so most realisations give the same weight up to FP32
  rounding; a path whose branch flips on a rounding difference diverges;
* independent streams: every per-pixel estimate agrees within 3 combined
  standard errors (failure fraction consistent with 0.27 %, mean z ~ 0);
* closed-form FP64 slabs: Beer-Lambert, isothermal absorbing slab radiance
  and flux, thin single-scattering slab.
"""
import math

import numpy as np
import pytest
from scipy.special import expn

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu

# Tolerance of a matched realisation: FP32 transport against FP64
MATCH_RTOL = 2e-3


def requests():
    out = []
    sc, rq = S.config_c1(scale=12 / 64, spp=8)
    out.append(("xwave_sw", sc, rq, 0b111))
    sc, rq = S.config_c2(scale=8 / 128, spp=16, cloud_def=(16, 16, 8))
    out.append(("flux_lw", sc, rq, 0b100))
    sc, rq = S.config_c3(scale=8 / 512, spp=4, cloud_def=(32, 32, 8), nbands=6, nquad=3)
    out.append(("image_cie", sc, rq, 0b111))
    sc, rq = S.config_c1(scale=8 / 64, spp=8)
    rq.mode = S.MODE_FLUX_SW
    rq.rect_pos, rq.rect_tgt, rq.rect_up, rq.rect_size = (1600, 1600, 0), (1600, 1600, 1), (0, 1, 0), (3200, 3200)
    out.append(("flux_sw", sc, rq, 0b111))
    sc, rq = S.config_c2(scale=8 / 128, spp=16, cloud_def=(16, 16, 8))
    rq.mode = S.MODE_XWAVE_LW
    rq.cam_pos, rq.cam_tgt, rq.cam_up = (800, 800, 10), (900, 900, 1500), (0, 1, 0)
    out.append(("xwave_lw", sc, rq, 0b100))
    return out


@pytest.mark.parametrize("name,scene,req,props", requests(), ids=lambda v: v if isinstance(v, str) else "")
def test_matched_stream_realisations(gpu_lib, oracle_lib, name, scene, req, props):
    gs = gpu_lib.GpuScene(scene, props)
    os_ = oracle_lib.OracleScene(scene, props)
    npix = req.width * req.height
    wg = gs.realisation_weights(req, 0, npix)
    wc = os_.realisation_weights(req, 0, npix)
    # rejected samples (NaN) are the same on both sides
    np.testing.assert_array_equal(np.isnan(wg), np.isnan(wc))
    ok = ~np.isnan(wc)
    g, c = wg[ok], wc[ok]
    scale = max(np.abs(c).mean(), 1e-300)
    close = np.abs(g - c) <= MATCH_RTOL * np.maximum(np.abs(c), 1e-6 * scale)
    frac = close.mean()
    print(f"{name}: {frac:.4f} of {close.size} realisations match within {MATCH_RTOL}")
    assert frac >= 0.9, frac


def estimates(buf, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        n = buf["n"].astype(np.float64)
        E = buf["sum"] / np.maximum(n, 1)
        V = np.maximum(buf["sum2"] / np.maximum(n, 1) - E * E, 0)
        return [(E.ravel(), np.sqrt(V / np.maximum(n, 1)).ravel())]
    if mode == S.MODE_IMAGE_CIE:
        return [(buf[c].ravel(), buf[c + "_se"].ravel()) for c in ("X", "Y", "Z")]
    return [(buf["L"].ravel(), buf["L_se"].ravel())]


def three_sigma(est_g, est_c):
    zs = []
    for (Eg, SEg), (Ec, SEc) in zip(est_g, est_c):
        s = np.sqrt(SEg ** 2 + SEc ** 2)
        m = s > 0
        zs.append((Eg[m] - Ec[m]) / s[m])
    z = np.concatenate(zs)
    return z


@pytest.mark.parametrize("name,scene,req,props", requests(), ids=lambda v: v if isinstance(v, str) else "")
def test_independent_three_sigma(gpu_lib, oracle_lib, name, scene, req, props):
    req.spp = max(req.spp, 128 if req.mode != S.MODE_IMAGE_CIE else 48)
    gs = gpu_lib.GpuScene(scene, props)
    os_ = oracle_lib.OracleScene(scene, props)
    rg = S.Request(**{**req.__dict__, "seed": 1001})
    rc = S.Request(**{**req.__dict__, "seed": 2002})
    bg, st = gs.draw_map(rg)
    bc, _ = os_.draw_map(rc)
    z = three_sigma(estimates(bg, req.mode), estimates(bc, req.mode))
    n = z.size
    assert n > 0
    fail = np.mean(np.abs(z) > 3)
    print(f"{name}: {n} estimates, |z|>3 fraction {fail:.4f}, mean z {z.mean():+.3f}, "
          f"stats {st}")
    # heavy-tailed weights make SE estimates noisy at low spp: allow 3x the
    # Gaussian 0.27 % plus binomial noise, and a mean z within 5/sqrt(n)
    assert fail <= 3 * 0.0027 + 3 * math.sqrt(0.0027 / n) + 1.0 / n
    assert abs(z.mean()) < 5.0 / math.sqrt(n) + 0.05


def test_beer_lambert_direct_gpu(gpu_lib, oracle_lib):
    k, H, el = 2e-4, 3000.0, 50.0
    sc = S.homogeneous_slab(k_abs=k, top=H, sun_elevation=el)
    gs = gpu_lib.GpuScene(sc)
    mu = math.sin(math.radians(el))
    sd = np.array([math.cos(math.radians(el)), 0.0, mu])
    z0 = np.array([0.0, 250.0, 1200.0])
    pos = np.stack([np.zeros(3), np.zeros(3), z0], axis=1)
    w = gs.radiance_sw(pos, np.tile(sd, (3, 1)), np.full(3, 550.0), np.zeros(3), np.zeros(3),
                       mask=gpu_lib.DIRECT)
    Lsun = oracle_lib.lib().ora_planck_monochromatic(550e-9, 5778.0)
    expect = Lsun * np.exp(-float(np.float32(k)) * (H - z0) / mu)
    # FP32 distances, FP64 optical depth: error ~ 1e-6 relative
    np.testing.assert_allclose(w, expect, rtol=2e-6)


def test_isothermal_slab_radiance_gpu(gpu_lib, oracle_lib):
    k, H, T = 3e-4, 2000.0, 260.0
    sc = S.homogeneous_slab(k_abs=k, top=H, temperature=T, band=(9000.0, 11000.0), ground_temperature=0.0)
    gs = gpu_lib.GpuScene(sc, 0b100)
    n = 1 << 20
    th = math.radians(35.0)
    d = np.array([math.sin(th), 0.0, math.cos(th)])
    w = gs.radiance_lw(np.zeros((n, 3)), np.tile(d, (n, 1)), np.full(n, 10000.0), np.zeros(n),
                       np.zeros(n), seed=7)
    B = oracle_lib.lib().ora_planck_monochromatic(10e-6, T)
    expect = B * (1.0 - math.exp(-float(np.float32(k)) * H / math.cos(th)))
    se = w.std() / math.sqrt(n)
    print("isothermal radiance", w.mean(), expect, se)
    assert abs(w.mean() - expect) < 4 * se


def test_isothermal_slab_flux_gpu(gpu_lib, oracle_lib):
    k, H, T = 2e-4, 2500.0, 270.0
    tau = float(np.float32(k)) * H
    sc = S.homogeneous_slab(k_abs=k, top=H, temperature=T, band=(9000.0, 11000.0), ground_temperature=0.0)
    gs = gpu_lib.GpuScene(sc, 0b100)
    req = S.Request(mode=S.MODE_FLUX_LW, width=16, height=16, spp=4096, wlen_range=(10000.0, 10000.0),
                    ref_temperature=290.0, rect_pos=(0, 0, 0), rect_tgt=(0, 0, 1), rect_up=(0, 1, 0),
                    rect_size=(100.0, 100.0), seed=11)
    buf, _ = gs.draw_map(req)
    tot, tot2, n = buf["sum"].sum(), buf["sum2"].sum(), buf["n"].sum()
    E = tot / n
    se = math.sqrt(max(tot2 / n - E * E, 0) / n)
    B = oracle_lib.lib().ora_planck_monochromatic(10e-6, T)
    expect = math.pi * B * (1.0 - 2.0 * expn(3, tau)) * 1e-9
    print("isothermal flux", E, expect, se, "error", (E - expect) / expect)
    assert abs(E - expect) < 4 * se


def test_single_scattering_slab_gpu(gpu_lib, oracle_lib):
    ks, H, el = 1e-5, 1000.0, 60.0
    tau = ks * H
    sc = S.homogeneous_slab(k_abs=0.0, k_sca=ks, top=H, sun_elevation=el, ground_reflectivity=0.0)
    gs = gpu_lib.GpuScene(sc)
    n = 1 << 21
    w = gs.radiance_sw(np.zeros((n, 3)), np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, 550.0),
                       np.zeros(n), np.zeros(n), mask=gpu_lib.DIFFUSE, seed=3)
    Lsun = oracle_lib.lib().ora_planck_monochromatic(550e-9, 5778.0)
    om = 2 * math.pi * (1 - math.cos(4.6524e-3))
    mu0 = math.sin(math.radians(el))
    p = 3 / (16 * math.pi) * (1 + mu0 ** 2)
    L1 = Lsun * om * p * (math.exp(-tau) - math.exp(-tau / mu0)) / (1 / mu0 - 1)
    se = w.std() / math.sqrt(n)
    print("single scattering", w.mean(), L1, se, "rel", w.mean() / L1 - 1)
    assert abs(w.mean() - L1) < 2 * tau * L1 + 4 * se
