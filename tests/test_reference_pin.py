"""The oracle pinned to the reference's own code (CPU).

oracle/_ref/libhtrdr_ref.so holds the reference's atmosphere hot-path C files
compiled unmodified (src/atmosphere/htrdr_atmosphere_compute_radiance_{sw,lw}.c,
src/atmosphere/htrdr_atmosphere_draw_map.c, ..._sun.c,
src/core/htrdr_ran_wlen_{planck,cie_xyz}.c, src/core/htrdr_spectral.c,
src/core/htrdr_rectangle.c, src/core/htrdr_buffer.c) over project-written
shims of their absent dependencies, which answer with the oracle's medium,
octrees and random streams (oracle/ref).  Both consume one stream per
(pixel, realisation) in the reference's draw order, so:

* every realisation weight of the oracle equals the reference's to within
  FP64 rounding (the only differences left are the order of a few products);
* per-pixel estimates, standard errors and LW brightness temperatures agree
  to the same precision, and the reference's dump_buffer text equals what
  htrdr_gpu_write_image prints for the reference's own buffer;
* with independent streams the two agree within 3 combined standard errors
  at the full flux-map size.

The library is built from the reference tree when it is present; the tests
are skipped where neither the tree nor a built library is available.
"""
import math
import os
import sys

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_ref_golden as G  # noqa: E402

# FP64 on both sides: the relative difference allowed for one realisation
REL = 1e-6


@pytest.fixture(scope="module")
def ref_lib():
    from oracle import reference as R
    if not R.available():
        pytest.skip("compiled reference oracle unavailable (no reference tree, no built library)")
    return R


def cases():
    return G.reference_cases()


def _ids(v):
    return v if isinstance(v, str) else ""


@pytest.mark.parametrize("name,scene,req,props", cases(), ids=_ids)
def test_oracle_realisations_equal_the_reference(ref_lib, oracle_lib, name, scene, req, props):
    npix = req.width * req.height
    wr = ref_lib.RefScene(scene, props).realisation_weights(req, 0, npix)
    wo = oracle_lib.OracleScene(scene, props).realisation_weights(req, 0, npix)
    np.testing.assert_array_equal(np.isnan(wr), np.isnan(wo))  # same rejected probes
    ok = ~np.isnan(wr)
    r, o = wr[ok], wo[ok]
    rel = np.abs(o - r) / np.maximum(np.abs(r), 1e-300)
    frac = float(np.mean(rel <= REL))
    print(f"{name}: {ok.sum()} realisations, {frac:.4f} within {REL}, "
          f"{np.mean(o == r):.4f} bit-equal, max rel {rel.max():.2e}")
    assert np.all(r >= 0)
    assert frac == 1.0, (frac, rel.max())


def _estimates(buf, mode):
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        n = np.maximum(buf["n"].astype(np.float64), 1)
        E = buf["sum"] / n
        return [(E, np.sqrt(np.maximum(buf["sum2"] / n - E * E, 0) / n))]
    if mode == S.MODE_IMAGE_CIE:
        return [(buf[c], buf[c + "_se"]) for c in ("X", "Y", "Z")]
    return [(buf["L"], buf["L_se"])]


@pytest.mark.parametrize("name,scene,req,props", cases(), ids=_ids)
def test_oracle_maps_equal_the_reference(ref_lib, oracle_lib, name, scene, req, props):
    """The reference's atmosphere_draw_map (its pixel callbacks accumulating
    spp realisations, SE, brightness temperature) against the oracle's."""
    br = ref_lib.RefScene(scene, props).draw_map(req)
    bo, _ = oracle_lib.OracleScene(scene, props).draw_map(req)
    if req.mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        np.testing.assert_array_equal(br["n"], bo["n"])
    np.testing.assert_array_equal(br["t_n"], bo["t_n"])
    for (Er, SEr), (Eo, SEo) in zip(_estimates(br, req.mode), _estimates(bo, req.mode)):
        np.testing.assert_allclose(Eo, Er, rtol=REL, atol=0)
        np.testing.assert_allclose(SEo, SEr, rtol=1e-4, atol=1e-12 * float(np.abs(Er).max()))
    if req.mode == S.MODE_XWAVE_LW:  # htrdr_brightness_temperature (src/core/htrdr_spectral.c:31-89)
        assert np.all(br["Tb"] > 0)
        np.testing.assert_allclose(bo["Tb"], br["Tb"], rtol=1e-6, atol=0)
        np.testing.assert_allclose(bo["Tb_se"], br["Tb_se"], rtol=1e-3, atol=1e-6)


@pytest.mark.parametrize("name,scene,req,props", cases()[:5], ids=_ids)
def test_reference_dump_equals_the_image_writer(ref_lib, tmp_path, name, scene, req, props):
    """dump_buffer of the reference (src/atmosphere/htrdr_atmosphere_draw_map.c:477-587)
    and htrdr_gpu_write_image print the same bytes for the same pixels."""
    from htrdr_kmin_b200 import api, build
    build.build()
    ref_path = str(tmp_path / "ref.txt")
    ours_path = str(tmp_path / "ours.txt")
    buf = ref_lib.RefScene(scene, props).draw_map(req, dump_path=ref_path)
    mine = np.frombuffer(buf.tobytes(), dtype=api.pixel_dtype(req.mode)).reshape(buf.shape)
    api.write_image(req.mode, mine, ours_path)
    with open(ref_path, "rb") as f:
        ref_bytes = f.read()
    with open(ours_path, "rb") as f:
        ours_bytes = f.read()
    assert ref_bytes.startswith(b"%d %d\n" % (req.width, req.height))
    assert ours_bytes == ref_bytes


def test_full_size_flux_map_three_sigma(ref_lib, oracle_lib):
    """The LW flux map at its full size (128 x 128 probes, 16 x 8 correlated-k,
    64 x 64 x 32 cloud) at 16 realisations per probe: the reference and the
    oracle on independent streams agree within 3 combined standard errors."""
    sc, rq = S.config_c2(spp=16)
    br = ref_lib.RefScene(sc, 0b100).draw_map(S.Request(**{**rq.__dict__, "seed": 71}))
    bo, _ = oracle_lib.OracleScene(sc, 0b100).draw_map(S.Request(**{**rq.__dict__, "seed": 72}))
    (Er, SEr), = _estimates(br, rq.mode)
    (Eo, SEo), = _estimates(bo, rq.mode)
    s = np.sqrt(SEr ** 2 + SEo ** 2)
    m = s > 0
    z = ((Eo - Er)[m] / s[m]).ravel()
    n = z.size
    fail = float(np.mean(np.abs(z) > 3))
    print(f"full-size flux map: {n} probes, |z|>3 fraction {fail:.4f}, mean z {z.mean():+.4f}")
    assert n > 16000
    assert fail <= 3 * 0.0027 + 3 * math.sqrt(0.0027 / n)
    assert abs(z.mean()) < 5.0 / math.sqrt(n) + 0.02


@pytest.mark.parametrize("name,scene,req,props", cases(), ids=_ids)
def test_golden_vectors_are_the_reference_outputs(ref_lib, name, scene, req, props):
    """tests/golden/reference_realisations.npz (read by the GPU tests) holds
    what the compiled reference computes now."""
    golden = np.load(G.OUT)
    rs = ref_lib.RefScene(scene, props)
    npix = req.width * req.height
    np.testing.assert_array_equal(rs.realisation_weights(req, 0, npix), golden[f"{name}/weights"])
    mq = S.Request(**{**req.__dict__, "seed": G.MAP_SEED, "spp": G.MAP_SPP[name]})
    for k, v in G.map_fields(rs.draw_map(mq), req.mode).items():
        np.testing.assert_array_equal(v, golden[f"{name}/map_{k}"])


def _batched_cases():
    """The request kinds of the batched workloads (8 bands x 4 points, SW and
    LW bands in one scene, repeated power-law cloud) on a reduced scene."""
    sc = S.batched_scenes(scale=1 / 16)[1]
    reqs = S.batched_requests(n=2, side_range=(6, 6), spp_range=(8, 8))
    return [("batched_sw", sc, reqs[0][1], 0b111), ("batched_lw", sc, reqs[1][1], 0b111)]


@pytest.mark.parametrize("name,scene,req,props", _batched_cases(), ids=_ids)
def test_batched_kinds_equal_the_reference(ref_lib, oracle_lib, name, scene, req, props):
    npix = req.width * req.height
    wr = ref_lib.RefScene(scene, props).realisation_weights(req, 0, npix)
    wo = oracle_lib.OracleScene(scene, props).realisation_weights(req, 0, npix)
    np.testing.assert_array_equal(np.isnan(wr), np.isnan(wo))
    rel = np.abs(wo - wr) / np.maximum(np.abs(wr), 1e-300)
    print(f"{name}: {wr.size} realisations, max rel {np.nanmax(rel):.2e}")
    assert np.nanmax(rel) <= REL
