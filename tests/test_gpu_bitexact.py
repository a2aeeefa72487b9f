"""Bit-exact integer work, CUDA library vs CPU oracle on identical inputs:
majorant octrees (node arrays byte for byte), octree point location, band
lookup, quadrature-point selection and the wavelength CDF searches."""
import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu


def small_scenes():
    c1, _ = S.config_c1()
    c2, _ = S.config_c2(cloud_def=(32, 32, 16))
    c3, _ = S.config_c3(cloud_def=(48, 40, 12), nbands=4, nquad=3)
    capped, _ = S.config_c1()
    capped.grid_max_definition = (8, 16, 4)
    nomerge, _ = S.config_c1()
    nomerge.optical_thickness = 0.0
    ragged, _ = S.config_c3(cloud_def=(37, 5, 9), nbands=2, nquad=2)
    return [("c1", c1, 0b111), ("c2", c2, 0b100), ("c3", c3, 0b111), ("capped", capped, 0b111),
            ("nomerge", nomerge, 0b111), ("ragged", ragged, 0b111)]


@pytest.mark.parametrize("name,scene,props", small_scenes(), ids=lambda v: v if isinstance(v, str) else "")
def test_octrees_identical(gpu_lib, oracle_lib, name, scene, props):
    gs = gpu_lib.GpuScene(scene, props)
    os_ = oracle_lib.OracleScene(scene, props)
    assert gs.depth() == os_.depth()
    for b in range(scene.nbands):
        for q in range(int(scene.nquads[b])):
            for p in range(3):
                if not props & (1 << p):
                    continue
                g = gs.tree(b, q, p)
                c = os_.tree(b, q, p)
                assert len(g) == len(c), (name, b, q, p)
                assert g.tobytes() == c.tobytes(), (name, b, q, p)
                # structural sanity: kmin <= kmax everywhere
                assert np.all(g["kmin"] <= g["kmax"])


def test_gpu_builder_matches_host_builder(gpu_lib):
    """The GPU octree builder and the host builder emit the same node arrays
    (and both match the oracle above) on a multi-band scene with -V and a
    ragged grid."""
    import time
    scene, _ = S.config_c3(cloud_def=(96, 80, 24), nbands=5, nquad=4)
    scene.grid_max_definition = (64, 0, 0)
    t0 = time.time()
    g = gpu_lib.GpuScene(scene)
    t1 = time.time()
    h = gpu_lib.GpuScene(scene, octree_on_host=True)
    t2 = time.time()
    print(f"octrees: GPU build {t1 - t0:.3f} s, host build {t2 - t1:.3f} s, {g.device_bytes / 1e6:.1f} MB")
    for b in range(scene.nbands):
        for q in range(int(scene.nquads[b])):
            for p in range(3):
                assert g.tree(b, q, p).tobytes() == h.tree(b, q, p).tobytes(), (b, q, p)


def test_locate_leaf_identical(gpu_lib, oracle_lib):
    scene, _ = S.config_c3(cloud_def=(48, 40, 12), nbands=2, nquad=2)
    gs = gpu_lib.GpuScene(scene)
    os_ = oracle_lib.OracleScene(scene)
    nx, ny, nz = scene.cloud_def
    cells = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                     -1).reshape(-1, 3).astype(np.uint32)
    for prop in (0, 1, 2):
        node, level = gs.locate_leaf(1, 1, prop, cells)
        sel = np.random.default_rng(prop).choice(len(cells), 500, replace=False)
        for i in sel:
            n, lv = os_.locate_leaf(1, 1, prop, cells[i])
            assert (int(node[i]), int(level[i])) == (n, lv)
        tree = gs.tree(1, 1, prop)
        assert np.all(tree["child"][node] == 0xFFFFFFFF)  # always a leaf


def test_find_band_and_quadrature_identical(gpu_lib, oracle_lib):
    scene, _ = S.config_c2(cloud_def=(4, 4, 2))
    gs = gpu_lib.GpuScene(scene, 0b100)
    os_ = oracle_lib.OracleScene(scene, 0b100)
    rng = np.random.default_rng(5)
    edges = np.concatenate([scene.band_lo, scene.band_hi])
    wl = np.concatenate([rng.uniform(2900.0, 101000.0, 4000), edges, np.nextafter(edges, 0),
                         np.nextafter(edges, np.inf)])
    g = gs.find_band(wl)
    c = np.array([os_.find_band(w) for w in wl], dtype=np.uint32)
    np.testing.assert_array_equal(g, c)
    iband = rng.integers(0, scene.nbands, 4000).astype(np.uint32)
    cum = np.cumsum(scene.quad_w.reshape(scene.nbands, -1), axis=1)
    r = np.concatenate([rng.random(4000), cum[iband % scene.nbands, 3]])
    ib = np.concatenate([iband, iband]).astype(np.uint32)
    g = gs.sample_quad(r, ib)
    c = np.array([os_.sample_quad(float(x), int(b)) for x, b in zip(r, ib)], dtype=np.uint32)
    np.testing.assert_array_equal(g, c)


@pytest.mark.parametrize("mode", [S.MODE_FLUX_LW, S.MODE_XWAVE_SW, S.MODE_IMAGE_CIE])
def test_wavelength_cdf_search_identical(gpu_lib, oracle_lib, mode):
    if mode == S.MODE_FLUX_LW:
        scene, req = S.config_c2(cloud_def=(4, 4, 2))
        props = 0b100
    elif mode == S.MODE_IMAGE_CIE:
        scene, req = S.config_c3(cloud_def=(4, 4, 2), nbands=30, nquad=2)
        props = 0b111
    else:
        scene, req = S.config_c3(cloud_def=(4, 4, 2), nbands=30, nquad=2)
        req.mode = S.MODE_XWAVE_SW
        req.wlen_range = (400.0, 700.0)
        props = 0b111
    gs = gpu_lib.GpuScene(scene, props)
    os_ = oracle_lib.OracleScene(scene, props)
    rng = np.random.default_rng(9)
    r0 = rng.random(20000)
    r1 = rng.random(20000)
    for ch in (0, 1, 2) if mode == S.MODE_IMAGE_CIE else (0,):
        gcb, gwl, gpdf = gs.sample_wavelength(req, ch, r0, r1)
        ccb, cwl, cpdf = os_.sample_wavelength(req, ch, r0, r1)
        np.testing.assert_array_equal(gcb, ccb)
        np.testing.assert_allclose(gwl, cwl, rtol=1e-12)
        np.testing.assert_allclose(gpdf, cpdf, rtol=1e-12)
