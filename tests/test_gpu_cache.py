"""The majorant-octree cache of option -O (htrdr_gpu_scene_create_cached).

* a first creation builds the octrees and writes the cache; a second one
  loads it: every tree is byte-identical and the realisation weights are
  bit-identical;
* a cache is loaded whatever -T and -V say (the doc of -O: they are ignored
  when the cache is used), and is refused for another medium (one cloud cell
  changed) or a file that is not a cache;
* the host and the GPU builders write caches that load to the same trees.
"""
import dataclasses
import os

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

pytestmark = pytest.mark.gpu


def _scene():
    sc, rq = S.config_c3(scale=8 / 512, spp=4, cloud_def=(32, 32, 8), nbands=3, nquad=2)
    return sc, rq


def _trees(gs, sc):
    out = []
    for b in range(sc.nbands):
        for q in range(int(sc.nquads[b])):
            for p in range(3):
                out.append(gs.tree(b, q, p))
    return out


def test_cache_round_trip(gpu_lib, tmp_path):
    sc, rq = _scene()
    path = str(tmp_path / "octrees.cache")
    built = gpu_lib.GpuScene(sc, 0b111, cache_path=path)
    assert os.path.getsize(path) > 64
    loaded = gpu_lib.GpuScene(sc, 0b111, cache_path=path)
    plain = gpu_lib.GpuScene(sc, 0b111)
    for a, b, c in zip(_trees(built, sc), _trees(loaded, sc), _trees(plain, sc)):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a, c)
    npix = rq.width * rq.height
    wa = built.realisation_weights(rq, 0, npix)
    wb = loaded.realisation_weights(rq, 0, npix)
    np.testing.assert_array_equal(wa.view(np.uint64), wb.view(np.uint64))


def test_cache_ignores_T_and_V(gpu_lib, tmp_path):
    sc, _ = _scene()
    path = str(tmp_path / "octrees.cache")
    first = gpu_lib.GpuScene(sc, 0b100, cache_path=path)
    other = dataclasses.replace(sc, optical_thickness=10.0, grid_max_definition=(8, 8, 8))
    rebuilt = gpu_lib.GpuScene(other, 0b100)
    loaded = gpu_lib.GpuScene(other, 0b100, cache_path=path)
    t_first, t_rebuilt, t_loaded = first.tree(0, 0, 2), rebuilt.tree(0, 0, 2), loaded.tree(0, 0, 2)
    assert t_first.shape != t_rebuilt.shape  # the options do change the build
    np.testing.assert_array_equal(t_loaded, t_first)


def test_cache_refuses_other_inputs(gpu_lib, tmp_path):
    sc, _ = _scene()
    path = str(tmp_path / "octrees.cache")
    gpu_lib.GpuScene(sc, 0b111, cache_path=path)
    lwc = sc.cloud_lwc.copy()
    lwc[3, 5, 7] += 1e-4
    other = dataclasses.replace(sc, cloud_lwc=lwc)
    with pytest.raises(gpu_lib.HtrdrError, match="other inputs"):
        gpu_lib.GpuScene(other, 0b111, cache_path=path)
    with pytest.raises(gpu_lib.HtrdrError, match="other inputs"):
        gpu_lib.GpuScene(sc, 0b100, cache_path=path)  # other octree properties
    bad = tmp_path / "not_a_cache"
    bad.write_bytes(b"x" * 200)
    with pytest.raises(gpu_lib.HtrdrError, match="not an octree cache"):
        gpu_lib.GpuScene(sc, 0b111, cache_path=str(bad))


def test_cache_host_and_gpu_builders(gpu_lib, tmp_path):
    sc, _ = _scene()
    p_gpu, p_host = str(tmp_path / "gpu.cache"), str(tmp_path / "host.cache")
    gpu_lib.GpuScene(sc, 0b111, cache_path=p_gpu)
    gpu_lib.GpuScene(sc, 0b111, octree_on_host=True, cache_path=p_host)
    a = gpu_lib.GpuScene(sc, 0b111, cache_path=p_gpu)
    b = gpu_lib.GpuScene(sc, 0b111, cache_path=p_host)
    for x, y in zip(_trees(a, sc), _trees(b, sc)):
        np.testing.assert_array_equal(x, y)


def test_cache_truncated(gpu_lib, tmp_path):
    sc, _ = _scene()
    path = tmp_path / "octrees.cache"
    gpu_lib.GpuScene(sc, 0b100, cache_path=str(path))
    data = path.read_bytes()
    path.write_bytes(data[:-16])
    with pytest.raises(gpu_lib.HtrdrError, match="size does not match"):
        gpu_lib.GpuScene(sc, 0b100, cache_path=str(path))
