"""Ground geometry (no GPU): the htrdr-obj reader and the oracle's mesh
queries and transport.

* the reader: polygon fans, negative indices, interfaces shared by groups,
  front:back and front:thin:back groups, materials and BRDF tables;
* ray queries on a flat quad against their closed-form answers: distance,
  the primitive left by the ray (self-hit), the range, the repeated tile;
* a flat repeated mesh with one material gives the plane ground's weights
  realisation by realisation (both draw the canonical that picks a BRDF at
  every surface event, as htrdr_mtl_create_bsdf does; the hit distances are
  FP32 on both) and so estimates the same radiance.
"""
import math

import numpy as np
import pytest

from htrdr_kmin_b200 import scene as S

FLAT_OBJ = """
v 0 0 0
v 1000 0 0
v 1000 1000 0
v 0 1000 0
usemtl air:ground
f 1 4 3 2
"""


def flat_mesh(refl=0.2, T=288.0, repeat=True, specular=False):
    mats = {"air": None, "ground": (T, [(500.0, "specular" if specular else "lambertian", refl)])}
    return S.parse_htrdr_obj(FLAT_OBJ, mats, sky_mtl="air", repeat=repeat)


def test_parse_htrdr_obj():
    obj = """# comment
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 2 0 0
usemtl a:b
f 1 2 3 4
usemtl a:c:b
f -1 -4 -3
usemtl a:b
f 1/1 3/3 2/2
"""
    mats = {"a": None, "b": (280.0, [(700.0, "lambertian", 0.3), (400.0, "specular", 0.1)]),
            "c": (300.0, [(500.0, "lambertian", 0.5)])}
    m = S.parse_htrdr_obj(obj, mats, sky_mtl="a")
    assert m.verts.shape == (5, 3)
    np.testing.assert_array_equal(m.tris, [[0, 1, 2], [0, 2, 3], [4, 1, 2], [0, 2, 1]])
    np.testing.assert_array_equal(m.tri_iface, [0, 0, 1, 0])
    np.testing.assert_array_equal(m.ifaces, [[0, S.NO_ID, 1], [0, 2, 1]])
    np.testing.assert_array_equal(m.mtl_nbrdf, [0, 2, 1])
    np.testing.assert_array_equal(m.mtl_temperature, [-1.0, 280.0, 300.0])
    # each material's table is sorted by wavelength
    np.testing.assert_array_equal(m.mtl_brdf, [[400.0, 1.0, 0.1], [700.0, 0.0, 0.3],
                                               [500.0, 0.0, 0.5]])
    assert m.sky_mtl == 0
    with pytest.raises(ValueError):
        S.parse_htrdr_obj("v 0 0 0\nf 1 1 1\n", mats)
    with pytest.raises(ValueError):
        S.parse_htrdr_obj("usemtl a:zzz\n", mats)


def test_terrain_winding_and_groups():
    m = S.with_terrain(S.config_c1(scale=12 / 64, spp=1)[0], n=8).ground_mesh
    v = m.verts[m.tris].astype(np.float64)
    N = np.cross(v[:, 2] - v[:, 0], v[:, 1] - v[:, 0])
    assert (N[:, 2] > 0).all()  # the front side (atmosphere) faces up
    assert set(np.unique(m.tri_iface)) == {0, 1}
    assert m.ifaces[:, 0].tolist() == [0, 0] and m.sky_mtl == 0


def _trace(os_, rays, tmax, from_prim=None, from_edge=None):
    n = len(rays)
    fp = np.full(n, S.NO_ID, np.uint32) if from_prim is None else from_prim
    fe = np.zeros(n, np.uint8) if from_edge is None else from_edge
    return os_.ground_trace(np.asarray(rays, np.float32), np.asarray(tmax, np.float32), fp, fe)


def _flat_scene(mesh):
    sc = S.homogeneous_slab(k_abs=1e-5, k_sca=1e-4, top=2000.0, ground_reflectivity=0.2,
                            ground_temperature=288.0)
    sc.ground_mesh = mesh
    return sc


def test_oracle_mesh_queries(oracle_lib):
    os_ = oracle_lib.OracleScene(_flat_scene(flat_mesh(repeat=False)))
    big = 1e30
    rays = [[300, 200, 50, 0, 0, -1],        # straight down: 50 m
            [300, 200, 50, 0, 0, 1],         # up: nothing
            [300, 200, 50, 0.6, 0, -0.8],    # slanted: 62.5 m
            [1500, 200, 50, 0, 0, -1],       # outside the quad
            [300, 200, -10, 0, 0, 1]]        # from below: 10 m, back side
    prim, dist = _trace(os_, rays, [big, big, big, big, big])
    assert prim[1] == S.NO_ID and prim[3] == S.NO_ID
    assert dist[1] == -1.0 and dist[3] == -1.0
    np.testing.assert_allclose(dist[[0, 2, 4]], [50.0, 62.5, 10.0], rtol=1e-6)
    assert prim[0] != S.NO_ID and prim[4] == prim[0]
    # the range is exclusive of its end
    p2, d2 = _trace(os_, rays[:1], [50.0])
    assert p2[0] == S.NO_ID
    p3, _ = _trace(os_, rays[:1], [50.001])
    assert p3[0] == prim[0]
    # a ray leaving a primitive never hits it again (self-hit rule), and a
    # hit at the start of the range is excluded
    p4, _ = _trace(os_, [[300, 200, 10, 0, 0, -1]], [big], np.array([prim[0]], np.uint32))
    assert p4[0] == S.NO_ID
    p5, _ = _trace(os_, [[300, 200, 10, 0, 0, -1]], [big])
    assert p5[0] == prim[0]
    p6, _ = _trace(os_, [[300, 200, 0, 0, 0, -1]], [big])
    assert p6[0] == S.NO_ID


def test_oracle_mesh_repeat(oracle_lib):
    os_ = oracle_lib.OracleScene(_flat_scene(flat_mesh(repeat=True)))
    rays = [[12345.5, -7777.25, 80, 0, 0, -1], [-2500, 300, 100, 0.6, 0.0, -0.8],
            [300, 200, 50, 0, 0, 1]]
    prim, dist = _trace(os_, rays, [1e30] * 3)
    np.testing.assert_allclose(dist[:2], [80.0, 125.0], rtol=1e-5)
    assert prim[2] == S.NO_ID
    # long grazing ray crossing many tiles before it comes down
    prim, dist = _trace(os_, [[100, 100, 100, 0.999, 0.0, -math.sqrt(1 - 0.999 ** 2)]], [1e30])
    expect = 100.0 / math.sqrt(1 - 0.999 ** 2)
    if expect / 1000.0 < 30:  # within the slab walk's 32 steps
        assert prim[0] != S.NO_ID
        np.testing.assert_allclose(dist[0], expect, rtol=1e-4)


def _three_sigma(bufs_a, bufs_b, keys):
    zs = []
    for k, se in keys:
        a, b = bufs_a[k].ravel(), bufs_b[k].ravel()
        s = np.sqrt(bufs_a[se].ravel() ** 2 + bufs_b[se].ravel() ** 2)
        m = s > 0
        zs.append((a[m] - b[m]) / s[m])
    return np.concatenate(zs)


@pytest.mark.parametrize("lw,specular", [(False, False), (True, False), (False, True)],
                         ids=["sw", "lw", "sw_specular"])
def test_flat_mesh_matches_plane(oracle_lib, lw, specular):
    """A flat repeated mesh = the plane ground (same BRDF, temperature)."""
    O = oracle_lib
    if lw:
        sc = S.homogeneous_slab(k_abs=2e-4, k_sca=1e-4, top=2000.0, temperature=260.0,
                                band=(9500.0, 10500.0), ground_reflectivity=0.3,
                                ground_temperature=288.0)
        rq = S.Request(mode=S.MODE_XWAVE_LW, width=6, height=6, spp=4000,
                       wlen_range=(10000.0, 10000.0), ref_temperature=288.0,
                       cam_pos=(100.0, 100.0, 500.0), cam_tgt=(400.0, 600.0, 0.0),
                       cam_up=(0.0, 0.0, 1.0), fov_deg=60.0, seed=7)
        mesh = flat_mesh(refl=0.3, T=288.0)
    else:
        sc = S.homogeneous_slab(k_abs=2e-5, k_sca=3e-4, top=2000.0, ground_reflectivity=0.4,
                                ground_temperature=288.0, sun_elevation=50.0)
        rq = S.Request(mode=S.MODE_XWAVE_SW, width=6, height=6, spp=4000,
                       wlen_range=(550.0, 550.0), cam_pos=(100.0, 100.0, 500.0),
                       cam_tgt=(400.0, 600.0, 0.0), cam_up=(0.0, 0.0, 1.0), fov_deg=60.0,
                       seed=7)
        mesh = flat_mesh(refl=0.4, T=288.0, specular=specular)
        if specular:
            sc.ground_brdf = S.BRDF_SPECULAR
    plane = O.OracleScene(sc)
    sm = _flat_scene(mesh)
    sm.layer_T, sm.gas_ka, sm.gas_ks = sc.layer_T, sc.gas_ka, sc.gas_ks
    sm.band_lo, sm.band_hi, sm.sun_elevation = sc.band_lo, sc.band_hi, sc.sun_elevation
    meshed = O.OracleScene(sm)
    npix = rq.width * rq.height
    wa = plane.realisation_weights(S.Request(**{**rq.__dict__, "spp": 200}), 0, npix)
    wb = meshed.realisation_weights(S.Request(**{**rq.__dict__, "spp": 200}), 0, npix)
    rel = np.abs(wa - wb) / np.maximum(np.abs(wa), 1e-300)
    assert np.all(rel <= 1e-6), rel.max()  # same streams, same events
    a, _ = plane.draw_map(rq)
    b, _ = meshed.draw_map(rq)
    assert np.all(a["L"] > 0) and np.all(b["L"] > 0)
    z = _three_sigma(a, b, [("L", "L_se")])
    print(f"{'lw' if lw else 'sw'}: max |z| {np.abs(z).max():.2f}, mean z {z.mean():.2f}")
    assert np.abs(z).max() < 4.0
    assert abs(z.mean()) < 3.0 / math.sqrt(len(z)) + 0.5


def test_flux_probe_rejection_under_terrain(oracle_lib):
    """Flux probes under the terrain surface are rejected (NaN weight),
    probes above it are kept."""
    O = oracle_lib
    sc = S.homogeneous_slab(k_abs=1e-5, k_sca=1e-4, top=2000.0)
    sc = S.with_terrain(sc, size=1000.0, n=8, amp=150.0, repeat=True)
    rq = S.Request(mode=S.MODE_FLUX_SW, width=4, height=4, spp=64, wlen_range=(550.0, 550.0),
                   rect_pos=(500.0, 500.0, 75.0), rect_tgt=(500.0, 500.0, 76.0),
                   rect_up=(0.0, 1.0, 0.0), rect_size=(1000.0, 1000.0), seed=3)
    w = O.OracleScene(sc).realisation_weights(rq, 0, rq.width * rq.height)
    rej = np.isnan(w).mean()
    assert 0.05 < rej < 0.95, rej


def test_parse_htrdr_materials():
    text = """# the example list of doc/htrdr-materials.5, with its BRDF tables
grass   /opt/materials/A001.mrumtl 300
sand    /opt/materials/B002.mrumtl 300   # trailing comment

air     none
"""
    tables = {"/opt/materials/A001.mrumtl": [(400.0, "lambertian", 0.05), (700.0, "lambertian", 0.4)],
              "/opt/materials/B002.mrumtl": [(550.0, "specular", 0.3)]}
    mats = S.parse_htrdr_materials(text, tables)
    assert list(mats) == ["grass", "sand", "air"]
    assert mats["air"] is None
    assert mats["grass"] == (300.0, tables["/opt/materials/A001.mrumtl"])
    m = S.parse_htrdr_obj(FLAT_OBJ.replace("air:ground", "air:grass"), mats, sky_mtl="air")
    np.testing.assert_array_equal(m.mtl_nbrdf, [2, 1, 0])
    np.testing.assert_array_equal(m.mtl_temperature, [300.0, 300.0, -1.0])
    assert m.sky_mtl == 2 and m.ifaces.tolist() == [[2, S.NO_ID, 0]]
    for bad in ("grass /x 300\ngrass /x 300\n", "grass /x\n", "grass /missing 300\n",
                "grass /x -4\n"):
        with pytest.raises(ValueError):
            S.parse_htrdr_materials(bad, {"/x": [(500.0, "lambertian", 0.1)]})
    with pytest.raises(ValueError):
        S.parse_htrdr_materials("g /x 300\n", {"/x": [(500.0, "glossy", 0.1)]})


def test_htrdr_obj_doc_examples():
    """The two examples of doc/htrdr-obj.5: a thin sheet of paper between
    air and concrete, and a wooden cube against a brick along Z."""
    paper = """v -1.0  -1.0  0
v -1.0   1.0  0
v  1.0  -1.0  0
v  1.0   1.0  0

usemtl air:paper:concrete
f 1 2 3
f 3 2 4
"""
    lam = (300.0, [(500.0, "lambertian", 0.5)])
    m = S.parse_htrdr_obj(paper, {"air": None, "paper": lam, "concrete": lam})
    assert m.ifaces.tolist() == [[0, 1, 2]] and m.tri_iface.tolist() == [0, 0]
    v = m.verts[m.tris].astype(np.float64)
    N = np.cross(v[:, 2] - v[:, 0], v[:, 1] - v[:, 0])
    assert np.all(N[:, 2] > 0)  # vertices clockwise seen from +z: the front faces +z
    cube = "\n".join(f"v {x} {y} {z}" for z in (0, 1) for y in (0, 1) for x in (0, 1)) + """
usemtl wood:air
f 1 3 2
f 2 3 4
f 1 5 3
f 3 5 7
f 5 6 7
f 7 6 8
f 4 8 2
f 2 8 6

usemtl wood:brick
f 3 7 4
f 4 7 8
f 1 2 5
f 5 2 6
"""
    m = S.parse_htrdr_obj(cube, {"wood": lam, "air": None, "brick": lam}, sky_mtl="air")
    assert m.tris.shape == (12, 3) and m.verts.shape == (8, 3)
    assert m.ifaces.tolist() == [[0, S.NO_ID, 1], [0, S.NO_ID, 2]]
    assert m.tri_iface.tolist() == [0] * 8 + [1] * 4
    # every face's front side (the wood) is inside the cube: the normal
    # (v2 - v0) x (v1 - v0) of the clockwise convention points inwards
    v = m.verts[m.tris].astype(np.float64)
    N = np.cross(v[:, 2] - v[:, 0], v[:, 1] - v[:, 0])
    out = v.mean(axis=1) - 0.5
    assert np.all(np.einsum("ij,ij->i", N, out) < 0)


def test_black_mesh_emits_planck(oracle_lib):
    """Closed form on the mesh: under a transparent atmosphere a camera that
    sees only a black (reflectivity 0) repeated mesh at temperature T
    measures B(lambda, T) exactly, every realisation."""
    O = oracle_lib
    T = 300.0
    sc = S.homogeneous_slab(k_abs=1e-30, k_sca=0.0, top=2000.0, temperature=250.0,
                            band=(9500.0, 10500.0))
    sc.ground_mesh = flat_mesh(refl=0.0, T=T, repeat=True)
    rq = S.Request(mode=S.MODE_XWAVE_LW, width=4, height=4, spp=8, wlen_range=(10000.0, 10000.0),
                   ref_temperature=T, cam_pos=(200.0, 300.0, 500.0), cam_tgt=(250.0, 350.0, 0.0),
                   cam_up=(0.0, 1.0, 0.0), fov_deg=30.0, seed=3)
    w = O.OracleScene(sc).realisation_weights(rq, 0, 16)
    B = O.lib().ora_planck_monochromatic(10000e-9, T)
    # weight = radiance / pdf(lambda) with a Dirac spectral domain: pdf 1 per nm
    np.testing.assert_allclose(w, B * 1e-9, rtol=1e-9)
