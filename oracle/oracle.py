"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: a plain-C, FP64-transport restatement of the
reference's atmosphere path, used by tests/, the smoke check and the CPU
baseline of bench.py.  Pinned to the reference's own code compiled unmodified
(oracle/reference.py, tests/test_reference_pin.py: equal realisation by
realisation) and to closed-form FP64 solutions (tests/test_oracle_pins.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

KA, KS, KEXT = 0, 1, 2
DIRECT, DIFFUSE, ALL = 1, 2, 3


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP); make skips it when
    the library is up to date.  Without make (or a compiler) an existing build
    is used as is."""
    try:
        subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []), check=True)
    except (OSError, subprocess.CalledProcessError):
        if not os.path.exists(_LIB_PATH):
            raise
    return _LIB_PATH


class SceneDesc(C.Structure):
    _fields_ = [
        ("nlayers", C.c_uint32), ("layer_z", C.POINTER(C.c_double)),
        ("layer_T", C.POINTER(C.c_float)), ("nbands", C.c_uint32),
        ("band_lo", C.POINTER(C.c_double)), ("band_hi", C.POINTER(C.c_double)),
        ("nquads", C.POINTER(C.c_uint32)), ("quad_w", C.POINTER(C.c_double)),
        ("gas_ka", C.POINTER(C.c_float)), ("gas_ks", C.POINTER(C.c_float)),
        ("cloud_def", C.c_uint32 * 3), ("cloud_lower", C.c_double * 3),
        ("cloud_cell", C.c_double * 3), ("cloud_lwc", C.POINTER(C.c_float)),
        ("cloud_sigma_ext", C.POINTER(C.c_float)), ("cloud_ssa", C.POINTER(C.c_float)),
        ("cloud_g", C.POINTER(C.c_float)), ("repeat_clouds", C.c_int32),
        ("optical_thickness", C.c_double), ("grid_max_definition", C.c_uint32 * 3),
        ("has_ground", C.c_int32), ("ground_brdf", C.c_int32),
        ("ground_reflectivity", C.c_double), ("ground_temperature", C.c_double),
        ("sun_azimuth", C.c_double), ("sun_elevation", C.c_double),
        ("props_mask", C.c_uint32),
        ("ground_nverts", C.c_uint32), ("ground_verts", C.POINTER(C.c_float)),
        ("ground_ntris", C.c_uint32), ("ground_tris", C.POINTER(C.c_uint32)),
        ("ground_tri_iface", C.POINTER(C.c_uint32)), ("ground_nifaces", C.c_uint32),
        ("ground_ifaces", C.POINTER(C.c_uint32)), ("ground_nmtls", C.c_uint32),
        ("ground_mtl_temperature", C.POINTER(C.c_double)),
        ("ground_mtl_nbrdf", C.POINTER(C.c_uint32)), ("ground_mtl_brdf", C.POINTER(C.c_double)),
        ("repeat_ground", C.c_int32), ("ground_sky_mtl", C.c_uint32),
    ]


class RequestDesc(C.Structure):
    _fields_ = [
        ("mode", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32),
        ("spp", C.c_uint32), ("wlen_range", C.c_double * 2), ("ref_temperature", C.c_double),
        ("camera_type", C.c_int32), ("cam_pos", C.c_double * 3), ("cam_tgt", C.c_double * 3),
        ("cam_up", C.c_double * 3), ("fov_deg", C.c_double), ("lens_radius", C.c_double),
        ("focal_dst", C.c_double), ("ortho_height", C.c_double),
        ("rect_pos", C.c_double * 3), ("rect_tgt", C.c_double * 3), ("rect_up", C.c_double * 3),
        ("rect_size", C.c_double * 2), ("seed", C.c_uint32),
    ]


class Node(C.Structure):
    _fields_ = [("kmin", C.c_float), ("kmax", C.c_float), ("child", C.c_uint32), ("pad", C.c_uint32)]


class Counters(C.Structure):
    _fields_ = [("nseg", C.c_uint64), ("nnode", C.c_uint64), ("ntc", C.c_uint64),
                ("nreal", C.c_uint64)]


NODE_DTYPE = np.dtype([("kmin", "<f4"), ("kmax", "<f4"), ("child", "<u4"), ("pad", "<u4")])
PIXEL_XWAVE = np.dtype([("L", "<f8"), ("L_se", "<f8"), ("Tb", "<f8"), ("Tb_se", "<f8"),
                        ("t_sum", "<f8"), ("t_sum2", "<f8"), ("t_n", "<u8"), ("t_nfail", "<u8")])
PIXEL_FLUX = np.dtype([("sum", "<f8"), ("sum2", "<f8"), ("n", "<u8"), ("nfail", "<u8"),
                       ("t_sum", "<f8"), ("t_sum2", "<f8"), ("t_n", "<u8"), ("t_nfail", "<u8")])
PIXEL_IMAGE = np.dtype([("X", "<f8"), ("X_se", "<f8"), ("Y", "<f8"), ("Y_se", "<f8"),
                        ("Z", "<f8"), ("Z_se", "<f8"),
                        ("t_sum", "<f8"), ("t_sum2", "<f8"), ("t_n", "<u8"), ("t_nfail", "<u8")])


def pixel_dtype(mode: int) -> np.dtype:
    return PIXEL_IMAGE if mode == 2 else (PIXEL_FLUX if mode in (3, 4) else PIXEL_XWAVE)


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        L.ora_scene_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]
        L.ora_scene_release.argtypes = [C.c_void_p]
        L.ora_scene_tree.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_int,
                                     C.POINTER(C.POINTER(Node))]
        L.ora_scene_tree.restype = C.c_size_t
        L.ora_scene_tree_depth.argtypes = [C.c_void_p]
        L.ora_scene_tree_depth.restype = C.c_uint32
        L.ora_find_band.argtypes = [C.c_void_p, C.c_double]
        L.ora_find_band.restype = C.c_size_t
        L.ora_sample_quad.argtypes = [C.c_void_p, C.c_double, C.c_size_t]
        L.ora_sample_quad.restype = C.c_size_t
        L.ora_locate_leaf.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_int,
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint32)]
        L.ora_draw_map.argtypes = [C.c_void_p, C.POINTER(RequestDesc), C.c_void_p, C.c_size_t,
                                   C.c_size_t, C.c_size_t, C.c_int, C.POINTER(Counters)]
        L.ora_realisation_weights.argtypes = [C.c_void_p, C.POINTER(RequestDesc), C.c_size_t,
                                              C.c_size_t, C.POINTER(C.c_double), C.c_int]
        L.ora_radiance_batch.argtypes = [C.c_void_p, C.c_int, C.c_size_t,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint32), C.c_int, C.c_uint32,
                                         C.POINTER(C.c_double), C.c_int]
        L.ora_sample_wavelength.argtypes = [C.c_void_p, C.POINTER(RequestDesc), C.c_int,
                                            C.c_size_t, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ora_ground_trace_batch.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_float),
                                             C.POINTER(C.c_float), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint8), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_float)]
        for name in ("ora_wiebelt",):
            getattr(L, name).argtypes = [C.c_double]
            getattr(L, name).restype = C.c_double
        for name in ("ora_blackbody_fraction", "ora_planck_interval", "ora_planck"):
            getattr(L, name).argtypes = [C.c_double, C.c_double, C.c_double]
            getattr(L, name).restype = C.c_double
        L.ora_planck_monochromatic.argtypes = [C.c_double, C.c_double]
        L.ora_planck_monochromatic.restype = C.c_double
        L.ora_radiance_temperature.argtypes = [C.c_double, C.c_double, C.c_double]
        L.ora_radiance_temperature.restype = C.c_double
        L.ora_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint32)]
        L.ora_fit_bar_1931.argtypes = [C.c_int, C.c_double]
        L.ora_fit_bar_1931.restype = C.c_double
    return _lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def scene_desc(scene, props_mask: int = 0b111):
    """The C description of a scene (SceneDesc) and the arrays it points to,
    which must stay alive while the description is in use."""
    scene.validate()
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a

    d = SceneDesc()
    d.nlayers = scene.nlayers
    d.layer_z = _p(arr(scene.layer_z, np.float64), C.c_double)
    d.layer_T = _p(arr(scene.layer_T, np.float32), C.c_float)
    d.nbands = scene.nbands
    d.band_lo = _p(arr(scene.band_lo, np.float64), C.c_double)
    d.band_hi = _p(arr(scene.band_hi, np.float64), C.c_double)
    d.nquads = _p(arr(scene.nquads, np.uint32), C.c_uint32)
    d.quad_w = _p(arr(scene.quad_w, np.float64), C.c_double)
    d.gas_ka = _p(arr(scene.gas_ka, np.float32), C.c_float)
    d.gas_ks = _p(arr(scene.gas_ks, np.float32), C.c_float)
    cd = scene.cloud_def
    for i in range(3):
        d.cloud_def[i] = cd[i]
        d.cloud_lower[i] = scene.cloud_lower[i]
        d.cloud_cell[i] = scene.cloud_cell[i]
        d.grid_max_definition[i] = scene.grid_max_definition[i]
    if scene.cloud_lwc is not None:
        d.cloud_lwc = _p(arr(scene.cloud_lwc, np.float32), C.c_float)
    nb = scene.nbands
    zeros = np.zeros(nb)
    d.cloud_sigma_ext = _p(arr(scene.cloud_sigma_ext if scene.cloud_sigma_ext is not None else zeros, np.float32), C.c_float)
    d.cloud_ssa = _p(arr(scene.cloud_ssa if scene.cloud_ssa is not None else zeros, np.float32), C.c_float)
    d.cloud_g = _p(arr(scene.cloud_g if scene.cloud_g is not None else zeros, np.float32), C.c_float)
    d.repeat_clouds = int(scene.repeat_clouds)
    d.optical_thickness = scene.optical_thickness
    d.has_ground = int(scene.has_ground)
    d.ground_brdf = int(scene.ground_brdf)
    d.ground_reflectivity = scene.ground_reflectivity
    d.ground_temperature = scene.ground_temperature
    d.sun_azimuth = scene.sun_azimuth
    d.sun_elevation = scene.sun_elevation
    d.props_mask = props_mask
    if scene.ground_mesh is not None:
        scene.ground_mesh.fill_desc(d, keep)
    return d, keep


class OracleScene:
    """A scene loaded into the oracle (majorant octrees built on creation)."""

    def __init__(self, scene, props_mask: int = 0b111):
        d, self._keep = scene_desc(scene, props_mask)
        self.scene = scene
        h = C.c_void_p()
        res = lib().ora_scene_create(C.byref(d), C.byref(h))
        if res != 0:
            raise RuntimeError(f"ora_scene_create failed: {res}")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib().ora_scene_release(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def tree(self, iband: int, iquad: int, prop: int) -> np.ndarray:
        ptr = C.POINTER(Node)()
        n = lib().ora_scene_tree(self.handle, iband, iquad, prop, C.byref(ptr))
        if n == 0:
            return np.zeros(0, dtype=NODE_DTYPE)
        buf = (C.c_char * (16 * n)).from_address(C.addressof(ptr.contents))
        return np.frombuffer(bytes(buf), dtype=NODE_DTYPE).copy()

    def depth(self) -> int:
        return int(lib().ora_scene_tree_depth(self.handle))

    def find_band(self, wlen: float) -> int:
        return int(lib().ora_find_band(self.handle, wlen))

    def sample_quad(self, r: float, iband: int) -> int:
        return int(lib().ora_sample_quad(self.handle, r, iband))

    def locate_leaf(self, iband, iquad, prop, cell):
        c = (C.c_uint32 * 3)(*[int(v) for v in cell])
        n, lv = C.c_uint32(), C.c_uint32()
        res = lib().ora_locate_leaf(self.handle, iband, iquad, prop, c, C.byref(n), C.byref(lv))
        if res != 0:
            raise ValueError(res)
        return int(n.value), int(lv.value)

    def draw_map(self, req, pix_begin: int = 0, pix_end: Optional[int] = None,
                 nthreads: int = 0):
        npix = req.width * req.height
        pix_end = npix if pix_end is None else pix_end
        dt = pixel_dtype(req.mode)
        buf = np.zeros((req.height, req.width), dtype=dt)
        cnt = Counters()
        rd = request_desc(req)
        res = lib().ora_draw_map(self.handle, C.byref(rd), buf.ctypes.data_as(C.c_void_p),
                                 req.width * dt.itemsize, pix_begin, pix_end, nthreads,
                                 C.byref(cnt))
        if res != 0:
            raise RuntimeError(f"ora_draw_map failed: {res}")
        return buf, {"nseg": cnt.nseg, "nnode": cnt.nnode, "ntc": cnt.ntc, "nreal": cnt.nreal}

    def sample_wavelength(self, req, channel: int, r0, r1):
        r0 = np.ascontiguousarray(r0, np.float64)
        r1 = np.ascontiguousarray(r1, np.float64)
        n = len(r0)
        cb = np.zeros(n, np.uint32)
        wl = np.zeros(n, np.float64)
        pdf = np.zeros(n, np.float64)
        rd = request_desc(req)
        res = lib().ora_sample_wavelength(self.handle, C.byref(rd), channel, n, _p(r0, C.c_double),
                                          _p(r1, C.c_double), _p(cb, C.c_uint32),
                                          _p(wl, C.c_double), _p(pdf, C.c_double))
        if res != 0:
            raise RuntimeError(res)
        return cb, wl, pdf

    def realisation_weights(self, req, pix_begin: int, pix_end: int, nthreads: int = 0):
        nr = req.realisations_per_pixel
        out = np.zeros((pix_end - pix_begin, nr), dtype=np.float64)
        rd = request_desc(req)
        res = lib().ora_realisation_weights(self.handle, C.byref(rd), pix_begin, pix_end,
                                            _p(out, C.c_double), nthreads)
        if res != 0:
            raise RuntimeError(res)
        return out

    def ground_trace(self, rays, tmax, from_prim, from_edge):
        """Ground-mesh queries (ora_ground.c): (primitive, distance) per ray."""
        rays = np.ascontiguousarray(rays, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        fp = np.ascontiguousarray(from_prim, np.uint32)
        fe = np.ascontiguousarray(from_edge, np.uint8)
        n = rays.shape[0]
        prim = np.zeros(n, np.uint32)
        dist = np.zeros(n, np.float32)
        res = lib().ora_ground_trace_batch(self.handle, n, _p(rays, C.c_float), _p(tmax, C.c_float),
                                           _p(fp, C.c_uint32), _p(fe, C.c_uint8),
                                           _p(prim, C.c_uint32), _p(dist, C.c_float))
        if res != 0:
            raise RuntimeError(f"ora_ground_trace_batch failed: {res}")
        return prim, dist

    def radiance(self, lw: bool, pos, dirs, wlen, iband, iquad, mask: int = ALL,
                 seed: int = 0, nthreads: int = 0) -> np.ndarray:
        n = len(wlen)
        pos = np.ascontiguousarray(pos, np.float64)
        dirs = np.ascontiguousarray(dirs, np.float64)
        wlen = np.ascontiguousarray(wlen, np.float64)
        iband = np.ascontiguousarray(iband, np.uint32)
        iquad = np.ascontiguousarray(iquad, np.uint32)
        out = np.zeros(n, np.float64)
        lib().ora_radiance_batch(self.handle, int(lw), n, _p(pos, C.c_double), _p(dirs, C.c_double),
                                 _p(wlen, C.c_double), _p(iband, C.c_uint32),
                                 _p(iquad, C.c_uint32), mask, seed, _p(out, C.c_double),
                                 nthreads)
        return out


def request_desc(req) -> RequestDesc:
    r = RequestDesc()
    r.mode = req.mode
    r.width, r.height, r.spp = req.width, req.height, req.spp
    r.wlen_range[0], r.wlen_range[1] = req.wlen_range
    r.ref_temperature = req.ref_temperature
    r.camera_type = req.camera_type
    for i in range(3):
        r.cam_pos[i], r.cam_tgt[i], r.cam_up[i] = req.cam_pos[i], req.cam_tgt[i], req.cam_up[i]
        r.rect_pos[i], r.rect_tgt[i], r.rect_up[i] = req.rect_pos[i], req.rect_tgt[i], req.rect_up[i]
    r.fov_deg, r.lens_radius, r.focal_dst, r.ortho_height = (
        req.fov_deg, req.lens_radius, req.focal_dst, req.ortho_height)
    r.rect_size[0], r.rect_size[1] = req.rect_size
    r.seed = req.seed
    return r


def philox(ctr, key) -> np.ndarray:
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().ora_philox4x32_10(c, k, o)
    return np.array(list(o), dtype=np.uint32)


def props_for_mode(mode: int) -> int:
    """Octrees a mode needs: SW walks use Ks, Ka and Kext; LW only Kext."""
    return 0b100 if mode in (1, 4) else 0b111
