"""Python mirror of the drop-in C ABI (include/htrdr_gpu.h), through ctypes.

The names follow the reference interface they replace:

* :meth:`GpuScene.draw_map` -- ``htrdr_draw_map`` with the atmosphere
  callbacks (src/core/htrdr_draw_map.h:89-93, src/atmosphere/htrdr_atmosphere_draw_map.c:592-641);
  returns the buffer of ``atmosphere_pixel_{xwave,flux,image}`` structs.
* :meth:`GpuScene.radiance_sw` / :meth:`GpuScene.radiance_lw` --
  ``atmosphere_compute_radiance_sw`` / ``_lw`` (src/atmosphere/htrdr_atmosphere_c.h:140-163).
* :class:`GpuScene` creation -- ``htsky_create`` (src/atmosphere/htrdr_atmosphere.c:366-382).

Errors are reported like the reference's ``res_T`` codes: a non-zero code
raises :class:`HtrdrError` carrying it.  There is no CPU fallback: without the
compiled library or without a GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import scene as S

_PKG = os.path.dirname(os.path.abspath(__file__))
# HTRDR_GPU_LIB: another build of the library (e.g. one compiled with other
# switches) in place of the in-tree one
LIB_PATH = os.environ.get("HTRDR_GPU_LIB") or os.path.join(_PKG, "lib", "libhtrdr_gpu.so")

RES_OK, RES_BAD_ARG, RES_MEM_ERR, RES_IO_ERR, RES_UNKNOWN_ERR, RES_BAD_OP = range(6)
KA, KS, KEXT = 0, 1, 2
DIRECT, DIFFUSE, ALL = 1, 2, 3

EXPORTED = [
    "htrdr_gpu_scene_create", "htrdr_gpu_scene_create_cached", "htrdr_gpu_scene_release", "htrdr_gpu_scene_device_bytes",
    "htrdr_gpu_scene_get_tree", "htrdr_gpu_scene_tree_depth", "htrdr_gpu_draw_map",
    "htrdr_gpu_draw_map_device", "htrdr_gpu_radiance_sw", "htrdr_gpu_radiance_lw",
    "htrdr_gpu_realisation_weights", "htrdr_gpu_find_band", "htrdr_gpu_sample_quad",
    "htrdr_gpu_locate_leaf", "htrdr_gpu_sample_wavelength", "htrdr_gpu_draw_maps_batched",
    "htrdr_gpu_draw_maps_batched_device", "htrdr_gpu_autotune", "htrdr_gpu_batch_create",
    "htrdr_gpu_batch_run", "htrdr_gpu_batch_release", "htrdr_gpu_server_create",
    "htrdr_gpu_server_submit", "htrdr_gpu_server_poll", "htrdr_gpu_server_wait",
    "htrdr_gpu_server_stats", "htrdr_gpu_server_release",
    "htrdr_gpu_default_tuning", "htrdr_gpu_version", "htrdr_gpu_device_count",
    "htrdr_gpu_last_error", "htrdr_gpu_scene_set_engine", "htrdr_gpu_mode_tuning",
    "htrdr_gpu_write_image", "htrdr_gpu_ground_trace", "htrdr_gpu_draw_map_noalloc",
    "htrdr_gpu_draw_map_accum_device", "htrdr_gpu_finalize_device",
    "htrdr_gpu_draw_maps_batched_accum_device", "htrdr_gpu_server_request_launches",
]

ENGINE_PERSISTENT, ENGINE_PLAIN, ENGINE_WAVEFRONT, ENGINE_SORTED = 0, 1, 2, 3


class HtrdrError(RuntimeError):
    def __init__(self, what: str, code: int, detail: str = ""):
        super().__init__(f"{what} failed with res_T {code}" + (f": {detail}" if detail else ""))
        self.code = code


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
        ("props_mask", C.c_uint32), ("octree_on_host", C.c_int32),
        ("ground_nverts", C.c_uint32), ("ground_verts", C.POINTER(C.c_float)),
        ("ground_ntris", C.c_uint32), ("ground_tris", C.POINTER(C.c_uint32)),
        ("ground_tri_iface", C.POINTER(C.c_uint32)), ("ground_nifaces", C.c_uint32),
        ("ground_ifaces", C.POINTER(C.c_uint32)), ("ground_nmtls", C.c_uint32),
        ("ground_mtl_temperature", C.POINTER(C.c_double)),
        ("ground_mtl_nbrdf", C.POINTER(C.c_uint32)), ("ground_mtl_brdf", C.POINTER(C.c_double)),
        ("repeat_ground", C.c_int32), ("ground_sky_mtl", C.c_uint32),
    ]


class Request(C.Structure):
    _fields_ = [
        ("mode", C.c_int32), ("width", C.c_uint32), ("height", C.c_uint32),
        ("spp", C.c_uint32), ("wlen_range", C.c_double * 2), ("ref_temperature", C.c_double),
        ("camera_type", C.c_int32), ("cam_pos", C.c_double * 3), ("cam_tgt", C.c_double * 3),
        ("cam_up", C.c_double * 3), ("fov_deg", C.c_double), ("lens_radius", C.c_double),
        ("focal_dst", C.c_double), ("ortho_height", C.c_double),
        ("rect_pos", C.c_double * 3), ("rect_tgt", C.c_double * 3), ("rect_up", C.c_double * 3),
        ("rect_size", C.c_double * 2), ("seed", C.c_uint32),
    ]


class BufferLayout(C.Structure):
    _fields_ = [("width", C.c_size_t), ("height", C.c_size_t), ("pitch", C.c_size_t),
                ("elmt_size", C.c_size_t), ("alignment", C.c_size_t)]


class Stats(C.Structure):
    _fields_ = [("realisations", C.c_uint64), ("segments", C.c_uint64), ("nodes", C.c_uint64),
                ("collisions", C.c_uint64), ("failures", C.c_uint64),
                ("kernel_ms", C.c_double), ("total_ms", C.c_double), ("launches", C.c_uint64),
                ("grid_bytes", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("block_size", C.c_uint32), ("queue_chunk", C.c_uint32),
                ("regroup_period", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("engine", C.c_uint32), ("wave_slots", C.c_uint32),
                ("trace_budget", C.c_uint32), ("wave_tail", C.c_uint32)]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("req", Request), ("layout", BufferLayout),
                ("buffer", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_size_t),
                ("round_target_ms", C.c_double), ("round_realisations", C.c_uint64),
                ("tuning", Tuning)]


class MapSummary(C.Structure):
    _fields_ = [("path_time_E", C.c_double), ("path_time_SE", C.c_double),
                ("flux_E", C.c_double), ("flux_SE", C.c_double),
                ("path_time_n", C.c_uint64), ("flux_n", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("rounds", C.c_uint64), ("realisations", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
                ("busy_ms", C.c_double), ("wall_ms", C.c_double), ("hbm_peak_bytes", C.c_size_t)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PIXEL_XWAVE = np.dtype([("L", "<f8"), ("L_se", "<f8"), ("Tb", "<f8"), ("Tb_se", "<f8"),
                        ("t_sum", "<f8"), ("t_sum2", "<f8"), ("t_n", "<u8"), ("t_nfail", "<u8")])
PIXEL_FLUX = np.dtype([("sum", "<f8"), ("sum2", "<f8"), ("n", "<u8"), ("nfail", "<u8"),
                       ("t_sum", "<f8"), ("t_sum2", "<f8"), ("t_n", "<u8"), ("t_nfail", "<u8")])
PIXEL_IMAGE = np.dtype([("X", "<f8"), ("X_se", "<f8"), ("Y", "<f8"), ("Y_se", "<f8"),
                        ("Z", "<f8"), ("Z_se", "<f8"),
                        ("t_sum", "<f8"), ("t_sum2", "<f8"), ("t_n", "<u8"), ("t_nfail", "<u8")])
NODE_DTYPE = np.dtype([("kmin", "<f4"), ("kmax", "<f4"), ("child", "<u4"), ("pad", "<u4")])


def pixel_dtype(mode: int) -> np.dtype:
    return PIXEL_IMAGE if mode == S.MODE_IMAGE_CIE else (
        PIXEL_FLUX if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW) else PIXEL_XWAVE)


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load the compiled library; raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m htrdr_kmin_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, sz, u32, i32, dp, up = C.c_void_p, C.c_size_t, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p
    L.htrdr_gpu_scene_create.argtypes = [C.c_int, C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]
    L.htrdr_gpu_scene_create_cached.argtypes = [C.c_int, C.POINTER(SceneDesc), C.c_char_p,
                                                C.POINTER(C.c_void_p)]
    L.htrdr_gpu_scene_release.argtypes = [vp]
    L.htrdr_gpu_scene_release.restype = None
    L.htrdr_gpu_scene_device_bytes.argtypes = [vp]
    L.htrdr_gpu_scene_device_bytes.restype = sz
    L.htrdr_gpu_scene_tree_depth.argtypes = [vp]
    L.htrdr_gpu_scene_tree_depth.restype = u32
    L.htrdr_gpu_scene_get_tree.argtypes = [vp, u32, u32, i32, vp, sz, C.POINTER(C.c_size_t)]
    L.htrdr_gpu_draw_map.argtypes = [vp, C.POINTER(Request), C.POINTER(BufferLayout), vp, C.POINTER(Stats)]
    L.htrdr_gpu_draw_map_device.argtypes = [vp, C.POINTER(Request), C.POINTER(BufferLayout), vp, C.POINTER(Stats)]
    L.htrdr_gpu_draw_map_accum_device.argtypes = [vp, C.POINTER(Request), vp, C.POINTER(Stats)]
    L.htrdr_gpu_finalize_device.argtypes = [vp, C.POINTER(Request), vp, C.POINTER(BufferLayout), vp]
    L.htrdr_gpu_radiance_sw.argtypes = [vp, sz, dp, dp, dp, up, up, i32, u32, dp]
    L.htrdr_gpu_radiance_lw.argtypes = [vp, sz, dp, dp, dp, up, up, u32, dp]
    L.htrdr_gpu_realisation_weights.argtypes = [vp, C.POINTER(Request), sz, sz, dp]
    L.htrdr_gpu_find_band.argtypes = [vp, sz, dp, up]
    L.htrdr_gpu_sample_quad.argtypes = [vp, sz, dp, up, up]
    L.htrdr_gpu_locate_leaf.argtypes = [vp, u32, u32, i32, sz, up, up, up]
    L.htrdr_gpu_sample_wavelength.argtypes = [vp, C.POINTER(Request), i32, sz, dp, dp, up, dp, dp]
    L.htrdr_gpu_draw_maps_batched.argtypes = [C.POINTER(BatchItem), sz, C.POINTER(Tuning), C.POINTER(Stats)]
    L.htrdr_gpu_draw_maps_batched_device.argtypes = [C.POINTER(BatchItem), sz, C.POINTER(Tuning), C.POINTER(Stats)]
    L.htrdr_gpu_draw_maps_batched_accum_device.argtypes = [C.POINTER(BatchItem), sz, C.POINTER(Tuning),
                                                           C.POINTER(Stats)]
    L.htrdr_gpu_autotune.argtypes = [C.POINTER(BatchItem), sz, C.POINTER(Tuning), C.POINTER(C.c_double)]
    L.htrdr_gpu_batch_create.argtypes = [C.POINTER(BatchItem), sz, C.POINTER(Tuning), C.POINTER(C.c_void_p)]
    L.htrdr_gpu_batch_run.argtypes = [vp, C.POINTER(Stats)]
    L.htrdr_gpu_batch_release.argtypes = [vp]
    L.htrdr_gpu_batch_release.restype = None
    L.htrdr_gpu_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]
    L.htrdr_gpu_server_submit.argtypes = [vp, vp, C.POINTER(Request), C.POINTER(BufferLayout), vp,
                                          C.POINTER(C.c_uint64)]
    L.htrdr_gpu_server_poll.argtypes = [vp, C.c_uint64, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.htrdr_gpu_server_wait.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(C.c_int)]
    L.htrdr_gpu_server_stats.argtypes = [vp, C.POINTER(ServerStats)]
    L.htrdr_gpu_server_request_launches.argtypes = [vp, C.c_uint64, C.POINTER(C.c_uint64),
                                                    C.POINTER(C.c_uint64)]
    L.htrdr_gpu_server_release.argtypes = [vp]
    L.htrdr_gpu_server_release.restype = None
    L.htrdr_gpu_default_tuning.argtypes = [C.POINTER(Tuning)]
    L.htrdr_gpu_default_tuning.restype = None
    L.htrdr_gpu_mode_tuning.argtypes = [i32, C.POINTER(Tuning)]
    L.htrdr_gpu_mode_tuning.restype = None
    L.htrdr_gpu_scene_set_engine.argtypes = [vp, i32, C.POINTER(Tuning)]
    L.htrdr_gpu_write_image.argtypes = [i32, C.POINTER(BufferLayout), vp, C.c_char_p,
                                        C.POINTER(MapSummary)]
    L.htrdr_gpu_ground_trace.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp]
    L.htrdr_gpu_version.restype = C.c_char_p
    L.htrdr_gpu_last_error.restype = C.c_char_p
    L.htrdr_gpu_device_count.restype = C.c_int
    _lib = L
    return L


def _check(res: int, what: str):
    if res != RES_OK:
        raise HtrdrError(what, res, lib().htrdr_gpu_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def to_request(req: S.Request) -> Request:
    r = Request()
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


def layout_for(req: S.Request) -> BufferLayout:
    dt = pixel_dtype(req.mode)
    lay = BufferLayout()
    lay.width, lay.height = req.width, req.height
    lay.pitch = req.width * dt.itemsize
    lay.elmt_size = dt.itemsize
    lay.alignment = 16
    return lay


def accum_records(req: S.Request) -> int:
    """Accumulator records of a map (htrdr_gpu_draw_map_accum_device): one
    per pixel and channel, then one per pixel for the time per realisation."""
    return req.width * req.height * ((3 if req.mode == S.MODE_IMAGE_CIE else 1) + 1)


def props_for_mode(mode: int) -> int:
    return 0b100 if mode in (S.MODE_XWAVE_LW, S.MODE_FLUX_LW) else 0b111


class GpuScene:
    """A scene resident in HBM with its majorant octrees (htsky_create)."""

    def __init__(self, scene: S.Scene, props_mask: int = 0b111, device: int = 0,
                 octree_on_host: bool = False, cache_path: Optional[str] = None):
        """cache_path: the octree cache of option -O (loaded when it holds
        this medium's octrees, written when it does not exist)."""
        scene.validate()
        self.scene = scene
        keep: List[np.ndarray] = []

        def arr(a, dt, ct):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ct))

        d = SceneDesc()
        d.nlayers = scene.nlayers
        d.layer_z = arr(scene.layer_z, np.float64, C.c_double)
        d.layer_T = arr(scene.layer_T, np.float32, C.c_float)
        d.nbands = scene.nbands
        d.band_lo = arr(scene.band_lo, np.float64, C.c_double)
        d.band_hi = arr(scene.band_hi, np.float64, C.c_double)
        d.nquads = arr(scene.nquads, np.uint32, C.c_uint32)
        d.quad_w = arr(scene.quad_w, np.float64, C.c_double)
        d.gas_ka = arr(scene.gas_ka, np.float32, C.c_float)
        d.gas_ks = arr(scene.gas_ks, np.float32, C.c_float)
        cd = scene.cloud_def
        for i in range(3):
            d.cloud_def[i] = cd[i]
            d.cloud_lower[i] = scene.cloud_lower[i]
            d.cloud_cell[i] = scene.cloud_cell[i]
            d.grid_max_definition[i] = scene.grid_max_definition[i]
        nb = scene.nbands
        if scene.cloud_lwc is not None:
            d.cloud_lwc = arr(scene.cloud_lwc, np.float32, C.c_float)
        d.cloud_sigma_ext = arr(scene.cloud_sigma_ext if scene.cloud_sigma_ext is not None else np.zeros(nb), np.float32, C.c_float)
        d.cloud_ssa = arr(scene.cloud_ssa if scene.cloud_ssa is not None else np.zeros(nb), np.float32, C.c_float)
        d.cloud_g = arr(scene.cloud_g if scene.cloud_g is not None else np.zeros(nb), np.float32, C.c_float)
        d.repeat_clouds = int(scene.repeat_clouds)
        d.optical_thickness = scene.optical_thickness
        d.has_ground = int(scene.has_ground)
        d.ground_brdf = int(scene.ground_brdf)
        d.ground_reflectivity = scene.ground_reflectivity
        d.ground_temperature = scene.ground_temperature
        d.sun_azimuth = scene.sun_azimuth
        d.sun_elevation = scene.sun_elevation
        d.props_mask = props_mask
        d.octree_on_host = int(octree_on_host)
        if scene.ground_mesh is not None:
            scene.ground_mesh.fill_desc(d, keep)
        h = C.c_void_p()
        if cache_path is not None:
            _check(lib().htrdr_gpu_scene_create_cached(device, C.byref(d), os.fsencode(cache_path),
                                                       C.byref(h)), "htrdr_gpu_scene_create_cached")
        else:
            _check(lib().htrdr_gpu_scene_create(device, C.byref(d), C.byref(h)), "htrdr_gpu_scene_create")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib().htrdr_gpu_scene_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(lib().htrdr_gpu_scene_device_bytes(self.handle))

    def depth(self) -> int:
        return int(lib().htrdr_gpu_scene_tree_depth(self.handle))

    def tree(self, iband: int, iquad: int, prop: int) -> np.ndarray:
        n = C.c_size_t()
        _check(lib().htrdr_gpu_scene_get_tree(self.handle, iband, iquad, prop, None, 0, C.byref(n)), "get_tree")
        out = np.zeros(n.value, dtype=NODE_DTYPE)
        if n.value:
            _check(lib().htrdr_gpu_scene_get_tree(self.handle, iband, iquad, prop, _ptr(out),
                                                  n.value, C.byref(n)), "get_tree")
        return out

    def set_engine(self, engine: int, tuning: Optional["Tuning"] = None):
        """Engine of draw_map on this scene: ENGINE_PERSISTENT, ENGINE_WAVEFRONT
        (tuning None: the mode's) or ENGINE_PLAIN.  Without a call, the
        mode's default tuning decides, engine included."""
        _check(lib().htrdr_gpu_scene_set_engine(self.handle, engine,
                                                C.byref(tuning) if tuning is not None else None),
               "htrdr_gpu_scene_set_engine")

    def draw_map(self, req: S.Request, device_out=None):
        """htrdr_draw_map: returns (pixel buffer [height, width], stats dict)."""
        r = to_request(req)
        lay = layout_for(req)
        st = Stats()
        if device_out is not None:
            _check(lib().htrdr_gpu_draw_map_device(self.handle, C.byref(r), C.byref(lay),
                                                   C.c_void_p(device_out), C.byref(st)),
                   "htrdr_gpu_draw_map_device")
            return None, st.as_dict()
        buf = np.zeros((req.height, req.width), dtype=pixel_dtype(req.mode))
        _check(lib().htrdr_gpu_draw_map(self.handle, C.byref(r), C.byref(lay), _ptr(buf), C.byref(st)),
               "htrdr_gpu_draw_map")
        return buf, st.as_dict()

    def draw_map_accum(self, req: S.Request, device_accum: int) -> dict:
        """The map's FP64 accumulators into device memory (accum_records(req)
        records of 32 bytes at `device_accum'); returns the stats."""
        r = to_request(req)
        st = Stats()
        _check(lib().htrdr_gpu_draw_map_accum_device(self.handle, C.byref(r), C.c_void_p(device_accum),
                                                     C.byref(st)), "htrdr_gpu_draw_map_accum_device")
        return st.as_dict()

    def finalize(self, req: S.Request, device_accum: int, device_out: int) -> None:
        """Pixel structs of the map (device memory) from its accumulators."""
        r = to_request(req)
        lay = layout_for(req)
        _check(lib().htrdr_gpu_finalize_device(self.handle, C.byref(r), C.c_void_p(device_accum),
                                               C.byref(lay), C.c_void_p(device_out)),
               "htrdr_gpu_finalize_device")

    def ground_trace(self, rays: np.ndarray, tmax: np.ndarray, from_prim: np.ndarray,
                     from_edge: np.ndarray):
        """Ground queries on the mesh: rays [n, 6] float32 (origin, direction),
        range [0, tmax), the primitive each ray leaves (NO_ID: none) and
        whether that hit lay on an edge.  Returns (primitive, distance)."""
        n = rays.shape[0]
        r = np.ascontiguousarray(rays, dtype=np.float32)
        t = np.ascontiguousarray(tmax, dtype=np.float32)
        fp = np.ascontiguousarray(from_prim, dtype=np.uint32)
        fe = np.ascontiguousarray(from_edge, dtype=np.uint8)
        prim = np.zeros(n, np.uint32)
        dist = np.zeros(n, np.float32)
        _check(lib().htrdr_gpu_ground_trace(self.handle, n, _ptr(r), _ptr(t), _ptr(fp), _ptr(fe),
                                            _ptr(prim), _ptr(dist)), "htrdr_gpu_ground_trace")
        return prim, dist

    def realisation_weights(self, req: S.Request, pix_begin: int, pix_end: int) -> np.ndarray:
        out = np.zeros((pix_end - pix_begin, req.realisations_per_pixel), np.float64)
        r = to_request(req)
        _check(lib().htrdr_gpu_realisation_weights(self.handle, C.byref(r), pix_begin, pix_end,
                                                   _ptr(out)), "realisation_weights")
        return out

    def _radiance(self, lw, pos, dirs, wlen, iband, iquad, mask, seed):
        pos = np.ascontiguousarray(pos, np.float64)
        dirs = np.ascontiguousarray(dirs, np.float64)
        wlen = np.ascontiguousarray(wlen, np.float64)
        iband = np.ascontiguousarray(iband, np.uint32)
        iquad = np.ascontiguousarray(iquad, np.uint32)
        n = len(wlen)
        out = np.zeros(n, np.float64)
        if lw:
            _check(lib().htrdr_gpu_radiance_lw(self.handle, n, _ptr(pos), _ptr(dirs), _ptr(wlen),
                                               _ptr(iband), _ptr(iquad), seed, _ptr(out)), "radiance_lw")
        else:
            _check(lib().htrdr_gpu_radiance_sw(self.handle, n, _ptr(pos), _ptr(dirs), _ptr(wlen),
                                               _ptr(iband), _ptr(iquad), mask, seed, _ptr(out)), "radiance_sw")
        return out

    def radiance_sw(self, pos, dirs, wlen, iband, iquad, mask: int = ALL, seed: int = 0):
        return self._radiance(False, pos, dirs, wlen, iband, iquad, mask, seed)

    def radiance_lw(self, pos, dirs, wlen, iband, iquad, seed: int = 0):
        return self._radiance(True, pos, dirs, wlen, iband, iquad, 0, seed)

    def find_band(self, wlen) -> np.ndarray:
        wlen = np.ascontiguousarray(wlen, np.float64)
        out = np.zeros(len(wlen), np.uint32)
        _check(lib().htrdr_gpu_find_band(self.handle, len(wlen), _ptr(wlen), _ptr(out)), "find_band")
        return out

    def sample_quad(self, r, iband) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        iband = np.ascontiguousarray(iband, np.uint32)
        out = np.zeros(len(r), np.uint32)
        _check(lib().htrdr_gpu_sample_quad(self.handle, len(r), _ptr(r), _ptr(iband), _ptr(out)), "sample_quad")
        return out

    def locate_leaf(self, iband: int, iquad: int, prop: int, cells) -> tuple:
        cells = np.ascontiguousarray(cells, np.uint32).reshape(-1, 3)
        n = len(cells)
        node = np.zeros(n, np.uint32)
        level = np.zeros(n, np.uint32)
        _check(lib().htrdr_gpu_locate_leaf(self.handle, iband, iquad, prop, n, _ptr(cells),
                                           _ptr(node), _ptr(level)), "locate_leaf")
        return node, level

    def sample_wavelength(self, req: S.Request, channel: int, r0, r1):
        r0 = np.ascontiguousarray(r0, np.float64)
        r1 = np.ascontiguousarray(r1, np.float64)
        n = len(r0)
        cb = np.zeros(n, np.uint32)
        wl = np.zeros(n, np.float64)
        pdf = np.zeros(n, np.float64)
        rq = to_request(req)
        _check(lib().htrdr_gpu_sample_wavelength(self.handle, C.byref(rq), channel, n, _ptr(r0),
                                                 _ptr(r1), _ptr(cb), _ptr(wl), _ptr(pdf)),
               "sample_wavelength")
        return cb, wl, pdf


def write_image(mode: int, buf: np.ndarray, path: str) -> dict:
    """Write a map (the pixel buffer draw_map returns) as an htrdr-image file;
    returns the run summaries (time per path, flux density)."""
    lay = BufferLayout()
    lay.width, lay.height = buf.shape[1], buf.shape[0]
    lay.elmt_size = buf.dtype.itemsize
    lay.pitch = buf.shape[1] * buf.dtype.itemsize
    lay.alignment = 8
    b = np.ascontiguousarray(buf)
    sm = MapSummary()
    _check(lib().htrdr_gpu_write_image(mode, C.byref(lay), b.ctypes.data, path.encode(), C.byref(sm)),
           "htrdr_gpu_write_image")
    return sm.as_dict()


def default_tuning() -> Tuning:
    t = Tuning()
    lib().htrdr_gpu_default_tuning(C.byref(t))
    return t


def mode_tuning(mode: int) -> Tuning:
    t = Tuning()
    lib().htrdr_gpu_mode_tuning(mode, C.byref(t))
    return t


def draw_maps_batched(items: Sequence[tuple], tuning: Optional[Tuning] = None):
    """Run many (GpuScene, Request) in one persistent kernel.  Returns the list
    of pixel buffers and the stats of the launch."""
    n = len(items)
    arr = (BatchItem * n)()
    bufs = []
    for i, (gs, req) in enumerate(items):
        b = np.zeros((req.height, req.width), dtype=pixel_dtype(req.mode))
        bufs.append(b)
        arr[i].scene = gs.handle
        arr[i].req = to_request(req)
        arr[i].layout = layout_for(req)
        arr[i].buffer = b.ctypes.data
    st = Stats()
    t = C.byref(tuning) if tuning is not None else None
    _check(lib().htrdr_gpu_draw_maps_batched(arr, n, t, C.byref(st)), "draw_maps_batched")
    return bufs, st.as_dict()


def autotune(items_device) -> tuple:
    """Pick the batched engine's tuning on a ctypes BatchItem array whose
    buffers are device memory.  Returns (Tuning, best kernel ms)."""
    t = Tuning()
    ms = C.c_double()
    _check(lib().htrdr_gpu_autotune(items_device, len(items_device), C.byref(t), C.byref(ms)),
           "htrdr_gpu_autotune")
    return t, ms.value


class Server:
    """Request loop with continuous batching (htrdr_gpu_server_*).

    ``submit`` returns a ticket; the map lands in a NumPy buffer returned by
    ``result`` once ``wait``/``poll`` report completion."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 << 30,
                 round_target_ms: float = 20.0, round_realisations: int = 0,
                 tuning: Optional[Tuning] = None):
        cfg = ServerConfig()
        cfg.device = device
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.round_target_ms = round_target_ms
        cfg.round_realisations = round_realisations
        cfg.tuning = tuning if tuning is not None else default_tuning()
        h = C.c_void_p()
        _check(lib().htrdr_gpu_server_create(C.byref(cfg), C.byref(h)), "htrdr_gpu_server_create")
        self.handle = h
        self._bufs = {}

    def submit(self, scene: "GpuScene", req: S.Request) -> int:
        buf = np.zeros((req.height, req.width), dtype=pixel_dtype(req.mode))
        r = to_request(req)
        lay = layout_for(req)
        t = C.c_uint64()
        _check(lib().htrdr_gpu_server_submit(self.handle, scene.handle, C.byref(r), C.byref(lay),
                                             _ptr(buf), C.byref(t)), "htrdr_gpu_server_submit")
        self._bufs[t.value] = buf
        return t.value

    def poll(self, ticket: int) -> bool:
        done, res = C.c_int(), C.c_int()
        _check(lib().htrdr_gpu_server_poll(self.handle, ticket, C.byref(done), C.byref(res)), "poll")
        if done.value and res.value != RES_OK:
            raise HtrdrError("request", res.value)
        return bool(done.value)

    def wait(self, ticket: int, timeout_s: float = 600.0) -> np.ndarray:
        res = C.c_int()
        _check(lib().htrdr_gpu_server_wait(self.handle, ticket, timeout_s, C.byref(res)), "wait")
        if res.value != RES_OK:
            raise HtrdrError("request", res.value)
        return self._bufs.pop(ticket)

    def launches(self, ticket: int) -> tuple:
        """(first, last) launch of the loop that carried the request."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().htrdr_gpu_server_request_launches(self.handle, ticket, C.byref(a), C.byref(b)),
               "htrdr_gpu_server_request_launches")
        return a.value, b.value

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().htrdr_gpu_server_stats(self.handle, C.byref(st)), "stats")
        return st.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            lib().htrdr_gpu_server_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count() -> int:
    return int(lib().htrdr_gpu_device_count())
