"""ctypes binding of the compiled reference oracle (oracle/_ref/libhtrdr_ref.so).

TEST INFRASTRUCTURE ONLY.  The library holds the reference's own atmosphere
hot-path C files -- src/atmosphere/htrdr_atmosphere_compute_radiance_sw.c,
..._lw.c, src/atmosphere/htrdr_atmosphere_draw_map.c,
src/atmosphere/htrdr_atmosphere_sun.c, src/core/htrdr_ran_wlen_planck.c,
src/core/htrdr_ran_wlen_cie_xyz.c, src/core/htrdr_spectral.c,
src/core/htrdr_rectangle.c and src/core/htrdr_buffer.c -- compiled unmodified
from the reference tree (oracle/ref/Makefile) against project-written shims of
their absent dependencies (rsys, star-sp, star-sf, star-3d, star-camera,
htsky: oracle/ref/include, oracle/ref/ref_shim.c).  The shims answer with the
oracle's own medium, octrees and random streams, so the library runs the
reference's event logic, draw order and accumulation over the oracle's
scenes: it pins the C restatement of oracle/ to the reference's code.

The reference tree is only needed to build the library; a built library is
used as is where the tree is absent.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from . import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libhtrdr_ref.so")
_REF_TREE = os.environ.get("HTRDR_REFERENCE_TREE", "/root/reference")


def build(force: bool = False) -> Optional[str]:
    """Compile the reference files with oracle/ref/Makefile when the reference
    tree is present; return the library path, or None when it can be neither
    built nor found."""
    if os.path.isdir(os.path.join(_REF_TREE, "src", "atmosphere")):
        subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "ref"), f"REF={_REF_TREE}"]
                       + (["-B"] if force else []), check=True)
    return _LIB_PATH if os.path.exists(_LIB_PATH) else None


def available() -> bool:
    return build() is not None


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = build()
        if path is None:
            raise RuntimeError("the compiled reference oracle is not built (no reference tree)")
        _lib = C.CDLL(path)
        L = _lib
        L.ref_scene_create.argtypes = [C.POINTER(O.SceneDesc), C.POINTER(C.c_void_p)]
        L.ref_scene_release.argtypes = [C.c_void_p]
        L.ref_draw_map.argtypes = [C.c_void_p, C.POINTER(O.RequestDesc), C.c_void_p, C.c_size_t,
                                   C.c_size_t, C.c_size_t, C.c_int, C.c_char_p]
        L.ref_realisation_weights.argtypes = [C.c_void_p, C.POINTER(O.RequestDesc), C.c_size_t,
                                              C.c_size_t, C.POINTER(C.c_double), C.c_int]
        L.ref_radiance_batch.argtypes = [C.c_void_p, C.c_int, C.c_size_t,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint32), C.c_int, C.c_uint32,
                                         C.POINTER(C.c_double), C.c_int]
    return _lib


class RefScene:
    """A scene run by the reference's own code (plane ground only)."""

    def __init__(self, scene, props_mask: int = 0b111):
        d, self._keep = O.scene_desc(scene, props_mask)
        self.scene = scene
        h = C.c_void_p()
        res = lib().ref_scene_create(C.byref(d), C.byref(h))
        if res != 0:
            raise RuntimeError(f"ref_scene_create failed: {res}")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib().ref_scene_release(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def draw_map(self, req, pix_begin: int = 0, pix_end: Optional[int] = None,
                 nthreads: int = 0, dump_path: Optional[str] = None):
        """The reference's atmosphere_draw_map: the map (pixels outside
        [pix_begin, pix_end) stay zero) and, with dump_path, its htrdr-image
        file as the reference's dump_buffer writes it."""
        npix = req.width * req.height
        pix_end = npix if pix_end is None else pix_end
        dt = O.pixel_dtype(req.mode)
        buf = np.zeros((req.height, req.width), dtype=dt)
        rd = O.request_desc(req)
        res = lib().ref_draw_map(self.handle, C.byref(rd), buf.ctypes.data_as(C.c_void_p),
                                 req.width * dt.itemsize, pix_begin, pix_end, nthreads,
                                 dump_path.encode() if dump_path else None)
        if res != 0:
            raise RuntimeError(f"ref_draw_map failed: {res}")
        return buf

    def realisation_weights(self, req, pix_begin: int, pix_end: int, nthreads: int = 0):
        nr = req.realisations_per_pixel
        out = np.zeros((pix_end - pix_begin, nr), dtype=np.float64)
        rd = O.request_desc(req)
        res = lib().ref_realisation_weights(self.handle, C.byref(rd), pix_begin, pix_end,
                                            out.ctypes.data_as(C.POINTER(C.c_double)), nthreads)
        if res != 0:
            raise RuntimeError(f"ref_realisation_weights failed: {res}")
        return out

    def radiance(self, lw: bool, pos, dirs, wlen, iband, iquad, mask: int = O.ALL,
                 seed: int = 0, nthreads: int = 0) -> np.ndarray:
        """atmosphere_compute_radiance_sw/_lw per ray, streams keyed like
        OracleScene.radiance."""
        n = len(wlen)
        pos = np.ascontiguousarray(pos, np.float64)
        dirs = np.ascontiguousarray(dirs, np.float64)
        wlen = np.ascontiguousarray(wlen, np.float64)
        iband = np.ascontiguousarray(iband, np.uint32)
        iquad = np.ascontiguousarray(iquad, np.uint32)
        out = np.zeros(n, np.float64)
        P = O._p
        res = lib().ref_radiance_batch(self.handle, int(lw), n, P(pos, C.c_double),
                                       P(dirs, C.c_double), P(wlen, C.c_double),
                                       P(iband, C.c_uint32), P(iquad, C.c_uint32), mask, seed,
                                       P(out, C.c_double), nthreads)
        if res != 0:
            raise RuntimeError(f"ref_radiance_batch failed: {res}")
        return out
