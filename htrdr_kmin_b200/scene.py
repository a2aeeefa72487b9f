"""Seeded synthetic scenes and render requests for the atmosphere path tracer.

The reference reads its medium from HTGOP (gas k-distribution), HTCP (LES
cloud grid) and HTMie (droplet optics) files through htsky
(src/atmosphere/htrdr_atmosphere.c:366-382).  None of those data sets exist
here, so the five workloads are generated from seeds.  One generator feeds
both the CUDA library and the CPU oracle, so both integrate the same medium.

Medium model (shared by every consumer of a :class:`Scene`):

* gas: ``nlayers`` horizontal layers between ``layer_z[i]`` and
  ``layer_z[i+1]`` metres; per (band, quadrature point, layer) absorption
  ``gas_ka`` and scattering ``gas_ks`` in 1/m, piecewise constant in z;
  temperature ``layer_T`` per layer.
* cloud: a cell grid ``cloud_lwc[z, y, x]`` (kg/m^3) whose lower corner is
  ``cloud_lower`` and cell size ``cloud_cell``; optionally repeated along X
  and Y (``repeat_clouds``, the ``-r`` flag of htrdr-atmosphere).  Per band:
  ``k_ext = lwc * cloud_sigma_ext``, single-scattering albedo ``cloud_ssa``
  and Henyey-Greenstein asymmetry ``cloud_g``.
* ground: the plane z = 0 with a Lambertian (or specular) BRDF of constant
  reflectivity and a temperature (emissivity = 1 - reflectivity).
* sun: azimuth/elevation in degrees (``-D`` flag).
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

# Output/spectral modes of htrdr_atmosphere_draw_map.c:438-475
MODE_XWAVE_SW = 0  # draw_pixel_xwave, shortwave   (draw_map.c:324-436)
MODE_XWAVE_LW = 1  # draw_pixel_xwave, longwave    (draw_map.c:324-436)
MODE_IMAGE_CIE = 2  # draw_pixel_image, CIE XYZ    (draw_map.c:109-207)
MODE_FLUX_SW = 3  # draw_pixel_flux, shortwave     (draw_map.c:209-322)
MODE_FLUX_LW = 4  # draw_pixel_flux, longwave      (draw_map.c:209-322)

CAMERA_PERSPECTIVE = 0
CAMERA_ORTHOGRAPHIC = 1

BRDF_LAMBERTIAN = 0
BRDF_SPECULAR = 1

# Seeds of the synthetic inputs
SEED_S1, SEED_S2, SEED_S3, SEED_S4, SEED_S5, SEED_S6 = 101, 202, 303, 404, 505, 606

RHO_WATER = 1000.0  # kg/m^3
R_EFF = 10e-6  # m
SIGMA_EXT_CLOUD = 3.0 / (2.0 * RHO_WATER * R_EFF)  # m^2/kg : k_ext = lwc*sigma


NO_ID = 0xFFFFFFFF


@dataclass
class GroundMesh:
    """Ground geometry (htrdr_atmosphere_ground_create,
    src/atmosphere/htrdr_atmosphere_ground.c:105-160): triangles with an
    interface each (front, thin, back material; NO_ID: none), materials with a
    temperature and BRDFs tabulated by wavelength.  A triangle is front-facing
    on the side from which its vertices are seen clockwise (doc/htrdr-obj.5)."""

    verts: np.ndarray        # float32 [nverts, 3] m
    tris: np.ndarray         # uint32 [ntris, 3]
    tri_iface: np.ndarray    # uint32 [ntris]
    ifaces: np.ndarray       # uint32 [nifaces, 3] front, thin, back
    mtl_temperature: np.ndarray  # float64 [nmtls] K
    mtl_nbrdf: np.ndarray    # uint32 [nmtls]
    mtl_brdf: np.ndarray     # float64 [sum nbrdf, 3] wavelength nm, type (0 Lambertian, 1 specular), reflectivity
    repeat: bool = False     # repeat the bounding box in X and Y
    sky_mtl: int = NO_ID     # material of the atmosphere (flux-probe rejection)
    mtl_names: Tuple[str, ...] = ()

    def fill_desc(self, d, keep: list) -> None:
        """Set the ground-mesh fields of a ctypes scene description (the CUDA
        library's or the oracle's: same field names)."""
        import ctypes as C

        def arr(a, dt, ct):
            a = np.ascontiguousarray(a, dtype=dt).reshape(-1)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ct))

        d.ground_nverts = int(self.verts.shape[0])
        d.ground_verts = arr(self.verts, np.float32, C.c_float)
        d.ground_ntris = int(self.tris.shape[0])
        d.ground_tris = arr(self.tris, np.uint32, C.c_uint32)
        d.ground_tri_iface = arr(self.tri_iface, np.uint32, C.c_uint32)
        d.ground_nifaces = int(self.ifaces.shape[0])
        d.ground_ifaces = arr(self.ifaces, np.uint32, C.c_uint32)
        d.ground_nmtls = int(self.mtl_temperature.shape[0])
        d.ground_mtl_temperature = arr(self.mtl_temperature, np.float64, C.c_double)
        d.ground_mtl_nbrdf = arr(self.mtl_nbrdf, np.uint32, C.c_uint32)
        d.ground_mtl_brdf = arr(self.mtl_brdf if self.mtl_brdf.size else np.zeros((1, 3)), np.float64, C.c_double)
        d.repeat_ground = int(self.repeat)
        d.ground_sky_mtl = int(self.sky_mtl)


def parse_htrdr_obj(obj_text: str, materials: dict, sky_mtl: str = "air",
                    repeat: bool = False) -> GroundMesh:
    """An htrdr-obj ground (doc/htrdr-obj.5): `v x y z`, `f i j k ...`
    (1-based or negative indices, polygons as fans), `usemtl front:back` or
    `usemtl front:thin:back`.  `materials' maps a material name to
    (temperature K, [(wavelength nm, "lambertian"|"specular", reflectivity),
    ...]) or to None for a semi-transparent material: the htrdr-materials
    list (doc/htrdr-materials.5) with the tabulated BRDFs given in place of
    its mrumtl files."""
    verts, tris, tri_iface = [], [], []
    iface_ids, ifaces = {}, []
    names = list(materials.keys())
    mid = {n: i for i, n in enumerate(names)}
    cur = None
    for raw in obj_text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        tok = line.split()
        if tok[0] == "v":
            verts.append([float(tok[1]), float(tok[2]), float(tok[3])])
        elif tok[0] == "usemtl":
            parts = " ".join(tok[1:]).split(":")
            if len(parts) == 2:
                front, thin, back = parts[0], None, parts[1]
            elif len(parts) == 3:
                front, thin, back = parts
            else:
                raise ValueError(f"usemtl `{' '.join(tok[1:])}': expected front:back or front:thin:back")
            key = (front, thin, back)
            for n in (front, back) + ((thin,) if thin else ()):
                if n not in mid:
                    raise ValueError(f"unknown material `{n}'")
            if key not in iface_ids:
                iface_ids[key] = len(ifaces)
                ifaces.append([mid[front], mid[thin] if thin else NO_ID, mid[back]])
            cur = iface_ids[key]
        elif tok[0] == "f":
            if cur is None:
                raise ValueError("a face outside any usemtl group")
            ids = []
            for t in tok[1:]:
                k = int(t.split("/")[0])
                ids.append(k - 1 if k > 0 else len(verts) + k)
            for j in range(1, len(ids) - 1):
                tris.append([ids[0], ids[j], ids[j + 1]])
                tri_iface.append(cur)
    temps, nbrdf, brdf = [], [], []
    for n in names:
        m = materials[n]
        if m is None:
            temps.append(-1.0)
            nbrdf.append(0)
            continue
        t, table = m
        temps.append(float(t))
        nbrdf.append(len(table))
        for wl, kind, refl in sorted(table):
            brdf.append([wl, 1.0 if kind == "specular" else 0.0, refl])
    return GroundMesh(verts=np.array(verts, dtype=np.float32), tris=np.array(tris, dtype=np.uint32),
                      tri_iface=np.array(tri_iface, dtype=np.uint32),
                      ifaces=np.array(ifaces, dtype=np.uint32).reshape(-1, 3),
                      mtl_temperature=np.array(temps, dtype=np.float64),
                      mtl_nbrdf=np.array(nbrdf, dtype=np.uint32),
                      mtl_brdf=np.array(brdf, dtype=np.float64).reshape(-1, 3), repeat=repeat,
                      sky_mtl=mid.get(sky_mtl, NO_ID), mtl_names=tuple(names))


def parse_htrdr_materials(text: str, brdf_tables: dict) -> dict:
    """An htrdr-materials list (doc/htrdr-materials.5): one material per
    line, `name none' for a semi-transparent material or `name path
    temperature' for an opaque one, `#' starting a comment.  `brdf_tables'
    maps each path to the BRDF table its mrumtl file holds, as
    [(wavelength nm, "lambertian"|"specular", reflectivity), ...].  Returns
    the materials dict that parse_htrdr_obj takes, in file order."""
    mats = {}
    for no, raw in enumerate(text.splitlines(), 1):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        tok = line.split()
        name = tok[0]
        if name in mats:
            raise ValueError(f"line {no}: material `{name}' listed twice")
        if len(tok) == 2 and tok[1] == "none":
            mats[name] = None
            continue
        if len(tok) != 3:
            raise ValueError(f"line {no}: expected `name none' or `name brdf-path temperature'")
        path, temperature = tok[1], float(tok[2])
        if not temperature >= 0.0:
            raise ValueError(f"line {no}: invalid temperature `{tok[2]}'")
        if path not in brdf_tables:
            raise ValueError(f"line {no}: no BRDF table for `{path}'")
        table = list(brdf_tables[path])
        for wl, kind, refl in table:
            if kind not in ("lambertian", "specular") or not 0.0 <= refl <= 1.0 or not wl > 0.0:
                raise ValueError(f"line {no}: invalid BRDF entry ({wl}, {kind}, {refl}) in `{path}'")
        mats[name] = (temperature, table)
    return mats


@dataclass
class Scene:
    layer_z: np.ndarray  # float64 [nlayers+1]
    layer_T: np.ndarray  # float32 [nlayers]
    band_lo: np.ndarray  # float64 [nbands] nm
    band_hi: np.ndarray  # float64 [nbands] nm
    nquads: np.ndarray  # uint32 [nbands]
    quad_w: np.ndarray  # float64 [sum nquads]
    gas_ka: np.ndarray  # float32 [sum nquads, nlayers]
    gas_ks: np.ndarray  # float32 [sum nquads, nlayers]
    cloud_lwc: Optional[np.ndarray]  # float32 [nz, ny, nx] or None
    cloud_lower: Tuple[float, float, float] = (0.0, 0.0, 1000.0)
    cloud_cell: Tuple[float, float, float] = (100.0, 100.0, 62.5)
    cloud_sigma_ext: Optional[np.ndarray] = None  # float32 [nbands]
    cloud_ssa: Optional[np.ndarray] = None  # float32 [nbands]
    cloud_g: Optional[np.ndarray] = None  # float32 [nbands]
    repeat_clouds: bool = False
    optical_thickness: float = 1.0  # -T
    grid_max_definition: Tuple[int, int, int] = (0, 0, 0)  # -V (0: cloud def)
    has_ground: bool = True
    ground_brdf: int = BRDF_LAMBERTIAN
    ground_reflectivity: float = 0.2
    ground_temperature: float = 288.0
    sun_azimuth: float = 0.0  # deg
    sun_elevation: float = 60.0  # deg
    name: str = "scene"
    ground_mesh: Optional[GroundMesh] = None  # replaces the plane ground when set

    @property
    def nlayers(self) -> int:
        return int(self.layer_T.shape[0])

    @property
    def nbands(self) -> int:
        return int(self.band_lo.shape[0])

    @property
    def cloud_def(self) -> Tuple[int, int, int]:
        if self.cloud_lwc is None:
            return (0, 0, 0)
        nz, ny, nx = self.cloud_lwc.shape
        return (int(nx), int(ny), int(nz))

    def quad_offset(self) -> np.ndarray:
        off = np.zeros(self.nbands + 1, dtype=np.int64)
        off[1:] = np.cumsum(self.nquads.astype(np.int64))
        return off

    def validate(self) -> None:
        assert self.layer_z.dtype == np.float64 and self.layer_z.ndim == 1
        assert np.all(np.diff(self.layer_z) > 0) and self.layer_z[0] == 0.0
        assert self.layer_T.shape == (self.layer_z.shape[0] - 1,)
        nq = int(self.nquads.sum())
        assert self.quad_w.shape == (nq,)
        assert self.gas_ka.shape == (nq, self.nlayers)
        assert self.gas_ks.shape == (nq, self.nlayers)
        assert np.all(self.band_lo < self.band_hi)
        assert np.all(self.band_hi[:-1] <= self.band_lo[1:])
        if self.cloud_lwc is not None:
            assert self.cloud_lwc.dtype == np.float32 and self.cloud_lwc.ndim == 3
            assert self.cloud_sigma_ext.shape == (self.nbands,)


@dataclass
class Request:
    """One htrdr-atmosphere run: sensor, spectral domain, output and spp."""

    mode: int
    width: int
    height: int
    spp: int
    wlen_range: Tuple[float, float] = (550.0, 550.0)  # nm (-s sw=|lw=)
    ref_temperature: float = 5778.0  # K (-s Tref=)
    # camera (-C / -P)
    camera_type: int = CAMERA_PERSPECTIVE
    cam_pos: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    cam_tgt: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    cam_up: Tuple[float, float, float] = (0.0, 0.0, 1.0)
    fov_deg: float = 70.0
    lens_radius: float = 0.0
    focal_dst: float = 1.0
    ortho_height: float = 1.0
    # flux sensor rectangle (-p)
    rect_pos: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rect_tgt: Tuple[float, float, float] = (0.0, 0.0, 1.0)
    rect_up: Tuple[float, float, float] = (0.0, 1.0, 0.0)
    rect_size: Tuple[float, float] = (1.0, 1.0)
    seed: int = 0
    name: str = "request"

    @property
    def realisations_per_pixel(self) -> int:
        return self.spp * (3 if self.mode == MODE_IMAGE_CIE else 1)

    @property
    def realisations(self) -> int:
        return self.width * self.height * self.realisations_per_pixel

    @property
    def pixel_size(self) -> int:
        """Bytes per pixel of the reference's pixel structs (htrdr_atmosphere_c.h:46-76)."""
        return 80 if self.mode == MODE_IMAGE_CIE else 64


# ---------------------------------------------------------------------------
# Building blocks
# ---------------------------------------------------------------------------
def rayleigh_ks0(wlen_nm: np.ndarray | float) -> np.ndarray | float:
    """Sea-level Rayleigh scattering coefficient (1/m), lambda^-4 law."""
    return 1.16e-5 * (550.0 / np.asarray(wlen_nm, dtype=np.float64)) ** 4


def layers_uniform(top: float = 50000.0, n: int = 50) -> np.ndarray:
    return np.linspace(0.0, top, n + 1, dtype=np.float64)


def temperature_profile(layer_z: np.ndarray) -> np.ndarray:
    """288 K at the surface, -6.5 K/km up to 11 km, isothermal above."""
    zmid = 0.5 * (layer_z[:-1] + layer_z[1:])
    t = 288.0 - 6.5e-3 * np.minimum(zmid, 11000.0)
    return t.astype(np.float32)


def lwc_lognormal(shape_zyx, seed: int, median_gm3: float = 0.2, sigma: float = 0.8) -> np.ndarray:
    rng = np.random.default_rng(seed)
    g = rng.standard_normal(shape_zyx)
    lwc = median_gm3 * 1e-3 * np.exp(sigma * g)  # kg/m^3
    return lwc.astype(np.float32)


def lwc_power_law(shape_zyx, seed: int, mean_gm3: float = 0.3, sigma: float = 0.8) -> np.ndarray:
    """Gaussian noise filtered to a k^-5/3 power spectrum, exponentiated and
    rescaled to the requested mean."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape_zyx
    noise = rng.standard_normal(shape_zyx)
    f = np.fft.rfftn(noise)
    kz = np.fft.fftfreq(nz)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    kx = np.fft.rfftfreq(nx)[None, None, :]
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    k[0, 0, 0] = 1.0
    amp = k ** (-5.0 / 6.0)  # power ~ k^-5/3
    amp[0, 0, 0] = 0.0
    g = np.fft.irfftn(f * amp, s=shape_zyx, axes=(0, 1, 2))
    g = (g - g.mean()) / (g.std() + 1e-30)
    field_ = np.exp(sigma * g)
    field_ *= (mean_gm3 * 1e-3) / field_.mean()
    return field_.astype(np.float32)


def gas_sw(layer_z: np.ndarray, band_lo, band_hi, nquads, seed: int,
           k0_range=(1e-6, 1e-3), scale_height: float = 8000.0):
    """Per (band, quad, layer) absorption k0*exp(-z/H) with k0 log-uniform,
    Rayleigh scattering with the same scale height."""
    rng = np.random.default_rng(seed)
    zmid = 0.5 * (layer_z[:-1] + layer_z[1:])
    prof = np.exp(-zmid / scale_height)
    rows_a, rows_s, w = [], [], []
    for b in range(len(band_lo)):
        lc = 0.5 * (band_lo[b] + band_hi[b])
        ks0 = rayleigh_ks0(lc)
        q = int(nquads[b])
        k0 = 10.0 ** rng.uniform(math.log10(k0_range[0]), math.log10(k0_range[1]), size=q)
        ww = rng.uniform(0.2, 1.0, size=q) if q > 1 else np.ones(1)
        w.append(ww / ww.sum())
        for iq in range(q):
            rows_a.append(k0[iq] * prof)
            rows_s.append(ks0 * prof)
    return (np.asarray(rows_a, dtype=np.float32), np.asarray(rows_s, dtype=np.float32),
            np.concatenate(w).astype(np.float64))


def gas_lw(layer_z: np.ndarray, band_lo, band_hi, nquads, seed: int,
           k_range=(1e-6, 1e2)):
    """Per (band, quad, layer) absorption log-uniform in k_range (1/m), seeded
    quadrature weights summing to 1, negligible Rayleigh scattering."""
    rng = np.random.default_rng(seed)
    nl = len(layer_z) - 1
    zmid = 0.5 * (layer_z[:-1] + layer_z[1:])
    rows_a, rows_s, w = [], [], []
    for b in range(len(band_lo)):
        lc = 0.5 * (band_lo[b] + band_hi[b])
        q = int(nquads[b])
        ww = rng.uniform(0.2, 1.0, size=q)
        w.append(ww / ww.sum())
        for iq in range(q):
            ka = 10.0 ** rng.uniform(math.log10(k_range[0]), math.log10(k_range[1]), size=nl)
            rows_a.append(ka)
            rows_s.append(rayleigh_ks0(lc) * np.exp(-zmid / 8000.0))
    return (np.asarray(rows_a, dtype=np.float32), np.asarray(rows_s, dtype=np.float32),
            np.concatenate(w).astype(np.float64))


def _cloud_optics(nbands: int, ssa: float, g: float = 0.85):
    return (np.full(nbands, SIGMA_EXT_CLOUD, dtype=np.float32),
            np.full(nbands, ssa, dtype=np.float32),
            np.full(nbands, g, dtype=np.float32))


# ---------------------------------------------------------------------------
# The five workloads
# ---------------------------------------------------------------------------
def config_c1(scale: float = 1.0, spp: Optional[int] = None) -> Tuple[Scene, Request]:
    """Shortwave image 64x64, 32 spp, one band at 550 nm with one quadrature
    point, 50 gas layers, 32x32x16 lognormal cloud, Lambertian ground 0.2,
    sun zenith 30 deg."""
    layer_z = layers_uniform()
    band_lo = np.array([545.0]); band_hi = np.array([555.0])
    nquads = np.array([1], dtype=np.uint32)
    ka, ks, w = gas_sw(layer_z, band_lo, band_hi, nquads, SEED_S1)
    lwc = lwc_lognormal((16, 32, 32), SEED_S2)
    sig, ssa, g = _cloud_optics(1, 0.999)
    scene = Scene(layer_z=layer_z, layer_T=temperature_profile(layer_z), band_lo=band_lo,
                  band_hi=band_hi, nquads=nquads, quad_w=w, gas_ka=ka, gas_ks=ks,
                  cloud_lwc=lwc, cloud_lower=(0.0, 0.0, 1000.0), cloud_cell=(100.0, 100.0, 62.5),
                  cloud_sigma_ext=sig, cloud_ssa=ssa, cloud_g=g, repeat_clouds=False,
                  ground_reflectivity=0.2, sun_azimuth=30.0, sun_elevation=60.0, name="c1")
    side = max(1, int(round(64 * scale)))
    req = Request(mode=MODE_XWAVE_SW, width=side, height=side, spp=spp or 32,
                  wlen_range=(550.0, 550.0), ref_temperature=5778.0,
                  cam_pos=(1600.0, -3000.0, 900.0), cam_tgt=(1600.0, 1600.0, 1500.0),
                  cam_up=(0.0, 0.0, 1.0), fov_deg=60.0, seed=1, name="c1_sw_image")
    return scene, req


def lw_bands(lo: float = 3000.0, hi: float = 100000.0, n: int = 16):
    edges = np.geomspace(lo, hi, n + 1)
    edges[0], edges[-1] = lo, hi
    return edges[:-1].copy(), edges[1:].copy()


def config_c2(scale: float = 1.0, spp: Optional[int] = None,
              cloud_def=(64, 64, 32)) -> Tuple[Scene, Request]:
    """Longwave flux map 128x128 probes at the ground, 256 realisations per
    probe, 16 bands x 8 quadrature points, per-layer k log-uniform in
    [1e-6, 1e2] 1/m, lapse-rate temperature, surface emissivity 0.95,
    64x64x32 lognormal cloud repeated along X and Y."""
    layer_z = layers_uniform()
    band_lo, band_hi = lw_bands(3000.0, 100000.0, 16)
    nquads = np.full(16, 8, dtype=np.uint32)
    ka, ks, w = gas_lw(layer_z, band_lo, band_hi, nquads, SEED_S1 + 7)
    nx, ny, nz = cloud_def
    lwc = lwc_lognormal((nz, ny, nx), SEED_S2 + 7)
    sig, ssa, g = _cloud_optics(16, 0.999)
    dz = 1000.0 / nz
    scene = Scene(layer_z=layer_z, layer_T=temperature_profile(layer_z), band_lo=band_lo,
                  band_hi=band_hi, nquads=nquads, quad_w=w, gas_ka=ka, gas_ks=ks,
                  cloud_lwc=lwc, cloud_lower=(0.0, 0.0, 1000.0), cloud_cell=(100.0, 100.0, dz),
                  cloud_sigma_ext=sig, cloud_ssa=ssa, cloud_g=g, repeat_clouds=True,
                  ground_reflectivity=0.05, ground_temperature=288.0, name="c2")
    side = max(1, int(round(128 * scale)))
    ext = nx * 100.0
    req = Request(mode=MODE_FLUX_LW, width=side, height=side, spp=spp or 256,
                  wlen_range=(3000.0, 100000.0), ref_temperature=290.0,
                  rect_pos=(0.5 * ext, 0.5 * ext, 0.0), rect_tgt=(0.5 * ext, 0.5 * ext, 1.0),
                  rect_up=(0.0, 1.0, 0.0), rect_size=(ext, ext), seed=2, name="c2_lw_flux")
    return scene, req


def config_c3(scale: float = 1.0, spp: Optional[int] = None,
              cloud_def=(256, 256, 64), nbands: int = 30, nquad: int = 16) -> Tuple[Scene, Request]:
    """CIE XYZ image 512x512, 64 spp x 3 channels, 30 bands x 16 quadrature
    points, 256x256x64 cloud of 50 m cells with a k^-5/3 LWC field."""
    layer_z = layers_uniform()
    edges = np.linspace(380.0, 780.0, nbands + 1)
    band_lo, band_hi = edges[:-1].copy(), edges[1:].copy()
    nquads = np.full(nbands, nquad, dtype=np.uint32)
    ka, ks, w = gas_sw(layer_z, band_lo, band_hi, nquads, SEED_S3 + 1)
    nx, ny, nz = cloud_def
    lwc = lwc_power_law((nz, ny, nx), SEED_S3)
    sig, ssa, g = _cloud_optics(nbands, 0.999)
    scene = Scene(layer_z=layer_z, layer_T=temperature_profile(layer_z), band_lo=band_lo,
                  band_hi=band_hi, nquads=nquads, quad_w=w, gas_ka=ka, gas_ks=ks,
                  cloud_lwc=lwc, cloud_lower=(0.0, 0.0, 1000.0), cloud_cell=(50.0, 50.0, 50.0),
                  cloud_sigma_ext=sig, cloud_ssa=ssa, cloud_g=g, repeat_clouds=False,
                  ground_reflectivity=0.2, sun_azimuth=120.0, sun_elevation=45.0, name="c3")
    side = max(1, int(round(512 * scale)))
    ex, ey = nx * 50.0, ny * 50.0
    req = Request(mode=MODE_IMAGE_CIE, width=side, height=side, spp=spp or 64,
                  wlen_range=(380.0, 780.0), ref_temperature=5778.0,
                  cam_pos=(0.5 * ex, -0.9 * ey, 1500.0), cam_tgt=(0.5 * ex, 0.5 * ey, 2200.0),
                  cam_up=(0.0, 0.0, 1.0), fov_deg=60.0, seed=3, name="c3_cie_image")
    return scene, req


def batched_scenes(scale: float = 1.0) -> List[Scene]:
    """The three cloud scenes of the batched/serving workloads (128^3,
    256x256x64, 512x512x128 at full scale), each with 4 SW bands x 4
    quadrature points over [500, 600] nm and 4 LW bands x 4 quadrature points
    over [8000, 12000] nm."""
    defs = [(128, 128, 128), (256, 256, 64), (512, 512, 128)]
    seeds = [SEED_S4, SEED_S5, SEED_S6]
    scenes = []
    for d, s in zip(defs, seeds):
        nx, ny, nz = (max(2, int(round(v * scale))) for v in d)
        layer_z = layers_uniform()
        sw_lo = np.linspace(500.0, 600.0, 5)
        lw_e = np.linspace(8000.0, 12000.0, 5)
        band_lo = np.concatenate([sw_lo[:-1], lw_e[:-1]])
        band_hi = np.concatenate([sw_lo[1:], lw_e[1:]])
        nquads = np.full(8, 4, dtype=np.uint32)
        ka_s, ks_s, w_s = gas_sw(layer_z, band_lo[:4], band_hi[:4], nquads[:4], s)
        ka_l, ks_l, w_l = gas_lw(layer_z, band_lo[4:], band_hi[4:], nquads[4:], s + 1,
                                 k_range=(1e-6, 1e-2))
        ka = np.concatenate([ka_s, ka_l]); ks = np.concatenate([ks_s, ks_l])
        w = np.concatenate([w_s, w_l])
        lwc = lwc_power_law((nz, ny, nx), s)
        sig = np.full(8, SIGMA_EXT_CLOUD, dtype=np.float32)
        ssa = np.full(8, 0.999, dtype=np.float32)  # the cloud recipe's albedo in every band
        g = np.full(8, 0.85, dtype=np.float32)
        cell = 6400.0 / max(nx, ny) if scale != 1.0 else 50.0
        dz = 1000.0 / nz  # a 1 km thick cloud layer based at 1 km
        scenes.append(Scene(layer_z=layer_z, layer_T=temperature_profile(layer_z),
                            band_lo=band_lo, band_hi=band_hi, nquads=nquads, quad_w=w,
                            gas_ka=ka, gas_ks=ks, cloud_lwc=lwc,
                            cloud_lower=(0.0, 0.0, 1000.0), cloud_cell=(cell, cell, dz),
                            cloud_sigma_ext=sig, cloud_ssa=ssa, cloud_g=g,
                            repeat_clouds=True, ground_reflectivity=0.2,
                            sun_azimuth=45.0, sun_elevation=50.0,
                            name=f"batch_{nx}x{ny}x{nz}"))
    return scenes


def batched_requests(n: int = 64, seed: int = SEED_S4, side_range=(32, 1024),
                     spp_range=(16, 1024), nscenes: int = 3) -> List[Tuple[int, Request]]:
    """Uneven request mix: image side and spp log-uniform, 50 % SW / 50 % LW,
    each on one of the batched scenes.  Returns (scene index, request)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        side = int(round(math.exp(rng.uniform(math.log(side_range[0]), math.log(side_range[1])))))
        spp = int(round(math.exp(rng.uniform(math.log(spp_range[0]), math.log(spp_range[1])))))
        sw = (i % 2) == 0
        isc = int(rng.integers(0, nscenes))
        if sw:
            req = Request(mode=MODE_XWAVE_SW, width=side, height=side, spp=spp,
                          wlen_range=(500.0, 600.0), ref_temperature=5778.0,
                          cam_pos=(3200.0, -4000.0, 1200.0), cam_tgt=(3200.0, 3200.0, 2500.0),
                          fov_deg=60.0, seed=1000 + i, name=f"req{i}_sw")
        else:
            req = Request(mode=MODE_XWAVE_LW, width=side, height=side, spp=spp,
                          wlen_range=(8000.0, 12000.0), ref_temperature=290.0,
                          cam_pos=(3200.0, 3200.0, 10.0), cam_tgt=(3300.0, 3300.0, 3000.0),
                          fov_deg=60.0, seed=1000 + i, name=f"req{i}_lw")
        out.append((isc, req))
    return out


def homogeneous_slab(k_abs: float, k_sca: float = 0.0, top: float = 1000.0,
                     temperature: float = 250.0, band=(545.0, 555.0), ground_reflectivity=0.0,
                     ground_temperature: float = 0.0, has_ground: bool = True,
                     sun_elevation: float = 60.0) -> Scene:
    """One homogeneous layer [0, top] with no cloud: the closed-form cases
    (Beer-Lambert transmissivity, isothermal slab emission, single scattering)."""
    layer_z = np.array([0.0, top], dtype=np.float64)
    return Scene(layer_z=layer_z, layer_T=np.array([temperature], dtype=np.float32),
                 band_lo=np.array([band[0]]), band_hi=np.array([band[1]]),
                 nquads=np.array([1], dtype=np.uint32), quad_w=np.array([1.0]),
                 gas_ka=np.array([[k_abs]], dtype=np.float32),
                 gas_ks=np.array([[k_sca]], dtype=np.float32), cloud_lwc=None,
                 cloud_sigma_ext=np.zeros(1, np.float32), cloud_ssa=np.zeros(1, np.float32),
                 cloud_g=np.zeros(1, np.float32), has_ground=has_ground,
                 ground_reflectivity=ground_reflectivity, ground_temperature=ground_temperature,
                 sun_elevation=sun_elevation, name="slab")


def with_cloud_box(scene: Scene, lwc: np.ndarray, lower, cell, ssa: float, g: float,
                   repeat: bool = False) -> Scene:
    s = dataclasses.replace(scene)
    s.cloud_lwc = lwc.astype(np.float32)
    s.cloud_lower = tuple(lower)
    s.cloud_cell = tuple(cell)
    s.cloud_sigma_ext = np.full(scene.nbands, SIGMA_EXT_CLOUD, np.float32)
    s.cloud_ssa = np.full(scene.nbands, ssa, np.float32)
    s.cloud_g = np.full(scene.nbands, g, np.float32)
    s.repeat_clouds = repeat
    return s


def terrain_materials() -> dict:
    """Materials of the synthetic terrain: the semi-transparent atmosphere,
    a Lambertian soil with a tabulated spectral reflectivity and a specular
    water surface (htrdr-materials list with its BRDF tables inline)."""
    return {
        "air": None,
        "soil": (290.0, [(300.0, "lambertian", 0.08), (550.0, "lambertian", 0.25),
                         (900.0, "lambertian", 0.40), (8000.0, "lambertian", 0.05)]),
        "water": (285.0, [(400.0, "specular", 0.06), (10000.0, "specular", 0.02)]),
    }


def terrain_obj(size: float = 3200.0, n: int = 16, amp: float = 150.0, seed: int = SEED_S5,
                origin=(0.0, 0.0), water_below: float = 0.35) -> str:
    """An htrdr-obj heightfield over [ox, ox+size] x [oy, oy+size]: n x n
    quads of two triangles, heights a seeded sum of sines in [0, amp], the
    quads whose mean height is under `water_below' x amp in the water
    group, the others soil.  Triangles are clockwise seen from above so the
    atmosphere is on their front side (`usemtl air:soil')."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(1.0, 3.0, size=(3, 2)) * 2.0 * math.pi / size
    ph = rng.uniform(0.0, 2.0 * math.pi, size=3)
    xs = origin[0] + np.linspace(0.0, size, n + 1)
    ys = origin[1] + np.linspace(0.0, size, n + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    H = sum(np.sin(k[i, 0] * X + k[i, 1] * Y + ph[i]) for i in range(3))
    H = (H - H.min()) / max(float(np.ptp(H)), 1e-9) * amp
    lines = [f"v {X[j, i]:.3f} {Y[j, i]:.3f} {H[j, i]:.3f}" for j in range(n + 1) for i in range(n + 1)]
    groups = {"air:soil": [], "air:water": []}
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i + 1
            b, c, d = a + 1, a + (n + 1), a + (n + 1) + 1
            key = "air:water" if H[j:j + 2, i:i + 2].mean() < water_below * amp else "air:soil"
            # (a, c, b) and (b, c, d) are clockwise seen from +z
            groups[key].append(f"f {a} {c} {b}")
            groups[key].append(f"f {b} {c} {d}")
    for key, faces in groups.items():
        if faces:
            lines.append(f"usemtl {key}")
            lines.extend(faces)
    return "\n".join(lines) + "\n"


def with_terrain(scene: Scene, size: float = 3200.0, n: int = 16, amp: float = 150.0,
                 seed: int = SEED_S5, repeat: bool = True) -> Scene:
    """The scene over the synthetic terrain (replacing its plane ground)."""
    s = dataclasses.replace(scene)
    s.ground_mesh = parse_htrdr_obj(terrain_obj(size, n, amp, seed), terrain_materials(),
                                    sky_mtl="air", repeat=repeat)
    return s
