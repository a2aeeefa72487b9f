"""Golden vectors of the reference's own code for the GPU parity tests.

Run where the reference tree is present (it builds oracle/_ref, the
reference's atmosphere hot-path C files compiled unmodified over the oracle's
scenes; see oracle/reference.py):

    python tests/golden/make_ref_golden.py

It writes tests/golden/reference_realisations.npz with, for every parity case
of reference_cases():

* ``<case>/weights``: the weight of every realisation of the map (one stream
  per (pixel, realisation), request seed), NaN for rejected probes;
* ``<case>/map_*``: the reference's atmosphere_draw_map of the same request at
  seed ``MAP_SEED`` and ``MAP_SPP`` realisations per pixel (per-pixel
  estimates and standard errors, and the brightness temperature of LW images).

The GPU tests compare the CUDA path with these vectors realisation by
realisation and pixel by pixel without the reference tree (it is absent on the
GPU machines)."""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from htrdr_kmin_b200 import scene as S  # noqa: E402

OUT = os.path.join(HERE, "reference_realisations.npz")
MAP_SEED = 4242
MAP_SPP = {"xwave_sw": 256, "flux_lw": 256, "image_cie": 64, "flux_sw": 256, "xwave_lw": 256,
           "xwave_sw_specular": 256}


def reference_cases():
    """(name, scene, request, octree properties) of the parity cases: the five
    output modes on reduced scenes and a specular ground."""
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
    sc, rq = S.config_c1(scale=8 / 64, spp=8)
    sc.ground_brdf, sc.ground_reflectivity = 1, 0.6
    rq.cam_tgt = (1600.0, 1600.0, 0.0)
    out.append(("xwave_sw_specular", sc, rq, 0b111))
    return out


def map_fields(buf, mode):
    """Per-pixel estimates of a pixel buffer: {name: array}."""
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        n = np.maximum(buf["n"].astype(np.float64), 1)
        E = buf["sum"] / n
        return {"E": E, "SE": np.sqrt(np.maximum(buf["sum2"] / n - E * E, 0) / n),
                "n": buf["n"].astype(np.int64)}
    if mode == S.MODE_IMAGE_CIE:
        return {c: buf[c] for c in ("X", "X_se", "Y", "Y_se", "Z", "Z_se")}
    return {"E": buf["L"], "SE": buf["L_se"], "Tb": buf["Tb"], "Tb_se": buf["Tb_se"]}


def main():
    from oracle import reference as R
    if not R.available():
        raise SystemExit("the compiled reference oracle cannot be built here (no reference tree)")
    data = {}
    for name, sc, rq, props in reference_cases():
        rs = R.RefScene(sc, props)
        npix = rq.width * rq.height
        data[f"{name}/weights"] = rs.realisation_weights(rq, 0, npix)
        mq = S.Request(**{**rq.__dict__, "seed": MAP_SEED, "spp": MAP_SPP[name]})
        for k, v in map_fields(rs.draw_map(mq), rq.mode).items():
            data[f"{name}/map_{k}"] = np.asarray(v)
        rs.close()
        print(f"{name}: {data[f'{name}/weights'].size} realisations")
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
