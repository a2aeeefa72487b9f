"""Writes the htrdr-image golden fixtures: for each output mode, a seeded
5x3 pixel buffer (`image_<mode>.npy', the reference's pixel structs) and the
text the reference's dump_buffer prints for it (`image_<mode>.txt'),
restated in Python (src/atmosphere/htrdr_atmosphere_draw_map.c:477-641).

    python tests/golden/make_image_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import test_image_writer as T  # noqa: E402
from htrdr_kmin_b200 import scene as S  # noqa: E402

MODES = {"xwave_sw": S.MODE_XWAVE_SW, "xwave_lw": S.MODE_XWAVE_LW, "image_cie": S.MODE_IMAGE_CIE,
         "flux_sw": S.MODE_FLUX_SW, "flux_lw": S.MODE_FLUX_LW}


def main():
    for name, mode in MODES.items():
        buf = T._random_map(mode, 5, 3, seed=100 + mode)
        np.save(os.path.join(HERE, f"image_{name}.npy"), buf)
        text, _, _ = T._reference_text(mode, buf)
        with open(os.path.join(HERE, f"image_{name}.txt"), "w") as f:
            f.write(text)


if __name__ == "__main__":
    main()
