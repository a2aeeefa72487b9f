"""htrdr_gpu_write_image: the htrdr-image file of a map and the run summaries,
checked byte for byte against a Python restatement of the reference's
dump_buffer / dump_accum (src/atmosphere/htrdr_atmosphere_draw_map.c:477-641)
on seeded pixel buffers of every mode, empty pixels included.  Host code
only: no GPU needed."""
import math
import os

import numpy as np
import pytest

from htrdr_kmin_b200 import api, build
from htrdr_kmin_b200 import scene as S


def _estimate(s, s2, n):
    # htrdr_accum_get_estimation (src/core/htrdr_accum.h:48-66)
    if n == 0:
        return 0.0, 0.0
    e = s / n
    return e, math.sqrt(max(s2 / n - e * e, 0.0) / n)


def _dump_accum(s, s2, n, total):
    if n == 0:
        return "0 0 "
    e, se = _estimate(s, s2, n)
    if total is not None:
        total[0] += s
        total[1] += s2
        total[2] += n
    return "%g %g " % (e, se)


def _reference_text(mode, buf):
    time_t, flux_t = [0.0, 0.0, 0], [0.0, 0.0, 0]
    out = ["%d %d\n" % (buf.shape[1], buf.shape[0])]
    for y in range(buf.shape[0]):
        for x in range(buf.shape[1]):
            p = buf[y, x]
            if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
                line = _dump_accum(p["sum"], p["sum2"], int(p["n"]), flux_t) + "0 0 0 0 "
            elif mode == S.MODE_IMAGE_CIE:
                line = "%g %g " % (p["X"], p["X_se"]) + "%g %g " % (p["Y"], p["Y_se"]) \
                    + "%g %g " % (p["Z"], p["Z_se"])
            else:
                line = "%g %g %f %f 0 0 " % (p["Tb"], p["Tb_se"], p["L"], p["L_se"])
            line += _dump_accum(p["t_sum"], p["t_sum2"], int(p["t_n"]), time_t)
            out.append(line + "\n")
        out.append("\n")
    return "".join(out), time_t, flux_t


def _random_map(mode, w, h, seed):
    rng = np.random.default_rng(seed)
    buf = np.zeros((h, w), dtype=api.pixel_dtype(mode))
    n = rng.integers(0, 300, size=(h, w))
    n[0, 0] = 0  # an empty pixel prints "0 0"
    wsum = rng.lognormal(0, 2, size=(h, w)) * n
    buf["t_n"] = n
    buf["t_sum"] = rng.uniform(1, 50, size=(h, w)) * n
    buf["t_sum2"] = buf["t_sum"] ** 2 / np.maximum(n, 1) * rng.uniform(1, 2, size=(h, w))
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        buf["n"] = n
        buf["sum"] = wsum
        buf["sum2"] = wsum ** 2 / np.maximum(n, 1) * rng.uniform(1, 3, size=(h, w))
    elif mode == S.MODE_IMAGE_CIE:
        for c in "XYZ":
            buf[c] = rng.lognormal(-8, 1, size=(h, w))
            buf[c + "_se"] = buf[c] * rng.uniform(0, 0.2, size=(h, w))
    else:
        buf["L"] = rng.lognormal(-5, 2, size=(h, w))
        buf["L_se"] = buf["L"] * rng.uniform(0, 0.2, size=(h, w))
        buf["Tb"] = rng.uniform(200, 300, size=(h, w))
        buf["Tb_se"] = rng.uniform(0, 3, size=(h, w))
    return buf


@pytest.mark.parametrize("mode", [S.MODE_XWAVE_SW, S.MODE_XWAVE_LW, S.MODE_IMAGE_CIE,
                                  S.MODE_FLUX_SW, S.MODE_FLUX_LW])
def test_image_file_matches_reference_dump(tmp_path, mode):
    build.build()
    buf = _random_map(mode, 13, 7, seed=mode + 1)
    path = str(tmp_path / "map.txt")
    summary = api.write_image(mode, buf, path)
    with open(path) as f:
        got = f.read()
    want, time_t, flux_t = _reference_text(mode, buf)
    assert got == want
    e, se = _estimate(*time_t)
    assert summary["path_time_n"] == time_t[2]
    assert summary["path_time_E"] == pytest.approx(e, rel=1e-12)
    assert summary["path_time_SE"] == pytest.approx(se, rel=1e-12)
    if mode in (S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        e, se = _estimate(*flux_t)
        assert summary["flux_n"] == flux_t[2]
        assert summary["flux_E"] == pytest.approx(e, rel=1e-12)
    else:
        assert summary["flux_n"] == 0


def test_image_writer_rejects_bad_arguments(tmp_path):
    buf = _random_map(S.MODE_XWAVE_SW, 4, 3, seed=0)
    with pytest.raises(api.HtrdrError) as e:
        api.write_image(S.MODE_IMAGE_CIE, buf, str(tmp_path / "x.txt"))  # wrong pixel size
    assert e.value.code == api.RES_BAD_ARG
    with pytest.raises(api.HtrdrError) as e:
        api.write_image(S.MODE_XWAVE_SW, buf, os.path.join(str(tmp_path), "no", "such", "dir.txt"))
    assert e.value.code == api.RES_IO_ERR


@pytest.mark.parametrize("name", ["xwave_sw", "xwave_lw", "image_cie", "flux_sw", "flux_lw"])
def test_image_golden_fixtures(tmp_path, name):
    """The writer's output for the committed pixel buffers equals the
    committed text (tests/golden, made by make_image_golden.py)."""
    build.build()
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    mode = {"xwave_sw": S.MODE_XWAVE_SW, "xwave_lw": S.MODE_XWAVE_LW, "image_cie": S.MODE_IMAGE_CIE,
            "flux_sw": S.MODE_FLUX_SW, "flux_lw": S.MODE_FLUX_LW}[name]
    buf = np.load(os.path.join(golden, f"image_{name}.npy"))
    assert buf.dtype == api.pixel_dtype(mode)
    path = str(tmp_path / "map.txt")
    api.write_image(mode, buf, path)
    with open(path) as f, open(os.path.join(golden, f"image_{name}.txt")) as g:
        assert f.read() == g.read()
