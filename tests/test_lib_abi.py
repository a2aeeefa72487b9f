"""The C-ABI library loads, exports every function include/htrdr_gpu.h
declares, and refuses to compute without a GPU (no CPU fallback).  No GPU
needed."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from htrdr_kmin_b200 import api, build
from htrdr_kmin_b200 import scene as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "htrdr_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(htrdr_gpu_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_function():
    path = build.build()
    lib = C.CDLL(path)
    names = header_functions()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(api.EXPORTED) <= set(names)


def test_version_and_no_device_behaviour():
    L = api.lib()
    assert b"sm_100a" in L.htrdr_gpu_version()
    ndev = api.device_count()
    if ndev == 0:
        # no CPU fallback: creating a scene without a device is refused
        sc, _ = S.config_c1(scale=0.125)
        with pytest.raises(api.HtrdrError) as e:
            api.GpuScene(sc)
        assert e.value.code == api.RES_BAD_OP


def test_bad_arguments_are_rejected_before_any_device_work():
    L = api.lib()
    h = C.c_void_p()
    assert L.htrdr_gpu_scene_create(0, None, C.byref(h)) == api.RES_BAD_ARG
    st = api.Stats()
    assert L.htrdr_gpu_draw_map(None, None, None, None, C.byref(st)) == api.RES_BAD_ARG
    assert L.htrdr_gpu_draw_maps_batched(None, 0, None, None) == api.RES_BAD_ARG


def test_pixel_layouts_match_reference_structs():
    # atmosphere_pixel_xwave / _flux / _image (src/atmosphere/htrdr_atmosphere_c.h:46-76)
    assert api.PIXEL_XWAVE.itemsize == 64
    assert api.PIXEL_FLUX.itemsize == 64
    assert api.PIXEL_IMAGE.itemsize == 80
    assert C.sizeof(api.BufferLayout) == 40


def test_engine_selection_and_mode_tuning_host_checks():
    L = api.lib()
    # a scene is required; unknown engines and invalid tunings are refused
    assert L.htrdr_gpu_scene_set_engine(None, api.ENGINE_PLAIN, None) == api.RES_BAD_ARG
    lw = api.mode_tuning(S.MODE_FLUX_LW)
    sw = api.mode_tuning(S.MODE_XWAVE_SW)
    cie = api.mode_tuning(S.MODE_IMAGE_CIE)
    for t in (lw, sw, cie):
        assert t.block_size % 32 == 0 and 0 < t.block_size <= 512 and t.queue_chunk >= 1
    # every mode on the wavefront (LW walks run whole in its trace stage); the
    # tail megakernel takes over earlier for LW and CIE than for SW
    assert lw.engine == sw.engine == cie.engine == api.ENGINE_WAVEFRONT
    assert sw.wave_tail > 0 and cie.wave_tail > 0 and lw.wave_tail > 0
    assert lw.wave_tail == cie.wave_tail > sw.wave_tail
    assert lw.trace_budget == sw.trace_budget == cie.trace_budget == 256


def test_tuning_struct_and_engine_fields():
    # struct htrdr_gpu_tuning: eight uint32 fields, the engine among them
    assert C.sizeof(api.Tuning) == 32
    t = api.default_tuning()
    assert t.engine == api.ENGINE_PERSISTENT and t.wave_slots == 0 and t.trace_budget == 0
    for mode in (S.MODE_XWAVE_SW, S.MODE_XWAVE_LW, S.MODE_IMAGE_CIE, S.MODE_FLUX_SW, S.MODE_FLUX_LW):
        assert api.mode_tuning(mode).engine in (api.ENGINE_PERSISTENT, api.ENGINE_WAVEFRONT)


@pytest.mark.parametrize("struct,mirror", [
    ("htrdr_gpu_scene_desc", "SceneDesc"), ("htrdr_gpu_request", "Request"),
    ("htrdr_gpu_buffer_layout", "BufferLayout"), ("htrdr_gpu_stats", "Stats"),
    ("htrdr_gpu_map_summary", "MapSummary"), ("htrdr_gpu_batch_item", "BatchItem"),
    ("htrdr_gpu_tuning", "Tuning"), ("htrdr_gpu_server_config", "ServerConfig"),
    ("htrdr_gpu_server_stats", "ServerStats")])
def test_struct_layout_matches_header(tmp_path, struct, mirror):
    """Every field of the ctypes mirror sits at the C struct's offset."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    cls = getattr(api, mirror)
    names = [f[0] for f in cls._fields_]
    src = ["#include <stddef.h>", "#include <stdio.h>", '#include "htrdr_gpu.h"', "int main(void) {",
           f'  printf("%zu\\n", sizeof(struct {struct}));']
    src += [f'  printf("%zu\\n", offsetof(struct {struct}, {n}));' for n in names]
    src += ["  return 0;", "}"]
    (tmp_path / "l.c").write_text("\n".join(src))
    exe = tmp_path / "l"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(tmp_path / "l.c"), "-o", str(exe)],
                   check=True)
    out = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert out[0] == C.sizeof(cls)
    assert out[1:] == [getattr(cls, n).offset for n in names]


def test_c_caller(tmp_path):
    """A strict-C99 caller (tests/c/abi_caller.c) compiles against the header
    with every warning as an error, links the library and checks the calls
    that need no device."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lib = build.build()
    exe = tmp_path / "abi_caller"
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Wpedantic", "-Werror",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "abi_caller.c"),
                    "-L", libdir, "-lhtrdr_gpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "map.txt")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "abi_caller ok" in r.stdout
