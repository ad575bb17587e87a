"""The C ABI without a GPU: the library loads, exports every function include/heatflow_b200.h declares, and its
record layouts match the header (ctypes mirror vs a C compiler)."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "heatflow_b200.h")


def _lib_path():
    from heatflow_mpm import _build
    if not os.path.exists(_build.OUT):
        if shutil.which("nvcc") is None:
            pytest.skip("libheatflow_b200.so not built and nvcc unavailable")
        _build.build()
    return _build.OUT


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(hf_\w+)\s*\(", src, flags=re.M)))


def test_exports_every_declared_function():
    lib = C.CDLL(_lib_path())
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_pure_functions_without_gpu():
    from heatflow_mpm import _lib
    L = _lib.load()
    assert L.hf_abi_version() == 1
    assert L.hf_cells_per_chunk() == 1024
    assert L.hf_chunks_for(96) == 864 and L.hf_chunks_for(10) == 1
    assert L.hf_tiles_for(96) == 864 and L.hf_tiles_for(48) == 144
    assert L.hf_workspace_bytes(1, 864, 864) > 6 * 8 * 864


def test_record_layout_matches_header(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc unavailable")
    from heatflow_mpm import _lib
    prog = tmp_path / "sizes.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\nint main(){printf("%%zu %%zu %%zu %%zu %%zu %%zu '
                    '%%zu %%zu %%zu\\n",sizeof(hf_scene),sizeof(hf_plan),sizeof(hf_scene_state),offsetof(hf_scene,T),'
                    'offsetof(hf_scene,state),offsetof(hf_scene_state,rhs_mean),sizeof(hf_heater_geometry),'
                    'offsetof(hf_heater_geometry,m_face),offsetof(hf_heater_geometry,sphere_c));return 0;}\n' % HEADER)
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", str(prog), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    want = [C.sizeof(_lib.Scene), C.sizeof(_lib.Plan), C.sizeof(_lib.SceneState), _lib.Scene.T.offset,
            _lib.Scene.state.offset, _lib.SceneState.rhs_mean.offset, C.sizeof(_lib.HeaterGeometry),
            _lib.HeaterGeometry.m_face.offset, _lib.HeaterGeometry.sphere_c.offset]
    assert [int(x) for x in got] == want


def test_heater_masks_bit_exact_vs_reference():
    """heatflow_mpm.heater reproduces the reference Heater.masks (golden SHA-256 of every output array)."""
    import ast
    import glob
    import hashlib
    import numpy as np
    from heatflow_mpm.heater import Heater
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    files = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "heater_*.npz")))
    assert len(files) >= 8
    for f in files:
        g = np.load(f)
        kw = ast.literal_eval(str(g["kwargs"]))
        L, h, n = float(g["L"]), float(g["h"]), int(g["n"])
        cell, solid, source, rate, kf, mf, geom = Heater(**kw).masks(n, h, (L / 2, L / 2), float(g["rho"]))
        arrs = dict(cell=cell.astype(np.int8), solid=solid, source=source, kx=kf[0], ky=kf[1], kz=kf[2], mx=mf[0],
                    my=mf[1], mz=mf[2])
        for k, v in arrs.items():
            assert sha(v) == str(g["sha_" + k]), (f, k)
        assert rate == float(g["rate"])
        assert np.array_equal(np.bincount(cell.ravel(), minlength=5), g["counts"])
        assert np.array_equal(np.array(geom["centre"]), g["centre"])
