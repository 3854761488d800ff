"""The C ABI library loads and exports every entry point its header declares
(no compute calls: these run without a GPU)."""

import ctypes
import os
import re

import numpy as np
import pytest

import snogray_b200 as sb
from snogray_b200 import scenes


def test_library_is_in_tree_and_loads():
    assert os.path.exists(sb.LIB_PATH)
    assert sb.version().startswith("snogray_b200")


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(sb.LIB_PATH)
    names = sb.exported_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_header_structs_match_ctypes_layout():
    # Sizes the Python binding assumes for the C structs.
    assert ctypes.sizeof(sb.SnogCamera) == 14 * 4
    assert ctypes.sizeof(sb.SnogRenderParams) == 8 * 4 + 8 + 2 * 4
    assert scenes.MAT_DTYPE.itemsize == 4 * 14
    assert scenes.SPHERE_DTYPE.itemsize == 20
    assert scenes.TRIPAR_DTYPE.itemsize == 44


def test_invalid_scene_is_rejected_with_status():
    sd = scenes.cornell_box()
    sd.tri_mat = sd.tri_mat.copy()
    sd.triangles = sd.triangles.copy()
    sd.triangles[0, 0] = 999                      # vertex index out of range
    with pytest.raises(sb.SnogError) as e:
        sb.Scene(sd, device=False)
    assert e.value.code == sb.SNOG_EINVAL
    assert "out of range" in str(e.value)


def test_non_monotone_parts_rejected():
    with pytest.raises(ValueError):
        sb.SceneData(materials=scenes.cornell_box().materials,
                     vertices=np.zeros((3, 3), np.float32),
                     triangles=np.array([[0, 1, 2], [0, 1, 2]], np.uint32),
                     tri_mat=np.array([1, 0], np.uint32))


def test_host_only_scene_refuses_tracing():
    with sb.Scene(scenes.cornell_box(), device=False) as sc:
        with pytest.raises(sb.SnogError) as e:
            sc.trace(scenes.random_rays(4), 2)
        assert "host-only" in str(e.value)
