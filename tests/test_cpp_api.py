"""The reference-shaped C++ API (include/snogray_b200.hpp): a C++ program
(tests/cpp/cornell_api.cc) builds the Cornell box with SurfaceGroup / Mesh /
Sphere / Tripar / Lambert / Glass / Glow / Camera / RenderMgr and renders it.

CPU: the header compiles against the C ABI, links the library, and the
flattened scene builds the same octree as the Python scene description.
GPU: its render equals the Python binding's render of the same scene, camera
and parameters (same library call, so only float summation order differs:
rtol 1e-4, atol 1e-5).
"""

import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import snogray_b200 as sb
from snogray_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(ROOT, "snogray_b200")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


@pytest.fixture(scope="module")
def cornell_api(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("cpp") / "cornell_api")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{os.path.join(ROOT, 'include')}", f"-I{CUDA_INC}",
           os.path.join(HERE, "cpp", "cornell_api.cc"), f"-L{LIBDIR}", "-lsnogray_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_scene_matches_python_scene(cornell_api):
    out = subprocess.run([cornell_api, "host"], check=True, capture_output=True, text=True)
    got = json.loads(out.stdout)
    info = sb.Scene(scenes.cornell_box(), device=False).info()
    for k, v in got.items():
        assert info[k] == v, k


def test_cpp_errors_become_exceptions(cornell_api):
    out = subprocess.run([cornell_api, "render", "0", "0", "1", os.devnull], capture_output=True, text=True)
    assert out.returncode == 1 and "error:" in out.stderr


@pytest.mark.gpu
def test_cpp_render_matches_python_render(cornell_api, tmp_path):
    w, h, spp, seed = 48, 40, 16, 3
    f32 = str(tmp_path / "img.f32")
    out = subprocess.run([cornell_api, "render", str(w), str(h), str(spp), f32, str(seed)], check=True,
                         capture_output=True, text=True)
    rec = json.loads(out.stdout)
    img = np.fromfile(f32, np.float32).reshape(h, w, 3)
    c = rec["camera"]
    cam = scenes.Camera()
    cam.pos, cam.forward, cam.right, cam.up = (np.array(c[3 * k:3 * k + 3], np.float32) for k in range(4))
    cam.tan_half_fov_x, cam.tan_half_fov_y = c[12], c[13]
    with sb.Scene(scenes.cornell_box()) as sc:
        ref, st = sc.render(cam, scenes.cornell_params(w, h, spp, seed=seed))
    assert rec["paths"] == st["paths"]
    assert np.isfinite(img).all() and img.mean() > 0
    assert np.allclose(img, ref, rtol=1e-4, atol=1e-5), np.abs(img - ref).max()


# ---- PLY meshes through load_ply_file (tests/cpp/ply_api.cc) -----------------

def _ply_scene_file(tmp_path):
    """The smooth mesh scene's triangles and vertex normals as a binary PLY,
    and the same scene as the Python description: one Cook-Torrance part,
    right-handed, lit by the scene's area light."""
    from test_ply import write_ply
    sd = scenes.mesh_scene(smooth=True)
    # The reference's PLY loader keeps a normal only if some component is
    # positive (and fails on the file otherwise): keep the sphere's upper cap
    # and the floor, whose normals all point up.
    keep = sd.normals[:, 1] > 0.05
    tri_ok = keep[sd.triangles].all(1)
    remap = np.cumsum(keep) - 1
    sd = sb.SceneData(materials=sd.materials, vertices=sd.vertices[keep], normals=sd.normals[keep],
                      triangles=remap[sd.triangles[tri_ok]].astype(np.uint32),
                      tri_mat=sd.tri_mat[tri_ok], tripars=sd.tripars, right_handed=True)
    path = str(tmp_path / "mesh.ply")
    props = [("x", "float"), ("y", "float"), ("z", "float"), ("nx", "float"), ("ny", "float"), ("nz", "float")]
    write_ply(path, "binary_little_endian", props, np.concatenate([sd.vertices, sd.normals], 1),
              sd.triangles.tolist(), face_types=("uchar", "uint"))
    mats = scenes._mats([scenes.material(scenes.MAT_COOK_TORRANCE, (0.7, 0.3, 0.2), (1, 1, 1), m=0.2, ior_n=1.5),
                         scenes.material(scenes.MAT_GLOW, (10.0, 10.0, 10.0))])
    tripars = sd.tripars.copy()
    tripars["mat"] = 1
    v, n, t = sb.load_ply(path)
    py = sb.SceneData(materials=mats, vertices=v, triangles=t, tri_mat=np.zeros(len(t), np.uint32),
                      tripars=tripars, normals=n, right_handed=True)
    return path, py


@pytest.fixture(scope="module")
def ply_api(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("cpp") / "ply_api")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{os.path.join(ROOT, 'include')}", f"-I{CUDA_INC}",
           os.path.join(HERE, "cpp", "ply_api.cc"), f"-L{LIBDIR}", "-lsnogray_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_ply_scene_matches_python_scene(ply_api, tmp_path):
    path, py = _ply_scene_file(tmp_path)
    out = subprocess.run([ply_api, "host", path], check=True, capture_output=True, text=True)
    got = json.loads(out.stdout)
    info = sb.Scene(py, device=False).info()
    for k, v in got.items():
        assert info[k] == v, k


@pytest.mark.gpu
def test_cpp_ply_render_matches_python_render(ply_api, tmp_path):
    path, py = _ply_scene_file(tmp_path)
    w, h, spp, seed = 40, 40, 16, 5
    f32 = str(tmp_path / "img.f32")
    out = subprocess.run([ply_api, "render", path, str(w), str(h), str(spp), f32, str(seed)], check=True,
                         capture_output=True, text=True)
    rec = json.loads(out.stdout)
    img = np.fromfile(f32, np.float32).reshape(h, w, 3)
    c = rec["camera"]
    cam = scenes.Camera()
    cam.pos, cam.forward, cam.right, cam.up = (np.array(c[3 * k:3 * k + 3], np.float32) for k in range(4))
    cam.tan_half_fov_x, cam.tan_half_fov_y = c[12], c[13]
    with sb.Scene(py) as sc:
        ref, st = sc.render(cam, scenes.mesh_params(w, h, spp, seed=seed))
    assert rec["paths"] == st["paths"]
    assert np.isfinite(img).all() and img.mean() > 0
    assert np.allclose(img, ref, rtol=1e-4, atol=1e-5), np.abs(img - ref).max()


# ---- partial renders: RenderPattern, sample-based output, 5-argument render --

LIMIT = dict(w=64, h=48, spp=16, lx=10, ly=8, lw=30, lh=20)


@pytest.mark.gpu
def test_cpp_limit_render_matches_python_window(cornell_api, tmp_path):
    """The reference driver's --limit set-up through the 5-argument
    RenderMgr::render gives the same image as the C ABI's window render, and
    fills the reference's RenderStats fields."""
    c = LIMIT
    f32 = str(tmp_path / "img.f32")
    out = subprocess.run([cornell_api, "limit", str(c["w"]), str(c["h"]), str(c["spp"]), str(c["lx"]), str(c["ly"]),
                          str(c["lw"]), str(c["lh"]), f32, "5"], check=True, capture_output=True, text=True)
    rec = json.loads(out.stdout)
    img = np.fromfile(f32, np.float32).reshape(c["lh"], c["lw"], 3)
    cam = scenes.cornell_camera(c["w"], c["h"])
    pattern = (c["lx"] - 2, c["ly"] - 2, c["lw"] + 4, c["lh"] + 4)
    with sb.Scene(scenes.cornell_box()) as sc:
        ref, st = sc.render_window(cam, scenes.cornell_params(c["w"], c["h"], c["spp"], seed=5), pattern,
                                   (c["lx"], c["ly"], c["lw"], c["lh"]))
    assert rec["paths"] == st["paths"] == (c["lw"] + 4) * (c["lh"] + 4) * c["spp"]
    assert np.isfinite(img).all() and img.mean() > 0
    assert np.allclose(img, ref, rtol=1e-4, atol=1e-5), np.abs(img - ref).max()
    assert rec["scene_intersect_calls"] == rec["closest_rays"] == st["closest_rays"] >= rec["paths"]
    assert rec["scene_shadow_tests"] == st["shadow_rays"] > 0
    assert rec["illum_calls"] > 0
    for k in ("intersect_nodes", "intersect_tests", "shadow_nodes", "shadow_tests"):
        assert rec[k] > 0, k
    # every query visits at least the root
    assert rec["intersect_nodes"] >= rec["scene_intersect_calls"]
