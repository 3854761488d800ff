"""Full path tracing on the GPU against the reference renderer (statistical).

Bar, per the reference's own image comparison (snogdiff: mean over all pixel
components, mean squared error, snogdiff.cc:133-190):
  * per-channel image means within 3 standard errors of the reference's,
    the SE combining the spread of K independent renders on each side;
  * RMSE against a 4096-spp reference render within 5% of the CPU render's
    RMSE at equal spp (median over K renders: firefly-heavy scenes make the
    mean of the RMSE too noisy to resolve 5% at this K).
Fixtures: tests/golden/render_*.npz, from the reference compiled in place.
"""

import math

import numpy as np
import pytest

from gen_golden import RENDER_CASES
from snogray_b200 import Scene, scenes

pytestmark = pytest.mark.gpu

K_GPU = 64


def _render_k(name, k, seed0=1):
    make_scene, make_cam, make_params, w, h, spp = RENDER_CASES[name]
    sd = make_scene()
    cam = make_cam(w, h)
    imgs = []
    with Scene(sd) as sc:
        for i in range(k):
            p = make_params(w, h, spp, seed=seed0 + i)
            img, st = sc.render(cam, p)
            imgs.append(img)
    return sd, np.array(imgs), st


@pytest.mark.parametrize("name", sorted(RENDER_CASES))
def test_image_mean_within_3se(name, golden):
    g = golden(f"render_{name}.npz")
    sd, imgs, st = _render_k(name, max(K_GPU, int(g["k"])))
    assert scenes.scene_digest(sd) == str(g["scene_digest"])
    assert imgs.shape[1:] == (int(g["height"]), int(g["width"]), 3)
    assert np.isfinite(imgs).all() and (imgs >= 0).all()
    means = imgs.reshape(len(imgs), -1, 3).mean(1)
    m_gpu = means.mean(0)
    se_gpu = means.std(0, ddof=1) / math.sqrt(len(means))
    se = np.sqrt(se_gpu ** 2 + g["se"] ** 2)
    z = np.abs(m_gpu - g["mean"]) / se
    assert (z < 3).all(), f"means gpu {m_gpu} ref {g['mean']} z {z}"


@pytest.mark.parametrize("name", sorted(RENDER_CASES))
def test_rmse_vs_ground_truth(name, golden):
    g = golden(f"render_{name}.npz")
    _, imgs, _ = _render_k(name, max(K_GPU, int(g["k"])), seed0=100000)
    gt = g["gt"].astype(np.float32)
    rmse = np.sqrt(((imgs - gt[None]) ** 2).reshape(len(imgs), -1).mean(1))
    gpu, cpu = float(np.median(rmse)), float(np.median(g["rmse"]))
    assert gpu <= 1.05 * cpu, f"median RMSE gpu {gpu:.4f} vs cpu {cpu:.4f}"


def test_render_is_deterministic_per_seed():
    sd = scenes.cornell_box()
    cam = scenes.cornell_camera(32, 32)
    with Scene(sd) as sc:
        a, _ = sc.render(cam, scenes.cornell_params(32, 32, 4, seed=7))
        b, _ = sc.render(cam, scenes.cornell_params(32, 32, 4, seed=7))
        c, _ = sc.render(cam, scenes.cornell_params(32, 32, 4, seed=8))
    # shadow contributions reach a path's radiance through float atomics, so
    # equal seeds agree up to the order of two additions per vertex
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
    assert np.abs(a - c).mean() > 1e-3


def test_render_stats_and_waves():
    """A job split into many waves gives the same image statistics as one
    wave (wave size is an implementation detail)."""
    import os
    sd = scenes.cornell_box()
    cam = scenes.cornell_camera(48, 40)
    p = scenes.cornell_params(48, 40, 16, seed=3)
    with Scene(sd) as sc:
        img1, st1 = sc.render(cam, p)
    os.environ["SNOG_WAVE_PATHS"] = str(52 * 16 * 7)    # 7 pattern rows per wave
    try:
        with Scene(sd) as sc:
            img2, st2 = sc.render(cam, p)
    finally:
        del os.environ["SNOG_WAVE_PATHS"]
    assert st1["paths"] == st2["paths"] == 52 * 44 * 16
    assert st2["waves"] > 1 and st1["waves"] == 1
    # identical per-path random streams, so identical images up to float
    # summation order in the splat
    assert np.allclose(img1, img2, rtol=1e-5, atol=1e-6)


def test_terrain_full_size_means_within_3se(golden):
    """The terrain workload at its stated size (2,093,058 triangles, 200
    spheres, 1024x512 sky, 1920x1080, depth 16) against K reference renders
    at the same low spp: per-channel image means within 3 standard errors,
    and the means of a 6 x 8 grid of tiles within 4.5 (48 tiles x 3 channels
    compared at once)."""
    from gen_golden import TERRAIN_FULL, tile_means
    g = golden("render_terrain_full.npz")
    c = TERRAIN_FULL
    sd = scenes.terrain_scene()
    assert scenes.scene_digest(sd) == str(g["scene_digest"])
    cam = scenes.terrain_camera(c["width"], c["height"])
    k = int(g["k"])
    means, tiles = [], []
    with Scene(sd) as sc:
        for i in range(k):
            img, _ = sc.render(cam, scenes.terrain_params(c["width"], c["height"], int(g["spp"]), seed=500 + i))
            assert np.isfinite(img).all() and (img >= 0).all()
            means.append(img.reshape(-1, 3).mean(0))
            tiles.append(tile_means(img, c["tiles"]))
    for ours, ref, bar in ((np.array(means), g["means"], 3.0), (np.array(tiles), g["tiles"], 4.5)):
        se = np.sqrt(ours.var(0, ddof=1) / len(ours) + ref.var(0, ddof=1) / len(ref))
        z = np.abs(ours.mean(0) - ref.mean(0)) / np.maximum(se, 1e-12)
        assert (z < bar).all(), f"max z {z.max():.2f} at {np.unravel_index(z.argmax(), z.shape)}"


def test_fifth_nested_medium_is_an_error():
    """The path state holds four media; a path entering a fifth nested glass
    ends the render with an error instead of dropping a medium silently
    (the reference's media list is unbounded, material/media.cc:76-118)."""
    mats = scenes._mats([scenes.material(scenes.MAT_LAMBERT, (0.5, 0.5, 0.5))] +
                        [scenes.material(scenes.MAT_GLASS, ior_n=1.2 + 0.1 * k) for k in range(5)] +
                        [scenes.material(scenes.MAT_GLOW, (5.0, 5.0, 5.0))])
    sph = np.zeros(6, scenes.SPHERE_DTYPE)
    for k, r in enumerate((0.4, 0.32, 0.24, 0.16, 0.08)):
        sph[k] = ((0.5, 0.5, 0.5), r, 1 + k)
    sph[5] = ((0.5, 0.5, -1.5), 0.3, 6)
    sd = scenes.SceneData(materials=mats, spheres=sph)
    cam = scenes.Camera()
    cam.move((0.5, 0.5, -1.0))
    cam.point((0.5, 0.5, 0.5), (0, 1, 0))
    cam.set_vert_fov(math.radians(10.0), 1.0)
    import snogray_b200 as sb
    with Scene(sd) as sc:
        with pytest.raises(sb.SnogError) as ei:
            sc.render(cam, scenes.RenderParams(16, 16, 4, max_path_len=12))
    assert ei.value.code == sb.SNOG_EINVAL and "fifth nested medium" in str(ei.value)
