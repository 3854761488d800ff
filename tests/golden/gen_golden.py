"""Generate the golden fixtures in tests/golden/ from the snogray reference.

Runs the reference renderer compiled in place from its own sources
(oracle/_ref/snog_ref_parity: -O2 -ffp-contract=off, IEEE single precision in
source order) through its own C++ API (oracle/ref_harness.cc).  The reference
tree exists only on the development machine, so the outputs are committed;
the GPU box and the CPU test suite read them.

Each scene is regenerated at test time from its generator and seed and pinned
by a sha256 digest of its arrays, so the fixtures hold only ids, distances,
octree digests and image statistics, not geometry.

    python tests/golden/gen_golden.py            # all fixtures
"""

from __future__ import annotations

import hashlib
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from snogray_b200 import scenes  # noqa: E402
import spec  # noqa: E402


def edge_rays(sd, n_rand, seed):
    """Rays that exercise the corners of the traversal: axis-aligned and
    zero directions, origins on the root cube's planes, zero and short
    extents, plus random rays."""
    rng = np.random.default_rng(seed)
    rays = [scenes.random_rays(n_rand, seed=seed)]
    lo = sd.vertices.min(0) if len(sd.vertices) else np.zeros(3)
    hi = sd.vertices.max(0) if len(sd.vertices) else np.ones(3)
    k = 512
    o = rng.uniform(lo - 0.05, hi + 0.05, (k, 3)).astype(np.float32)
    axes = np.eye(3, dtype=np.float32)
    d = np.concatenate([axes, -axes])[rng.integers(0, 6, k)]
    soa = np.empty((7, k), np.float32)
    soa[0:3], soa[3:6], soa[6] = o.T, d.T, np.inf
    rays.append(soa)
    # origins snapped to the octree midplanes of the unit cube
    o2 = rng.uniform(0, 1, (k, 3)).astype(np.float32)
    o2[:, rng.integers(0, 3)] = 0.5
    dd = rng.normal(size=(k, 3)).astype(np.float32)
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    soa2 = np.empty((7, k), np.float32)
    soa2[0:3], soa2[3:6] = o2.T, dd.T
    soa2[6] = np.where(np.arange(k) % 4 == 0, 0.0, np.where(np.arange(k) % 4 == 1, 0.05, np.inf))
    rays.append(soa2)
    z = np.zeros((7, 16), np.float32)       # zero directions
    z[0:3] = rng.uniform(0, 1, (3, 16))
    z[6] = np.inf
    rays.append(z)
    return np.concatenate(rays, axis=1)


def camera_film_locs(w, h, seed):
    """Film locations of one jittered sample per pixel, as
    Renderer::render_packet forms them (render-mgr/renderer.cc:84):
    u = x / width, v = (height - y) / height, in float32."""
    rng = np.random.default_rng(seed)
    n = w * h
    px = (np.arange(n) % w + rng.uniform(0, 1, n)).astype(np.float32)
    py = (np.arange(n) // w + rng.uniform(0, 1, n)).astype(np.float32)
    u = px / np.float32(w)
    v = (np.float32(h) - py) / np.float32(h)
    return u, v


def eye_dirs(cam, u, v):
    """Camera::eye_vec (camera/camera.h:384-389) in float32, in the order the
    camera kernels evaluate it: forward + right x tan_x + up y tan_y."""
    x = (np.float32(2) * u - np.float32(1)).astype(np.float32)
    y = (np.float32(2) * v - np.float32(1)).astype(np.float32)
    f, r, up = (np.asarray(a, np.float32) for a in (cam.forward, cam.right, cam.up))
    return (f[None] + (r[None] * x[:, None]) * np.float32(cam.tan_half_fov_x)
            + (up[None] * y[:, None]) * np.float32(cam.tan_half_fov_y)).astype(np.float32)


def camera_rays(cam, w, h, max_trace, seed):
    """Eye rays as Camera::eye_ray makes them for jittered film positions
    (camera/camera.cc:108-160): unnormalised direction, t1 = max_trace."""
    u, v = camera_film_locs(w, h, seed)
    n = w * h
    d = eye_dirs(cam, u, v)
    soa = np.empty((7, n), np.float32)
    soa[0:3] = np.asarray(cam.pos, np.float32)[:, None]
    soa[3:6] = d.T
    soa[6] = max_trace
    return soa


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


TRACE_CASES = {
    # name: (scene factory, ray factory, n_closest fraction)
    "mixed": (lambda: scenes.mixed_scene(4000, 300, 200, seed=5),
              lambda sd: edge_rays(sd, 12000, seed=31)),
    "soup": (lambda: scenes.random_triangles(20000, seed=2),
             lambda sd: scenes.random_rays(16384, seed=3)),
    "terrain": (lambda: scenes.terrain_scene(n=96, n_spheres=40, seed=11, env_w=64, env_h=32),
                lambda sd: edge_rays(sd, 8000, seed=37)),
    "cornell_camera": (lambda: scenes.cornell_box(),
                       lambda sd: camera_rays(scenes.cornell_camera(64, 64), 64, 64,
                                              np.float32(4.0), seed=41)),
    # a right-handed mesh (PLY convention): normals e1 x e2
    "mesh_flat": (lambda: scenes.mesh_scene(smooth=False),
                  lambda sd: np.concatenate([camera_rays(scenes.mesh_camera(48, 48), 48, 48,
                                                         np.float32(4.0), seed=43),
                                             edge_rays(sd, 4000, seed=47)], 1)),
}


# Per-sample shading: probes through each camera's film (spec.camera_probes)
# with random BSDF and light parameters, evaluated by the reference's
# Bsdf::sample / eval and light samplers' sample / eval (harness mode
# `samples`).  The scenes cover Lambert, Cook-Torrance, Mirror (conductor,
# dielectric over Lambert, zero reflectance) and Glass materials, smooth
# mesh normals, and tripar, sphere, point, spot, far and envmap lights.
SAMPLE_CASES = {
    "cornell": (scenes.cornell_box, lambda: scenes.cornell_camera(64, 64)),
    "mirror": (scenes.mirror_scene, lambda: scenes.cornell_camera(64, 64)),
    "spot_far": (scenes.spot_far_scene, lambda: scenes.spot_far_camera(64, 64)),
    "terrain": (lambda: scenes.terrain_scene(n=96, n_spheres=40, seed=11, env_w=64, env_h=32),
                lambda: scenes.terrain_camera(64, 48)),
    "mesh_smooth": (lambda: scenes.mesh_scene(smooth=True), lambda: scenes.mesh_camera(48, 48)),
    "nested_glass": (scenes.nested_glass_scene, lambda: scenes.cornell_camera(64, 64)),
}
SAMPLE_PROBES = 2048


def filter_offsets():
    """Offsets for the image filter: the knots (0, +-0.5, +-1, +-1.5, +-2 and
    just inside and outside the radius) on both axes, plus uniform random
    points over [-2.5, 2.5]^2."""
    knots = np.array([0, 0.5, 1, 1.5, 2, 1.999, 2.001, 0.999, 1.001, 2.5], np.float32)
    knots = np.concatenate([knots, -knots])
    gx, gy = np.meshgrid(knots, knots)
    rnd = np.random.default_rng(59).uniform(-2.5, 2.5, (4096, 2)).astype(np.float32)
    return np.concatenate([np.stack([gx.ravel(), gy.ravel()], 1), rnd]).astype(np.float32)


# Cameras whose eye rays are pinned: (scene, camera, film width, height).
CAMERA_CASES = {
    "cornell": (scenes.cornell_box, lambda: scenes.cornell_camera(64, 64), 64, 64),
    "terrain": (lambda: scenes.terrain_scene(n=96, n_spheres=40, seed=11, env_w=64, env_h=32),
                lambda: scenes.terrain_camera(96, 54), 96, 54),
}


def gen_camera():
    out = {}
    for name, (mk, cam, w, h) in CAMERA_CASES.items():
        u, v = camera_film_locs(w, h, seed=61)
        out[name] = spec.ref_eye_dirs(mk(), cam(), u, v)
    np.savez_compressed(os.path.join(HERE, "camera_eye_rays.npz"), **out)
    print("camera_eye_rays:", {k: v.shape for k, v in out.items()})


def gen_filter():
    xy = filter_offsets()
    v, info = spec.ref_filter(xy)
    np.savez_compressed(os.path.join(HERE, "filter_mitchell.npz"), xy=xy, val=v,
                        b=np.float32(info["b"]), c=np.float32(info["c"]), radius=np.float32(info["x_radius"]))
    print(f"filter_mitchell: {len(xy)} offsets, b {info['b']}, c {info['c']}, radius {info['x_radius']}")


def gen_samples(name):
    mk, cam = SAMPLE_CASES[name]
    sd = mk()
    probes = spec.camera_probes(cam(), SAMPLE_PROBES, seed=53)
    nl, head, lights = spec.ref_samples(sd, probes)
    np.savez_compressed(os.path.join(HERE, f"samples_{name}.npz"), probes=probes, head=head, lights=lights,
                        n_lights=np.uint32(nl), scene_digest=scenes.scene_digest(sd))
    print(f"samples_{name}: {int(head[:, 0].sum())} hits of {len(probes)}, {nl} lights")


def gen_trace(name):
    make_scene, make_rays = TRACE_CASES[name]
    sd = make_scene()
    rays = make_rays(sd)
    n = rays.shape[1]
    n_closest = n // 2
    prim, t, nrm, stats, _ = spec.ref_trace(sd, rays, n_closest, threads=8)
    oc = spec.ref_octree(sd)
    hit = np.nonzero(prim[:n_closest] >= 0)[0]
    np.savez_compressed(
        os.path.join(HERE, f"trace_{name}.npz"), prim=prim, t=t, normal_hit=nrm[hit],
        closest_nodes=stats["closest"]["node_calls"], any_nodes=stats["any"]["node_calls"],
        scene_digest=scenes.scene_digest(sd), rays_digest=digest(rays), n_closest=n_closest,
        oct_children_digest=digest(oc["children"]), oct_heads_digest=digest(oc["heads"]),
        oct_list_digest=digest(oc["list"]), oct_origin=oc["origin"], oct_size=oc["size"],
        oct_nodes=len(oc["heads"]))
    hit = (prim[:n_closest] >= 0).mean(), (prim[n_closest:] >= 0).mean()
    print(f"trace_{name}: {n} rays, hit rate closest {hit[0]:.3f} any {hit[1]:.3f}, "
          f"{len(oc['heads'])} nodes")


def image_stats(imgs):
    """Per-channel image means over K independent renders and their standard
    error (snogdiff's mean, snogdiff.cc:133-190)."""
    means = np.array([im.reshape(-1, 3).mean(0) for im in imgs])
    return means.mean(0), means.std(0, ddof=1) / math.sqrt(len(imgs))


RENDER_CASES = {
    "cornell": (scenes.cornell_box, scenes.cornell_camera, scenes.cornell_params, 128, 128, 16),
    "terrain": (lambda: scenes.terrain_scene(n=96, n_spheres=40, seed=11, env_w=256, env_h=128),
                scenes.terrain_camera, scenes.terrain_params, 64, 48, 16),
    # right-handed meshes, with vertex normals and flat
    "mesh_smooth": (lambda: scenes.mesh_scene(smooth=True), scenes.mesh_camera, scenes.mesh_params,
                    64, 64, 16),
    "mesh_flat": (lambda: scenes.mesh_scene(smooth=False), scenes.mesh_camera, scenes.mesh_params,
                  64, 64, 16),
    # the direct-lighting integrator (glass: reflection and transmission both recurse)
    "cornell_direct": (scenes.cornell_box, scenes.cornell_camera, scenes.direct_params, 96, 96, 16),
    "mesh_flat_direct": (lambda: scenes.mesh_scene(smooth=False), scenes.mesh_camera, scenes.direct_params,
                         64, 64, 16),
    # the Cornell workload at its stated size: 256x256, 16 spp, max depth 8
    "cornell256": (scenes.cornell_box, scenes.cornell_camera, scenes.cornell_params, 256, 256, 16),
    # Mirror (conductor, dielectric over Lambert, zero reflectance), a sphere
    # light and an omni point light; both integrators
    "mirror": (scenes.mirror_scene, scenes.cornell_camera, scenes.mirror_params, 64, 64, 16),
    "mirror_direct": (scenes.mirror_scene, scenes.cornell_camera, scenes.direct_params, 64, 64, 16),
    # a spotlight with a fringe and two far lights (angle 0 and 8 degrees)
    "spot_far": (scenes.spot_far_scene, scenes.spot_far_camera, scenes.mirror_params, 64, 64, 16),
    "spot_far_direct": (scenes.spot_far_scene, scenes.spot_far_camera, scenes.direct_params, 64, 64, 16),
    # four nested glass media
    "nested_glass": (scenes.nested_glass_scene, scenes.cornell_camera, scenes.nested_glass_params,
                     64, 64, 16),
}


# Renders per side for cases whose median RMSE is too spread at 64 to resolve
# the 5 % bar (caustics through faceted or nested glass, small bright lights
# seen in mirrors: bootstrap SDs of the median of 2-15 % at 64).
RENDER_K = {"mesh_flat_direct": 1024, "mirror": 256, "mirror_direct": 256, "spot_far": 1024,
            "spot_far_direct": 2048, "nested_glass": 1024, "cornell256": 1024}


def gen_render(name, k=None, gt_spp=4096):
    k = k or RENDER_K.get(name, 64)
    make_scene, make_cam, make_params, w, h, spp = RENDER_CASES[name]
    sd = make_scene()
    cam = make_cam(w, h)
    params = make_params(w, h, spp)
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(8) as ex:
        futs = [ex.submit(spec.ref_render, sd, cam, params, 1, i) for i in range(k)]
        res = [f.result() for f in futs]
    imgs = [r[0] for r in res]
    mean, se = image_stats(imgs)
    gt, info = spec.ref_render(sd, cam, params, threads=8, seed_skip=1000, spp=gt_spp)
    # RMSE of each spp-S reference render against the ground truth.
    rmse = np.array([np.sqrt(((im - gt) ** 2).mean()) for im in imgs])
    np.savez_compressed(os.path.join(HERE, f"render_{name}.npz"),
                        mean=mean, se=se, rmse=rmse, gt=gt.astype(np.float16), k=k, spp=spp,
                        gt_spp=gt_spp, width=w, height=h, scene_digest=scenes.scene_digest(sd),
                        ref_mpaths=np.array([r[1]["mpaths_per_s"] for r in res]))
    print(f"render_{name}: mean {mean} se {se} rmse {rmse.mean():.4f}+-{rmse.std():.4f} "
          f"gt {info['seconds']:.1f}s")


# The terrain workload at its stated size (2,093,058 triangles, 200 spheres,
# 1024x512 sky, 1920x1080, max depth 16), rendered K times at a low spp;
# each render is reduced to its per-channel mean and the means of a grid of
# TILES tiles.
TERRAIN_FULL = dict(k=32, spp=2, width=1920, height=1080, tiles=(6, 8))


def tile_means(img, tiles):
    ty, tx = tiles
    h, w, _ = img.shape
    return img.reshape(ty, h // ty, tx, w // tx, 3).mean((1, 3)).reshape(-1, 3)


def gen_terrain_full():
    c = TERRAIN_FULL
    sd = scenes.terrain_scene()
    cam = scenes.terrain_camera(c["width"], c["height"])
    params = scenes.terrain_params(c["width"], c["height"], c["spp"])
    red = lambda im: np.concatenate([im.reshape(-1, 3).mean(0)[None], tile_means(im, c["tiles"])])
    outs, infos = spec.ref_render_repeat(sd, cam, params, c["k"], threads=os.cpu_count() or 8, reduce=red)
    stats = np.array(outs)                       # (k, 1 + tiles, 3)
    np.savez_compressed(os.path.join(HERE, "render_terrain_full.npz"), means=stats[:, 0], tiles=stats[:, 1:],
                        k=c["k"], spp=c["spp"], width=c["width"], height=c["height"],
                        tile_grid=np.array(c["tiles"]), scene_digest=scenes.scene_digest(sd),
                        ref_seconds=np.array([i["seconds"] for i in infos]))
    m = stats[:, 0]
    print(f"render_terrain_full: mean {m.mean(0)} se {m.std(0, ddof=1) / math.sqrt(len(m))}")


if __name__ == "__main__":
    if not spec.have_ref():
        spec.build(["ref"])
    which = sys.argv[1:] or ["trace", "render", "terrain_full", "samples", "filter", "camera"]
    if "terrain_full" in which:
        gen_terrain_full()
    if "trace" in which:
        for nm in TRACE_CASES:
            gen_trace(nm)
    if "render" in which:
        for nm in RENDER_CASES:
            gen_render(nm)
    if "filter" in which:
        gen_filter()
    if "camera" in which:
        gen_camera()
    if "samples" in which:
        for nm in SAMPLE_CASES:
            gen_samples(nm)
    for nm in which:
        if nm in RENDER_CASES:
            gen_render(nm)
    with open(os.path.join(HERE, "README.txt"), "w") as f:
        f.write("Golden fixtures made by tests/golden/gen_golden.py from the snogray reference\n"
                "compiled in place (oracle/Makefile, parity flavour).  Regenerate with:\n"
                "    python tests/golden/gen_golden.py\n")
