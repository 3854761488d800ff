"""Oracle-side tooling: scene-spec files and the reference harness runner.

TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference legs import this module.  It writes the scene-spec and
ray-batch files read by oracle/ref_harness.cc (the reference renderer driven
through its own C++ API) and by the restatement in oracle/port.cc, runs those
programs, and parses their output.  The layout matches oracle/scene_spec.h.
"""

from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference source tree; SNOGRAY_REFERENCE overrides the default location.
REFERENCE_TREE = os.environ.get("SNOGRAY_REFERENCE", "/root/reference")


def _scenes_module():
    """snogray_b200/scenes.py (numpy only) without importing the package,
    whose __init__ maps the CUDA library."""
    import importlib.util
    import sys
    name = "snogray_b200.scenes"
    if name in sys.modules:
        return sys.modules[name]
    if "_snog_scenes_file" in sys.modules:
        return sys.modules["_snog_scenes_file"]
    path = os.path.join(os.path.dirname(HERE), "snogray_b200", "scenes.py")
    spec_ = importlib.util.spec_from_file_location("_snog_scenes_file", path)
    mod = importlib.util.module_from_spec(spec_)
    sys.modules["_snog_scenes_file"] = mod
    spec_.loader.exec_module(mod)
    return mod


def ref_binary(flavour="parity"):
    return os.path.join(REF_DIR, f"snog_ref_{flavour}")


def port_binary():
    return os.path.join(REF_DIR, "snog_port")


def have_ref(flavour="parity"):
    return os.access(ref_binary(flavour), os.X_OK)


def build(targets=("all",), quiet=True):
    """Build the oracle.  The reference flavours need the reference tree,
    which exists only on the development machine; the restatement builds
    anywhere with g++."""
    tg = list(targets)
    if "all" in tg and not os.path.isdir(REFERENCE_TREE):
        tg = ["port"]
    out = subprocess.run(["make", "-C", HERE, "-j8", f"REF={REFERENCE_TREE}", *tg], capture_output=True,
                         text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    return out


def ensure_port():
    if not os.access(port_binary(), os.X_OK):
        build(["port"])
    return port_binary()


def write_spec(path, scene, camera=None, params=None):
    """Write SCENE (snogray_b200.scenes.SceneData) with CAMERA and PARAMS.
    The scene module is loaded from its file, so writing a spec never loads
    the product's CUDA library."""
    sc = _scenes_module()
    params = params or sc.RenderParams()
    camera = camera or sc.Camera()
    env = scene.envmap
    env_h, env_w = (env.shape[0], env.shape[1]) if env is not None else (0, 0)
    hdr = bytearray()
    hdr += b"SNOGSPC1"
    hdr += np.array([len(scene.materials), len(scene.vertices), len(scene.triangles),
                     len(scene.spheres), len(scene.tripars), len(scene.point_lights),
                     len(scene.far_lights), env_w, env_h], "<u4").tobytes()
    hdr += np.asarray(scene.env_frame, "<f4").reshape(9).tobytes()
    for v in (camera.pos, camera.forward, camera.right, camera.up):
        hdr += np.asarray(v, "<f4").reshape(3).tobytes()
    hdr += np.array([camera.tan_half_fov_x, camera.tan_half_fov_y], "<f4").tobytes()
    hdr += np.array([params.width, params.height, params.spp, params.min_path_len,
                     params.max_path_len, params.direct_samples], "<u4").tobytes()
    hdr += np.array([params.min_trace, params.bg_alpha], "<f4").tobytes()
    normals = getattr(scene, "normals", None)
    hdr += np.array([1 if normals is not None else 0, 1 if getattr(scene, "right_handed", False) else 0,
                     getattr(params, "integrator", 0)], "<u4").tobytes()
    hdr += np.zeros(5, "<u4").tobytes()
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(np.ascontiguousarray(scene.materials).tobytes())
        f.write(np.ascontiguousarray(scene.vertices, "<f4").tobytes())
        f.write(np.ascontiguousarray(scene.triangles, "<u4").tobytes())
        f.write(np.ascontiguousarray(scene.tri_mat, "<u4").tobytes())
        f.write(np.ascontiguousarray(scene.spheres).tobytes())
        f.write(np.ascontiguousarray(scene.tripars).tobytes())
        f.write(np.ascontiguousarray(scene.point_lights).tobytes())
        f.write(np.ascontiguousarray(scene.far_lights).tobytes())
        if env is not None:
            f.write(np.ascontiguousarray(env, "<f4").tobytes())
        if normals is not None:
            f.write(np.ascontiguousarray(normals, "<f4").reshape(-1, 3).tobytes())


def write_rays(path, soa, n_closest):
    soa = np.ascontiguousarray(soa, np.float32)
    n = soa.shape[1]
    with open(path, "wb") as f:
        f.write(np.array([n, n_closest], "<u4").tobytes())
        f.write(soa.tobytes())


def _run(cmd, timeout=3600):
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if out.returncode != 0:
        raise RuntimeError(f"{cmd[0]} failed ({out.returncode}): {out.stderr[-2000:]}")
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    return json.loads(lines[-1]) if lines else {}


def read_octree(path):
    raw = np.fromfile(path, np.uint8)
    hdr_f = raw[:16].view("<f4")
    n_nodes, n_list = raw[16:24].view("<u4")
    nodes = raw[24:24 + 36 * n_nodes].view("<u4").reshape(n_nodes, 9)
    lst = raw[24 + 36 * n_nodes:24 + 36 * n_nodes + 4 * n_list].view("<i4")
    return {"origin": hdr_f[:3].copy(), "size": float(hdr_f[3]), "children": nodes[:, :8].copy(),
            "heads": nodes[:, 8].copy(), "list": lst.copy()}


def read_trace(path, n):
    raw = np.fromfile(path, np.uint8)
    prim = raw[:4 * n].view("<i4").copy()
    t = raw[4 * n:8 * n].view("<f4").copy()
    nrm = raw[8 * n:20 * n].view("<f4").reshape(n, 3).copy()
    st = raw[20 * n:20 * n + 80].view("<u8").reshape(2, 5)
    keys = ["surface_tests", "surface_hits", "neg_cache_hits", "neg_cache_collisions", "node_calls"]
    return prim, t, nrm, {"closest": dict(zip(keys, map(int, st[0]))),
                          "any": dict(zip(keys, map(int, st[1])))}


def read_pfm(path):
    with open(path, "rb") as f:
        kind = f.readline().strip()
        w, h = map(int, f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), "<f4" if scale < 0 else ">f4")
    ch = 3 if kind == b"PF" else 1
    img = data.reshape(h, w, ch).astype(np.float32)
    return img[::-1].copy()     # PFM stores the bottom row first


def ref_octree(scene, flavour="parity", tmpdir=None):
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, op = os.path.join(d, "s.spec"), os.path.join(d, "o.bin")
        write_spec(sp, scene)
        stats = _run([ref_binary(flavour), "octree", sp, op])
        oc = read_octree(op)
    oc["stats"] = stats
    return oc


def ref_ply(path, flavour="parity", tmpdir=None):
    """The reference's load_ply_file on PATH: {"vertices", "normals", "triangles"}
    (normals: one row per normal the mesh kept) or {"error": message}."""
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        op = os.path.join(d, "p.bin")
        _run([ref_binary(flavour), "ply", path, op])
        with open(op, "rb") as f:
            data = f.read()
    head, _, rest = data.partition(b"\n")
    if head.startswith(b"ERR"):
        return {"error": head[4:].decode()}
    nv, nn, nt = np.frombuffer(rest[:12], "<u4")
    off = 12
    verts = np.frombuffer(rest[off:off + 12 * nv], "<f4").reshape(nv, 3)
    off += 12 * nv
    nrm = np.frombuffer(rest[off:off + 12 * nn], "<f4").reshape(nn, 3)
    off += 12 * nn
    tris = np.frombuffer(rest[off:off + 12 * nt], "<u4").reshape(nt, 3)
    return {"vertices": verts, "normals": nrm, "triangles": tris}


def ref_trace(scene, soa, n_closest, threads=8, flavour="parity", tmpdir=None):
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, rp, op = (os.path.join(d, x) for x in ("s.spec", "r.bin", "o.bin"))
        write_spec(sp, scene)
        write_rays(rp, soa, n_closest)
        info = _run([ref_binary(flavour), "trace", sp, rp, op, str(threads)])
        prim, t, nrm, stats = read_trace(op, soa.shape[1])
    return prim, t, nrm, stats, info


def ref_render(scene, camera, params, threads=1, seed_skip=0, spp=0, row0=0, rows=0,
               flavour="parity", tmpdir=None, timeout=7200):
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, op = os.path.join(d, "s.spec"), os.path.join(d, "o.pfm")
        write_spec(sp, scene, camera, params)
        info = _run([ref_binary(flavour), "render", sp, op, str(threads), str(seed_skip),
                     str(spp), str(row0), str(rows)], timeout=timeout)
        img = read_pfm(op)
    return img, info


def ref_render_repeat(scene, camera, params, repeat, threads=8, spp=0, flavour="parity", tmpdir=None,
                      timeout=7200, reduce=None):
    """REPEAT independent renders of one job in one reference process (the
    scene and its octree are built once; every render's RenderContexts draw
    fresh seeds).  Returns ([reduce(image) for each render], [info per
    render]); REDUCE defaults to the identity."""
    reduce = reduce or (lambda im: im)
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, op = os.path.join(d, "s.spec"), os.path.join(d, "o.pfm")
        write_spec(sp, scene, camera, params)
        out = subprocess.run([ref_binary(flavour), "render", sp, op, str(threads), "0", str(spp), "0", "0",
                              str(repeat), "1"], capture_output=True, text=True, timeout=timeout)
        if out.returncode != 0:
            raise RuntimeError(f"reference render failed ({out.returncode}): {out.stderr[-2000:]}")
        infos = [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]
        outs = [reduce(read_pfm(f"{op}.{r}.pfm")) for r in range(repeat)]
    return outs, infos


def port_trace(scene, soa, n_closest, threads=8, tmpdir=None):
    """Closest/any-hit through the restatement (oracle/port.cc)."""
    exe = ensure_port()
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, rp, op = (os.path.join(d, x) for x in ("s.spec", "r.bin", "o.bin"))
        write_spec(sp, scene)
        write_rays(rp, soa, n_closest)
        info = _run([exe, "trace", sp, rp, op, str(threads)])
        prim, t, nrm, stats = read_trace(op, soa.shape[1])
    return prim, t, nrm, stats, info


def port_octree(scene, tmpdir=None):
    exe = ensure_port()
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, op = os.path.join(d, "s.spec"), os.path.join(d, "o.bin")
        write_spec(sp, scene)
        stats = _run([exe, "octree", sp, op])
        oc = read_octree(op)
    oc["stats"] = stats
    return oc


PROBE_HEAD, PROBE_LIGHT = 9, 18     # oracle/ref_harness.cc kProbeHead, kProbeLight


def camera_probes(camera, n, seed=0):
    """N probes of SCENE's camera: rays through uniform random points of the
    film (unit directions, extent [0, 1e30]) with uniform random BSDF and
    light parameters.  Returns an (n, 12) float32 array in the layout the
    harness's samples mode reads."""
    rng = np.random.default_rng(seed)
    fx = rng.uniform(-1, 1, n).astype(np.float32)
    fy = rng.uniform(-1, 1, n).astype(np.float32)
    fwd, right, up = (np.asarray(v, np.float64) for v in (camera.forward, camera.right, camera.up))
    d = (fwd[None] + (fx * camera.tan_half_fov_x)[:, None] * right[None] +
         (fy * camera.tan_half_fov_y)[:, None] * up[None])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    pr = np.zeros((n, 12), np.float32)
    pr[:, 0:3] = np.asarray(camera.pos, np.float32)[None]
    pr[:, 3] = 0.0
    pr[:, 4:7] = d.astype(np.float32)
    pr[:, 7] = 1e30
    pr[:, 8:12] = rng.random((n, 4), np.float32)
    return pr


def read_samples(path):
    """(n_lights, head (n, 9), lights (n, n_lights, 18)) from a samples file."""
    raw = np.fromfile(path, np.uint8)
    n, nl = raw[:8].view("<u4")
    res = raw[8:].view("<f4").reshape(int(n), PROBE_HEAD + PROBE_LIGHT * int(nl))
    return int(nl), res[:, :PROBE_HEAD].copy(), res[:, PROBE_HEAD:].reshape(int(n), int(nl), PROBE_LIGHT).copy()


def ref_samples(scene, probes, flavour="parity", tmpdir=None):
    """The reference's Bsdf::sample / eval and light samplers' sample / eval
    at the probes' hits (harness mode `samples`)."""
    probes = np.ascontiguousarray(probes, np.float32)
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, pp, op = (os.path.join(d, x) for x in ("s.spec", "p.bin", "o.bin"))
        write_spec(sp, scene)
        with open(pp, "wb") as f:
            f.write(np.array([len(probes)], "<u4").tobytes())
            f.write(probes.tobytes())
        _run([ref_binary(flavour), "samples", sp, pp, op])
        return read_samples(op)


def ref_filter(xy, flavour="parity", tmpdir=None):
    """The reference's image filter, ImageMitchellFilt::val (x, y), at the
    (n, 2) offsets XY.  Returns (values, info: b, c, radii)."""
    xy = np.ascontiguousarray(xy, np.float32)
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        ip, op = os.path.join(d, "xy.bin"), os.path.join(d, "v.bin")
        with open(ip, "wb") as f:
            f.write(np.array([len(xy)], "<u4").tobytes())
            f.write(xy.tobytes())
        info = _run([ref_binary(flavour), "filter", ip, op])
        return np.fromfile(op, "<f4").copy(), info


def ref_eye_dirs(scene, camera, u, v, flavour="parity", tmpdir=None):
    """The reference's Camera::eye_ray directions (eye_vec, not normalised)
    for CAMERA at film locations (U, V); returns an (n, 3) float32 array."""
    uv = np.ascontiguousarray(np.stack([u, v], 1), np.float32)
    with tempfile.TemporaryDirectory(dir=tmpdir) as d:
        sp, ip, op = (os.path.join(d, x) for x in ("s.spec", "uv.bin", "d.bin"))
        write_spec(sp, scene, camera)
        with open(ip, "wb") as f:
            f.write(np.array([len(uv)], "<u4").tobytes())
            f.write(uv.tobytes())
        _run([ref_binary(flavour), "camera", sp, ip, op])
        return np.fromfile(op, "<f4").reshape(-1, 3).copy()
