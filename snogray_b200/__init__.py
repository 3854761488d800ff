"""snogray_b200 -- B200 path-tracing backend for snogray's render path.

Python face of the C ABI in include/snogray_b200.h (loaded with ctypes from
the in-tree libsnogray_b200.so).  There is no fallback: if the shared library
is missing or fails to load, importing this package raises.

    from snogray_b200 import Scene, scenes
    sd = scenes.cornell_box()
    with Scene(sd) as sc:
        img, stats = sc.render(scenes.cornell_camera(256, 256), scenes.cornell_params())
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import scenes  # noqa: F401  (re-exported)
from .scenes import Camera, RenderParams, SceneData

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsnogray_b200.so")

SNOG_OK, SNOG_EINVAL, SNOG_ENOMEM, SNOG_ECUDA, SNOG_ETIMEOUT, SNOG_EBUSY, SNOG_ENOTFOUND, \
    SNOG_ECANCELED = range(8)


class SnogError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"snogray_b200 error {code}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m snogray_b200.build`")
    return C.CDLL(LIB_PATH)


_lib = _load()


# --- C structs (must match include/snogray_b200.h) -------------------------

class SnogSceneDesc(C.Structure):
    _fields_ = [("n_materials", C.c_uint32), ("materials", C.c_void_p),
                ("n_vertices", C.c_uint32), ("vertices", C.c_void_p),
                ("n_triangles", C.c_uint32), ("triangles", C.c_void_p),
                ("tri_material", C.c_void_p),
                ("n_spheres", C.c_uint32), ("spheres", C.c_void_p),
                ("n_tripars", C.c_uint32), ("tripars", C.c_void_p),
                ("n_point_lights", C.c_uint32), ("point_lights", C.c_void_p),
                ("n_far_lights", C.c_uint32), ("far_lights", C.c_void_p),
                ("env_width", C.c_uint32), ("env_height", C.c_uint32),
                ("env_rgb", C.c_void_p), ("env_frame", C.c_float * 9),
                ("vertex_normals", C.c_void_p), ("mesh_right_handed", C.c_uint32)]


class SnogPlyMesh(C.Structure):
    _fields_ = [("n_vertices", C.c_uint32), ("vertices", C.POINTER(C.c_float)),
                ("normals", C.POINTER(C.c_float)), ("n_triangles", C.c_uint32),
                ("triangles", C.POINTER(C.c_uint32))]


class SnogCamera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("tan_half_fov_x", C.c_float), ("tan_half_fov_y", C.c_float)]


class SnogRenderParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("min_path_len", C.c_uint32), ("max_path_len", C.c_uint32),
                ("direct_samples", C.c_uint32), ("min_trace", C.c_float), ("bg_alpha", C.c_float),
                ("seed", C.c_uint64), ("integrator", C.c_uint32), ("flags", C.c_uint32)]


SNOG_RENDER_COUNT_TRAVERSAL = 1


class SnogRenderWindow(C.Structure):
    _fields_ = [("pat_x", C.c_int32), ("pat_y", C.c_int32), ("pat_width", C.c_uint32),
                ("pat_height", C.c_uint32), ("out_x", C.c_int32), ("out_y", C.c_int32),
                ("out_width", C.c_uint32), ("out_height", C.c_uint32)]


class SnogSceneInfo(C.Structure):
    _fields_ = [("n_nodes", C.c_uint32), ("n_plist", C.c_uint32), ("max_depth", C.c_uint32),
                ("n_leaf_nodes", C.c_uint32), ("n_triangles", C.c_uint32),
                ("n_spheres", C.c_uint32), ("n_tripars", C.c_uint32), ("n_lights", C.c_uint32),
                ("n_list_surfaces", C.c_uint64), ("origin", C.c_float * 3), ("size", C.c_float),
                ("bbox_min", C.c_float * 3), ("bbox_max", C.c_float * 3), ("horizon", C.c_float),
                ("device_bytes", C.c_uint64), ("build_ms", C.c_double), ("pair_lists", C.c_uint32),
                ("reserved", C.c_uint32)]


class SnogRenderStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("device_ms", C.c_double), ("waves", C.c_uint32), ("kernel_launches", C.c_uint32),
                ("closest_ms", C.c_double), ("shadow_ms", C.c_double), ("shade_ms", C.c_double),
                ("other_ms", C.c_double), ("closest_launches", C.c_uint32),
                ("shadow_launches", C.c_uint32), ("closest_nodes", C.c_uint64),
                ("closest_tests", C.c_uint64), ("shadow_nodes", C.c_uint64),
                ("shadow_tests", C.c_uint64), ("illum_calls", C.c_uint64)]


class SnogEngineConfig(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("item_paths", C.c_uint32), ("ring_items", C.c_uint32),
                ("max_jobs", C.c_uint32), ("max_lights", C.c_uint32), ("iters_per_launch", C.c_uint32),
                ("max_scenes", C.c_uint32), ("reserved", C.c_uint32), ("mem_budget", C.c_uint64)]


class SnogJobStats(C.Structure):
    _fields_ = [("submit_ms", C.c_double), ("admit_ms", C.c_double), ("start_ms", C.c_double),
                ("finish_ms", C.c_double), ("paths", C.c_uint64), ("status", C.c_int32)]


class SnogBatchStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("wall_ms", C.c_double), ("kernel_launches", C.c_uint32), ("iterations", C.c_uint32),
                ("closest_ms", C.c_double), ("shadow_ms", C.c_double), ("shade_ms", C.c_double),
                ("other_ms", C.c_double)]


def _sig(name, res, *args):
    try:
        f = getattr(_lib, name)
    except AttributeError:
        def missing(*_a, _name=name):
            raise SnogError(SNOG_EINVAL, f"{_name} is not exported by {LIB_PATH}")
        return missing
    f.restype = res
    f.argtypes = list(args)
    return f


_P = C.c_void_p
_lib_version = _sig("snog_version", C.c_char_p)
_last_error = _sig("snog_last_error", C.c_char_p)
_init = _sig("snog_init", C.c_int, C.c_int)
_scene_create = _sig("snog_scene_create", C.c_int, C.POINTER(SnogSceneDesc), C.POINTER(_P))
_scene_build_host = _sig("snog_scene_build_host", C.c_int, C.POINTER(SnogSceneDesc), C.POINTER(_P))
_scene_create_ex = _sig("snog_scene_create_ex", C.c_int, C.POINTER(SnogSceneDesc), C.c_uint32, C.POINTER(_P))
_scene_destroy = _sig("snog_scene_destroy", C.c_int, _P)
_scene_info = _sig("snog_scene_info", C.c_int, _P, C.POINTER(SnogSceneInfo))
_scene_octree = _sig("snog_scene_octree", C.c_int, _P, _P, _P, _P)
_trace = _sig("snog_trace", C.c_int, _P, _P, C.c_uint32, C.c_uint32, _P, _P, _P, _P)
_trace_device = _sig("snog_trace_device", C.c_int, _P, _P, C.c_uint32, C.c_uint32, _P, _P, _P, _P)
_sample_probe = _sig("snog_sample_probe", C.c_int, _P, _P, _P, C.c_uint32, _P)
_render = _sig("snog_render", C.c_int, _P, C.POINTER(SnogCamera), C.POINTER(SnogRenderParams), _P,
               C.POINTER(SnogRenderStats))
_render_device = _sig("snog_render_device", C.c_int, _P, C.POINTER(SnogCamera),
                      C.POINTER(SnogRenderParams), _P, _P, C.POINTER(SnogRenderStats))
_render_window = _sig("snog_render_window", C.c_int, _P, C.POINTER(SnogCamera), C.POINTER(SnogRenderParams),
                      C.POINTER(SnogRenderWindow), _P, C.POINTER(SnogRenderStats))


_engine_default = _sig("snog_engine_default_config", C.c_int, C.POINTER(SnogEngineConfig))
_render_batch = _sig("snog_render_batch", C.c_int, C.POINTER(_P), C.POINTER(SnogCamera),
                     C.POINTER(SnogRenderParams), C.c_uint32, C.POINTER(_P), C.c_int,
                     C.POINTER(SnogEngineConfig), C.POINTER(SnogBatchStats))
_engine_create = _sig("snog_engine_create", C.c_int, C.POINTER(SnogEngineConfig), _P, C.POINTER(_P))
_engine_render = _sig("snog_engine_render", C.c_int, _P, C.POINTER(_P), C.POINTER(SnogCamera),
                      C.POINTER(SnogRenderParams), C.c_uint32, C.POINTER(_P), C.c_int,
                      C.POINTER(SnogBatchStats))
_engine_destroy = _sig("snog_engine_destroy", C.c_int, _P)
_engine_autotune = _sig("snog_engine_autotune", C.c_int, C.POINTER(_P), C.POINTER(SnogCamera),
                        C.POINTER(SnogRenderParams), C.c_uint32, C.c_uint32,
                        C.POINTER(SnogEngineConfig), C.POINTER(SnogEngineConfig),
                        C.POINTER(C.c_double))
_server_create = _sig("snog_server_create", C.c_int, C.POINTER(SnogEngineConfig), C.POINTER(_P))
_server_add_scene = _sig("snog_server_add_scene", C.c_int, _P, _P, C.POINTER(C.c_uint32))
_server_submit = _sig("snog_server_submit", C.c_int, _P, C.c_uint32, C.POINTER(SnogCamera),
                      C.POINTER(SnogRenderParams), _P, C.POINTER(C.c_uint64))
_server_poll = _sig("snog_server_poll", C.c_int, _P, C.c_uint64, C.POINTER(SnogJobStats))
_server_wait = _sig("snog_server_wait", C.c_int, _P, C.c_uint64, C.c_uint32, C.POINTER(SnogJobStats))
_server_cancel = _sig("snog_server_cancel", C.c_int, _P, C.c_uint64)
_server_pause = _sig("snog_server_pause", C.c_int, _P, C.c_uint64)
_server_resume = _sig("snog_server_resume", C.c_int, _P, C.c_uint64)
_server_checkpoint = _sig("snog_server_checkpoint", C.c_int, _P, C.c_uint64, C.c_char_p, C.c_uint32)
_server_submit_resume = _sig("snog_server_submit_resume", C.c_int, _P, C.c_uint32, C.c_char_p,
                             C.c_void_p, C.POINTER(C.c_uint64))
_server_destroy = _sig("snog_server_destroy", C.c_int, _P)


def _check(rc):
    if rc != SNOG_OK:
        raise SnogError(rc, _last_error().decode(errors="replace"))


def version():
    return _lib_version().decode()


def init(device=0):
    _check(_init(device))


def _ptr(a):
    return None if a is None or a.size == 0 else a.ctypes.data


def camera_struct(cam: Camera) -> SnogCamera:
    c = SnogCamera()
    for name in ("pos", "forward", "right", "up"):
        getattr(c, name)[:] = [float(x) for x in np.asarray(getattr(cam, name), np.float32)]
    c.tan_half_fov_x = cam.tan_half_fov_x
    c.tan_half_fov_y = cam.tan_half_fov_y
    return c


def params_struct(p: RenderParams) -> SnogRenderParams:
    return SnogRenderParams(p.width, p.height, p.spp, p.min_path_len, p.max_path_len,
                            p.direct_samples, p.min_trace, p.bg_alpha, p.seed, p.integrator,
                            getattr(p, "flags", 0))


class Scene:
    """A scene resident on the device (or host-only, for inspecting the
    octree).  Mirrors the reference's GlobalRenderState/Scene pair: built
    once from the surfaces and lights, then rendered or traced."""

    OCTREE_AUTO, OCTREE_HOST, OCTREE_DEVICE = 0, 1, 2
    LISTS = {"probe": 0, "single": 1 << 8, "paired": 2 << 8}   # SNOG_LISTS_*

    def __init__(self, data: SceneData, device=True, octree=0, lists="probe"):
        """OCTREE picks the octree builder of a device scene (snog_scene_create_ex):
        OCTREE_AUTO, OCTREE_HOST or OCTREE_DEVICE; a host-only scene
        (DEVICE=False) always uses the host builder.  LISTS picks how the
        closest-hit traversal deals node lists to lanes: "probe" (decided
        from random rays at creation), "single" or "paired"; results are the
        same in every mode."""
        if lists not in self.LISTS:
            raise ValueError(f"lists must be one of {sorted(self.LISTS)}")
        self.data = data
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a

        d = SnogSceneDesc()
        m = arr(data.materials, data.materials.dtype)
        d.n_materials, d.materials = len(m), _ptr(m)
        v = arr(data.vertices, np.float32)
        d.n_vertices, d.vertices = len(data.vertices), _ptr(v)
        t = arr(data.triangles, np.uint32)
        tm = arr(data.tri_mat, np.uint32)
        d.n_triangles, d.triangles, d.tri_material = len(data.triangles), _ptr(t), _ptr(tm)
        s = arr(data.spheres, data.spheres.dtype)
        d.n_spheres, d.spheres = len(s), _ptr(s)
        tp = arr(data.tripars, data.tripars.dtype)
        d.n_tripars, d.tripars = len(tp), _ptr(tp)
        pl = arr(data.point_lights, data.point_lights.dtype)
        d.n_point_lights, d.point_lights = len(pl), _ptr(pl)
        fl = arr(data.far_lights, data.far_lights.dtype)
        d.n_far_lights, d.far_lights = len(fl), _ptr(fl)
        if data.envmap is not None:
            e = arr(data.envmap, np.float32)
            d.env_height, d.env_width = e.shape[0], e.shape[1]
            d.env_rgb = _ptr(e)
        d.env_frame[:] = [float(x) for x in np.asarray(data.env_frame, np.float32).reshape(9)]
        if data.normals is not None:
            nrm = arr(data.normals, np.float32)
            if nrm.shape != data.vertices.shape:
                raise ValueError("normals must have one (x, y, z) per vertex")
            d.vertex_normals = _ptr(nrm)
        d.mesh_right_handed = 1 if data.right_handed else 0
        h = _P()
        if device:
            _check(_scene_create_ex(C.byref(d), octree | self.LISTS[lists], C.byref(h)))
        else:
            _check(_scene_build_host(C.byref(d), C.byref(h)))
        self._h = h
        self.on_device = device

    def close(self):
        if getattr(self, "_h", None):
            _check(_scene_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def info(self):
        i = SnogSceneInfo()
        _check(_scene_info(self._h, C.byref(i)))
        return {f: (list(getattr(i, f)) if isinstance(getattr(i, f), C.Array) else getattr(i, f))
                for f, _ in SnogSceneInfo._fields_}

    def octree(self):
        """(origin, size, children[n,8], heads[n], plist) with plist entries as
        primitive ids, -1 ending each list -- the reference's Octree arrays."""
        inf = self.info()
        ch = np.zeros((inf["n_nodes"], 8), np.uint32)
        hd = np.zeros(inf["n_nodes"], np.uint32)
        pl = np.zeros(inf["n_plist"], np.int32)
        _check(_scene_octree(self._h, _ptr(ch), _ptr(hd), _ptr(pl)))
        return {"origin": np.array(inf["origin"], np.float32), "size": inf["size"],
                "children": ch, "heads": hd, "list": pl}

    def trace(self, rays_soa, n_closest, want_normal=False):
        """Closest/any-hit queries for a (7, n) float32 SoA batch in host
        memory.  Returns (prim, t, normal or None, counters)."""
        rays = np.ascontiguousarray(rays_soa, np.float32)
        n = rays.shape[1]
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        nrm = np.empty((n, 3), np.float32) if want_normal else None
        cnt = np.zeros(4, np.uint64)
        _check(_trace(self._h, _ptr(rays), n, n_closest, _ptr(prim), _ptr(t), _ptr(nrm), _ptr(cnt)))
        return prim, t, nrm, {"closest_nodes": int(cnt[0]), "closest_tests": int(cnt[1]),
                              "any_nodes": int(cnt[2]), "any_tests": int(cnt[3])}

    def sample_probe(self, probes, extra=None):
        """The shading functions at given parameters (snog_sample_probe):
        PROBES is (n, 12) float32 (origin, t0 = 0, unit direction, t1, BSDF
        u v, light u v); EXTRA is (n, n_lights) or None.  Returns (head
        (n, 9), lights (n, n_lights, 18)) in the layout the header documents."""
        pr = np.ascontiguousarray(probes, np.float32)
        n = pr.shape[0]
        nl = self.info()["n_lights"]
        ex = None if extra is None else np.ascontiguousarray(extra, np.float32).reshape(n, nl)
        out = np.zeros((n, 9 + 18 * nl), np.float32)
        _check(_sample_probe(self._h, _ptr(pr), _ptr(ex), n, _ptr(out)))
        return out[:, :9].copy(), out[:, 9:].reshape(n, nl, 18).copy()

    def trace_device(self, d_rays, n, n_closest, d_prim, d_t=None, d_normal=None, stream=None):
        """Device-pointer variant (integers, e.g. torch tensor .data_ptr())."""
        _check(_trace_device(self._h, d_rays, n, n_closest, d_prim, d_t, d_normal, stream))

    def render(self, camera: Camera, params: RenderParams):
        """Render to a (height, width, 3) float32 image in host memory."""
        out = np.empty((params.height, params.width, 3), np.float32)
        st = SnogRenderStats()
        cs, ps = camera_struct(camera), params_struct(params)
        _check(_render(self._h, C.byref(cs), C.byref(ps), _ptr(out), C.byref(st)))
        return out, {f: getattr(st, f) for f, _ in SnogRenderStats._fields_}

    def render_window(self, camera: Camera, params: RenderParams, pattern, output):
        """Render the film rectangle PATTERN = (left_x, top_y, width, height)
        into the output window OUTPUT = (base_x, base_y, width, height) of
        the params.width x params.height film (the reference's
        RenderMgr::render with a RenderPattern and a sample-based
        ImageSampledOutput).  Returns ((out_h, out_w, 3) image, stats)."""
        win = SnogRenderWindow(int(pattern[0]), int(pattern[1]), int(pattern[2]), int(pattern[3]),
                               int(output[0]), int(output[1]), int(output[2]), int(output[3]))
        out = np.empty((int(output[3]), int(output[2]), 3), np.float32)
        st = SnogRenderStats()
        cs, ps = camera_struct(camera), params_struct(params)
        _check(_render_window(self._h, C.byref(cs), C.byref(ps), C.byref(win), _ptr(out), C.byref(st)))
        return out, {f: getattr(st, f) for f, _ in SnogRenderStats._fields_}

    def render_device(self, camera: Camera, params: RenderParams, d_out, stream=None,
                      want_stats=False):
        st = SnogRenderStats()
        cs, ps = camera_struct(camera), params_struct(params)
        _check(_render_device(self._h, C.byref(cs), C.byref(ps), d_out, stream,
                              C.byref(st) if want_stats else None))
        return {f: getattr(st, f) for f, _ in SnogRenderStats._fields_} if want_stats else None


def engine_config(**kw):
    """The engine's default configuration with fields overridden by KW."""
    c = SnogEngineConfig()
    _check(_engine_default(C.byref(c)))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _job_arrays(jobs):
    n = len(jobs)
    scenes = (_P * n)(*[j[0].handle for j in jobs])
    cams = (SnogCamera * n)(*[camera_struct(j[1]) for j in jobs])
    prms = (SnogRenderParams * n)(*[params_struct(j[2]) for j in jobs])
    return n, scenes, cams, prms


def _out_arrays(jobs, outs):
    if outs is None:
        outs = [np.empty((j[2].height, j[2].width, 3), np.float32) for j in jobs]
        ptrs = [o.ctypes.data for o in outs]
    else:   # device pointers (ints) or arrays
        ptrs = [o if isinstance(o, int) else o.ctypes.data for o in outs]
    return outs, (_P * len(jobs))(*ptrs)


def _batch_stats(st):
    return {f: getattr(st, f) for f, _ in SnogBatchStats._fields_}


def render_batch(jobs, config=None):
    """Render [(Scene, Camera, RenderParams), ...] together on the streaming
    engine.  Returns (list of (H, W, 3) float32 images, stats dict)."""
    n, scenes, cams, prms = _job_arrays(jobs)
    outs, optr = _out_arrays(jobs, None)
    st = SnogBatchStats()
    _check(_render_batch(scenes, cams, prms, n, optr, 0, C.byref(config) if config else None,
                         C.byref(st)))
    return outs, _batch_stats(st)


def autotune(jobs, sample_jobs=0, base=None):
    """Engine configuration tuned on a sample of JOBS; returns (config, Mpaths/s on the sample)."""
    n, scenes, cams, prms = _job_arrays(jobs)
    best = SnogEngineConfig()
    rate = C.c_double()
    _check(_engine_autotune(scenes, cams, prms, n, sample_jobs, C.byref(base) if base else None,
                            C.byref(best), C.byref(rate)))
    return best, rate.value


class Engine:
    """A persistent streaming engine (snog_engine_*): queues and CUDA graph
    stay allocated between batches.  STREAM: a cudaStream_t as int, or 0."""

    def __init__(self, config=None, stream=0):
        h = _P()
        _check(_engine_create(C.byref(config) if config else None, stream or None, C.byref(h)))
        self._h = h

    def render(self, jobs, device_outs=None, host_outs=None):
        """Render JOBS to completion.  Images go to DEVICE_OUTS (device
        pointers, one per job), else to HOST_OUTS ((H, W, 3) float32 arrays,
        e.g. pinned), else to new host arrays, which are returned."""
        n, scenes, cams, prms = _job_arrays(jobs)
        outs, optr = _out_arrays(jobs, device_outs if device_outs else host_outs)
        st = SnogBatchStats()
        _check(_engine_render(self._h, scenes, cams, prms, n, optr, 1 if device_outs else 0,
                              C.byref(st)))
        return (None if device_outs else outs), _batch_stats(st)

    def close(self):
        if getattr(self, "_h", None):
            _check(_engine_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """A render server (snog_server_*): scenes stay resident, jobs submitted
    at any time join the running wavefront (continuous batching)."""

    def __init__(self, config=None):
        h = _P()
        _check(_server_create(C.byref(config) if config else None, C.byref(h)))
        self._h = h
        self._outs = {}
        self._scenes = []

    def add_scene(self, scene: Scene):
        slot = C.c_uint32()
        _check(_server_add_scene(self._h, scene.handle, C.byref(slot)))
        self._scenes.append(scene)
        return slot.value

    def submit(self, slot, camera: Camera, params: RenderParams):
        out = np.empty((params.height, params.width, 3), np.float32)
        jid = C.c_uint64()
        cs, ps = camera_struct(camera), params_struct(params)
        _check(_server_submit(self._h, slot, C.byref(cs), C.byref(ps), out.ctypes.data, C.byref(jid)))
        self._outs[jid.value] = out
        return jid.value

    @staticmethod
    def _stats(st):
        return {f: getattr(st, f) for f, _ in SnogJobStats._fields_}

    def poll(self, job):
        st = SnogJobStats()
        rc = _server_poll(self._h, job, C.byref(st))
        if rc == SNOG_EBUSY:
            return None
        _check(rc)
        return self._outs.pop(job), self._stats(st)

    def wait(self, job, timeout_ms=60000):
        st = SnogJobStats()
        _check(_server_wait(self._h, job, timeout_ms, C.byref(st)))
        return self._outs.pop(job), self._stats(st)

    def cancel(self, job):
        _check(_server_cancel(self._h, job))

    def pause(self, job):
        """Stop starting JOB's paths; those in flight finish (snog_server_pause)."""
        _check(_server_pause(self._h, job))

    def resume(self, job):
        _check(_server_resume(self._h, job))

    def checkpoint(self, job, path, timeout_ms=60000):
        """Write paused JOB's finished paths to PATH (snog_server_checkpoint)."""
        _check(_server_checkpoint(self._h, job, os.fsencode(path), timeout_ms))

    def submit_resume(self, slot, path):
        """A job continuing the checkpoint in PATH; its image goes where
        wait() returns it, like submit()."""
        with open(path, "rb") as f:
            head = f.read(8 + C.sizeof(SnogCamera) + C.sizeof(SnogRenderParams))
        ps = SnogRenderParams.from_buffer_copy(head[8 + C.sizeof(SnogCamera):])
        out = np.empty((ps.height, ps.width, 3), np.float32)
        jid = C.c_uint64()
        _check(_server_submit_resume(self._h, slot, os.fsencode(path), out.ctypes.data, C.byref(jid)))
        self._outs[jid.value] = out
        return jid.value

    def close(self):
        if getattr(self, "_h", None):
            _check(_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_ply_load = _sig("snog_ply_load", C.c_int, C.c_char_p, C.POINTER(SnogPlyMesh))
_ply_free = _sig("snog_ply_free", C.c_int, C.POINTER(SnogPlyMesh))


def load_ply(path):
    """Read a PLY mesh with the reference's rules (snog_ply_load).  Returns
    (vertices (n, 3) float32, normals (n, 3) float32 or None, triangles (m, 3)
    uint32); the mesh is right-handed."""
    m = SnogPlyMesh()
    _check(_ply_load(os.fsencode(path), C.byref(m)))
    try:
        nv, nt = m.n_vertices, m.n_triangles
        verts = np.ctypeslib.as_array(m.vertices, (nv * 3,)).reshape(nv, 3).copy() if nv else \
            np.zeros((0, 3), np.float32)
        nrm = (np.ctypeslib.as_array(m.normals, (nv * 3,)).reshape(nv, 3).copy()
               if bool(m.normals) and nv else None)
        tris = np.ctypeslib.as_array(m.triangles, (nt * 3,)).reshape(nt, 3).copy() if nt else \
            np.zeros((0, 3), np.uint32)
    finally:
        _ply_free(C.byref(m))
    return verts, nrm, tris


def exported_symbols():
    """Names declared in include/snogray_b200.h (for the ABI check)."""
    import re
    hdr = os.path.join(os.path.dirname(_HERE), "include", "snogray_b200.h")
    with open(hdr) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(snog_\w+)\s*\(", text, re.M)))


__all__ = ["Scene", "SceneData", "Camera", "RenderParams", "SnogError", "scenes", "init",
           "version", "exported_symbols", "load_ply", "LIB_PATH"]
