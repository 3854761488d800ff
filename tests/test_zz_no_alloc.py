"""snog_render_device_noalloc: the render entry point that allocates no device
memory, for hosts that own all device memory themselves or cannot let
cudaMalloc / cudaFree stall the device.  Its working memory is one fixed
device array inside the library, shared by all calls.

Checked through the C ABI: two calls in a row (different jobs, so the second
must not see the first's leftovers) each match the allocating entry point,
snog_render_device, on the same job; so does a job several times larger than
one wave of the array, which the call renders in many waves (the pixel rows
of consecutive waves meet in the filter's accumulator); a call on a new job
size leaves the device's free memory unchanged; jobs beyond the array's
limits -- too many pixels, or too many samples per pixel for one wave -- are
refused with a clear error.  Images agree up to float summation order (the
two entry points split the job into different waves, and shadow
contributions arrive through atomics): rtol 1e-5, atol 1e-6, as the other
multi-wave render tests.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    import snogray_b200 as sb
    fn = ctypes.CDLL(sb.LIB_PATH).snog_render_device_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(sb.SnogCamera), ctypes.POINTER(sb.SnogRenderParams),
                   ctypes.c_void_p, ctypes.c_void_p]
    return fn


def test_noalloc_matches_allocating_render_on_two_calls():
    import torch
    import snogray_b200 as sb
    from snogray_b200 import scenes
    fn = _noalloc_fn()
    jobs = [(96, 80, 8, 11), (64, 48, 4, 12)]
    with sb.Scene(scenes.cornell_box()) as sc:
        for w, h, spp, seed in jobs:
            cam = scenes.cornell_camera(w, h)
            p = scenes.cornell_params(w, h, spp, seed=seed)
            ref = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
            sc.render_device(cam, p, ref.data_ptr())
            out = torch.full((h, w, 3), float("nan"), dtype=torch.float32, device="cuda")
            cs, ps = sb.camera_struct(cam), sb.params_struct(p)
            rc = fn(sc.handle, ctypes.byref(cs), ctypes.byref(ps), out.data_ptr(), None)
            assert rc == sb.SNOG_OK, sb._last_error().decode()
            torch.cuda.synchronize()
            a, b = out.cpu().numpy(), ref.cpu().numpy()
            assert np.isfinite(a).all()
            assert np.allclose(a, b, rtol=1e-5, atol=1e-6), np.abs(a - b).max()


def _render_both(fn, sc, cam, p):
    import torch
    import snogray_b200 as sb
    ref = torch.empty((p.height, p.width, 3), dtype=torch.float32, device="cuda")
    sc.render_device(cam, p, ref.data_ptr())
    out = torch.full((p.height, p.width, 3), float("nan"), dtype=torch.float32, device="cuda")
    cs, ps = sb.camera_struct(cam), sb.params_struct(p)
    rc = fn(sc.handle, ctypes.byref(cs), ctypes.byref(ps), out.data_ptr(), None)
    assert rc == sb.SNOG_OK, sb._last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy(), ref.cpu().numpy()


def test_noalloc_many_waves_match_allocating_render():
    """132 x 132 pattern pixels x 64 spp = 1.1M paths: about six waves of the
    array's path state (some 190k paths with one light)."""
    import snogray_b200 as sb
    from snogray_b200 import scenes
    fn = _noalloc_fn()
    w = h = 128
    with sb.Scene(scenes.cornell_box()) as sc:
        a, b = _render_both(fn, sc, scenes.cornell_camera(w, h), scenes.cornell_params(w, h, 64, seed=21))
    assert np.isfinite(a).all() and a.mean() > 0.05
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6), np.abs(a - b).max()


def test_noalloc_leaves_free_device_memory_unchanged():
    import torch
    import snogray_b200 as sb
    from snogray_b200 import scenes
    fn = _noalloc_fn()
    with sb.Scene(scenes.cornell_box()) as sc:
        outs = {}
        for w, h in ((40, 32), (72, 56)):
            outs[w] = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()

        def call(w, h, spp):
            cs = sb.camera_struct(scenes.cornell_camera(w, h))
            ps = sb.params_struct(scenes.cornell_params(w, h, spp, seed=2))
            rc = fn(sc.handle, ctypes.byref(cs), ctypes.byref(ps), outs[w].data_ptr(), None)
            assert rc == sb.SNOG_OK, sb._last_error().decode()
            torch.cuda.synchronize()

        # The first call on the device looks up the array's address and loads
        # the kernels this job size uses (the same spp: the same kernels).
        call(40, 32, 8)
        free0, _ = torch.cuda.mem_get_info()
        call(72, 56, 8)                      # a new job size
        free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"


def test_noalloc_refuses_samples_beyond_one_wave():
    """With two lights and 64 light samples each a vertex needs 256 shadow
    rays: one wave of the array then holds some 3,700 paths, fewer than one
    pixel's 4096 samples."""
    import torch
    import snogray_b200 as sb
    from snogray_b200 import scenes
    fn = _noalloc_fn()
    w = h = 8
    with sb.Scene(scenes.mirror_scene()) as sc:
        assert sc.info()["n_lights"] == 2
        out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        cs = sb.camera_struct(scenes.cornell_camera(w, h))
        p = scenes.mirror_params(w, h, 4096)
        p.direct_samples = 64
        ps = sb.params_struct(p)
        rc = fn(sc.handle, ctypes.byref(cs), ctypes.byref(ps), out.data_ptr(), None)
        assert rc == sb.SNOG_EINVAL
        assert "do not fit the no-alloc scratch" in sb._last_error().decode()


def test_noalloc_refuses_jobs_beyond_its_scratch():
    import torch
    import snogray_b200 as sb
    from snogray_b200 import scenes
    fn = _noalloc_fn()
    w, h = 1200, 1000                                   # 1.2M pixels > the 1M limit
    with sb.Scene(scenes.cornell_box()) as sc:
        out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        cs = sb.camera_struct(scenes.cornell_camera(w, h))
        ps = sb.params_struct(scenes.cornell_params(w, h, 1))
        rc = fn(sc.handle, ctypes.byref(cs), ctypes.byref(ps), out.data_ptr(), None)
        assert rc == sb.SNOG_EINVAL
        assert "no-alloc limit" in sb._last_error().decode()
