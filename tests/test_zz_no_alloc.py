"""snog_render_device_noalloc: the render entry point that allocates no device
memory, for hosts that own all device memory themselves or cannot let
cudaMalloc / cudaFree stall the device.  Its working memory is one fixed
device array inside the library, shared by all calls.

Checked through the C ABI: two calls in a row (different jobs, so the second
must not see the first's leftovers) each match the allocating entry point,
snog_render_device, on the same job; a job beyond the array's limit is refused
with a clear error.  Images agree up to float summation order (the two entry
points split the job into different waves, and shadow contributions arrive
through atomics): rtol 1e-5, atol 1e-6, as the other multi-wave render tests.
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
