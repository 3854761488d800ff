"""Eye rays, pinned to the reference.

The camera kernels (k_camera, k_e_regen) form a sample's film location as
Renderer::render_packet does (render-mgr/renderer.cc:84) and its direction as
Camera::eye_vec (camera/camera.h:384-389), in float32 in that order.  The
golden generator's restatement of those two steps (gen_golden.eye_dirs) makes
the Cornell camera rays that the device traces bit-exactly
(tests/test_trace_gpu.py, trace_cornell_camera.npz); this test pins the
restatement to the reference's own Camera::eye_ray, bit for bit, on two
cameras (tests/golden/camera_eye_rays.npz, harness mode `camera`).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import spec
from gen_golden import CAMERA_CASES, camera_film_locs, eye_dirs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(CAMERA_CASES))
def test_eye_directions_equal_reference_eye_rays(name):
    g = np.load(os.path.join(GOLDEN, "camera_eye_rays.npz"))
    mk, cam, w, h = CAMERA_CASES[name]
    u, v = camera_film_locs(w, h, seed=61)
    assert np.array_equal(eye_dirs(cam(), u, v), g[name])
    if spec.have_ref():
        assert np.array_equal(spec.ref_eye_dirs(mk(), cam(), u, v), g[name])
