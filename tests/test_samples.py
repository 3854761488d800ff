"""Per-sample parity of the path's shading functions.

The renderers draw sample parameters from their own generator, so images are
compared statistically (test_render_gpu.py).  Here the parameters are inputs:
for probes through each fixture scene's camera (a ray, a BSDF parameter and a
light parameter), the device's Bsdf::sample / Bsdf::eval and every light
sampler's sample / eval (snog_sample_probe) are compared, sample by sample,
with the reference's functions at the same parameters
(tests/golden/samples_*.npz, from oracle/ref_harness.cc mode `samples`:
material/bsdf.h:158-168, light/light-sampler.h).  The sphere light's extra
random number (light/sphere-light-sampler.cc:90) is the one the reference
drew, fed to the device.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import spec
from gen_golden import SAMPLE_CASES
from snogray_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Floats computed in a different order (and CUDA's versus glibc's
# transcendental functions) agree to a few ulps: over the six scenes 92-100 %
# of the values are bit-equal, the largest relative difference is 1.2e-4
# (a Cook-Torrance eval near grazing, where nearby values cancel) and the
# largest direction difference 3.3e-7.  The bars leave a margin of 4 and 30.
RTOL, ATOL_DIR = 5e-4, 1e-5

# Head: hit, BSDF sample val[3] pdf dir[3] flags.  Per light: sample val[3]
# pdf dir[3] dist extra; BSDF eval val[3] pdf; light eval val[3] pdf dist.
# Per quantity: where, value columns, direction columns, the pdf column that
# says whether there is a sample (a sample of pdf 0 is "no sample": its
# direction means nothing -- the reference leaves it (0, 0, 0), the device
# (0, 0, 1) -- so directions are compared where either side has a sample).
QUANTITIES = {
    "bsdf_sample": ("head", [1, 2, 3, 4], [5, 6, 7], 4),
    "light_sample": ("light", [0, 1, 2, 3, 7], [4, 5, 6], 3),
    "bsdf_eval": ("light", [9, 10, 11, 12], [], None),
    "light_eval": ("light", [13, 14, 15, 16, 17], [], None),
}


def load(name):
    return np.load(os.path.join(GOLDEN, f"samples_{name}.npz"))


def _close(a, b, cols_val, cols_dir, col_pdf):
    ok = np.ones(a.shape[:-1], bool)
    for c in cols_val:
        x, y = a[..., c].astype(np.float64), b[..., c].astype(np.float64)
        ok &= np.abs(x - y) <= RTOL * np.maximum(np.abs(x), np.abs(y)) + 1e-30
    if cols_dir:
        sampled = (a[..., col_pdf] != 0) | (b[..., col_pdf] != 0)
        for c in cols_dir:
            ok &= ~sampled | (np.abs(a[..., c] - b[..., c]) <= ATOL_DIR)
    return ok


def mismatches(g, head, lights):
    """Per quantity: (rows compared, rows outside tolerance) over hit probes,
    plus the exact checks (hit, BSDF sample flags)."""
    rh, rl = g["head"], g["lights"]
    hit = rh[:, 0] > 0
    out = {"hit_differs": int((rh[:, 0] != head[:, 0]).sum()),
           "flags_differ": int((rh[hit, 8] != head[hit, 8]).sum())}
    for q, (where, vals, dirs, pdf) in QUANTITIES.items():
        a, b = (rh, head) if where == "head" else (rl, lights)
        ok = _close(a, b, vals, dirs, pdf)
        if where == "head":
            ok, used = ok[hit], hit.sum()
        else:
            ok, used = ok[hit], hit.sum() * a.shape[1]
        out[q] = (int(used), int((~ok).sum()))
    return out


def sampled_rows(g):
    """Hit probes whose BSDF sample, and (probe, light) pairs whose light
    sample, the reference made (pdf > 0)."""
    hit = g["head"][:, 0] > 0
    return int((g["head"][hit, 4] > 0).sum()), int((g["lights"][hit, :, 3] > 0).sum())


@pytest.mark.parametrize("name", sorted(SAMPLE_CASES))
def test_fixture_pins_scene_probes_and_reference(name):
    g = load(name)
    mk, cam = SAMPLE_CASES[name]
    sd = mk()
    assert str(g["scene_digest"]) == scenes.scene_digest(sd)
    assert np.array_equal(g["probes"], spec.camera_probes(cam(), len(g["probes"]), seed=53))
    hit = g["head"][:, 0] > 0
    assert hit.sum() > 500
    # every light gets samples, and the BSDF samples cover their classes
    assert (g["lights"][hit, :, 3] > 0).any(axis=0).all()
    assert (g["head"][hit, 4] > 0).mean() > 0.9
    if spec.have_ref():
        nl, head, lights = spec.ref_samples(sd, g["probes"][:256])
        assert nl == int(g["n_lights"])
        assert np.array_equal(head, g["head"][:256])
        assert np.array_equal(lights, g["lights"][:256])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SAMPLE_CASES))
def test_device_shading_matches_reference_per_sample(name):
    import snogray_b200 as sb
    g = load(name)
    mk, _ = SAMPLE_CASES[name]
    with sb.Scene(mk()) as sc:
        assert sc.info()["n_lights"] == int(g["n_lights"])
        head, lights = sc.sample_probe(g["probes"], extra=g["lights"][:, :, 8])
    m = mismatches(g, head, lights)
    assert m["hit_differs"] == 0 and m["flags_differ"] == 0, m
    for q in QUANTITIES:
        assert m[q][1] == 0, (q, m)


def test_probe_refusals_before_device_work():
    """snog_sample_probe refuses a host-only scene and null arguments with
    SNOG_EINVAL before it touches the device."""
    import ctypes

    import snogray_b200 as sb
    g = load("cornell")
    with sb.Scene(scenes.cornell_box(), device=False) as sc:
        with pytest.raises(sb.SnogError) as e:
            sc.sample_probe(g["probes"][:4])
        assert e.value.code == sb.SNOG_EINVAL and "host-only" in str(e.value)
        out = np.zeros(64, np.float32)
        assert sb._sample_probe(sc.handle, None, None, 4, out.ctypes.data_as(ctypes.c_void_p)) == sb.SNOG_EINVAL
    assert sb._sample_probe(None, None, None, 0, None) == sb.SNOG_EINVAL
