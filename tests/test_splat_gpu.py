"""The Mitchell-filter splat (ImageFilterConv::add_sample,
image/image-filter-conv.h:109-186, and the resolve of
image/image-sampled-output.cc:79-123) against a float64 restatement, on
synthetic samples.

A checkpoint whose paths are all finished carries every sample of a job --
per path the radiance and alpha (Tint) and the film jitter -- so a job resumed
from it traces nothing and only splats.  Writing such a checkpoint from
seeded random samples gives the device splat known input; the image must
equal the restatement's up to float32 summation order.  The samples include
zero and partial alpha and radiance bright enough for the negative-lobe clamp
(neg_clamp = -0.1), and the sample counts cover every lane-group width the
splat kernel is compiled for (1, 2, 4, 8, 16 and 32 lanes per target pixel,
with counts that do not fill a group).
"""

import numpy as np
import pytest

import snogray_b200 as sb
from snogray_b200 import scenes

pytestmark = pytest.mark.gpu

B = C = 1.0 / 3.0


def mitchell1(x):
    """The Mitchell-Netravali filter with B = C = 1/3, radius 2
    (image/image-mitchell-filt.h:50-65), elementwise in float64."""
    x = np.abs(x)
    outer = ((-B - 6 * C) * x ** 3 + (6 * B + 30 * C) * x ** 2 + (-12 * B - 48 * C) * x + (8 * B + 24 * C)) / 6
    inner = ((12 - 9 * B - 6 * C) * x ** 3 + (-18 + 12 * B + 6 * C) * x ** 2 + (6 - 2 * B)) / 6
    return np.where(x > 2, 0.0, np.where(x > 1, outer, inner))


def ref_splat(w, h, spp, result, jit):
    """Gather of every target pixel over the samples of its 5x5 pattern
    neighbourhood (the pattern has a 2-pixel margin), then the resolve."""
    pw = w + 4
    res = result.astype(np.float64).reshape(h + 4, pw, spp, 4)
    jt = jit.astype(np.float64).reshape(h + 4, pw, spp, 2)
    acc = np.zeros((h, w, 4))
    wsum = np.zeros((h, w))
    ty, tx = np.mgrid[0:h, 0:w]
    for dy in range(-2, 3):
        for dx in range(-2, 3):
            r = res[ty + dy + 2, tx + dx + 2]                  # (h, w, spp, 4)
            j = jt[ty + dy + 2, tx + dx + 2]
            sx = (tx + dx)[..., None] + j[..., 0]
            sy = (ty + dy)[..., None] + j[..., 1]
            wt = mitchell1(sx - (tx[..., None] + 0.5)) * mitchell1(sy - (ty[..., None] + 0.5))
            c = r[..., :3] * r[..., 3:4] * wt[..., None]
            a = r[..., 3] * wt
            mc = c.min(-1)
            clamp = (wt < 0) & (mc < -0.1)
            sc = np.where(clamp, -0.1 / np.where(clamp, mc, 1.0), 1.0)
            acc[..., :3] += (c * sc[..., None]).sum(2)
            acc[..., 3] += (a * sc).sum(2)
            wsum += (wt * sc).sum(2)
    scale = np.where((wsum > 0) & (wsum != 1), 1.0 / np.where(wsum > 0, wsum, 1.0), 1.0)
    acc *= scale[..., None]
    al = np.clip(acc[..., 3], 0, 1)
    rgb = np.maximum(acc[..., :3], 0)
    rgb = np.where(((al != 0) & (al != 1))[..., None], rgb / np.where(al > 0, al, 1.0)[..., None], rgb)
    return rgb


def synthetic_samples(n, seed):
    rng = np.random.default_rng(seed)
    result = np.empty((n, 4), np.float32)
    result[:, :3] = rng.uniform(0, 1, (n, 3))
    bright = rng.random(n) < 0.1
    result[bright, :3] *= 40.0                          # reaches the negative-lobe clamp
    result[:, 3] = rng.choice(np.array([1.0, 1.0, 1.0, 0.5, 0.0], np.float32), n)
    jit = rng.random((n, 2)).astype(np.float32)
    return result, jit


def write_all_done_checkpoint(path, sc, cam, params, result, jit):
    """Checkpoint file of a job whose every path is finished: "SNOGCKP1", the
    job's SnogCamera and SnogRenderParams, total and finished paths, the
    scene's fingerprint (surfaces | octree nodes << 32), then the samples."""
    inf = sc.info()
    check = (inf["n_triangles"] + inf["n_spheres"] + inf["n_tripars"]) | (inf["n_nodes"] << 32)
    total = (params.width + 4) * (params.height + 4) * params.spp
    assert len(result) == len(jit) == total
    with open(path, "wb") as f:
        f.write(b"SNOGCKP1")
        f.write(bytes(sb.camera_struct(cam)))
        f.write(bytes(sb.params_struct(params)))
        f.write(np.array([total, total, check], "<u8").tobytes())
        f.write(np.ascontiguousarray(result, "<f4").tobytes())
        f.write(np.ascontiguousarray(jit, "<f4").tobytes())


@pytest.fixture(scope="module")
def cornell():
    sb.init(0)
    with sb.Scene(scenes.cornell_box()) as sc:
        yield sc


@pytest.mark.parametrize("spp", [1, 2, 3, 5, 8, 13, 16, 33, 64])
def test_device_splat_equals_restatement(cornell, tmp_path, spp):
    w, h = 23, 17
    cam = scenes.cornell_camera(w, h)
    params = scenes.cornell_params(w, h, spp, seed=spp)
    result, jit = synthetic_samples((w + 4) * (h + 4) * spp, seed=1000 + spp)
    path = str(tmp_path / "all_done.ckp")
    write_all_done_checkpoint(path, cornell, cam, params, result, jit)
    with sb.Server(sb.engine_config(slots=1 << 16, item_paths=1 << 12)) as srv:
        slot = srv.add_scene(cornell)
        img, st = srv.wait(srv.submit_resume(slot, path), timeout_ms=60000)
    assert st["status"] == sb.SNOG_OK
    ref = ref_splat(w, h, spp, result, jit)
    assert img.shape == ref.shape
    # float32 sums of up to 25 x 64 terms, some 40x brighter than the result
    assert np.allclose(img, ref, rtol=1e-3, atol=1e-4), np.abs(img - ref).max()
