"""The streaming engine (batched and served rendering) on the GPU.

A job's random streams are keyed by (seed, path index in the job, dimension),
not by where or when it runs, so a job rendered in a batch, in a server mix,
or alone through the plain renderer produces the same image up to the order
of float additions (shadow contributions arrive through atomics, samples are
gathered in a different order): rtol 1e-4, atol 1e-5 here.
"""

import time

import numpy as np
import pytest

import snogray_b200 as sb
from snogray_b200 import scenes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-5


def _jobs():
    cornell = sb.Scene(scenes.cornell_box())
    terrain = sb.Scene(scenes.terrain_scene(n=64, n_spheres=20, seed=3, env_w=64, env_h=32))
    soup = sb.Scene(scenes.soup_scene(3000, 5))
    rng = np.random.default_rng(0)
    return [
        (cornell, scenes.cornell_camera(48, 40), scenes.cornell_params(48, 40, 8, seed=3)),
        (terrain, scenes.terrain_camera(64, 36), scenes.terrain_params(64, 36, 4, seed=4)),
        (soup, scenes.orbit_camera(40, 40, rng), sb.RenderParams(40, 40, 16, 3, 8, 1, seed=5)),
        (cornell, scenes.cornell_camera(32, 32), scenes.cornell_params(32, 32, 16, seed=6)),
    ]


def test_batch_matches_plain_renders():
    jobs = _jobs()
    imgs, st = sb.render_batch(jobs)
    assert st["paths"] == sum(p.width * p.height * p.spp for _, _, p in jobs)
    assert st["closest_rays"] > 0 and st["shadow_rays"] > 0
    for (sc, cam, p), img in zip(jobs, imgs):
        ref, _ = sc.render(cam, p)
        assert np.isfinite(img).all()
        assert np.allclose(img, ref, rtol=RTOL, atol=ATOL), np.abs(img - ref).max()


def test_batch_with_tiny_queues_and_ring():
    """Few slots and small items: many regeneration rounds, ring wrap-around,
    jobs interleaved item by item -- same images."""
    jobs = _jobs()[:3]
    cfg = sb.engine_config(slots=4096, item_paths=1000, ring_items=16, iters_per_launch=1)
    imgs, _ = sb.render_batch(jobs, cfg)
    for (sc, cam, p), img in zip(jobs, imgs):
        ref, _ = sc.render(cam, p)
        assert np.allclose(img, ref, rtol=RTOL, atol=ATOL), np.abs(img - ref).max()


def test_server_result_same_alone_and_in_mix():
    jobs = _jobs()
    cfg = sb.engine_config(slots=1 << 16, item_paths=4096)
    with sb.Server(cfg) as srv:
        slots = {}
        for sc, _, _ in jobs:
            if id(sc) not in slots:
                slots[id(sc)] = srv.add_scene(sc)
        # job 0 alone
        j = srv.submit(slots[id(jobs[0][0])], jobs[0][1], jobs[0][2])
        alone, st = srv.wait(j)
        assert st["status"] == 0 and st["finish_ms"] >= st["start_ms"] >= st["admit_ms"] >= st["submit_ms"]
        # job 0 again, arriving while the others run
        ids = []
        for k in (1, 2, 0, 3):
            sc, cam, p = jobs[k]
            ids.append((k, srv.submit(slots[id(sc)], cam, p)))
            time.sleep(0.002)
        outs = {k: srv.wait(jid) for k, jid in ids}
    assert np.allclose(outs[0][0], alone, rtol=RTOL, atol=ATOL)
    for k, (img, st) in outs.items():
        ref, _ = jobs[k][0].render(jobs[k][1], jobs[k][2])
        assert np.allclose(img, ref, rtol=RTOL, atol=ATOL)
        assert st["paths"] == jobs[k][2].width * jobs[k][2].height * jobs[k][2].spp


def test_server_cancel_and_timeouts():
    sc = sb.Scene(scenes.cornell_box())
    with sb.Server(sb.engine_config(slots=1 << 14, item_paths=1024)) as srv:
        slot = srv.add_scene(sc)
        big = srv.submit(slot, scenes.cornell_camera(256, 256), scenes.cornell_params(256, 256, 64))
        small = srv.submit(slot, scenes.cornell_camera(16, 16), scenes.cornell_params(16, 16, 4))
        srv.cancel(big)
        img, st = srv.wait(small)
        assert st["status"] == 0 and img.mean() > 0
        with pytest.raises(sb.SnogError) as e:
            srv.wait(big)
        assert e.value.code == sb.SNOG_ECANCELED
        with pytest.raises(sb.SnogError) as e:
            srv.poll(987654)
        assert e.value.code == sb.SNOG_ENOTFOUND
        # a wait that runs out returns SNOG_ETIMEOUT and leaves the job running
        j = srv.submit(slot, scenes.cornell_camera(128, 128), scenes.cornell_params(128, 128, 64))
        with pytest.raises(sb.SnogError) as e:
            srv.wait(j, timeout_ms=0)
        assert e.value.code == sb.SNOG_ETIMEOUT
        img, st = srv.wait(j, timeout_ms=120000)
        assert st["status"] == 0
