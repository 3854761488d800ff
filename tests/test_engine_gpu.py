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
        (soup, scenes.orbit_camera(40, 40, rng), sb.RenderParams(40, 40, 16, 3, 8, 2, seed=5)),
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


def test_persistent_engine_reuse_and_device_outputs():
    import torch
    jobs = _jobs()
    with sb.Engine(sb.engine_config(slots=1 << 18, item_paths=1 << 13)) as eng:
        a, st_a = eng.render(jobs)
        b, st_b = eng.render(jobs[::-1])          # other scene slots, same images
        outs = [torch.empty((p.height, p.width, 3), dtype=torch.float32, device="cuda") for _, _, p in jobs]
        none, st_c = eng.render(jobs, device_outs=[o.data_ptr() for o in outs])
        torch.cuda.synchronize()
    assert none is None
    assert st_a["paths"] == st_b["paths"] == st_c["paths"]
    for k, (sc, cam, p) in enumerate(jobs):
        ref, _ = sc.render(cam, p)
        assert np.allclose(a[k], ref, rtol=RTOL, atol=ATOL)
        assert np.allclose(b[len(jobs) - 1 - k], ref, rtol=RTOL, atol=ATOL)
        assert np.allclose(outs[k].cpu().numpy(), ref, rtol=RTOL, atol=ATOL)


def test_profiled_batch_reports_kernel_times(monkeypatch):
    jobs = _jobs()[:2]
    monkeypatch.setenv("SNOG_PROFILE_KERNELS", "1")
    imgs, st = sb.render_batch(jobs)
    assert st["iterations"] > 0 and st["closest_ms"] > 0 and st["shadow_ms"] > 0 and st["shade_ms"] > 0
    for (sc, cam, p), img in zip(jobs, imgs):
        ref, _ = sc.render(cam, p)
        assert np.allclose(img, ref, rtol=RTOL, atol=ATOL)


def test_autotune_returns_a_working_config():
    jobs = _jobs()
    cfg, rate = sb.autotune(jobs, sample_jobs=4)
    assert rate > 0
    assert cfg.slots >= 1024 and cfg.item_paths > 0 and cfg.iters_per_launch > 0
    imgs, _ = sb.render_batch(jobs, cfg)
    for (sc, cam, p), img in zip(jobs, imgs):
        ref, _ = sc.render(cam, p)
        assert np.allclose(img, ref, rtol=RTOL, atol=ATOL)


def test_many_scenes_in_one_batch():
    """More distinct scenes than jobs slots of the default table size: a
    uneven batch of small soups (the batched workload in miniature)."""
    rng = np.random.default_rng(9)
    jobs = []
    for k in range(40):
        n = int(rng.integers(200, 3000))
        res = int(rng.choice([16, 24, 32]))
        jobs.append((sb.Scene(scenes.soup_scene(n, 100 + k)), scenes.orbit_camera(res, res, rng),
                     sb.RenderParams(res, res, int(rng.choice([1, 4, 8])), seed=k)))
    imgs, st = sb.render_batch(jobs, sb.engine_config(slots=1 << 14, item_paths=512, max_scenes=64))
    for (sc, cam, p), img in zip(jobs, imgs):
        ref, _ = sc.render(cam, p)
        assert np.allclose(img, ref, rtol=RTOL, atol=ATOL)


def test_direct_integrator_spawn_ring_overflow_is_unbiased(golden):
    """The direct integrator starts a second ray where glass both reflects and
    transmits; with a tiny queue the spawn ring is full most of the time and
    vertices keep one of their two rays at twice the weight.  Image means stay
    within 3 standard errors of the reference's (render_cornell_direct)."""
    import math
    g = golden("render_cornell_direct.npz")
    w, h, spp = int(g["width"]), int(g["height"]), int(g["spp"])
    cfg = sb.engine_config(slots=4096, item_paths=1024, ring_items=256)
    means = []
    with sb.Scene(scenes.cornell_box()) as sc:
        cam = scenes.cornell_camera(w, h)
        for k in range(32):
            imgs, st = sb.render_batch([(sc, cam, scenes.direct_params(w, h, spp, seed=100 + k))], config=cfg)
            means.append(imgs[0].reshape(-1, 3).mean(0))
    means = np.array(means)
    m = means.mean(0)
    se = np.sqrt((means.std(0, ddof=1) / math.sqrt(len(means))) ** 2 + g["se"] ** 2)
    z = np.abs(m - g["mean"]) / se
    assert (z < 3).all(), f"means {m} ref {g['mean']} z {z}"


def test_direct_integrator_same_through_plain_batch_and_server():
    sd = scenes.cornell_box()
    cam = scenes.cornell_camera(40, 32)
    p = scenes.direct_params(40, 32, 8, seed=5)
    with sb.Scene(sd) as sc:
        plain, st = sc.render(cam, p)
        batch, _ = sb.render_batch([(sc, cam, p)])
        with sb.Server() as srv:
            served, sst = srv.wait(srv.submit(srv.add_scene(sc), cam, p))
    assert st["paths"] == 44 * 36 * 8 and st["shadow_rays"] > 0
    assert np.isfinite(plain).all() and plain.mean() > 0.05
    for img in (batch[0], served):
        assert np.allclose(img, plain, rtol=1e-5, atol=1e-6), np.abs(img - plain).max()



def test_list_dealing_modes_give_identical_results():
    """Dealing node lists one entry per lane and two per lane finds the same
    hits in the same order, on a scene of long lists (a random-triangle soup)
    and one of short lists (the terrain): the same traversal counts, exactly
    (a different hit would change the rest of its path), and the same images
    on the plain renderer and the engine up to the order in which shadow
    rays' contributions are added (float atomics: rtol 1e-4, the bar of the
    engine-vs-plain tests)."""
    import dataclasses
    cases = [(scenes.soup_scene(300_000, seed=25), scenes.orbit_camera(48, 40, np.random.default_rng(5)),
              sb.RenderParams(48, 40, 4, seed=3)),
             (scenes.terrain_scene(n=256, n_spheres=20, env_w=64, env_h=32), scenes.terrain_camera(40, 32),
              scenes.terrain_params(40, 32, 4, seed=4))]
    for sd, cam, p in cases:
        with sb.Scene(sd, lists="single") as one, sb.Scene(sd, lists="paired") as two:
            assert one.info()["pair_lists"] == 0 and two.info()["pair_lists"] == 1
            counted = dataclasses.replace(p, flags=sb.SNOG_RENDER_COUNT_TRAVERSAL)
            img1, st1 = one.render(cam, counted)
            img2, st2 = two.render(cam, counted)
            assert np.allclose(img1, img2, rtol=1e-4, atol=1e-5), np.abs(img1 - img2).max()
            assert st1["closest_tests"] > 0
            for k in ("closest_rays", "closest_nodes", "closest_tests", "shadow_nodes", "shadow_tests"):
                assert st1[k] == st2[k], k
            e1, _ = sb.render_batch([(one, cam, p)])
            e2, _ = sb.render_batch([(two, cam, p)])
            assert np.allclose(e1[0], e2[0], rtol=1e-4, atol=1e-5), np.abs(e1[0] - e2[0]).max()


def test_list_dealing_chosen_per_scene():
    """The closest-hit traversal deals list entries in pairs for scenes whose
    rays meet long lists (a random-triangle soup), one by one otherwise (the
    terrain); either way a job's image is its plain render's."""
    with sb.Scene(scenes.soup_scene(1_000_000, seed=25)) as soup, \
            sb.Scene(scenes.terrain_scene(n=256, n_spheres=20, env_w=64, env_h=32)) as terrain:
        assert soup.info()["pair_lists"] == 1
        assert terrain.info()["pair_lists"] == 0
        jobs = [(soup, scenes.orbit_camera(48, 40, np.random.default_rng(5)), sb.RenderParams(48, 40, 4, seed=3)),
                (terrain, scenes.terrain_camera(40, 32), scenes.terrain_params(40, 32, 4, seed=4))]
        imgs, _ = sb.render_batch(jobs)
        for (sc, cam, p), img in zip(jobs, imgs):
            ref, _ = sc.render(cam, p)
            assert np.allclose(img, ref, rtol=1e-4, atol=1e-5), np.abs(img - ref).max()
