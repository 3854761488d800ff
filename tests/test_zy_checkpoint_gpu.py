"""Preemption and checkpoints of resident jobs on the render server.

A job paused part-way, written to a checkpoint file and continued by another
server (a fresh one, as after a restart) gives the image of the same job
rendered without interruption: path streams are keyed by the job's seed and
the path index, so the resumed job traces exactly the paths the checkpoint
lacks.  Shadow rays add their contributions with float atomics, so equal jobs
agree up to the order of those additions (rtol 1e-5, as in the renderer's
determinism test).  Paused jobs free the device for other jobs.
"""

import ctypes
import os
import time

import numpy as np
import pytest

import snogray_b200 as sb
from snogray_b200 import scenes

pytestmark = pytest.mark.gpu

CKP_HEAD = 8 + ctypes.sizeof(sb.SnogCamera) + ctypes.sizeof(sb.SnogRenderParams)   # magic, camera, params


def _job(w=1024, h=1024, spp=64, seed=9):
    return scenes.cornell_camera(w, h), scenes.cornell_params(w, h, spp, seed=seed)


def _counts(path):
    with open(path, "rb") as f:
        f.seek(CKP_HEAD)
        total, done = np.frombuffer(f.read(16), "<u8")
    return int(total), int(done)


def _cfg():
    # a small queue, so a job is pushed a few queue-windows at a time
    return sb.engine_config(slots=1 << 18, item_paths=1 << 14)


@pytest.fixture(scope="module")
def cornell():
    sb.init(0)
    with sb.Scene(scenes.cornell_box()) as sc:
        yield sc


def _uninterrupted(sc, cam, params):
    with sb.Server(_cfg()) as srv:
        slot = srv.add_scene(sc)
        return srv.wait(srv.submit(slot, cam, params), timeout_ms=600000)[0]


def test_checkpoint_resumed_in_new_server_equals_uninterrupted(cornell, tmp_path):
    cam, params = _job()
    path = str(tmp_path / "job.ckp")
    with sb.Server(_cfg()) as srv:
        slot = srv.add_scene(cornell)
        jid = srv.submit(slot, cam, params)
        time.sleep(0.02)
        srv.pause(jid)
        srv.checkpoint(jid, path)
        total, done = _counts(path)
        assert 0 < done < total, (done, total)
        srv.cancel(jid)
    with sb.Server(_cfg()) as srv2:
        slot = srv2.add_scene(cornell)
        img, st = srv2.wait(srv2.submit_resume(slot, path), timeout_ms=600000)
    assert st["status"] == sb.SNOG_OK
    full = _uninterrupted(cornell, cam, params)
    assert np.isfinite(img).all() and img.mean() > 0.05
    assert np.allclose(img, full, rtol=1e-5, atol=1e-6), np.abs(img - full).max()


def test_paused_job_lets_others_run_then_resumes(cornell, tmp_path):
    cam, params = _job(seed=21)
    cam_s, params_s = _job(64, 64, 4, seed=22)
    with sb.Server(_cfg()) as srv:
        slot = srv.add_scene(cornell)
        big = srv.submit(slot, cam, params)
        time.sleep(0.02)
        srv.pause(big)
        small = srv.submit(slot, cam_s, params_s)
        img_s, st_s = srv.wait(small, timeout_ms=120000)
        assert st_s["status"] == sb.SNOG_OK
        assert srv.poll(big) is None                 # still paused
        srv.resume(big)
        img_b, st_b = srv.wait(big, timeout_ms=600000)
    assert st_b["status"] == sb.SNOG_OK
    full = _uninterrupted(cornell, cam, params)
    assert np.allclose(img_b, full, rtol=1e-5, atol=1e-6)


def test_checkpoint_errors(cornell, tmp_path):
    cam, params = _job(256, 256, 16, seed=3)
    path = str(tmp_path / "a.ckp")
    with sb.Server(_cfg()) as srv:
        slot = srv.add_scene(cornell)
        jid = srv.submit(slot, cam, params)
        with pytest.raises(sb.SnogError) as e:          # not paused
            srv.checkpoint(jid, path, timeout_ms=100)
        assert e.value.code == sb.SNOG_EINVAL
        srv.pause(jid)
        srv.checkpoint(jid, path)
        with pytest.raises(sb.SnogError) as e:
            srv.checkpoint(12345, path)
        assert e.value.code == sb.SNOG_ENOTFOUND
        srv.cancel(jid)
        with sb.Scene(scenes.mixed_scene(500, 20, 20, seed=1)) as other:
            oslot = srv.add_scene(other)
            jbad = srv.submit_resume(oslot, path)
            with pytest.raises(sb.SnogError) as e:       # taken on another scene
                srv.wait(jbad)
            assert "different scene" in str(e.value)
        bad = str(tmp_path / "bad.ckp")
        with open(path, "rb") as f:
            data = f.read()
        with open(bad, "wb") as f:
            f.write(data[:-8])                           # truncated
        with pytest.raises(sb.SnogError) as e:
            srv.submit_resume(slot, bad)
        assert e.value.code == sb.SNOG_EINVAL
        # a header whose path counts disagree with the job or with the file:
        # refused before anything is sized from them
        for total_delta, done_value in ((1, None), (0, 1 << 31)):
            forged = bytearray(data)
            total, done = np.frombuffer(bytes(forged[CKP_HEAD:CKP_HEAD + 16]), "<u8")
            forged[CKP_HEAD:CKP_HEAD + 8] = np.uint64(total + total_delta).tobytes()
            if done_value is not None:
                forged[CKP_HEAD + 8:CKP_HEAD + 16] = np.uint64(min(done_value, total)).tobytes()
            with open(bad, "wb") as f:
                f.write(bytes(forged))
            with pytest.raises(sb.SnogError) as e:
                srv.submit_resume(slot, bad)
            assert e.value.code == sb.SNOG_EINVAL and "complete snogray_b200 checkpoint" in str(e.value)
