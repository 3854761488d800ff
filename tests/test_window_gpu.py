"""Partial renders (the reference's --limit: a RenderPattern with the
filter margin and an output window with a sample base, snogray.lua:442-454,
543-560) through snog_render_window.

* the whole-image window is snog_render itself (same paths, same streams);
* a limited window renders the same image as the full render's window, in
  distribution (different path indices, so different streams): per-channel
  window means within 4 standard errors over K seeds each side;
* output pixels beyond the filter's reach of the pattern get no sample;
* the direct integrator (streaming engine) takes windows too;
* malformed windows are refused.
"""

import math

import numpy as np
import pytest

import snogray_b200 as sb
from snogray_b200 import scenes

pytestmark = pytest.mark.gpu

W, H, SPP = 64, 48, 16


@pytest.fixture(scope="module")
def cornell():
    with sb.Scene(scenes.cornell_box()) as sc:
        yield sc


def test_whole_image_window_is_the_render(cornell):
    cam = scenes.cornell_camera(W, H)
    p = scenes.cornell_params(W, H, SPP, seed=11)
    full, st = cornell.render(cam, p)
    win, stw = cornell.render_window(cam, p, (-2, -2, W + 4, H + 4), (0, 0, W, H))
    assert st["paths"] == stw["paths"]
    assert np.allclose(full, win, rtol=1e-5, atol=1e-6)


def test_limit_window_matches_full_render(cornell):
    lx, ly, lw, lh = 10, 8, 30, 20
    cam = scenes.cornell_camera(W, H)
    k = 16
    a, b = [], []
    for i in range(k):
        full, _ = cornell.render(cam, scenes.cornell_params(W, H, SPP, seed=100 + i))
        a.append(full[ly:ly + lh, lx:lx + lw].reshape(-1, 3).mean(0))
        win, st = cornell.render_window(cam, scenes.cornell_params(W, H, SPP, seed=200 + i),
                                        (lx - 2, ly - 2, lw + 4, lh + 4), (lx, ly, lw, lh))
        assert win.shape == (lh, lw, 3) and st["paths"] == (lw + 4) * (lh + 4) * SPP
        b.append(win.reshape(-1, 3).mean(0))
    a, b = np.array(a), np.array(b)
    se = np.sqrt(a.var(0, ddof=1) / k + b.var(0, ddof=1) / k)
    z = np.abs(a.mean(0) - b.mean(0)) / se
    assert (z < 4).all(), (a.mean(0), b.mean(0), z)


def test_pixels_beyond_the_pattern_get_no_samples(cornell):
    cam = scenes.cornell_camera(W, H)
    img, st = cornell.render_window(cam, scenes.cornell_params(W, H, SPP, seed=3), (20, 15, 6, 5), (0, 0, W, H))
    assert st["paths"] == 6 * 5 * SPP
    yy, xx = np.mgrid[0:H, 0:W]
    # a sample in pattern pixel p reaches the output pixels within 2 of p
    reach = (xx >= 18) & (xx < 28) & (yy >= 13) & (yy < 22)
    assert (img[~reach] == 0).all()
    assert (img[15:20, 20:26].sum(-1) > 0).all()


def test_direct_integrator_window(cornell):
    cam = scenes.cornell_camera(W, H)
    p = scenes.direct_params(W, H, 8, seed=4, light_samples=2)
    full, _ = cornell.render(cam, p)
    win, _ = cornell.render_window(cam, p, (-2, -2, W + 4, H + 4), (0, 0, W, H))
    # same paths on the same engine: equal up to the order of float atomics
    assert np.allclose(full, win, rtol=1e-4, atol=1e-5)
    part, st = cornell.render_window(cam, p, (8, 6, 24, 20), (10, 8, 20, 16))
    assert part.shape == (16, 20, 3) and np.isfinite(part).all() and part.mean() > 0
    assert st["paths"] == 24 * 20 * 8


@pytest.mark.parametrize("bad", [
    ((0, 0, 0, 10), (0, 0, 10, 10)),          # empty pattern
    ((0, 0, 10, 10), (0, 0, 10, 0)),          # empty output
    ((-(1 << 21), 0, 10, 10), (0, 0, 10, 10)),  # offset out of range
])
def test_bad_windows_are_refused(cornell, bad):
    cam = scenes.cornell_camera(W, H)
    with pytest.raises(sb.SnogError) as ei:
        cornell.render_window(cam, scenes.cornell_params(W, H, 4), *bad)
    assert ei.value.code == sb.SNOG_EINVAL
