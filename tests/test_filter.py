"""The image output's filter, pinned to the reference.

The device splat (k_splat, k_resolve) is compared in tests/test_splat_gpu.py
with a float64 restatement of the Mitchell-Netravali filter.  This CPU test
pins that restatement to the reference's own filter, ImageMitchellFilt::val
(image/image-mitchell-filt.h:45-65, default b = c = 1/3, radius 2), evaluated
by the reference compiled in place (tests/golden/filter_mitchell.npz, harness
mode `filter`): at the knots of both axes and 4096 random offsets over the
filter's support and beyond.
"""

from __future__ import annotations

import os

import numpy as np

import spec
from gen_golden import filter_offsets
from test_splat_gpu import B, C, mitchell1

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_restatement_equals_reference_filter():
    g = np.load(os.path.join(GOLDEN, "filter_mitchell.npz"))
    assert np.array_equal(g["xy"], filter_offsets())
    assert np.float32(B) == g["b"] and np.float32(C) == g["c"] and g["radius"] == 2.0
    xy = g["xy"].astype(np.float64)
    mine = mitchell1(xy[:, 0]) * mitchell1(xy[:, 1])
    # The reference evaluates in float32: a few ulps of the largest value (0.79).
    assert np.abs(mine - g["val"]).max() < 2e-6
    # zero outside the radius, negative lobes inside it
    outside = np.abs(xy).max(1) > 2.0
    assert (g["val"][outside] == 0).all()
    assert (g["val"] < 0).any()


def test_fixture_is_the_live_reference():
    if not spec.have_ref():
        return
    g = np.load(os.path.join(GOLDEN, "filter_mitchell.npz"))
    v, _ = spec.ref_filter(g["xy"])
    assert np.array_equal(v, g["val"])
