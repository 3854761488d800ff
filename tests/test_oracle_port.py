"""Pin the oracle's restatement (oracle/port.cc) to the reference.

The restatement is what the GPU tests check the CUDA path against at sizes
no fixture can hold, so it must itself reproduce the reference: octree arrays,
hit ids, hit distances bit for bit, and the reference's node-call counts
(the restatement recurses exactly as space/octree.cc:175-300 does).
"""

import hashlib

import numpy as np
import pytest

import spec
from gen_golden import TRACE_CASES
from snogray_b200 import scenes


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(TRACE_CASES))
def test_port_octree_matches_reference(name, golden):
    g = golden(f"trace_{name}.npz")
    sd = TRACE_CASES[name][0]()
    oc = spec.port_octree(sd)
    assert _digest(oc["children"]) == str(g["oct_children_digest"])
    assert _digest(oc["heads"]) == str(g["oct_heads_digest"])
    assert _digest(oc["list"]) == str(g["oct_list_digest"])
    assert np.array_equal(oc["origin"], g["oct_origin"])


@pytest.mark.parametrize("name", sorted(TRACE_CASES))
def test_port_trace_matches_reference(name, golden):
    g = golden(f"trace_{name}.npz")
    make_scene, make_rays = TRACE_CASES[name]
    sd = make_scene()
    rays = make_rays(sd)
    nc = int(g["n_closest"])
    prim, t, _, st, _ = spec.port_trace(sd, rays, nc, threads=4)
    assert np.array_equal(prim, g["prim"])
    hit = np.nonzero(prim[:nc] >= 0)[0]
    assert np.array_equal(t[hit].view(np.uint32), g["t"][hit].view(np.uint32))
    assert st["closest"]["node_calls"] == int(g["closest_nodes"])
    assert st["any"]["node_calls"] == int(g["any_nodes"])


def test_port_miss_and_empty_cases():
    sd = scenes.cornell_box()
    rays = np.zeros((7, 3), np.float32)
    rays[0:3, 0] = (5, 5, 5)                       # outside, pointing away
    rays[3:6, 0] = (1, 0, 0)
    rays[0:3, 1] = (0.5, 0.5, 0.5)                 # zero direction hits nothing
    rays[0:3, 2] = (0.5, 0.5, 0.5)                 # zero extent hits nothing
    rays[3:6, 2] = (0, 1, 0)
    rays[6] = (np.inf, np.inf, 0.0)
    prim, _, _, _, _ = spec.port_trace(sd, rays, 3, threads=1)
    assert (prim == -1).all()
