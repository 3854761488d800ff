"""The product's octree builder against the reference's octree.

The node arrays (BFS order, children, list heads), the packed surface lists,
the root cube origin and size must be the reference's exactly
(space/octree-builder.cc:173-650): hit ids depend on them.  Golden digests come
from the reference compiled in place (tests/golden/gen_golden.py); when the
compiled reference is present it is also run live on further scenes.
"""

import hashlib

import numpy as np
import pytest

import spec
from gen_golden import TRACE_CASES
from snogray_b200 import Scene, scenes


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(TRACE_CASES))
def test_octree_matches_reference_fixture(name, golden):
    g = golden(f"trace_{name}.npz")
    sd = TRACE_CASES[name][0]()
    assert scenes.scene_digest(sd) == str(g["scene_digest"]), "scene generator drifted"
    with Scene(sd, device=False) as sc:
        oc = sc.octree()
        info = sc.info()
    assert len(oc["heads"]) == int(g["oct_nodes"])
    assert np.array_equal(oc["origin"], g["oct_origin"])
    assert np.float32(oc["size"]) == np.float32(g["oct_size"])
    assert _digest(oc["children"]) == str(g["oct_children_digest"])
    assert _digest(oc["heads"]) == str(g["oct_heads_digest"])
    assert _digest(oc["list"]) == str(g["oct_list_digest"])
    assert info["max_depth"] >= 1


LIVE = [
    lambda: scenes.cornell_box(),
    lambda: scenes.random_triangles(3000, seed=17, edge_lo=0.0, edge_hi=0.3),
    lambda: scenes.mixed_scene(500, 500, 500, seed=23),
    lambda: scenes.soup_scene(5000, 4),
    lambda: scenes.terrain_scene(n=48, n_spheres=10, seed=3, env_w=32, env_h=16),
]


@pytest.mark.skipif(not spec.have_ref(), reason="compiled reference not present")
@pytest.mark.parametrize("k", range(len(LIVE)))
def test_octree_matches_live_reference(k):
    sd = LIVE[k]()
    ref = spec.ref_octree(sd)
    with Scene(sd, device=False) as sc:
        mine = sc.octree()
    for key in ("children", "heads", "list", "origin"):
        assert np.array_equal(ref[key], mine[key]), key
    assert np.float32(ref["size"]) == np.float32(mine["size"])


def test_degenerate_triangles_left_out():
    # A zero-area triangle is not inserted (surface/mesh.cc:833-846).
    sd = scenes.random_triangles(50, seed=1)
    v = sd.vertices.copy()
    v[5] = v[3]                                  # triangle 1 collapses to a segment
    sd.vertices = v
    with Scene(sd, device=False) as sc:
        oc = sc.octree()
    assert 1 not in set(oc["list"].tolist())
    assert 0 in set(oc["list"].tolist())


def test_empty_scene_rejected():
    sd = scenes.cornell_box()
    sd.vertices = np.zeros((0, 3), np.float32)
    sd.triangles = np.zeros((0, 3), np.uint32)
    sd.tri_mat = np.zeros(0, np.uint32)
    sd.spheres = sd.spheres[:0]
    sd.tripars = sd.tripars[:0]
    import snogray_b200 as sb
    with pytest.raises(sb.SnogError):
        Scene(sd, device=False)


@pytest.mark.parametrize("mode", [3, 3 << 8, 1 << 10, 0xff])
def test_unknown_scene_modes_refused_before_any_device_work(mode):
    """snog_scene_create_ex refuses an unknown octree builder or list
    dealing (SNOG_LISTS_*) before it touches the device."""
    import snogray_b200 as sb
    with pytest.raises(sb.SnogError) as e:
        Scene(scenes.cornell_box(), octree=mode)
    assert e.value.code == sb.SNOG_EINVAL
    with pytest.raises(ValueError):
        Scene(scenes.cornell_box(), lists="triple")


def test_glass_media_are_shared_and_bounded():
    """Glass materials with equal ior and absorption share one medium; more
    than 31 distinct media is refused (the path state's medium ids are 5
    bits)."""
    import snogray_b200 as sb
    base = scenes.random_triangles(8, seed=1)
    same = scenes._mats([scenes.material(scenes.MAT_GLASS, ior_n=1.5) for _ in range(40)])
    sph = np.zeros(40, scenes.SPHERE_DTYPE)
    sph["center"] = np.linspace(0, 1, 40)[:, None]
    sph["radius"] = 0.01
    sph["mat"] = np.arange(40)
    sd = scenes.SceneData(materials=same, vertices=base.vertices, triangles=base.triangles,
                          tri_mat=np.zeros(8, np.uint32), spheres=sph)
    sb.Scene(sd, device=False).close()
    sd.materials = scenes._mats([scenes.material(scenes.MAT_GLASS, ior_n=1.1 + 0.01 * k) for k in range(40)])
    with pytest.raises(sb.SnogError) as ei:
        sb.Scene(sd, device=False)
    assert ei.value.code == sb.SNOG_EINVAL and "31 distinct" in str(ei.value)
